// Internal declarations shared by the host code and the CUDA kernels of libvct.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/vct.h"

namespace vct {

// Error reporting: the last message per host thread.
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
// The geometry limits every entry point that takes a vct_geometry applies
// (views, channels, grid size, pixel size, xfactor); `who` prefixes the
// error message.  Returns VCT_OK or VCT_E_ARG.
int check_geometry(const vct_geometry* g, const char* who);

#define VCT_CUDA(call)                                     \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return vct::cuda_fail(e_, #call); \
  } while (0)

// Index checks of the bounds build (libvct_bounds.so, -DVCT_BOUNDS=1): an
// access whose check fails is skipped and counted, with the largest failing
// source line, in its translation unit's counters, which
// vct_bounds_violations reads and clears.  Nothing traps.  In the product
// build VCT_INDEX_OK(c) is `true` and the checks compile away.
#ifndef VCT_BOUNDS
#define VCT_BOUNDS 0
#endif
#if defined(__CUDACC__)
#if VCT_BOUNDS
static __device__ unsigned int vct_bounds_hits_;
static __device__ int vct_bounds_line_;
static __host__ __device__ __forceinline__ bool vct_index_ok_(bool ok, int line) {
#if defined(__CUDA_ARCH__)
  if (!ok) {
    atomicAdd(&vct_bounds_hits_, 1u);
    atomicMax(&vct_bounds_line_, line);
  }
#endif
  return ok;
}
#define VCT_INDEX_OK(cond) vct::vct_index_ok_((cond), __LINE__)
// Defines the translation unit's reader: (hits, largest line), then clears.
#define VCT_BOUNDS_READER(name)                                                        \
  int name(unsigned int* hits, int* line) {                                            \
    VCT_CUDA(cudaMemcpyFromSymbol(hits, vct_bounds_hits_, sizeof(unsigned int)));      \
    VCT_CUDA(cudaMemcpyFromSymbol(line, vct_bounds_line_, sizeof(int)));              \
    const unsigned int z = 0;                                                          \
    VCT_CUDA(cudaMemcpyToSymbol(vct_bounds_hits_, &z, sizeof z));                      \
    VCT_CUDA(cudaMemcpyToSymbol(vct_bounds_line_, &z, sizeof z));                      \
    return VCT_OK;                                                                     \
  }
#else
#define VCT_INDEX_OK(cond) true
#define VCT_BOUNDS_READER(name)              \
  int name(unsigned int* hits, int* line) { \
    *hits = 0;                               \
    *line = 0;                               \
    return VCT_OK;                           \
  }
#endif
#endif
// The readers, one per instrumented translation unit.
int bounds_forward(unsigned int* hits, int* line);
int bounds_adjoint(unsigned int* hits, int* line);
int bounds_fbp(unsigned int* hits, int* line);
int bounds_lengthproj(unsigned int* hits, int* line);
int bounds_measured(unsigned int* hits, int* line);

// Geometry constants derived once per context; every field is computed on the
// host with the reference's own expression order so the device walk sees
// bit-identical inputs.
struct DevGeom {
  int N;           // recon_size
  int nxm;         // (int)(N*0.5)                MB/reprojection_TOMO.cpp:25
  double s;        // pixel_cm (reconScale)
  double lim;      // double(nxm)*reconScale      :79
  double rmax;     // N*0.5*1.0                   :37 (pixels, compared with cm)
  int rmax_active; // 1 when a segment midpoint can reach rmax (pixel >= ~0.707 cm)
  double sid;      // DIST_BTWN_SRC_AND_ISOCENT_CM
  int views_used;  // views/2*2                    :35
  int views;       // projImgHeight
  int width;       // projImgWidth
  int C;           // end_channel - start_channel
  int start;       // start_channel
  double dens_div; // stored density units per g/cm^3 (1000: the reference's maps)
};

// Packed maps: one 16-byte record per pixel, 8 int16 materials (unused
// materials 0).  Negative densities are stored as 0: the reference gives
// them zero weight (MB/reprojection_TOMO.cpp:151-155).  The grid is padded
// by kMapPad cells on every side (see vct_forward.cu).
struct alignas(16) PixelRec {
  int16_t m[8];
};
constexpr int kMapPad = 2;
inline size_t padded_pixels(int N) { return (size_t)(N + 2 * kMapPad) * (size_t)(N + 2 * kMapPad); }
// The device map buffer holds the row-major padded grid followed by its
// transposed copy.
inline size_t map_records(int N) { return 2 * padded_pixels(N); }

struct FwdStats {
  unsigned int max_bits;  // float bits of the maximum (values are >= 0)
  unsigned int min_bits;  // float bits of the minimum
  unsigned long long segments;
  unsigned int pad;
};

struct Workspace;  // device buffers, defined in vct_host.cpp

// Launchers (vct_forward.cu / vct_fbp.cu).  All enqueue on `st`.
int launch_pack_maps(const int16_t* d_maps, int M, int N, PixelRec* d_packed, cudaStream_t st);
int launch_forward(const DevGeom& g, const PixelRec* d_maps, int M, const double* d_mu_tab,
                   const float* d_pdf, int NE, const double* d_cos, const double* d_sin,
                   const double* d_det_ox, const double* d_det_oy, int sum_mode, int fast, float* d_out,
                   double* d_lint, FwdStats* d_stats, cudaStream_t st, int v0 = 0, int v1 = -1,
                   const int* d_exact = nullptr, int nexact = 0);
// The rays whose fast-walk plan is the exact walk (geometry only): with
// d_list == nullptr only their count (*d_count); else up to cap of them.
// launch_forward given that list walks them a warp per ray after the rest.
int launch_exact_list(const DevGeom& g, const double* d_cos, const double* d_sin, const double* d_px0,
                      const double* d_py0, int* d_list, int cap, int* d_count, cudaStream_t st);
// One slice of a batched forward (vct_batch.cpp): its geometry, device
// tables and outputs.  tile0 is the index of its first ray tile.
struct FwdJob {
  DevGeom g;
  const PixelRec* maps;
  const double* mu;  // [NE][M] mu*log2(e)/xfactor
  const float* pdf;
  const double* cos_t;
  const double* sin_t;
  const double* px0;
  const double* py0;
  float* out;        // [views][width]
  FwdStats* stats;
  const int* exact;  // the rays the fast walk hands back (walked a warp per ray after the rest), or NULL
  int nexact;
  unsigned int tile0;
  int NE, fast;
};
// d_xfirst: prefix sums [njobs + 1] of the jobs' nexact (total nexact_total).
int launch_forward_batch(const FwdJob* d_jobs, int njobs, int M, int tile_rays, unsigned int ntiles, int ne_max,
                         int grid, unsigned int* d_counter, const unsigned int* d_xfirst, unsigned int nexact_total,
                         cudaStream_t st);
int forward_batch_occupancy(int M, int ne_max, int* blocks_per_sm);
int launch_normalize_noise(const DevGeom& g, const float* d_in, float* d_out, const FwdStats* d_stats,
                           int pad_zero, double sigma, uint64_t seed, cudaStream_t st, int r0 = 0, int r1 = -1);
// The batch engine's launches after the forward (vct_batch.cpp): one launch
// per stage runs the blocks of every job.  A PostJob holds one job's
// arguments of the single-slice normalisation/noise and FBP kernels; per
// stage, first[stage * (n + 1) + j] is the index of job j's first block
// (prefix sums; first[.. + n] is the stage's block count).  The blocks do
// exactly what the single-slice launches do, so results are bit-identical.
struct PostJob {
  float* sino;            // [V][W]: un-normalised in, normalised (+ noise) out
  const FwdStats* stats;
  int V, W, pad_zero;
  double sigma;
  unsigned int key0, key1;
  float* img;             // [N][N], or NULL (no FBP)
  const double* coeff;    // weight factors [C]
  const float* h0;        // filter kernel [2C-1], then the row factors [C]
  const float2* cs;       // (cos, sin) per view
  float* q;               // filtered sinogram [V][C]
  float2* q2;             // its interpolation pairs [V][C] (quarter-turn jobs), or NULL
  int C, start, N, sym, win;
  float scale, sid, inv_dbeta, center, out_scale;
};
enum { kPostNorm = 0, kPostWeight, kPostFilter, kPostBpSym, kPostBpGen, kPostStages };  // kPostWeight: no blocks (fused into the filter)
// Block counts of one job per stage (0 where the stage does not apply).
void post_job_blocks(const PostJob& j, unsigned int blocks[kPostStages]);
// The backprojector's launch parameters of one slice (as launch_fbp_backproject
// derives them): fills C, start, N, sym, win, scale, sid, inv_dbeta, center,
// out_scale.
void fbp_bp_params(int V, int W, int start, int C, int N, double pixel_cm, double sid, double max_beta, int xfactor,
                   PostJob* j);
int launch_normalize_noise_batch(const PostJob* d_jobs, const unsigned int* d_first, int n, unsigned int nblocks,
                                 cudaStream_t st);
// weight, filter and the two backprojectors; cmax: largest channel count,
// winmax: largest staged window of a general-backprojector job.
int launch_fbp_batch(const PostJob* d_jobs, const unsigned int* d_first, int n, const unsigned int nblocks[kPostStages],
                     int cmax, int winmax, int view_groups, cudaStream_t st);
// Map packing of many slices in one launch: job j packs maps[j] (N[j]) into
// out[j]; first[j] is its first block.
struct PackJob {
  const int16_t* maps;
  PixelRec* out;
  int N;
};
int launch_pack_maps_batch(const PackJob* d_jobs, const unsigned int* d_first, int n, int M, unsigned int nblocks,
                           cudaStream_t st);
unsigned int pack_maps_blocks(int N);
// bh_alpha != 0: beam-hardening correction of the line integrals on the way.
int launch_fbp_weight(const float* d_sino, int V, int W, int start, int C, const double* d_coeff,
                      float* d_g, cudaStream_t st, double bh_alpha = 0.0, double bh_beta = 0.0);
int launch_beam_hardening(float* d_p, long long n, double alpha, double beta, cudaStream_t st);
// launch_fbp_weight + launch_fbp_filter in one pass (the weighted sinogram is
// not stored).
int launch_fbp_weight_filter(const float* d_sino, int W, int start, const double* d_coeff, double bh_alpha,
                             double bh_beta, const float* d_h0, const float* d_cm, int V, int C, int in_mode,
                             float* d_q, float2* d_q2, cudaStream_t st);
// d_q2 (optional): the filtered rows also as interpolation pairs
// (q[c], q[c+1]) [V][C], for the quarter-turn backprojector.
int launch_fbp_filter(const float* d_g, const float* d_h0, const float* d_cm, int V, int C, int in_mode,
                      float* d_q, cudaStream_t st, float2* d_q2 = nullptr);
// view_groups: how many warp groups split the views of the quarter-turn
// backprojector (2, 4 or 8; other values mean 4).
// band0..band1: the image rows [band0, band1) of the general backprojector,
// or the orbit rows [band0, band1) of [0, N/2) of the quarter-turn one
// (fbp_band_count); pixels outside the band are not written.
int fbp_band_count(int V, int N);
// d_q2 (optional): the pairs of launch_fbp_filter, read by the quarter-turn
// backprojector instead of two loads from d_q.
int launch_fbp_backproject(const float* d_q, int V, int C, int N, double pixel_cm, double sid,
                           double max_beta, int xfactor, const float* d_cs, float* d_img,
                           cudaStream_t st, int view_groups = 4, int band0 = 0, int band1 = -1,
                           const float2* d_q2 = nullptr);
// Transposes of the three FBP steps (vct_fbp.cu).
size_t fbp_backproject_t_scratch(int V, int C, int N);  // 64-bit words of d_acc
int launch_fbp_backproject_t(const float* d_u, int V, int C, int N, double pixel_cm, double sid, double max_beta,
                             int xfactor, const float* d_cs, unsigned long long* d_acc, float* d_qb,
                             cudaStream_t st);
int launch_fbp_filter_t(const float* d_q, const float* d_h0, const float* d_cm, int V, int C, float* d_g,
                        cudaStream_t st);
int launch_fbp_weight_t(const float* d_g, int V, int W, int start, int C, const double* d_coeff, float* d_lam,
                        cudaStream_t st);

// lengthproj_TOMO (vct_lengthproj.cu): geometry of one slice.
struct LpGeom {
  int N, V, W, start_ch, end_ch;
  int start, count, nrot;  // first view, views used, whole rotations before it
  int first, stride;       // rows first + k*stride, k < count (lengthproj_TOMO: 0, 1)
  int round_tables;        // 1: chord and channel rounded to float (lengthproj_TOMO_2)
  double s, sid, dsrc, diso, R, iso, dalpha;
};
int launch_lengthproj(const LpGeom& q, const double* d_cos, const double* d_sin, const float* d_proj, float* d_npf,
                      cudaStream_t st);

// The reference's iterative step (vct_ir.cu).
int launch_ir_update(int N, const float* d_before, const float* d_prior, const float* d_npf, const float* d_npf_re,
                     double wbefore, double w_tv, double w_prior, int ite, int thinout, float* d_after,
                     cudaStream_t st);
int squdiff_scratch_doubles();
int launch_squdiff(const float* d_p, const float* d_r, int W, int start, int C, int first, int stride, int rows,
                   int quad, double* d_part, double* d_out, cudaStream_t st);

// Adjoint (vct_adjoint.cu).  Ray kinds of the per-ray walk record.
constexpr int kAdjRayNone = 0;   // no segment
constexpr int kAdjRayFast = 1;   // fast walk: lumped segment + chords in a major-index range
constexpr int kAdjRayExact = 2;  // exact walk (scattered in fixed point)

// The gather splits each tile's views into kAdjChunks consecutive ranges,
// each a separate work item with its own partial sums (summed in order by
// the fold), so the items spread evenly over the resident blocks.
#ifndef VCT_ADJ_CHUNKS
#define VCT_ADJ_CHUNKS 2
#endif
constexpr int kAdjChunks = VCT_ADJ_CHUNKS;
// The ranges used for M elements: kAdjChunks up to 6 elements, one above (at
// 8 elements the batch's gather lost more to the split, in registers, than
// the single slice gained).
#if defined(__CUDACC__)
__host__ __device__
#endif
constexpr int adj_chunks(int M) { return M <= 6 ? kAdjChunks : 1; }

struct AdjGeom {
  int N, nxm, C, start, views_used;
  int log2_terms;     // bound on log2(terms per pixel) of the exact-walk scatter
  double s, sid, iso, inv_dalpha;
  double lmax;        // longest possible segment (cm)
};

int launch_adj_plan(const DevGeom& g, const double* d_cos, const double* d_sin, const double* d_px0,
                    const double* d_py0, int4* d_rec, int* d_special, int* d_nspecial, cudaStream_t st);
int adj_forward_blocks(const DevGeom& g);
int launch_adj_forward(const DevGeom& g, const PixelRec* d_maps, int M, const double* d_mu_l2, const float* d_pdf,
                       int NE, double ynorm, const double* d_cos, const double* d_sin, const double* d_px0,
                       const double* d_py0, const int4* d_rec, const double* d_lsp, int mode, const float* d_meas,
                       const float* d_wts, float* d_g, double* d_loss_part, unsigned int* d_gmax, cudaStream_t st);
// Line integrals [nspecial][M] of the rays the fast walk hands back (the
// exact walk, one warp per ray); adj_forward reads them for those rays.
int launch_adj_lines(const DevGeom& g, int M, const PixelRec* d_maps, const double* d_cos, const double* d_sin,
                     const double* d_px0, const double* d_py0, const int* d_special, int nspecial_host, double* d_lsp,
                     cudaStream_t st);
int launch_adj_loss(const double* d_part, int n, double* d_out, cudaStream_t st);
int launch_adj_special(const DevGeom& g, int M, const double* d_cos, const double* d_sin, const double* d_px0,
                       const double* d_py0, const int* d_special, const int* d_nspecial, int nspecial_host,
                       const float* d_g, const unsigned int* d_gmax, double lmax, int log2_terms,
                       unsigned long long* d_acc, cudaStream_t st);
int launch_adj_gmax(int M, const int* d_special, const int* d_nspecial, int nspecial_host, const float* d_g,
                    unsigned int* d_gmax, cudaStream_t st);
int adj_pick_tile(const AdjGeom& a, double lim);
// Gather into d_ext [M][N+1][N+1] (cells -1..N-1), then fold into d_grad
// [M][N][N] together with the exact-walk rays' fixed-point sums (d_sacc may
// be NULL).  Two launches.
// Per (tile, view) records of the gather (geometry only, once per context):
// their size in bytes, and the kernel that fills them (window overflow sets
// bit 0 of *d_status).
size_t adj_tileview_bytes(const AdjGeom& a, int tile);
int launch_adj_tiles(const AdjGeom& a, int tile, const double* d_cos, const double* d_sin, const int4* d_rec,
                     void* d_tv, int* d_status, cudaStream_t st);
int launch_adj_gather(const AdjGeom& a, int M, int tile, const double* d_cos, const double* d_sin,
                      const double2* d_dir, const int4* d_rec, const float* d_g, const void* d_tv, float* d_ext,
                      cudaStream_t st);
// Cells at index -1 onto index 0 and the exact-walk rays' fixed-point sums
// added: d_ext [M][N+1][N+1] -> d_grad [M][N][N].
int launch_adj_fold(const AdjGeom& a, int M, const unsigned long long* d_sacc, const unsigned int* d_gmax,
                    const float* d_ext, float* d_grad, cudaStream_t st);

// Loss and gradient of many slices, one launch per stage (vct_batch.cpp):
// the arguments of one job's vct_forward_adjoint_dev.  Per stage,
// first[stage * (n + 1) + j] is job j's first block (prefix sums); the
// persistent forward takes 128-ray tiles from a counter (tile0: the job's
// first tile).  Each block does what the single-slice launch does, in the
// same order, so losses and gradients are bit-identical.
struct AdjJob {
  DevGeom g;
  AdjGeom a;
  const PixelRec* maps;
  const double* mu;  // [NE][M] mu*log2(e)/xfactor
  const float* pdf;
  int NE;
  double ynorm;
  const double* cos_t;
  const double* sin_t;
  const double* px0;
  const double* py0;
  const double2* dir;
  const int4* rec;
  const void* tv;    // the gather's per (tile, view) records (the batch's tile shape)
  const float* meas;
  const float* wts;
  float* gr;         // ray factors [rays][M]
  double* part;      // loss partials, one per 128-ray tile
  double* loss;
  unsigned int* gmax;
  const int* special;
  int nspecial;
  double* lsp;       // exact-walk rays' line integrals [nspecial][M]
  unsigned long long* sacc;  // exact-walk sums [M][N][N], NULL without exact-walk rays
  double lmax;
  int log2_terms;
  float* ext;        // [kAdjChunks][M][N+1][N+1]
  float* grad;       // [M][N][N]
  unsigned int tile0;
};
// Stages; the gather has one stage per tile shape (a job's own shape,
// adj_pick_tile), kAdjStGather + shape.
enum { kAdjStReset = 0, kAdjStLines, kAdjStLoss, kAdjStSpecial, kAdjStGather, kAdjStFold = kAdjStGather + 4, kAdjStages };
// Block counts of one job per stage for its gather tile shape and M elements.
void adj_job_blocks(const AdjJob& j, int M, int tile, unsigned int blocks[kAdjStages]);
// 128-ray tiles of one job's persistent forward.
#if defined(__CUDACC__)
__host__ __device__
#endif
unsigned int adj_job_ray_tiles(const DevGeom& g);
// The exact-walk scatter runs on `side` (forked after the loss sums with
// ev_fork, joined before the fold with ev_join) so that it overlaps the
// gather; side == st runs everything in order on st.
int launch_adj_batch(const AdjJob* d_jobs, const unsigned int* d_first, int n, int M, int ne_max,
                     unsigned int ntiles_ray, const unsigned int nblocks[kAdjStages], unsigned int* d_counter,
                     cudaStream_t st, cudaStream_t side = nullptr, cudaEvent_t ev_fork = nullptr,
                     cudaEvent_t ev_join = nullptr);

}  // namespace vct
