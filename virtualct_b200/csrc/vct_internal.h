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

#define VCT_CUDA(call)                                     \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return vct::cuda_fail(e_, #call); \
  } while (0)

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
                   double* d_lint, FwdStats* d_stats, cudaStream_t st);
int launch_normalize_noise(const DevGeom& g, const float* d_in, float* d_out, const FwdStats* d_stats,
                           int pad_zero, double sigma, uint64_t seed, cudaStream_t st);
int launch_fbp_weight(const float* d_sino, int V, int W, int start, int C, const double* d_coeff,
                      float* d_g, cudaStream_t st);
int launch_fbp_filter(const float* d_g, const float* d_h0, const float* d_cm, int V, int C, int in_mode,
                      float* d_q, cudaStream_t st);
int launch_fbp_backproject(const float* d_q, int V, int C, int N, double pixel_cm, double sid,
                           double max_beta, int xfactor, const float* d_cs, float* d_img,
                           cudaStream_t st);

}  // namespace vct
