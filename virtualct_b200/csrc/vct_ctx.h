// The context behind vct_ctx* (include/vct.h), shared by the host code
// (vct_host.cpp) and the batch engine (vct_batch.cpp).
#pragma once
#include <cuda_runtime.h>

#include "vct_internal.h"

namespace vct {
// Device buffer that grows on demand.
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  int ensure(size_t count) {
    if (count <= n && p) return VCT_OK;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    VCT_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
    n = count;
    return VCT_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};
// Copy streams, events and double buffers of vct_mbfpa_many, made on its
// first call.
struct Pipe {
  cudaStream_t in = nullptr, out = nullptr;
  cudaEvent_t start = nullptr, ev_in[2] = {}, ev_packed[2] = {}, ev_done[2] = {}, ev_out[2] = {};
  DBuf<int16_t> stage[2];
  DBuf<float> sino[2];
  ~Pipe() {
    for (int s = 0; s < 2; s++) {
      stage[s].release();
      sino[s].release();
      for (cudaEvent_t e : {ev_in[s], ev_packed[s], ev_done[s], ev_out[s]})
        if (e) cudaEventDestroy(e);
    }
    if (start) cudaEventDestroy(start);
    if (in) cudaStreamDestroy(in);
    if (out) cudaStreamDestroy(out);
  }
};
// Per-stage device times of one entry-point call (vct_set_stage_timing):
// an event on the call's stream before its first stage and after each
// stage.  Off by default; when off, begin() and mark() do nothing.
struct StageTimer {
  static constexpr int kMax = 16;
  int on = 0;
  int n = 0;
  const char* name[kMax] = {};
  cudaEvent_t ev[kMax + 1] = {};
  void begin(cudaStream_t s) {
    n = 0;
    if (on) cudaEventRecord(ev[0], s);
  }
  void mark(const char* stage, cudaStream_t s) {
    if (!on || n >= kMax) return;
    name[n] = stage;
    cudaEventRecord(ev[++n], s);
  }
  ~StageTimer() {
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};
}  // namespace vct

struct vct_ctx {
  int device = 0;
  vct_geometry geo{};
  vct::DevGeom dg{};
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  long long launches = 0;
  // geometry tables
  vct::DBuf<double> cos_t, sin_t, det_px0, det_py0;
  vct::DBuf<float> cs_f;  // (cos, sin) pairs in float for the backprojector
  // MBFPA
  int M = 0, NE = 0;
  double ynorm = 0.0;  // sum of the pdf as uploaded (the un-attenuated intensity)
  int maps_ready = 0, spectrum_ready = 0;
  int sum_mode = VCT_SUM_COMPENSATED;
  int walk_mode = VCT_WALK_FAST;
  vct::DBuf<int16_t> maps_raw;
  vct::DBuf<vct::PixelRec> maps;
  vct::DBuf<double> mu_scaled;  // [NE][M], mu/xfactor (reference summation)
  vct::DBuf<double> mu_log2;    // [NE][M], mu*log2(e)/xfactor (compensated summation)
  vct::DBuf<float> pdf;
  vct::DBuf<float> full, out;   // [views][width]
  vct::DBuf<vct::FwdStats> stats;       // [0] live, [1] the reset value
  vct::FwdStats* h_stats = nullptr;  // pinned
  long long last_segments = 0;
  // FBP
  vct::DBuf<double> fbp_coeff;  // SID*cos((k-cw)*dbeta)*dbeta
  vct::DBuf<float> fbp_h[3];    // per filter (1 Ram-Lak, 2 Shepp-Logan): h0[2C-1] + row factors[C]
  vct::DBuf<float> fbp_g, fbp_q, fbp_sino, fbp_img;
  vct::DBuf<float2> fbp_q2;  // filtered rows as interpolation pairs (quarter-turn backprojector)
  vct::DBuf<unsigned long long> fbp_tacc;  // FBP transpose: fixed-point row sums + max|u|
  double bh_alpha = 0.0, bh_beta = 0.0;
  vct::DBuf<double> sq_part;  // calc_squdiff_quad block partials
  vct::DBuf<float> ir_proj, ir_reproj, ir_img;  // iterative step: sinograms [V][W], images 5 x [N][N]
  vct::DBuf<double> ir_out;  // beam-hardening correction in the FBP (alpha 0: off)
  // Adjoint: per-ray walk plans (geometry only), ray factors, fixed-point
  // accumulator of the exact-walk rays, loss partials.
  int adj_ready = 0, adj_nspecial = 0, adj_tile = -1;
  vct::AdjGeom ag{};
  vct::DBuf<int4> adj_rec;
  vct::DBuf<int> adj_special, adj_ints;  // ints: [0] special count, [1] status
  // The rays the fast walk hands back (geometry only, listed by vct_create):
  // [0] their count, then the rays; the forward walks them a warp per ray.
  vct::DBuf<int> fwd_exact;
  int fwd_nexact = 0;
  vct::DBuf<double2> adj_dir;
  vct::DBuf<float4> adj_tv;  // per (tile, view) records of the gather
  vct::DBuf<float> adj_g;
  vct::DBuf<double> adj_part, adj_loss;
  vct::DBuf<unsigned int> adj_gmax;
  vct::DBuf<unsigned long long> adj_sacc;
  vct::DBuf<double> adj_lsp;  // exact-walk rays' line integrals [nspecial][M]
  vct::DBuf<float> adj_meas, adj_wts, adj_grad;
  vct::DBuf<float> adj_ext;  // [kAdjChunks][M][N+1][N+1] gather partial sums before the fold
  vct::Pipe* pipe = nullptr;  // vct_mbfpa_many
  vct::StageTimer timer;      // vct_set_stage_timing
};


namespace vct {
// Internal helpers of vct_host.cpp.
int ctx_check(vct_ctx* c);
int ctx_build_filter(vct_ctx* c, int filter);
int ctx_pad_zero(const vct_ctx* c);
int ctx_fbp(vct_ctx* c, const float* d_sino, int filter, float* d_img, int view_groups);
int ctx_adj_prepare(vct_ctx* c);
int ctx_adj_run(vct_ctx* c, int mode, const float* d_meas, const float* d_wts, const float* d_g, float* d_grad,
                double* d_loss);
}  // namespace vct
