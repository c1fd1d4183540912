// Fan-beam FBP on sm_100a: filterSinogram (FBP/filterSinogramTOMO.cpp:205-275)
// and reconstructImage (FBP/reconstructImageTOMO.cpp:11-105) for one slice.
//
//   1. weight:   g[v][k] = -ln p[v][k] * SID*cos((k-cw)*dbeta) * dbeta, once per
//                sample (the reference re-evaluates the log inside its
//                609-long inner loop, i.e. 609 times per sample).
//   2. filter:   q[v][m] = sum_k h[m][k] g[v][k]; h is one kernel shifted
//                per row (times an edge-row factor), so each view is a 1-D
//                convolution, shared memory + register window, FP32 FMA.
//   3. backproject: pixel-driven, equiangular fan weight 1/L^2, linear
//                interpolation on the detector; 32 x 16 pixel tiles, views in
//                chunks with each view's detector window for the tile staged
//                in shared memory.
#include <cuda_runtime.h>

#include <algorithm>

#include "vct_internal.h"
#include "vct_fastmath.cuh"

namespace vct {

// ------------------------------------------------------------------ weight
// With bh_alpha != 0 the beam-hardening correction of
// MB/beam_hardening_correction.cpp:49-56 is applied on the way: the
// line integral y = -ln p becomes |y| + alpha |y|^beta (the reference program
// takes the logarithm in single precision, logf, and stores exp(-y') as float
// for the FBP to take -ln again; here y' goes straight into the weight).
__device__ __forceinline__ void fbp_weight_elem(const float* __restrict__ sino, long long i, int W, int start, int C,
                                                const double* __restrict__ coeff, double bh_alpha, double bh_beta,
                                                float* __restrict__ g) {
  const int v = (int)(i / C);
  const int k = (int)(i - (long long)v * C);
  const float pf = sino[(size_t)v * W + start + k];
  double y;
  if (bh_alpha != 0.0) {
    y = -(double)logf(pf);
    y = fabs(y) + bh_alpha * pow(fabs(y), bh_beta);
  } else {
    y = -log((double)pf);
  }
  g[i] = (float)(y * coeff[k]);
}

__global__ void fbp_weight_kernel(const float* __restrict__ sino, int V, int W, int start, int C,
                                  const double* __restrict__ coeff, double bh_alpha, double bh_beta,
                                  float* __restrict__ g) {
  const long long n = (long long)V * C;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  fbp_weight_elem(sino, i, W, start, C, coeff, bh_alpha, bh_beta, g);
}

int launch_fbp_weight(const float* d_sino, int V, int W, int start, int C, const double* d_coeff,
                        float* d_g, cudaStream_t st, double bh_alpha, double bh_beta) {
  const long long n = (long long)V * C;
  fbp_weight_kernel<<<(int)((n + 255) / 256), 256, 0, st>>>(d_sino, V, W, start, C, d_coeff, bh_alpha, bh_beta,
                                                             d_g);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// The correction on its own, in place: p <- (float)exp(-(|y| + alpha |y|^beta)),
// y = -logf(p), as MB/beam_hardening_correction.cpp:49-56.
__global__ void beam_hardening_kernel(float* __restrict__ p, long long n, double alpha, double beta) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double y = -(double)logf(p[i]);
    y = fabs(y) + alpha * pow(fabs(y), beta);
    p[i] = (float)exp(-y);
  }
}

int launch_beam_hardening(float* d_p, long long n, double alpha, double beta, cudaStream_t st) {
  if (n <= 0) return VCT_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  beam_hardening_kernel<<<(unsigned)blocks, 256, 0, st>>>(d_p, n, alpha, beta);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------------------------------ filter
// q[v][m] = sum_k h[m][k] g[v][k] (FBP/filterSinogramTOMO.cpp:233-243 with the
// constant factors folded into g).  prepareConstMap's rows are one kernel
// shifted, h[m][k] = c_m h0(m-k), with c_m = 1 except the renormalised edge
// rows (:114-123), so each view is a 1-D convolution: one block per view, g
// and h0 in shared memory.  Register tiling: each thread owns FC_R = 4
// consecutive outputs and takes k in chunks of 4; per chunk one 128-bit
// load of g (the same for every thread) and one aligned 128-bit load of
// the 4 new kernel values of a sliding window of 8, h0(m0 - k0 - 3 .. m0 -
// k0 + 4), feed 16 FMAs.  For each output k runs in ascending order, as in
// the reference.
// WEIGHT: the row is loaded straight from the sinogram and weighted on the
// way (the weight kernel's g = -ln p * coeff, optionally with the
// beam-hardening correction), so the weighted sinogram is never stored.
// TRANSPOSE: the transposed filter, g[v][k] = sum_m h0(m-k) c_m q[v][m]; h0
// is even (both kernels depend on |m-k| only), so it is the same convolution
// with the row factor applied to the input instead of the output.
// Outputs per thread (4 / 8 / 12 measured 28.6 / 31.4 / 34.0 us at 800 x 609
// with the sliding window, 30.4 us before it with 4: fewer threads per
// view's block hide less of the shared-load latency).
#ifndef VCT_FC_R
#define VCT_FC_R 4
#endif
constexpr int FC_R = VCT_FC_R, FC_TMAX = 256;
static_assert(FC_R % 4 == 0, "outputs per thread: a multiple of 4");

// Shared memory of one view: g padded to a multiple of 4 (+4 zeros), then
// h0(d) at index OFF + d for |d| <= C-1 (zero around it), OFF = 3 mod 4 so
// the window loads are 16-byte aligned.
__host__ __device__ inline int fc_cpad(int C) { return (C + 3) / 4 * 4; }
__host__ __device__ inline int fc_off(int C) { return fc_cpad(C) + 3; }
__host__ __device__ inline int fc_smem_floats(int C) { return (fc_cpad(C) + 4) + (fc_off(C) + fc_cpad(C) + 8); }
// Threads per block for C channels: one pass of 4 outputs each, up to 256.
inline int fc_threads(int C) {
  int t = ((C + FC_R - 1) / FC_R + 31) / 32 * 32;
  return t > FC_TMAX ? FC_TMAX : t;
}

template <bool TRANSPOSE, bool WEIGHT>
__device__ __forceinline__ void fbp_filter_view(const float* __restrict__ G, const float* __restrict__ h0,
                                                const float* __restrict__ cm, int v, int C, int in_mode,
                                                float* __restrict__ Q, float2* __restrict__ Q2, float* sm,
                                                int W = 0, int start = 0, const double* __restrict__ coeff = nullptr,
                                                double bh_alpha = 0.0, double bh_beta = 0.0) {
  const int cpad = fc_cpad(C), off = fc_off(C);
  float* sg = sm;              // [cpad + 4]
  float* sh = sm + cpad + 4;   // [off + cpad + 8]
  const int nt = blockDim.x;
  for (int k = threadIdx.x; k < cpad + 4; k += nt) {
    float gk = 0.0f;
    if (k < C) {
      if (WEIGHT) {
        const float pf = G[(size_t)v * W + start + k];
        double y;
        if (bh_alpha != 0.0) {
          y = -(double)logf(pf);
          y = fabs(y) + bh_alpha * pow(fabs(y), bh_beta);
        } else {
          y = -log((double)pf);
        }
        gk = (float)(y * coeff[k]);
      } else {
        gk = TRANSPOSE ? G[(size_t)v * C + k] * cm[k] : G[(size_t)v * C + k];
      }
    }
    sg[k] = gk;
  }
  for (int x = threadIdx.x; x < off + cpad + 8; x += nt) {
    const int d = x - off;
    sh[x] = (d > -C && d < C) ? h0[d + C - 1] : 0.0f;
  }
  __syncthreads();
  for (int m0 = threadIdx.x * FC_R; m0 < C; m0 += nt * FC_R) {
    float acc[FC_R];
#pragma unroll
    for (int j = 0; j < FC_R; j++) acc[j] = 0.0f;
    // The window h0(m0 - k0 - 3 + i), i < FC_R + 4, slides down by 4 per
    // chunk: the upper FC_R values are the previous chunk's lower ones, so
    // each chunk loads only 4 new kernel values (one 128-bit load).
    float w[FC_R + 4];
#pragma unroll
    for (int b = 1; b < FC_R / 4 + 1; b++) {
      const float4 wb = *reinterpret_cast<const float4*>(sh + off + m0 - 3 + 4 * b);
      w[4 * b] = wb.x;
      w[4 * b + 1] = wb.y;
      w[4 * b + 2] = wb.z;
      w[4 * b + 3] = wb.w;
    }
    // Loads one chunk ahead (sg has 4 zeros past cpad, and sh + off + m0 -
    // cpad - 3 = sh + m0), so the FMAs do not wait on shared memory.
    float4 g4n = *reinterpret_cast<const float4*>(sg);
    float4 wbn = *reinterpret_cast<const float4*>(sh + off + m0 - 3);
#pragma unroll 4
    for (int k0 = 0; k0 < cpad; k0 += 4) {
      const float4 g4 = g4n, wb = wbn;
      g4n = *reinterpret_cast<const float4*>(sg + k0 + 4);
      wbn = *reinterpret_cast<const float4*>(sh + off + m0 - k0 - 7);
      w[0] = wb.x;
      w[1] = wb.y;
      w[2] = wb.z;
      w[3] = wb.w;
      const float g[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < FC_R; j++) acc[j] = fmaf(w[j - i + 3], g[i], acc[j]);  // h0(m0 + j - (k0 + i))
#pragma unroll
      for (int i = FC_R + 3; i >= 4; i--) w[i] = w[i - 4];
    }
#pragma unroll
    for (int j = 0; j < FC_R; j++) {
      const int m = m0 + j;
      if (m >= C) break;
      if (TRANSPOSE) {
        Q[(size_t)v * C + m] = acc[j];
      } else {
        float q = acc[j] * cm[m];
        if (in_mode && (q < 1000.0f || q > 300000.0f)) q = 0.0f;  // :250-255
        Q[(size_t)v * C + m] = q;
      }
    }
  }
  if (Q2) {
    // The row again as interpolation pairs (q[m], q[m+1]), for the
    // quarter-turn backprojector's 8-byte loads; the block's writes above
    // are visible after the barrier.
    __syncthreads();
    const float* qr = Q + (size_t)v * C;
    for (int m = threadIdx.x; m < C; m += nt)
      Q2[(size_t)v * C + m] = make_float2(qr[m], m + 1 < C ? qr[m + 1] : 0.0f);
  }
}

template <bool TRANSPOSE>
__global__ void __launch_bounds__(FC_TMAX)
fbp_filter_kernel(const float* __restrict__ G, const float* __restrict__ h0, const float* __restrict__ cm,
                  int V, int C, int in_mode, float* __restrict__ Q, float2* __restrict__ Q2) {
  extern __shared__ __align__(16) float sm[];
  fbp_filter_view<TRANSPOSE, false>(G, h0, cm, blockIdx.x, C, in_mode, Q, Q2, sm);
}

// Weight and filter in one pass, from the sinogram [V][W].
__global__ void __launch_bounds__(FC_TMAX)
fbp_weight_filter_kernel(const float* __restrict__ sino, int W, int start, const double* __restrict__ coeff,
                         double bh_alpha, double bh_beta, const float* __restrict__ h0, const float* __restrict__ cm,
                         int V, int C, int in_mode, float* __restrict__ Q, float2* __restrict__ Q2) {
  extern __shared__ __align__(16) float sm[];
  fbp_filter_view<false, true>(sino, h0, cm, blockIdx.x, C, in_mode, Q, Q2, sm, W, start, coeff, bh_alpha, bh_beta);
}

static int filter_smem(int C, size_t* bytes) {
  *bytes = (size_t)fc_smem_floats(C) * sizeof(float);
  if (*bytes > 220 * 1024) return fail(VCT_E_UNSUPPORTED, "filter: channel count above the shared-memory limit");
  return VCT_OK;
}

int launch_fbp_filter(const float* d_g, const float* d_h0, const float* d_cm, int V, int C, int in_mode,
                      float* d_q, cudaStream_t st, float2* d_q2) {
  size_t smem;
  if (int rc = filter_smem(C, &smem)) return rc;
  VCT_CUDA(cudaFuncSetAttribute(fbp_filter_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fbp_filter_kernel<false><<<V, fc_threads(C), smem, st>>>(d_g, d_h0, d_cm, V, C, in_mode, d_q, d_q2);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int launch_fbp_weight_filter(const float* d_sino, int W, int start, const double* d_coeff, double bh_alpha,
                             double bh_beta, const float* d_h0, const float* d_cm, int V, int C, int in_mode,
                             float* d_q, float2* d_q2, cudaStream_t st) {
  size_t smem;
  if (int rc = filter_smem(C, &smem)) return rc;
  VCT_CUDA(cudaFuncSetAttribute(fbp_weight_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fbp_weight_filter_kernel<<<V, fc_threads(C), smem, st>>>(d_sino, W, start, d_coeff, bh_alpha, bh_beta, d_h0, d_cm,
                                                          V, C, in_mode, d_q, d_q2);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int launch_fbp_filter_t(const float* d_q, const float* d_h0, const float* d_cm, int V, int C, float* d_g,
                        cudaStream_t st) {
  size_t smem;
  if (int rc = filter_smem(C, &smem)) return rc;
  VCT_CUDA(cudaFuncSetAttribute(fbp_filter_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fbp_filter_kernel<true><<<V, fc_threads(C), smem, st>>>(d_q, d_h0, d_cm, V, C, 0, d_g, nullptr);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// Transposed weight: lam[v][start + k] = coeff[k] * g[v][k] (the linear part
// of the weight step, g = -ln p * coeff); other channels stay 0.
__global__ void fbp_weight_t_kernel(const float* __restrict__ g, int V, int W, int start, int C,
                                    const double* __restrict__ coeff, float* __restrict__ lam) {
  const long long n = (long long)V * W;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = (int)(i / W);
  const int k = (int)(i - (long long)v * W) - start;
  lam[i] = (k >= 0 && k < C) ? (float)((double)g[(size_t)v * C + k] * coeff[k]) : 0.0f;
}

int launch_fbp_weight_t(const float* d_g, int V, int W, int start, int C, const double* d_coeff, float* d_lam,
                        cudaStream_t st) {
  const long long n = (long long)V * W;
  fbp_weight_t_kernel<<<(int)((n + 255) / 256), 256, 0, st>>>(d_g, V, W, start, C, d_coeff, d_lam);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------------------------- backproject
// Fractional channel of pixel (xx, yy) cm in the view with (cos, sin):
// FBP/reconstructImageTOMO.cpp:67-72.
__device__ __forceinline__ float bp_channel(float xx, float yy, float c, float s, float sid,
                                            float inv_dbeta, float center, float* L2) {
  const float X = xx * c + yy * s;
  const float Y = -xx * s + yy * c;
  const float d = sid - Y;
  *L2 = d * d + X * X;
  return atan_small(__fdividef(X, d)) * inv_dbeta + center;
}

// 32 x 16 pixel tile per block, 256 threads, 2 pixels per thread (rows ty and
// ty+8).  Views go in chunks of BP_VC; for each view only the detector window
// the tile projects onto (from the tile's corner pixels, -2 channels) is
// staged in shared memory as pairs (q[i], q[i+1]), `win` entries wide, so the
// interpolation is one 8-byte load.
constexpr int BP_TX = 32, BP_TY = 8, BP_PIX = 2, BP_VC = 32;

__device__ __forceinline__ void fbp_bp_block(int bx, int by, const float* __restrict__ Q, int V, int C, int N,
                                             int win, float scale, float sid, float inv_dbeta, float center,
                                             float out_scale, const float2* __restrict__ cs, float* __restrict__ img,
                                             int row0, int row1, float2* sm2) {
  float2* sQ = sm2;                                        // [BP_VC][win] pairs
  float2* sCS = sQ + BP_VC * win;                          // [BP_VC]
  int* sOff = reinterpret_cast<int*>(sCS + BP_VC);         // [BP_VC]
  const int tid = threadIdx.y * BP_TX + threadIdx.x;
  const int x0 = bx * BP_TX, y0 = row0 + by * (BP_TY * BP_PIX);
  const int x = x0 + threadIdx.x;
  const float cp = (float)N / 2.0f - 0.5f;
  // Inscribed-circle mask (FBP/misc.cpp:20-36): (y-r)^2 + (x-r)^2 <= r^2.
  const double r = (double)(N - 1) / 2.0;
  const float xx = -((float)x - cp) * scale;
  float yy[BP_PIX], acc[BP_PIX];
  bool in[BP_PIX];
#pragma unroll
  for (int k = 0; k < BP_PIX; k++) {
    const int y = y0 + threadIdx.y + BP_TY * k;
    yy[k] = -((float)y - cp) * scale;
    in[k] = x < N && y < row1 && ((double)y - r) * ((double)y - r) + ((double)x - r) * ((double)x - r) <= r * r;
    acc[k] = 0.0f;
  }
  // A tile with no pixel inside the circle only writes zeros.
  const bool any = __syncthreads_or(in[0] || in[1]);
  const int use = any ? V / 2 * 2 : 0;  // usesinogram, :30
  // Tile corners (pixel centres) for the per-view windows.
  const int xe = min(x0 + BP_TX - 1, N - 1), ye = min(y0 + BP_TY * BP_PIX - 1, row1 - 1);
  const float cx0 = -((float)x0 - cp) * scale, cx1 = -((float)xe - cp) * scale;
  const float cy0 = -((float)y0 - cp) * scale, cy1 = -((float)ye - cp) * scale;
  for (int v0 = 0; v0 < use; v0 += BP_VC) {
    const int nv = min(BP_VC, use - v0);
    __syncthreads();
    if (tid < nv) {
      const float2 t = cs[v0 + tid];
      float L2;
      const float a = bp_channel(cx0, cy0, t.x, t.y, sid, inv_dbeta, center, &L2);
      const float b = bp_channel(cx1, cy0, t.x, t.y, sid, inv_dbeta, center, &L2);
      const float c2 = bp_channel(cx0, cy1, t.x, t.y, sid, inv_dbeta, center, &L2);
      const float d = bp_channel(cx1, cy1, t.x, t.y, sid, inv_dbeta, center, &L2);
      sOff[tid] = (int)floorf(fminf(fminf(a, b), fminf(c2, d))) - 2;
      sCS[tid] = t;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < nv; j += BP_TY) {
      const int off = sOff[j];
      const float* qrow = Q + (size_t)(v0 + j) * C;
      for (int k = threadIdx.x; k < win; k += BP_TX) {
        const int ch = off + k;
        const float q0 = (ch >= 0 && ch < C) ? qrow[ch] : 0.0f;
        const float q1 = (ch + 1 >= 0 && ch + 1 < C) ? qrow[ch + 1] : 0.0f;
        sQ[j * win + k] = make_float2(q0, q1);
      }
    }
    __syncthreads();
    for (int j = 0; j < nv; j++) {
      const float2 t = sCS[j];
      const int off = sOff[j];
      const float2* q = sQ + j * win;
      const float* qg = Q + (size_t)(v0 + j) * C;
#pragma unroll
      for (int k = 0; k < BP_PIX; k++) {
        float L2;
        const float fg = bp_channel(xx, yy[k], t.x, t.y, sid, inv_dbeta, center, &L2);
        // (int)(fGAM) truncates toward zero (:73): adding 2^23 with round-to-
        // zero leaves trunc(fg) in the low mantissa bits for 0 <= fg < 2^22;
        // fg in (-1, 0) truncates to 0 and is kept (w < 0, as the reference).
        const float big = __fadd_rz(fmaxf(fg, 0.0f), 8388608.0f);
        const int gi = fg > -1.0f ? (__float_as_int(big) - 0x4B000000) : -1;
        const float w = fg - (big - 8388608.0f);
        if (in[k] && gi >= 0 && gi < C - 1) {
          const int li = gi - off;
          float2 qq;
          if (li >= 0 && li < win) qq = q[li];
          else qq = make_float2(qg[gi], qg[gi + 1]);  // outside the staged window
          acc[k] += __fdividef(fmaf(w, qq.y - qq.x, qq.x), L2);
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < BP_PIX; k++) {
    const int y = y0 + threadIdx.y + BP_TY * k;
    if (x < N && y < row1) img[(size_t)y * N + x] = in[k] ? acc[k] * out_scale : 0.0f;
  }
}

__global__ void __launch_bounds__(BP_TX * BP_TY, 4)
fbp_bp_kernel(const float* __restrict__ Q, int V, int C, int N, int win, float scale, float sid,
              float inv_dbeta, float center, float out_scale, const float2* __restrict__ cs,
              float* __restrict__ img, int row0, int row1) {
  extern __shared__ float2 sm2[];
  fbp_bp_block(blockIdx.x, blockIdx.y, Q, V, C, N, win, scale, sid, inv_dbeta, center, out_scale, cs, img, row0,
               row1, sm2);
}

// Backprojection with the square grid's quarter-turn symmetry, for V
// divisible by 4 and even N.  Pixel (x, y) in view j and pixel
// (N-1-y, x) in view j + V/4 have the same rotated coordinates (X, Y): with
// beta' = beta + 90 deg, cos' = -sin, sin' = cos, and the pixel centre
// (xx, yy) maps to (-yy, xx).  So the geometry (X, Y, L^2, fractional
// channel) computed for p0 = (x, y) in view j also serves
//   p1 = (N-1-y, x) in view j+V/4, p2 = (N-1-x, N-1-y) in view j+V/2,
//   p3 = (y, N-1-x) in view j+3V/4   (views mod V);
// running j over all V views gives each of the four pixels every view, with
// a quarter of the geometry work.  Orbit representatives cover the top-left
// quadrant.
// The trig tables of the four views agree with the quarter-turn to double
// rounding, below the FP32 resolution of the geometry.
// 32 x 4 orbits per block; the base views are split over VS groups of warps
// (threadIdx.z; VS = 4 unless a batch's tuner picks another), summed in
// shared memory at the end.  The four filtered
// rows of each base view are read through the L1 cache (the 32 pixels of a
// warp read neighbouring channels).
constexpr int BS_TX = 32, BS_TY = 4, BS_VS = 4;  // BS_VS: the default view split
// (Also measured: the register cap for 4 blocks of 512 threads per SM, 32
// registers, 0.213 ms against 0.127 ms; each batch of U base views computing
// its geometry first and then issuing all 4U row loads unconditionally
// (clamped channels), U = 2 / 4 / 8 at 60 / 82 / 127 registers: 0.135 /
// 0.145 / 0.123 ms -- the last too close to pay for its register footprint
// in the batch's kernel; 32-bit row offsets instead of 64-bit ones, 0.135
// against 0.126 ms.)
#ifndef VCT_BP_UNROLL
#define VCT_BP_UNROLL 8
#endif

// One base view j of an orbit: the geometry (FBP/reconstructImageTOMO.cpp:
// 67-73) once, then the four rotated rows, row q at qbase + off[q] (views
// mod V, the offsets set by the caller for j's quarter).  PAIRS: Q2 holds
// (q[c], q[c+1]) pairs, one 8-byte load per row; else two loads from Q.
template <bool PAIRS>
__device__ __forceinline__ void bp_orbit_view(const float* __restrict__ Q, const float2* __restrict__ Q2, int C,
                                              float xx, float yy, float2 t, long long jrow, const long long off[4],
                                              float sid, float inv_dbeta, float center, float acc[4]) {
  const float X = xx * t.x + yy * t.y;
  const float Y = -xx * t.y + yy * t.x;
  const float d = sid - Y;
  const float rd = rcp_approx(d);
  const float fg = atan_small(X * rd) * inv_dbeta + center;
  const float iL2 = rcp_approx(fmaf(d, d, X * X));
  // (int)(fGAM) truncates toward zero: trunc(fg) via 2^23 with round-to-zero;
  // fg in (-1, 0) truncates to 0 and is kept (w < 0), as the reference.
  const float big = __fadd_rz(fmaxf(fg, 0.0f), 8388608.0f);
  const int gi = fg > -1.0f ? (__float_as_int(big) - 0x4B000000) : -1;
  const float w = fg - (big - 8388608.0f);
  if ((unsigned)gi < (unsigned)(C - 1)) {
    const long long base = jrow + gi;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float q0, q1;
      if (PAIRS) {
        const float2 p = __ldg(Q2 + base + off[q]);
        q0 = p.x;
        q1 = p.y;
      } else {
        const float* qr = Q + base + off[q];
        q0 = __ldg(qr);
        q1 = __ldg(qr + 1);
      }
      acc[q] = fmaf(fmaf(w, q1 - q0, q0), iL2, acc[q]);
    }
  }
}

template <int VS, bool PAIRS>
__device__ __forceinline__ void fbp_bp_sym_block(int bx, int by, const float* __restrict__ Q,
                                                 const float2* __restrict__ Q2, int V, int C, int N, float scale,
                                                 float sid, float inv_dbeta, float center, float out_scale,
                                                 const float2* __restrict__ cs, float* __restrict__ img, int y_lo,
                                                 int y_hi, float (*part)[4][BS_TX * BS_TY]) {
  const int H = N / 2, V4 = V / 4;
  const int x = bx * BS_TX + threadIdx.x;
  const int y = y_lo + by * BS_TY + threadIdx.y;  // orbit rows [y_lo, y_hi) of [0, N/2)
  const int lt = threadIdx.y * BS_TX + threadIdx.x;
  const int z = threadIdx.z;
  const double r = (double)(N - 1) / 2.0;
  // The circle mask (FBP/misc.cpp:20-36) is invariant under the quarter turn.
  const bool in = x < H && y < y_hi &&
                  ((double)y - r) * ((double)y - r) + ((double)x - r) * ((double)x - r) <= r * r;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  if (in) {
    const float cp = (float)N / 2.0f - 0.5f;
    const float xx = -((float)x - cp) * scale;
    const float yy = -((float)y - cp) * scale;
    const int jb = (int)((long long)V * z / VS), je = (int)((long long)V * (z + 1) / VS);
    // Base views in quarter `seg` (j in [seg V/4, (seg+1) V/4)): row q is
    // j + q V/4, less V where that passes V, i.e. where q + seg >= 4.
    for (int seg = 0; seg < 4; seg++) {
      const int s0 = max(jb, seg * V4), s1 = min(je, (seg + 1) * V4);
      if (s0 >= s1) continue;
      long long off[4];
#pragma unroll
      for (int q = 0; q < 4; q++) off[q] = (long long)(q * V4 - (q + seg >= 4 ? V : 0)) * C;
      int j = s0;
      // VCT_BP_UNROLL base views per iteration: their row loads are in flight together
      for (; j + VCT_BP_UNROLL - 1 < s1; j += VCT_BP_UNROLL) {
#pragma unroll
        for (int u = 0; u < VCT_BP_UNROLL; u++)
          bp_orbit_view<PAIRS>(Q, Q2, C, xx, yy, __ldg(cs + j + u), (long long)(j + u) * C, off, sid, inv_dbeta,
                               center, acc);
      }
      for (; j < s1; j++)
        bp_orbit_view<PAIRS>(Q, Q2, C, xx, yy, __ldg(cs + j), (long long)j * C, off, sid, inv_dbeta, center, acc);
    }
  }
  if (z > 0) {
#pragma unroll
    for (int q = 0; q < 4; q++) part[z - 1][q][lt] = acc[q];
  }
  __syncthreads();
  if (z == 0 && x < H && y < y_hi) {
    const int px[4] = {x, N - 1 - y, N - 1 - x, y};
    const int py[4] = {y, x, N - 1 - y, N - 1 - x};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float a = acc[q];
#pragma unroll
      for (int k = 0; k < VS - 1; k++) a += part[k][q][lt];
      img[(size_t)py[q] * N + px[q]] = in ? a * out_scale : 0.0f;
    }
  }
}

template <int VS, bool PAIRS>
__global__ void __launch_bounds__(BS_TX * BS_TY * VS)
fbp_bp_sym_kernel(const float* __restrict__ Q, const float2* __restrict__ Q2, int V, int C, int N, float scale,
                  float sid, float inv_dbeta, float center, float out_scale, const float2* __restrict__ cs,
                  float* __restrict__ img, int y_lo, int y_hi) {
  __shared__ float part[VS - 1][4][BS_TX * BS_TY];
  fbp_bp_sym_block<VS, PAIRS>(blockIdx.x, blockIdx.y, Q, Q2, V, C, N, scale, sid, inv_dbeta, center, out_scale, cs,
                              img, y_lo, y_hi, part);
}

// ------------------------------------------------- backprojection transpose
// qb[v][m] = out_scale * sum over mask pixels p of wt(p, v, m) u[p] / L2(p, v),
// wt = 1 - w where trunc(fg) = m and w where trunc(fg) = m - 1: the transpose
// of the interpolating backprojection above.  One thread per (view, bin)
// gathers, so no two threads write one output.  The pixels whose fractional
// channel fg lies in the bin's interval (m-1, m+1) -- from -1 for m <= 1,
// since (int) truncates (-1, 0) to 0 -- are the pixels between two rays from
// the source; each image row (or column, whichever the rays cross more
// steeply) meets that wedge in a short run found in closed form, and every
// pixel of the run is evaluated with the forward's own formula.
// SYM: the quarter-turn orbit of fbp_bp_sym_kernel -- the geometry of pixel p
// in view j is that of its rotations in views j + V/4, j + V/2, j + 3V/4, so
// one evaluation serves four outputs (V % 4 == 0, N even).
template <bool SYM>
__global__ void __launch_bounds__(128)
fbp_bp_t_kernel(const float* __restrict__ U, int V, int C, int N, float scale, float sid, float inv_dbeta,
                float dbeta_det, float center, float out_scale, const float2* __restrict__ cs,
                float* __restrict__ QB) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (m >= C) return;
  const float2 t = cs[j];
  const float c = t.x, s = t.y;
  const float cp = (float)N / 2.0f - 0.5f;
  // The wedge: fan angles of fg = lo and fg = m + 1 (a margin is added below).
  const float lo = m <= 1 ? -1.0f : (float)(m - 1);
  const float T1 = tanf((lo - center) * dbeta_det), T2 = tanf(((float)(m + 1) - center) * dbeta_det);
  const float Tm = 0.5f * (T1 + T2);
  const bool rows = fabsf(c - Tm * s) >= fabsf(s + Tm * c);
  const int V4 = V / 4;
  const int n1 = N - 1;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int line = 0; line < N; line++) {
    // Fixed coordinate of the line and the run of the other one.
    float a0, a1;
    if (rows) {
      const float yy = -((float)line - cp) * scale;
      const float x1 = (T1 * (sid - yy * c) - yy * s) / (c - T1 * s);
      const float x2 = (T2 * (sid - yy * c) - yy * s) / (c - T2 * s);
      a0 = cp - x1 / scale;
      a1 = cp - x2 / scale;
    } else {
      const float xx = -((float)line - cp) * scale;
      const float y1 = (T1 * (sid + xx * s) - xx * c) / (s + T1 * c);
      const float y2 = (T2 * (sid + xx * s) - xx * c) / (s + T2 * c);
      a0 = cp - y1 / scale;
      a1 = cp - y2 / scale;
    }
    const int k0 = max((int)floorf(fminf(a0, a1)) - 1, 0);
    const int k1 = min((int)ceilf(fmaxf(a0, a1)) + 1, n1);
    for (int k = k0; k <= k1; k++) {
      const int x = rows ? k : line, y = rows ? line : k;
      // Inscribed-circle mask, exactly: (2y-N+1)^2 + (2x-N+1)^2 <= (N-1)^2.
      const int dy2 = 2 * y - n1, dx2 = 2 * x - n1;
      if (dy2 * dy2 + dx2 * dx2 > n1 * n1) continue;
      const float xx = -((float)x - cp) * scale, yy = -((float)y - cp) * scale;
      float fg, iL2;
      if (SYM) {
        const float X = xx * c + yy * s;
        const float Y = -xx * s + yy * c;
        const float d = sid - Y;
        const float rd = rcp_approx(d);
        fg = atan_small(X * rd) * inv_dbeta + center;
        iL2 = rcp_approx(fmaf(d, d, X * X));
      } else {
        float L2;
        fg = bp_channel(xx, yy, c, s, sid, inv_dbeta, center, &L2);
        iL2 = __fdividef(1.0f, L2);
      }
      const float big = __fadd_rz(fmaxf(fg, 0.0f), 8388608.0f);
      const int gi = fg > -1.0f ? (__float_as_int(big) - 0x4B000000) : -1;
      const float w = fg - (big - 8388608.0f);
      if ((unsigned)gi >= (unsigned)(C - 1)) continue;
      float wt;
      if (gi == m) wt = 1.0f - w;
      else if (gi == m - 1) wt = w;
      else continue;
      wt *= iL2;
      if (SYM) {
        acc[0] = fmaf(wt, U[(size_t)y * N + x], acc[0]);
        acc[1] = fmaf(wt, U[(size_t)x * N + (n1 - y)], acc[1]);
        acc[2] = fmaf(wt, U[(size_t)(n1 - y) * N + (n1 - x)], acc[2]);
        acc[3] = fmaf(wt, U[(size_t)(n1 - x) * N + y], acc[3]);
      } else {
        acc[0] = fmaf(wt, U[(size_t)y * N + x], acc[0]);
      }
    }
  }
  if (SYM) {
#pragma unroll
    for (int q = 0; q < 4; q++) QB[(size_t)(j + q * V4) * C + m] = acc[q] * out_scale;
  } else {
    QB[(size_t)j * C + m] = acc[0] * out_scale;
  }
}

// Symmetric case as a scatter: the forward's own per-(orbit pixel, view)
// geometry, evaluated once (bp_orbit_view's formula), adds (1-w)/L^2 u and
// w/L^2 u to bins gi and gi+1 of the four rows of the orbit.  Block
// (b, part) owns rows b, b+V/4, b+V/2, b+3V/4 -- the rows base views
// b + i V/4 reach through the quarter turn -- and one part of the orbit
// pixels (at most BT_PART_PIXELS of them); it sums in shared memory and
// flushes to a global 64-bit accumulator.  Every sum is in integers (fixed
// point), so it does not depend on the order of the atomics and the result
// is the same from run to run.  The rotated pixels are read from a
// transposed copy of u, so every read is along a row.
// Parts of the orbit pixels per base view (blocks V/4 x parts): 2 / 4 / 8 /
// 16 / 32 / 64 measured 0.569 / 0.526 / 0.432 / 0.411 / 0.413 / 0.438 ms at
// 512^2 from 800 x 609 (output bit-identical).
#ifndef VCT_BT_PARTS
#define VCT_BT_PARTS 16
#endif
constexpr int BT_PARTS = VCT_BT_PARTS;
// Largest part: a shared slot (row, bin) then takes at most 4 x 4096 = 2^14
// adds (one per pixel of the part for each of the four base views).
constexpr int BT_PART_PIXELS = 4096;
// Fixed point: a contribution c becomes rint(c fx) with fx = 2^33 / (max|u|
// max 1/L^2), so |rint(c fx)| <= 2^33, split as h 2^17 + l with |h| <= 2^16
// and 0 <= l < 2^17: the slot sums of h and of l stay within 2^30 and 2^31
// (32-bit, no carries), and a part's total h 2^17 + l within 2^47.
constexpr float BT_FIX_BITS = 8589934592.0f;  // 2^33

// lo += l, hi += h for rint(v) = h 2^17 + l: rint(v) as a 64-bit integer,
// h = floor(rint(v) / 2^17) (|h| <= 2^16) and l its low 17 bits (0 <= l <
// 2^17, so a slot's sum of l stays below 2^14 x 2^17 = 2^31).  Both adds are
// fire-and-forget shared-memory atomics.  (Measured at 512^2 from 800 x 609:
// 0.85 ms with two-word 64-bit adds that carried through the returned low
// word, 1.86 ms with 64-bit atomics, 1.50 ms with float ones; h and l by two
// float roundings with the 1.5 * 2^23 constant instead of the 64-bit
// conversion, 0.338 ms against 0.310 ms, same sums.)
__device__ __forceinline__ void bt_add(int* lo, int* hi, float v) {
  const long long r = __float2ll_rn(v);
  atomicAdd(lo, (int)((unsigned int)r & 0x1FFFFu));
  atomicAdd(hi, (int)(r >> 17));
}

// ut[c][r] = u[r][c], N x N, 32 x 32 tiles through shared memory.
__global__ void transpose_kernel(const float* __restrict__ u, int N, float* __restrict__ ut) {
  __shared__ float tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = by + k, c = bx + threadIdx.x;
    if (r < N && c < N) tile[k][threadIdx.x] = u[(size_t)r * N + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = bx + k, r = by + threadIdx.x;
    if (r < N && c < N) ut[(size_t)c * N + r] = tile[threadIdx.x][k];
  }
}

__global__ void absmax_kernel(const float* __restrict__ u, long long n, unsigned int* __restrict__ out) {
  float m = 0.0f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(u[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(out, __float_as_uint(m));
}

__device__ __forceinline__ float bt_fixed_scale(const unsigned long long* umax_slot, float il2max) {
  const float um = __uint_as_float((unsigned int)*umax_slot);
  if (!(um > 0.0f)) return 1.0f;
  return (float)((double)BT_FIX_BITS / ((double)um * (double)il2max));  // 2^33 / max |c|
}

__global__ void __launch_bounds__(256)
fbp_bp_t_scatter_kernel(const float* __restrict__ U, const float* __restrict__ UT, int V, int C, int N, float scale,
                        float sid, float inv_dbeta, float center, float il2max, const float2* __restrict__ cs,
                        unsigned long long* __restrict__ acc) {
  extern __shared__ int s_lo[];  // [4][C] sums of l, then [4][C] sums of h
  int* s_hi = s_lo + 4 * C;
  const int b = blockIdx.x, part = blockIdx.y, parts = gridDim.y;
  const int V4 = V / 4, H = N / 2, n1 = N - 1;
  for (int i = threadIdx.x; i < 8 * C; i += blockDim.x) s_lo[i] = 0;
  const float fx = bt_fixed_scale(acc + (size_t)V * C, il2max);
  __syncthreads();
  const float cp = (float)N / 2.0f - 0.5f;
  const int np = H * H;
  const int o0 = (int)((long long)np * part / parts), o1 = (int)((long long)np * (part + 1) / parts);
  const int o_first = o0 + threadIdx.x;
  for (int i = 0; i < 4; i++) {
    const float2 t = __ldg(cs + b + i * V4);
    // Neighbouring lanes take neighbouring pixels across the rays (along x
    // when the view's rays run closer to y, else along y), so their bins
    // differ and their shared-memory adds do not collide.
    const bool alongy = fabsf(t.y) > fabsf(t.x);
    // Orbit pixel o = sl H + f, stepped by the block size without a division.
    int f = o_first % H, sl = o_first / H;
    for (int o = o_first; o < o1; o += blockDim.x) {
      const int x = alongy ? sl : f, y = alongy ? f : sl;
      f += blockDim.x;
      while (f >= H) f -= H, sl++;
      // Inscribed-circle mask, exactly: (2y-N+1)^2 + (2x-N+1)^2 <= (N-1)^2.
      const int dy2 = 2 * y - n1, dx2 = 2 * x - n1;
      if (dy2 * dy2 + dx2 * dx2 > n1 * n1) continue;
      const float xx = -((float)x - cp) * scale;
      const float yy = -((float)y - cp) * scale;
      // FBP/reconstructImageTOMO.cpp:67-73, as bp_orbit_view.
      const float X = xx * t.x + yy * t.y;
      const float Y = -xx * t.y + yy * t.x;
      const float d = sid - Y;
      const float rd = rcp_approx(d);
      const float fg = atan_small(X * rd) * inv_dbeta + center;
      const float iL2f = rcp_approx(fmaf(d, d, X * X)) * fx;
      const float big = __fadd_rz(fmaxf(fg, 0.0f), 8388608.0f);
      const int gi = fg > -1.0f ? (__float_as_int(big) - 0x4B000000) : -1;
      const float w = fg - (big - 8388608.0f);
      if ((unsigned)gi >= (unsigned)(C - 1)) continue;
      // u at the orbit's pixels (x, y), (n1-y, x), (n1-x, n1-y), (y, n1-x),
      // each read along a row of u or of its transposed copy ut.
      float uq[4];
      if (!alongy) {
        uq[0] = __ldg(U + (size_t)y * N + x);
        uq[1] = __ldg(UT + (size_t)(n1 - y) * N + x);
        uq[2] = __ldg(U + (size_t)(n1 - y) * N + (n1 - x));
        uq[3] = __ldg(UT + (size_t)y * N + (n1 - x));
      } else {
        uq[0] = __ldg(UT + (size_t)x * N + y);
        uq[1] = __ldg(U + (size_t)x * N + (n1 - y));
        uq[2] = __ldg(UT + (size_t)(n1 - x) * N + (n1 - y));
        uq[3] = __ldg(U + (size_t)(n1 - x) * N + y);
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float val = uq[q] * iL2f;                 // u / L^2 in fixed-point units
        const float c1 = w * val, c0 = val - c1;  // (1 - w) val and w val
        const int at = ((i + q) & 3) * C + gi;
        bt_add(s_lo + at, s_hi + at, c0);
        bt_add(s_lo + at + 1, s_hi + at + 1, c1);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * C; i += blockDim.x) {
    const long long v = (long long)s_hi[i] * 131072 + s_lo[i];
    if (v) atomicAdd(acc + (size_t)(b + (i / C) * V4) * C + (i % C), (unsigned long long)v);
  }
}

__global__ void fbp_bp_t_finish_kernel(const unsigned long long* __restrict__ acc, int V, int C, int N, float il2max,
                                       float out_scale, float* __restrict__ qb) {
  const float fx = bt_fixed_scale(acc + (size_t)V * C, il2max);
  const long long n = (long long)V * C;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    qb[i] = (float)((double)(long long)acc[i] / (double)fx) * out_scale;
}

// Scratch of the symmetric transpose: V*C fixed-point sums, the max|u| word,
// and the transposed image (N*N floats).
size_t fbp_backproject_t_scratch(int V, int C, int N) { return (size_t)V * C + 1 + ((size_t)N * N + 1) / 2; }

// Transpose of launch_fbp_backproject (same kernel choice, same geometry).
// Rows v >= V/2*2 of qb are 0, as the backprojection never reads them.
// d_acc: fbp_backproject_t_scratch(V, C, N) words, used by the symmetric case.
int launch_fbp_backproject_t(const float* d_u, int V, int C, int N, double pixel_cm, double sid, double max_beta,
                             int xfactor, const float* d_cs, unsigned long long* d_acc, float* d_qb,
                             cudaStream_t st) {
  const int half = (C - 1) / 2;
  const double dbeta_det = max_beta / half;
  const double dbeta = 2.0 * 3.141592653589793 / V;
  const int Vu = V / 2 * 2;
  const bool sym = V % 4 == 0 && N % 2 == 0;
  if (Vu < V) VCT_CUDA(cudaMemsetAsync(d_qb + (size_t)Vu * C, 0, (size_t)(V - Vu) * C * sizeof(float), st));
  dim3 grid((C + 127) / 128, sym ? V / 4 : Vu);
  if (grid.y == 0) return VCT_OK;
  if (sym) {
    // Largest 1/L^2 over the grid: the pixel centres lie within (N-1)/2
    // pixels * sqrt(2) of the isocentre; twice that bound for margin.
    const double reach = 0.5 * (N - 1) * pixel_cm * 1.4142135623730951;
    if (!(sid > reach)) return fail(VCT_E_UNSUPPORTED, "fbp transpose: the grid reaches the source");
    const float il2max = (float)(2.0 / ((sid - reach) * (sid - reach)));
    const size_t smem = (size_t)8 * C * sizeof(int);
    float* d_ut = reinterpret_cast<float*>(d_acc + (size_t)V * C + 1);
    VCT_CUDA(cudaMemsetAsync(d_acc, 0, ((size_t)V * C + 1) * sizeof(unsigned long long), st));
    absmax_kernel<<<148 * 4, 256, 0, st>>>(d_u, (long long)N * N, reinterpret_cast<unsigned int*>(d_acc + (size_t)V * C));
    transpose_kernel<<<dim3((N + 31) / 32, (N + 31) / 32), dim3(32, 8), 0, st>>>(d_u, N, d_ut);
    VCT_CUDA(cudaFuncSetAttribute(fbp_bp_t_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int parts = std::max(BT_PARTS, (int)(((long long)(N / 2) * (N / 2) + BT_PART_PIXELS - 1) / BT_PART_PIXELS));
    fbp_bp_t_scatter_kernel<<<dim3(V / 4, parts), 256, smem, st>>>(
        d_u, d_ut, V, C, N, (float)pixel_cm, (float)sid, (float)(1.0 / dbeta_det), (float)(C / 2), il2max,
        reinterpret_cast<const float2*>(d_cs), d_acc);
    fbp_bp_t_finish_kernel<<<148 * 4, 256, 0, st>>>(d_acc, V, C, N, il2max, (float)(dbeta * xfactor), d_qb);
  } else
    fbp_bp_t_kernel<false><<<grid, 128, 0, st>>>(d_u, V, C, N, (float)pixel_cm, (float)sid,
                                                 (float)(1.0 / dbeta_det), (float)dbeta_det, (float)(C / 2),
                                                 (float)(dbeta * xfactor), reinterpret_cast<const float2*>(d_cs), d_qb);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int fbp_band_count(int V, int N) { return (V % 4 == 0 && N % 2 == 0) ? N / 2 : N; }

void fbp_bp_params(int V, int W, int start, int C, int N, double pixel_cm, double sid, double max_beta, int xfactor,
                   PostJob* j) {
  const int half = (C - 1) / 2;
  const double dbeta_det = max_beta / half;
  const double dbeta = 2.0 * 3.141592653589793 / V;
  // Window: the angle a tile's diagonal subtends from the source at the
  // nearest approach of the reconstruction square, in channels, + margins.
  const double tile_cm = (double)BP_TX * pixel_cm * 1.41421356237;
  const double near_cm = sid - 0.5 * N * pixel_cm * 1.41421356237;
  int win = C + 4;
  if (near_cm > tile_cm) win = (int)(tile_cm / near_cm / dbeta_det) + 8;
  win = ((win + 31) / 32) * 32;
  if (win > C + 4) win = C + 4;
  j->V = V;
  j->W = W;
  j->C = C;
  j->start = start;
  j->N = N;
  j->sym = V % 4 == 0 && N % 2 == 0;
  j->win = win;
  j->scale = (float)pixel_cm;
  j->sid = (float)sid;
  j->inv_dbeta = (float)(1.0 / dbeta_det);
  j->center = (float)(C / 2);
  j->out_scale = (float)(dbeta * xfactor);
}

static size_t bp_gen_smem(int win) {
  return (size_t)BP_VC * win * sizeof(float2) + BP_VC * (sizeof(float2) + sizeof(int));
}

int launch_fbp_backproject(const float* d_q, int V, int C, int N, double pixel_cm, double sid,
                           double max_beta, int xfactor, const float* d_cs, float* d_img,
                           cudaStream_t st, int view_groups, int band0, int band1, const float2* d_q2) {
  if (band1 < 0) band1 = fbp_band_count(V, N);
  if (band0 < 0 || band0 > band1 || band1 > fbp_band_count(V, N))
    return fail(VCT_E_ARG, "fbp: band outside the image");
  if (band0 == band1) return VCT_OK;
  PostJob p{};
  fbp_bp_params(V, C, 0, C, N, pixel_cm, sid, max_beta, xfactor, &p);
  const float2* cs2 = reinterpret_cast<const float2*>(d_cs);
  if (p.sym) {
    const int H = N / 2;
    dim3 grid((H + BS_TX - 1) / BS_TX, (band1 - band0 + BS_TY - 1) / BS_TY);
#define VCT_SYM(vs, pairs)                                                                                \
  fbp_bp_sym_kernel<vs, pairs><<<grid, dim3(BS_TX, BS_TY, vs), 0, st>>>(d_q, d_q2, V, C, N, p.scale, p.sid, \
                                                                        p.inv_dbeta, p.center, p.out_scale, cs2, \
                                                                        d_img, band0, band1)
    if (d_q2) {
      switch (view_groups) {
        case 2: VCT_SYM(2, true); break;
        case 8: VCT_SYM(8, true); break;
        default: VCT_SYM(BS_VS, true); break;
      }
    } else {
      switch (view_groups) {
        case 2: VCT_SYM(2, false); break;
        case 8: VCT_SYM(8, false); break;
        default: VCT_SYM(BS_VS, false); break;
      }
    }
#undef VCT_SYM
    VCT_CUDA(cudaGetLastError());
    return VCT_OK;
  }
  dim3 grid((N + BP_TX - 1) / BP_TX, (band1 - band0 + BP_TY * BP_PIX - 1) / (BP_TY * BP_PIX));
  dim3 block(BP_TX, BP_TY);
  const size_t smem = bp_gen_smem(p.win);
  VCT_CUDA(cudaFuncSetAttribute(fbp_bp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fbp_bp_kernel<<<grid, block, smem, st>>>(d_q, V, C, N, p.win, p.scale, p.sid, p.inv_dbeta, p.center, p.out_scale,
                                           cs2, d_img, band0, band1);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------------------------------ batch
// Job of block b in a batched stage: the last j with first[j] <= b.
__device__ __forceinline__ int post_job_of(const unsigned int* __restrict__ first, int n, unsigned int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

void post_job_blocks(const PostJob& j, unsigned int blocks[kPostStages]) {
  blocks[kPostNorm] = (unsigned int)(((long long)j.V * j.W + 255) / 256);
  blocks[kPostWeight] = blocks[kPostFilter] = blocks[kPostBpSym] = blocks[kPostBpGen] = 0;
  if (!j.img) return;
  blocks[kPostFilter] = (unsigned int)j.V;  // weight applied on the filter's row load
  if (j.sym) {
    const int H = j.N / 2;
    blocks[kPostBpSym] = (unsigned int)(((H + BS_TX - 1) / BS_TX) * ((H + BS_TY - 1) / BS_TY));
  } else {
    blocks[kPostBpGen] = (unsigned int)(((j.N + BP_TX - 1) / BP_TX) * ((j.N + BP_TY * BP_PIX - 1) / (BP_TY * BP_PIX)));
  }
}

__global__ void __launch_bounds__(FC_TMAX) fbp_filter_batch_kernel(const PostJob* __restrict__ jobs,
                                                                   const unsigned int* __restrict__ first, int n) {
  extern __shared__ __align__(16) float sm[];
  const int jx = post_job_of(first, n, blockIdx.x);
  const PostJob& J = jobs[jx];
  fbp_filter_view<false, true>(J.sino, J.h0, J.h0 + 2 * J.C - 1, (int)(blockIdx.x - first[jx]), J.C, 0, J.q, J.q2,
                               sm, J.W, J.start, J.coeff, 0.0, 0.0);
}

template <int VS>
__global__ void __launch_bounds__(BS_TX * BS_TY * VS)
fbp_bp_sym_batch_kernel(const PostJob* __restrict__ jobs, const unsigned int* __restrict__ first, int n) {
  __shared__ float part[VS - 1][4][BS_TX * BS_TY];
  const int jx = post_job_of(first, n, blockIdx.x);
  const PostJob& J = jobs[jx];
  const int H = J.N / 2, nbx = (H + BS_TX - 1) / BS_TX;
  const int b = (int)(blockIdx.x - first[jx]);
  fbp_bp_sym_block<VS, true>(b % nbx, b / nbx, J.q, J.q2, J.V, J.C, J.N, J.scale, J.sid, J.inv_dbeta, J.center,
                             J.out_scale, J.cs, J.img, 0, H, part);
}

__global__ void __launch_bounds__(BP_TX * BP_TY, 4)
fbp_bp_batch_kernel(const PostJob* __restrict__ jobs, const unsigned int* __restrict__ first, int n) {
  extern __shared__ float2 sm2[];
  const int jx = post_job_of(first, n, blockIdx.x);
  const PostJob& J = jobs[jx];
  const int nbx = (J.N + BP_TX - 1) / BP_TX;
  const int b = (int)(blockIdx.x - first[jx]);
  fbp_bp_block(b % nbx, b / nbx, J.q, J.V, J.C, J.N, J.win, J.scale, J.sid, J.inv_dbeta, J.center, J.out_scale, J.cs,
               J.img, 0, J.N, sm2);
}

int launch_fbp_batch(const PostJob* d_jobs, const unsigned int* d_first, int n, const unsigned int nblocks[kPostStages],
                     int cmax, int winmax, int view_groups, cudaStream_t st) {
  const unsigned int* f = d_first;
  if (nblocks[kPostFilter]) {  // the weight is applied on the filter's row load
    size_t smem;
    if (int rc = filter_smem(cmax, &smem)) return rc;
    VCT_CUDA(cudaFuncSetAttribute(fbp_filter_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fbp_filter_batch_kernel<<<nblocks[kPostFilter], fc_threads(cmax), smem, st>>>(d_jobs, f + kPostFilter * (n + 1),
                                                                                  n);
    VCT_CUDA(cudaGetLastError());
  }
  if (nblocks[kPostBpSym]) {
    const unsigned int* fs = f + kPostBpSym * (n + 1);
    switch (view_groups) {
      case 2: fbp_bp_sym_batch_kernel<2><<<nblocks[kPostBpSym], dim3(BS_TX, BS_TY, 2), 0, st>>>(d_jobs, fs, n); break;
      case 8: fbp_bp_sym_batch_kernel<8><<<nblocks[kPostBpSym], dim3(BS_TX, BS_TY, 8), 0, st>>>(d_jobs, fs, n); break;
      default: fbp_bp_sym_batch_kernel<BS_VS><<<nblocks[kPostBpSym], dim3(BS_TX, BS_TY, BS_VS), 0, st>>>(d_jobs, fs, n); break;
    }
    VCT_CUDA(cudaGetLastError());
  }
  if (nblocks[kPostBpGen]) {
    const size_t smem = bp_gen_smem(winmax);
    VCT_CUDA(cudaFuncSetAttribute(fbp_bp_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fbp_bp_batch_kernel<<<nblocks[kPostBpGen], dim3(BP_TX, BP_TY), smem, st>>>(d_jobs, f + kPostBpGen * (n + 1), n);
    VCT_CUDA(cudaGetLastError());
  }
  return VCT_OK;
}

VCT_BOUNDS_READER(bounds_fbp)

}  // namespace vct
