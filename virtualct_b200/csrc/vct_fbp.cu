// Fan-beam FBP on sm_100a: filterSinogram (FBP/filterSinogramTOMO.cpp:205-275)
// and reconstructImage (FBP/reconstructImageTOMO.cpp:11-105) for one slice.
//
//   1. weight:   g[v][k] = -ln p[v][k] * SID*cos((k-cw)*dbeta) * dbeta, once per
//                sample (the reference re-evaluates the log inside its
//                609-long inner loop, i.e. 609 times per sample).
//   2. filter:   q[v][m] = sum_k h[m][k] g[v][k] -- a [V x C] x [C x C]^T
//                product, tiled through shared memory, FP32 FMA.
//   3. backproject: pixel-driven, equiangular fan weight 1/L^2, linear
//                interpolation on the detector; views staged in shared memory
//                in chunks; one thread per pixel.
#include <cuda_runtime.h>

#include "vct_internal.h"

namespace vct {

// ------------------------------------------------------------------ weight
__global__ void fbp_weight_kernel(const float* __restrict__ sino, int V, int W, int start, int C,
                                  const double* __restrict__ coeff, float* __restrict__ g) {
  const long long n = (long long)V * C;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = (int)(i / C);
  const int k = (int)(i - (long long)v * C);
  const double p = (double)sino[(size_t)v * W + start + k];
  g[i] = (float)(-log(p) * coeff[k]);
}

int launch_fbp_weight(const float* d_sino, int V, int W, int start, int C, const double* d_coeff,
                        float* d_g, cudaStream_t st) {
  const long long n = (long long)V * C;
  fbp_weight_kernel<<<(int)((n + 255) / 256), 256, 0, st>>>(d_sino, V, W, start, C, d_coeff, d_g);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------------------------------ filter
// Q[V][C] = G[V][C] * H[C][C]^T.  Block tile 32 views x 64 channels, k step
// 32; 128 threads, each owns a 4 x 4 register tile.
constexpr int FB_M = 32, FB_N = 64, FB_K = 32, FB_T = 128;

__global__ void __launch_bounds__(FB_T)
fbp_filter_kernel(const float* __restrict__ G, const float* __restrict__ H, int V, int C,
                  int in_mode, float* __restrict__ Q) {
  __shared__ float sG[FB_K][FB_M + 4];
  __shared__ float sH[FB_K][FB_N + 4];
  const int v0 = blockIdx.y * FB_M, m0 = blockIdx.x * FB_N;
  const int tx = threadIdx.x & 15;  // channel group (4 channels each)
  const int ty = threadIdx.x >> 4;  // view group (4 views each)
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
  for (int k0 = 0; k0 < C; k0 += FB_K) {
    // G tile: 32 views x 32 k -> transposed into sG[k][v].
    for (int e = threadIdx.x; e < FB_M * FB_K; e += FB_T) {
      int vv = e / FB_K, kk = e % FB_K;
      int v = v0 + vv, k = k0 + kk;
      sG[kk][vv] = (v < V && k < C) ? G[(size_t)v * C + k] : 0.0f;
    }
    // H tile: 64 rows m x 32 k -> sH[k][m].
    for (int e = threadIdx.x; e < FB_N * FB_K; e += FB_T) {
      int mm = e / FB_K, kk = e % FB_K;
      int m = m0 + mm, k = k0 + kk;
      sH[kk][mm] = (m < C && k < C) ? H[(size_t)m * C + k] : 0.0f;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < FB_K; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = sG[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = sH[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int v = v0 + ty * 4 + i;
    if (v >= V) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int m = m0 + tx + 16 * j;
      if (m >= C) continue;
      float q = acc[i][j];
      if (in_mode && (q < 1000.0f || q > 300000.0f)) q = 0.0f;  // :250-255
      Q[(size_t)v * C + m] = q;
    }
  }
}

int launch_fbp_filter(const float* d_g, const float* d_h, int V, int C, int in_mode, float* d_q,
                      cudaStream_t st) {
  dim3 grid((C + FB_N - 1) / FB_N, (V + FB_M - 1) / FB_M);
  fbp_filter_kernel<<<grid, FB_T, 0, st>>>(d_g, d_h, V, C, in_mode, d_q);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------------------------- backproject
constexpr int BP_TX = 16, BP_TY = 16, BP_VCHUNK = 16;

__global__ void __launch_bounds__(BP_TX * BP_TY)
fbp_bp_kernel(const float* __restrict__ Q, int V, int C, int N, float scale, float sid,
              float inv_dbeta_det, float center_ch, float out_scale, const float2* __restrict__ cs,
              float* __restrict__ img) {
  extern __shared__ float sm[];
  float* sQ = sm;                                           // [BP_VCHUNK][C]
  float2* sCS = reinterpret_cast<float2*>(sm + BP_VCHUNK * C);  // [BP_VCHUNK]
  const int x = blockIdx.x * BP_TX + threadIdx.x;
  const int y = blockIdx.y * BP_TY + threadIdx.y;
  const int tid = threadIdx.y * BP_TX + threadIdx.x;
  // Inscribed-circle mask (FBP/misc.cpp:20-36): (y-r)^2 + (x-r)^2 <= r^2.
  const double r = (double)(N - 1) / 2.0;
  const bool inside = x < N && y < N &&
                      ((double)y - r) * ((double)y - r) + ((double)x - r) * ((double)x - r) <= r * r;
  const float cp = (float)N / 2.0f - 0.5f;
  const float xx = -((float)x - cp) * scale;
  const float yy = -((float)y - cp) * scale;
  const int use = V / 2 * 2;  // usesinogram, :30
  float acc = 0.0f;
  for (int v0 = 0; v0 < use; v0 += BP_VCHUNK) {
    const int nv = min(BP_VCHUNK, use - v0);
    __syncthreads();
    for (int e = tid; e < nv * C; e += BP_TX * BP_TY) sQ[e] = Q[(size_t)v0 * C + e];
    if (tid < nv) sCS[tid] = cs[v0 + tid];
    __syncthreads();
    if (inside) {
      for (int j = 0; j < nv; j++) {
        const float2 t = sCS[j];  // (cos, sin)
        const float X = xx * t.x + yy * t.y;
        const float Y = -xx * t.y + yy * t.x;
        const float d = sid - Y;
        const float L2 = d * d + X * X;
        const float fg = atanf(__fdividef(X, d)) * inv_dbeta_det + center_ch;
        const int gi = (int)fg;  // truncation as (int)(fGAM), :73
        if (gi >= 0 && gi < C - 1) {
          const float w = fg - (float)gi;
          const float* q = sQ + j * C + gi;
          const float s1 = (1.0f - w) * q[0] + w * q[1];
          acc += __fdividef(s1, L2);
        }
      }
    }
  }
  if (x < N && y < N) img[(size_t)y * N + x] = inside ? acc * out_scale : 0.0f;
}

int launch_fbp_backproject(const float* d_q, int V, int C, int N, double pixel_cm, double sid,
                           double max_beta, int xfactor, const float* d_cs, float* d_img,
                           cudaStream_t st) {
  const int half = (C - 1) / 2;
  const double dbeta_det = max_beta / half;
  const double dbeta = 2.0 * 3.141592653589793 / V;
  dim3 grid((N + BP_TX - 1) / BP_TX, (N + BP_TY - 1) / BP_TY);
  dim3 block(BP_TX, BP_TY);
  const size_t smem = (size_t)BP_VCHUNK * C * sizeof(float) + BP_VCHUNK * sizeof(float2);
  VCT_CUDA(cudaFuncSetAttribute(fbp_bp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fbp_bp_kernel<<<grid, block, smem, st>>>(d_q, V, C, N, (float)pixel_cm, (float)sid,
                                           (float)(1.0 / dbeta_det), (float)(C / 2),
                                           (float)(dbeta * xfactor),
                                           reinterpret_cast<const float2*>(d_cs), d_img);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

}  // namespace vct
