// The reference's iterative step on sm_100a: the image update of
// IR_ImageTOMO (MB/IR_ImageTOMO.cpp:19-72) and the sinogram distances of
// calc_squdiff_quad (MB/main.cpp:111-134).  Together with lengthproj_TOMO_2
// (vct_lengthproj.cu) and the forward they make the step of MB/main.cpp:
// 432-600 that writes ReconImageRaw/*.
#include <cuda_runtime.h>
#include <math.h>

#include "vct_internal.h"

namespace vct {

// double_TV of MB/IR_ImageTOMO.cpp:10-17: the total-variation derivative at a
// pixel from its neighbours (a1 left, a2 right, a3 up, a4 down, a7 down-left,
// a8 up-right), float differences squared in float, roots in double.
__device__ __forceinline__ double tv_term(float a, float a1, float a2, float a3, float a4, float a7, float a8) {
  const double d1 = sqrt((double)(__fadd_rn(__fmul_rn(a - a2, a - a2), __fmul_rn(a - a4, a - a4)))) + 0.00000001;
  const double d2 = sqrt((double)(__fadd_rn(__fmul_rn(a - a1, a - a1), __fmul_rn(a1 - a7, a1 - a7)))) + 0.00000001;
  const double d3 = sqrt((double)(__fadd_rn(__fmul_rn(a3 - a8, a3 - a8), __fmul_rn(a - a3, a - a3)))) + 0.00000001;
  return (double)(__fadd_rn(a - a2, a - a4)) / d1 + (double)(a - a1) / d2 + (double)(a - a3) / d3;
}

// One update of the image (the first element's map, N x N): per mask pixel,
// lambda = w_tv * TV + w_prior * TV(image - prior) + 1e-6 (interior pixels),
// del_F = npf_re - npf/thinout + lambda; after = max(0, before + w * del_F)
// with w = wbefore, or before / (npf/thinout - lambda) past iteration 300.
// Pixels outside the mask keep `after` unchanged.
__global__ void ir_update_kernel(int N, const float* __restrict__ before, const float* __restrict__ prior,
                                 const float* __restrict__ npf, const float* __restrict__ npf_re, double wbefore,
                                 double w_tv, double w_prior, int ite, int thinout, float* __restrict__ after) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= N) return;
  const double r = (double)(N - 1) / 2.0;
  if (!(((double)y - r) * ((double)y - r) + ((double)x - r) * ((double)x - r) <= r * r)) return;
  const int k = y * N + x;
  double cost_tv = 0.0, cost_prior = 0.0;
  if (y < N - 1 && x < N - 1 && x > 0 && y > 0) {
    const int k1 = k - 1, k2 = k + 1, k3 = k - N, k4 = k + N, k7 = k + N - 1, k8 = k - N + 1;
    cost_tv = -tv_term(before[k], before[k1], before[k2], before[k3], before[k4], before[k7], before[k8]);
    const float p0 = prior ? prior[k] : 0.0f, p1 = prior ? prior[k1] : 0.0f, p2 = prior ? prior[k2] : 0.0f,
                p3 = prior ? prior[k3] : 0.0f, p4 = prior ? prior[k4] : 0.0f, p7 = prior ? prior[k7] : 0.0f,
                p8 = prior ? prior[k8] : 0.0f;
    cost_prior = -tv_term(before[k] - p0, before[k1] - p1, before[k2] - p2, before[k3] - p3, before[k4] - p4,
                          before[k7] - p7, before[k8] - p8);
  }
  const double lambda = w_tv * cost_tv + w_prior * cost_prior + 0.000001;
  const double del_F = npf_re[k] - npf[k] / thinout + lambda;
  double w = wbefore;
  if (ite > 300) w = before[k] / (npf[k] / thinout - lambda);
  float v = (float)(before[k] + w * del_F);
  if (v < 0.0f) v = 0.0f;
  after[k] = v;
}

int launch_ir_update(int N, const float* d_before, const float* d_prior, const float* d_npf, const float* d_npf_re,
                     double wbefore, double w_tv, double w_prior, int ite, int thinout, float* d_after,
                     cudaStream_t st) {
  dim3 grid((N + 127) / 128, N);
  ir_update_kernel<<<grid, 128, 0, st>>>(N, d_before, d_prior, d_npf, d_npf_re, wbefore, w_tv, w_prior, ite,
                                         thinout, d_after);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// calc_squdiff_quad: over rows thinnumb + j*thinout (j < count/thinout) and
// channels [start, end): objective = sum (double)(p - r)^2 (the difference
// in float), quadratic = sum 0.5 p ln(p/r)^2 (only when `quad`).  Per-block
// partials in a fixed order, then one block sums them: deterministic.
constexpr int kSqThreads = 256;

__global__ void squdiff_kernel(const float* __restrict__ p, const float* __restrict__ r, int W, int start, int C,
                               int first, int stride, int rows, int quad, double* __restrict__ part) {
  __shared__ double s_o[kSqThreads], s_q[kSqThreads];
  const long long n = (long long)rows * C;
  double o = 0.0, qd = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(i / C), c = (int)(i - (long long)j * C);
    const size_t idx = (size_t)(first + j * stride) * W + start + c;
    const double d = (double)(p[idx] - r[idx]);
    o += d * d;
    if (quad) {
      const double t = log((double)(p[idx] / r[idx]));
      qd += 0.5 * p[idx] * t * t;
    }
  }
  s_o[threadIdx.x] = o;
  s_q[threadIdx.x] = qd;
  __syncthreads();
  for (int w = kSqThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s_o[threadIdx.x] += s_o[threadIdx.x + w];
      s_q[threadIdx.x] += s_q[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s_o[0];
    part[2 * blockIdx.x + 1] = s_q[0];
  }
}

__global__ void squdiff_final_kernel(const double* __restrict__ part, int nb, double* __restrict__ out) {
  if (threadIdx.x == 0) {
    double o = 0.0, q = 0.0;
    for (int b = 0; b < nb; b++) {
      o += part[2 * b];
      q += part[2 * b + 1];
    }
    out[0] = o;
    out[1] = q;
  }
}

constexpr int kSqBlocks = 148;

int squdiff_scratch_doubles() { return 2 * kSqBlocks; }

int launch_squdiff(const float* d_p, const float* d_r, int W, int start, int C, int first, int stride, int rows,
                   int quad, double* d_part, double* d_out, cudaStream_t st) {
  squdiff_kernel<<<kSqBlocks, kSqThreads, 0, st>>>(d_p, d_r, W, start, C, first, stride, rows, quad, d_part);
  VCT_CUDA(cudaGetLastError());
  squdiff_final_kernel<<<1, 32, 0, st>>>(d_part, kSqBlocks, d_out);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

}  // namespace vct
