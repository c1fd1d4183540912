// Projected gradient-descent step on element densities, for iterative
// material decomposition driven by the adjoint (no counterpart in the
// reference; its own iterative update is a multiplicative ratio step).
#include <cuda_runtime.h>
#include <math.h>

#include "vct_internal.h"

namespace vct {

__global__ void descent_kernel(float* __restrict__ rho, const float* __restrict__ ga, const float* __restrict__ gb,
                               float step, double units, int16_t* __restrict__ maps, long long count) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    float g = ga[i];
    if (gb) g += gb[i];
    const float r = fmaxf(rho[i] - step * g, 0.0f);
    rho[i] = r;
    const double q = rint((double)r * units);
    maps[i] = (int16_t)(q > 32767.0 ? 32767.0 : q);
  }
}

// Diagonally scaled step: rho -= step * grad * scale, the scale table of one
// slice ([M][N][N]) applied to each of `count` entries modulo `period`.
__global__ void descent_scaled_kernel(float* __restrict__ rho, const float* __restrict__ grad,
                                      const float* __restrict__ scale, long long period, float step, double units,
                                      int16_t* __restrict__ maps, long long count) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const float r = fmaxf(rho[i] - step * (grad[i] * scale[i % period]), 0.0f);
    rho[i] = r;
    const double q = rint((double)r * units);
    maps[i] = (int16_t)(q > 32767.0 ? 32767.0 : q);
  }
}

}  // namespace vct

using namespace vct;

extern "C" int vct_descent_step_dev(float* d_rho, const float* d_grad_a, const float* d_grad_b, double step,
                                    double units, int16_t* d_maps, long long count, void* stream) {
  if (!d_rho || !d_grad_a || !d_maps || count < 0 || !(units > 0)) return fail(VCT_E_ARG, "vct_descent_step_dev: bad argument");
  if (count == 0) return VCT_OK;
  const long long blocks = (count + 255) / 256;
  descent_kernel<<<(unsigned)(blocks < 65535 * 16 ? blocks : 65535 * 16), 256, 0, (cudaStream_t)stream>>>(
      d_rho, d_grad_a, d_grad_b, (float)step, units, d_maps, count);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

extern "C" int vct_descent_step_scaled_dev(float* d_rho, const float* d_grad, const float* d_scale, long long period,
                                           double step, double units, int16_t* d_maps, long long count,
                                           void* stream) {
  if (!d_rho || !d_grad || !d_scale || !d_maps || count < 0 || period <= 0 || !(units > 0))
    return fail(VCT_E_ARG, "vct_descent_step_scaled_dev: bad argument");
  if (count == 0) return VCT_OK;
  const long long blocks = (count + 255) / 256;
  descent_scaled_kernel<<<(unsigned)(blocks < 65535 * 16 ? blocks : 65535 * 16), 256, 0, (cudaStream_t)stream>>>(
      d_rho, d_grad, d_scale, period, (float)step, units, d_maps, count);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}
