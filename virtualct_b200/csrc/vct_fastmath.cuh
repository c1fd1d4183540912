// Small float helpers shared by the backprojector (vct_fbp.cu) and the
// adjoint's channel search (vct_adjoint.cu).
#pragma once
#include <cuda_runtime.h>

namespace vct {

// atan(t) on |t| <= 0.5 as t*P(t^2), P of degree 5: a least-squares fit of
// atan(t)/t on Chebyshev nodes in t^2 (made for this kernel); max error
// 3.7e-8 rad in FP32.  Pixels inside the reconstruction circle see
// |t| = |X/(SID-Y)| < 0.45 at the default geometry; larger |t| is outside
// the fan and rejected by the channel test either way.
__device__ __forceinline__ float atan_small(float t) {
  const float u = t * t;
  float p = -0.05077829957008362f;
  p = fmaf(p, u, 0.10122803598642349f);
  p = fmaf(p, u, -0.14165857434272766f);
  p = fmaf(p, u, 0.19993248581886292f);
  p = fmaf(p, u, -0.3333319127559662f);
  p = fmaf(p, u, 1.0f);
  return t * p;
}

__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

}  // namespace vct
