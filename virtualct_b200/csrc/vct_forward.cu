// MBFPA forward projection on sm_100a.
//
// One thread walks one ray (view v, channel c) through the N x N grid exactly
// as MB/reprojection_TOMO.cpp:53-283 does -- same double-precision expressions
// in the same order, compiled with --fmad=false so no product is fused -- and
// accumulates the per-element line integrals L_m = sum_seg rho_m * len in FP64
// registers.  The walk is done once per ray for all energy bins (the
// reference repeats it for every bin, MB/main.cpp:492-506); the polyenergetic
// epilogue then evaluates sum_E pdf(E) * exp(-sum_m mu_m(E) L_m) with the
// mu table in shared memory.
//
// Maps are read as one 16-byte record (8 x int16) per pixel through the
// read-only path; at 512^2 the record array is 4 MB and stays L2-resident.
#include <cuda_runtime.h>

#include "vct_internal.h"
#include "vct_philox.h"

namespace vct {

// ---------------------------------------------------------------- map packing
__global__ void pack_maps_kernel(const int16_t* __restrict__ maps, int M, int n2,
                                 PixelRec* __restrict__ out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n2) return;
  PixelRec r;
#pragma unroll
  for (int m = 0; m < 8; m++) {
    int16_t v = m < M ? maps[(size_t)m * n2 + p] : (int16_t)0;
    r.m[m] = v < 0 ? (int16_t)0 : v;
  }
  out[p] = r;
}

int launch_pack_maps(const int16_t* d_maps, int M, int N, PixelRec* d_packed, cudaStream_t st) {
  int n2 = N * N;
  pack_maps_kernel<<<(n2 + 255) / 256, 256, 0, st>>>(d_maps, M, n2, d_packed);
  return cudaGetLastError() == cudaSuccess ? VCT_OK : cuda_fail(cudaGetLastError(), "pack_maps_kernel");
}

// ------------------------------------------------------------------ the walk
// (int)d as the reference's x86-64 build evaluates it (cvttsd2si): NaN and
// out-of-range values give INT_MIN, whereas the PTX conversion saturates and
// maps NaN to 0.  Only reachable on degenerate rays, but it keeps the
// rejection of NaN segments identical.
__device__ __forceinline__ int trunc_i32(double d) {
  return (d >= -2147483648.0 && d < 2147483648.0) ? __double2int_rz(d) : (int)0x80000000;
}

struct RayAcc {
  double L[8];
  int nseg;
};

template <int M>
__device__ __forceinline__ void gather_add(const PixelRec* __restrict__ maps, int pix, double rr,
                                           RayAcc& a) {
  const int4 w = __ldg(reinterpret_cast<const int4*>(maps) + pix);
  const unsigned int u[4] = {(unsigned)w.x, (unsigned)w.y, (unsigned)w.z, (unsigned)w.w};
#pragma unroll
  for (int m = 0; m < M; m++) {
    unsigned int s = (m & 1) ? (u[m >> 1] >> 16) : (u[m >> 1] & 0xffffu);
    // rho = (float)short/1000 as MB/main.cpp:103 (IEEE float division).
    float rho = __fdiv_rn((float)s, 1000.0f);
    a.L[m] = __fma_rn((double)rho, rr, a.L[m]);
  }
  a.nseg++;
}

// Segment emission of MB/reprojection_TOMO.cpp:145-163 / :171-189: length,
// midpoint pixel (truncating casts), bounds test, then the gather.
template <int M>
__device__ __forceinline__ void emit(const DevGeom& g, const PixelRec* __restrict__ maps, double xb0,
                                     double yb0, double xb1, double yb1, RayAcc& a) {
  double rr = sqrt((xb0 - xb1) * (xb0 - xb1) + (yb0 - yb1) * (yb0 - yb1));
  int xmc = trunc_i32((xb0 + xb1) * 0.5 / g.s + g.nxm);
  int ymc = trunc_i32((-yb0 - yb1) * 0.5 / g.s + g.nxm);
  if (xmc >= 0 && ymc >= 0 && xmc <= g.N - 1 && ymc <= g.N - 1) {
    if (g.rmax_active) {
      // ph = 0 for every element when the midpoint radius (cm) reaches rmax
      // (a pixel count), :150-155.
      double r = sqrt((xb0 + xb1) * (xb0 + xb1) + (-yb0 - yb1) * (-yb0 - yb1)) * 0.5;
      if (r >= g.rmax) return;
    }
    gather_add<M>(maps, xmc + ymc * g.N, rr, a);
  }
}

template <int M>
__device__ void walk_ray(const DevGeom& g, const PixelRec* __restrict__ maps, double cb, double sb,
                         double px0, double py0, RayAcc& a) {
  const double sx = g.sid * sb;  // :53
  const double sy = g.sid * cb;  // :54
  const double px = +px0 * cb + py0 * sb;  // :73
  const double py = -px0 * sb + py0 * cb;  // :74
  const double lim = g.lim;
  // Grid-square intersections, :76-101.
  double xx0 = 0, yy0 = 0, xx1 = 0, yy1 = 0;
  int m = 0;
  {
    double t;
    double yv = lim;
    t = (yv - sy) / (py - sy) * (px - sx) + sx;
    if (fabs(t) < lim) { if (m == 0) { xx0 = t; yy0 = yv; } else { xx1 = t; yy1 = yv; } m++; }
    yv = -lim;
    t = (yv - sy) / (py - sy) * (px - sx) + sx;
    if (fabs(t) < lim) { if (m == 0) { xx0 = t; yy0 = yv; } else if (m == 1) { xx1 = t; yy1 = yv; } m++; }
    double xv = lim;
    t = (xv - sx) / (px - sx) * (py - sy) + sy;
    if (fabs(t) < lim) { if (m == 0) { xx0 = xv; yy0 = t; } else if (m == 1) { xx1 = xv; yy1 = t; } m++; }
    xv = -lim;
    t = (xv - sx) / (px - sx) * (py - sy) + sy;
    if (fabs(t) < lim) { if (m == 0) { xx0 = xv; yy0 = t; } else if (m == 1) { xx1 = xv; yy1 = t; } m++; }
  }
  // A ray missing the square never enters the reference's walk loop.
  if (m < 2) return;
  double xi, yi, xf, yf;  // :103-108
  if ((xx0 - sx) * (xx0 - sx) + (yy0 - sy) * (yy0 - sy) + 0.0 <
      (xx1 - sx) * (xx1 - sx) + (yy1 - sy) * (yy1 - sy) + 0.0) {
    xi = xx0; yi = yy0; xf = xx1; yf = yy1;
  } else {
    xi = xx1; yi = yy1; xf = xx0; yf = yy0;
  }
  double xb0 = xi, yb0 = yi;
  const int max_steps = 4 * g.N + 64;  // a walk has at most ~N+2 steps
  if (fabs(xi - xf) > fabs(yi - yf)) {  // x-major, :113-200
    const double pha = (xf - xi) / fabs(xi - xf);
    int xin;
    if ((xi < 0 && (xf - xi) < 0) || (xi > 0 && (xf - xi) > 0))
      xin = trunc_i32((double)trunc_i32(xi) + (xf - xi) / fabs(xf - xi));
    else
      xin = trunc_i32(xi);
    double xii = xin;
    double yii = (xii - sx) / (px - sx) * (py - sy) + sy;
    int yma = 0;
    const double ydir = (yf - yi) / fabs(yf - yi);
    for (int ik = 0; ik < max_steps; ik++) {
      if (!(xii <= lim && xii >= -lim && yii <= lim && yii >= -lim)) break;
      xii = xin + pha * ik * g.s;
      const int ymb = yma;
      const double yj = yii;
      yii = (xii - sx) / (px - sx) * (py - sy) + sy;
      yma = trunc_i32(yii / g.s);
      if (ik != 0 && (yma != ymb || (yii / fabs(yii) != yj / fabs(yj)))) {
        double yiii;
        if ((yii < 0 && (yf - yi) < 0) || (yii > 0 && (yf - yi) > 0))
          yiii = (double)(yma * g.s);
        else
          yiii = (double)(yma * g.s) - ydir * g.s;
        const double xiii = (yiii - sy) / (py - sy) * (px - sx) + sx;
        const double chy = (xii - xiii) * (xii - xiii) + (yii - yiii) * (yii - yiii);
        if (chy != 0) {
          emit<M>(g, maps, xb0, yb0, xiii, yiii, a);
          xb0 = xiii;
          yb0 = yiii;
        }
      }
      emit<M>(g, maps, xb0, yb0, xii, yii, a);
      xb0 = xii;
      yb0 = yii;
    }
  } else {  // y-major, :201-283
    const double pha = (yf - yi) / fabs(yi - yf);
    int yin;
    if ((yi < 0 && (yf - yi) < 0) || (yi > 0 && (yf - yi) > 0))
      yin = trunc_i32((double)trunc_i32(yi) + (yf - yi) / fabs(yf - yi));
    else
      yin = trunc_i32(yi);
    double yii = yin;
    double xii = (yii - sy) / (py - sy) * (px - sx) + sx;
    int xma = 0;
    const double xdir = (xf - xi) / fabs(xf - xi);
    for (int ik = 0; ik < max_steps; ik++) {
      if (!(xii <= lim && xii >= -lim && yii <= lim && yii >= -lim)) break;
      yii = yin + pha * ik * g.s;
      const int xmb = xma;
      const double xj = xii;
      xii = (yii - sy) / (py - sy) * (px - sx) + sx;
      xma = trunc_i32(xii / g.s);
      if (ik != 0 && (xma != xmb || (xii / fabs(xii) != xj / fabs(xj)))) {
        double xiii;
        if ((xii < 0 && (xf - xi) < 0) || (xii > 0 && (xf - xi) > 0))
          xiii = (double)(xma * g.s);
        else
          xiii = (double)(xma * g.s) - xdir * g.s;
        const double yiii = (xiii - sx) / (px - sx) * (py - sy) + sy;
        const double chy = (xii - xiii) * (xii - xiii) + (yii - yiii) * (yii - yiii);
        if (chy != 0) {
          emit<M>(g, maps, xb0, yb0, xiii, yiii, a);
          xb0 = xiii;
          yb0 = yiii;
        }
      }
      emit<M>(g, maps, xb0, yb0, xii, yii, a);
      xb0 = xii;
      yb0 = yii;
    }
  }
}

// ------------------------------------------------------------- the kernel
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_ull(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kFwdThreads = 128;

template <int M, int SUM_MODE>
__global__ void __launch_bounds__(kFwdThreads)
forward_kernel(DevGeom g, const PixelRec* __restrict__ maps, const double* __restrict__ mu_scaled,
               const float* __restrict__ pdf, int NE, const double* __restrict__ cos_t,
               const double* __restrict__ sin_t, const double* __restrict__ det_px0,
               const double* __restrict__ det_py0, float* __restrict__ out,
               double* __restrict__ lint, FwdStats* __restrict__ stats) {
  extern __shared__ double smem[];
  double* s_mu = smem;                              // [NE][M]
  float* s_pdf = reinterpret_cast<float*>(smem + (size_t)NE * M);  // [NE]
  for (int i = threadIdx.x; i < NE * M; i += blockDim.x) s_mu[i] = mu_scaled[i];
  for (int i = threadIdx.x; i < NE; i += blockDim.x) s_pdf[i] = pdf[i];
  __syncthreads();

  const long long nrays = (long long)g.views_used * g.C;
  const long long ray = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = ray < nrays;
  float val = 0.0f;
  RayAcc a;
#pragma unroll
  for (int m = 0; m < 8; m++) a.L[m] = 0.0;
  a.nseg = 0;
  if (active) {
    const int v = (int)(ray / g.C);
    const int c = (int)(ray - (long long)v * g.C);
    walk_ray<M>(g, maps, cos_t[v], sin_t[v], det_px0[c], det_py0[c], a);
    if (lint) {
#pragma unroll
      for (int m = 0; m < M; m++) lint[ray * M + m] = a.L[m];
    }
    if (out) {
      float accf = 0.0f;
      double accd = 0.0;
      for (int e = 0; e < NE; e++) {
        double t = 0.0;
#pragma unroll
        for (int m = 0; m < M; m++) t = __fma_rn(s_mu[e * M + m], a.L[m], t);
        double intens = (double)s_pdf[e] * exp(-t);
        if (SUM_MODE == VCT_SUM_REFERENCE)
          accf = __fadd_rn(accf, (float)intens);
        else
          accd = __dadd_rn(accd, intens);
      }
      val = SUM_MODE == VCT_SUM_REFERENCE ? accf : (float)accd;
      out[(size_t)v * g.width + g.start + c] = val;
    }
  }
  // Block reductions: max/min of the output and the segment count.
  __shared__ float s_max[kFwdThreads / 32], s_min[kFwdThreads / 32];
  __shared__ unsigned long long s_seg[kFwdThreads / 32];
  float vmax = active ? val : 0.0f;
  float vmin = active ? val : 3.0e38f;
  unsigned long long ns = (unsigned long long)a.nseg;
  vmax = warp_max(vmax);
  vmin = warp_min(vmin);
  ns = warp_sum_ull(ns);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { s_max[wid] = vmax; s_min[wid] = vmin; s_seg[wid] = ns; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float bm = s_max[0], bn = s_min[0];
    unsigned long long bs = s_seg[0];
    for (int w = 1; w < kFwdThreads / 32; w++) {
      bm = fmaxf(bm, s_max[w]);
      bn = fminf(bn, s_min[w]);
      bs += s_seg[w];
    }
    // Non-negative floats order like their bit patterns.
    atomicMax(&stats->max_bits, __float_as_uint(bm));
    atomicMin(&stats->min_bits, __float_as_uint(bn));
    atomicAdd(&stats->segments, bs);
  }
}

template <int M>
static int launch_forward_m(const DevGeom& g, const PixelRec* d_maps, const double* d_mu,
                            const float* d_pdf, int NE, const double* d_cos, const double* d_sin,
                            const double* d_px0, const double* d_py0, int sum_mode, float* d_out,
                            double* d_lint, FwdStats* d_stats, cudaStream_t st) {
  const long long nrays = (long long)g.views_used * g.C;
  const int blocks = (int)((nrays + kFwdThreads - 1) / kFwdThreads);
  const size_t smem = (size_t)NE * M * sizeof(double) + (size_t)NE * sizeof(float);
  if (blocks == 0) return VCT_OK;
  if (sum_mode == VCT_SUM_REFERENCE) {
    auto k = forward_kernel<M, VCT_SUM_REFERENCE>;
    VCT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<blocks, kFwdThreads, smem, st>>>(g, d_maps, d_mu, d_pdf, NE, d_cos, d_sin, d_px0, d_py0,
                                          d_out, d_lint, d_stats);
  } else {
    auto k = forward_kernel<M, VCT_SUM_COMPENSATED>;
    VCT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<blocks, kFwdThreads, smem, st>>>(g, d_maps, d_mu, d_pdf, NE, d_cos, d_sin, d_px0, d_py0,
                                          d_out, d_lint, d_stats);
  }
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int launch_forward(const DevGeom& g, const PixelRec* d_maps, int M, const double* d_mu_scaled,
                   const float* d_pdf, int NE, const double* d_cos, const double* d_sin,
                   const double* d_det_ox, const double* d_det_oy, int sum_mode, float* d_out,
                   double* d_lint, FwdStats* d_stats, cudaStream_t st) {
  switch (M) {
#define VCT_CASE(mm) \
  case mm:           \
    return launch_forward_m<mm>(g, d_maps, d_mu_scaled, d_pdf, NE, d_cos, d_sin, d_det_ox, d_det_oy, sum_mode, d_out, d_lint, d_stats, st);
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default:
      return fail(VCT_E_ARG, "number of materials must be 1..8");
  }
}

// -------------------------------------------------- normalisation and noise
// MB/main.cpp:511-522 (divide by the float maximum) and gaussiannoise0
// (:51-76): p += sigma*z, p < 0 -> projection_min/10, p > 1 -> 1, with
// z = sqrt(-2 ln u1) sin(2 pi u2) (:46-49).  u1, u2 come from Philox4x32-10
// keyed by the 64-bit seed, counter (channel, view, 0, 0).
__global__ void normalize_noise_kernel(const float* __restrict__ in, float* __restrict__ out, int V,
                                       int W, const FwdStats* __restrict__ stats, int pad_zero,
                                       double sigma, uint32_t k0, uint32_t k1) {
  const long long n = (long long)V * W;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float pmax = __uint_as_float(stats->max_bits);
  float pmin_raw = __uint_as_float(stats->min_bits);
  if (pad_zero) pmin_raw = fminf(pmin_raw, 0.0f);
  const float p = __fdiv_rn(in[i], pmax);
  if (sigma <= 0.0) {
    out[i] = p;
    return;
  }
  const double pmin = (double)__fdiv_rn(pmin_raw, pmax);
  const int v = (int)(i / W);
  const int c = (int)(i - (long long)v * W);
  Philox4 ctr;
  ctr.v[0] = (uint32_t)c;
  ctr.v[1] = (uint32_t)v;
  ctr.v[2] = 0u;
  ctr.v[3] = 0u;
  const Philox4 r = philox4x32_10(ctr, k0, k1);
  const double u1 = u01_open(r.v[0], r.v[1]);
  const double u2 = u01_open(r.v[2], r.v[3]);
  const double z = sqrt(-2.0 * log(u1)) * sin(2.0 * 3.141592653589793 * u2);
  const double nstar = (double)p + sigma * z;
  float o = (float)nstar;
  if (nstar < 0) o = (float)(pmin / 10);
  if (nstar > 1.0) o = 1.0f;
  out[i] = o;
}

int launch_normalize_noise(const DevGeom& g, const float* d_in, float* d_out, const FwdStats* d_stats,
                           int pad_zero, double sigma, uint64_t seed, cudaStream_t st) {
  const long long n = (long long)g.views * g.width;
  const int threads = 256;
  const int blocks = (int)((n + threads - 1) / threads);
  normalize_noise_kernel<<<blocks, threads, 0, st>>>(d_in, d_out, g.views, g.width, d_stats, pad_zero,
                                                     sigma, (uint32_t)seed, (uint32_t)(seed >> 32));
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

}  // namespace vct
