// Adjoint of the MBFPA forward projector on sm_100a (no counterpart in the
// reference, which has no gradient).
//
// The forward model is the reference walk (MB/reprojection_TOMO.cpp:113-283)
// as a linear map A from element densities rho_m [N][N] (g/cm^3) to per-ray
// line integrals L_m = sum_seg rho_m(pixel) * len, followed by the
// polyenergetic intensity y = sum_E pdf(E) exp(-sum_m mu_m(E) L_m / xfactor).
// The loss is the reference's weighted log least squares (MB/main.cpp:125-126)
//     l = 1/2 sum_i w_i (ln(y_i / ynorm) - ln p_i)^2,   ynorm = sum_E pdf(E),
// over rays with p_i > 0 (w_i = p_i unless the caller gives weights), and
//     dl/drho_m = A^T g_m,   g_m,i = -w_i r_i D_m,i / y_i,
// D_m,i = sum_E pdf exp(...) mu_m(E) / xfactor.  A VJP mode takes dl/d(y/ynorm)
// from the caller instead of the loss.
//
// A^T is computed exactly for the walk, not for an idealised ray model.  For
// every ray the fast walk's plan (vct_walk.cuh) says which cells it covers:
//   - the lumped first segment (entry point to the first whole-cm major
//     gridline) goes to one pixel with one length;
//   - after it, whole major steps between two major cell indices, where each
//     cell receives the exact chord of the ray through it (cells at index -1
//     fold onto index 0, the reference's truncating cast; index N is dropped).
// The pixel-driven gather (adj_gather_kernel) evaluates, for every pixel and
// view, the chords of the few rays whose footprint covers it, tests the cell
// against the ray's major-index range, adds the lumped length where the pixel
// is the ray's lumped pixel, and accumulates g * len: no atomics, one thread
// per pixel, fixed order, hence deterministic.  Rays the fast walk hands to
// the exact walk (rays through the grid origin, where the reference's sign
// test divides 0/0) are scattered along the exact walk in 64-bit fixed point
// with integer atomics, whose sum does not depend on their order.
#include <cuda_runtime.h>
#include <math.h>

#include "vct_internal.h"
#include "vct_walk.cuh"

namespace vct {

// ------------------------------------------------------------- walk plans
// Per-ray record: x = kind | xmaj << 2; y = (maj_lo + 1) | (maj_hi + 1) << 16;
// z = lumped pixel (col | row << 16) or -1; w = lumped length (float bits, cm).
__global__ void adj_plan_kernel(DevGeom g, const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                                const double* __restrict__ det_px0, const double* __restrict__ det_py0,
                                int4* __restrict__ rec, int* __restrict__ special, int* __restrict__ nspecial) {
  const long long nrays = (long long)g.views_used * g.C;
  const long long ray = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (ray >= nrays) return;
  const int v = (int)(ray / g.C);
  const int c = (int)(ray - (long long)v * g.C);
  int4 o = make_int4(kAdjRayNone, 0, -1, 0);
  Ray r;
  if (ray_setup(g, cos_t[v], sin_t[v], det_px0[c], det_py0[c], r)) {
    FastPlan p;
    if (g.rmax_active)
      p.status = kPlanExact;
    else
      fast_plan(g, r, p);
    if (p.status == kPlanExact) {
      const int idx = atomicAdd(nspecial, 1);
      o.x = kAdjRayExact;
      o.y = idx;  // its place in the list (and in the line-integral buffer)
      special[idx] = (int)ray;
    } else if (p.status == kPlanWalk) {
      const int lo = min(p.maj0, p.majK), hi = max(p.maj0, p.majK);
      o.x = kAdjRayFast | (p.xmaj << 2);
      o.y = (lo + 1) | ((hi + 1) << 16);
      if (p.pix_lumped >= 0) {
        const int P = g.N + 2 * kPad;
        const int col = p.pix_lumped % P - kPad, row = p.pix_lumped / P - kPad;
        o.z = col | (row << 16);  // both in [0, N): no division to unpack
        o.w = __float_as_int((float)p.rr_first);
      }
    }
  }
  rec[ray] = o;
}

int launch_adj_plan(const DevGeom& g, const double* d_cos, const double* d_sin, const double* d_px0,
                    const double* d_py0, int4* d_rec, int* d_special, int* d_nspecial, cudaStream_t st) {
  const long long nrays = (long long)g.views_used * g.C;
  if (nrays == 0) return VCT_OK;
  VCT_CUDA(cudaMemsetAsync(d_nspecial, 0, sizeof(int), st));
  adj_plan_kernel<<<(unsigned)((nrays + 255) / 256), 256, 0, st>>>(g, d_cos, d_sin, d_px0, d_py0, d_rec, d_special,
                                                                   d_nspecial);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------------- forward with ray factors
// Fixed-point scale of the exact-walk scatter: every term |g * len| stays
// below 2^(62 - log2_terms), so the sum over at most 2^log2_terms terms fits
// a signed 64-bit integer.
__device__ __forceinline__ double special_scale(unsigned int gmax_bits, double lmax, int log2_terms) {
  const float gm = __uint_as_float(gmax_bits);
  if (!(gm > 0.0f)) return 1.0;
  const int e = ilogb((double)gm * lmax) + 1;  // gm * lmax < 2^e
  return ldexp(1.0, 62 - log2_terms - e);
}

__device__ __forceinline__ float ex2_approx_f(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr int kAdjFwdThreads = 128;

// One thread per ray: the walk (fast, or exact where the plan says so), then
// y and D_m over the energy bins (mu_l2 = mu * log2(e) / xfactor, 2^-x split
// as in the forward's compensated epilogue, FP64 sums), then the ray factors
// g_m.  MODE 0: loss (meas, optional weights); MODE 1: VJP (upstream
// dl/d(y/ynorm) in `meas`).  Per-block loss partials are summed in a fixed
// order.
// The ray's walk, y, D_m and ray factors g_m; returns its loss term (MODE 0).
template <int M, int MODE>
__device__ __forceinline__ double adj_forward_ray(const DevGeom& g, const PixelRec* __restrict__ maps,
                                                  const double* __restrict__ s_mu, const float* __restrict__ s_pdf,
                                                  int NE, double ynorm, const double* __restrict__ cos_t,
                                                  const double* __restrict__ sin_t,
                                                  const double* __restrict__ det_px0,
                                                  const double* __restrict__ det_py0, const int4* __restrict__ rec,
                                                  const double* __restrict__ lsp, const float* __restrict__ meas,
                                                  const float* __restrict__ wts,
                                                  float* __restrict__ gout, unsigned int* __restrict__ gmax_special,
                                                  long long ray) {
  double loss = 0.0;
  const int v = (int)(ray / g.C);
  const int c = (int)(ray - (long long)v * g.C);
  const int4 rc = rec[ray];
  const int kind = rc.x & 3;
  double L[8];
  if (kind == kAdjRayExact) {
    // walked beforehand by a whole warp (adj_lines_kernel)
#pragma unroll
    for (int m = 0; m < M; m++) L[m] = lsp[(size_t)rc.y * M + m];
  } else {
    RayAcc a;
    acc_init(a);
    if (kind == kAdjRayFast) {
      Ray r;
      ray_setup(g, cos_t[v], sin_t[v], det_px0[c], det_py0[c], r);
      walk_fast<M>(g, maps, r, a);
    }
    finish_lines<M>(a, L, g.dens_div);
  }
  double y = 0.0, D[M];
#pragma unroll
  for (int m = 0; m < M; m++) D[m] = 0.0;
  for (int e = 0; e < NE; e++) {
    double x = 0.0;
#pragma unroll
    for (int m = 0; m < M; m++) x = __fma_rn(s_mu[e * M + m], L[m], x);
    const int nI = __double2int_rd(x);
    if (nI <= 125) {
      const float fr = (float)(x - (double)nI);
      const float scale = __int_as_float((127 - nI) << 23);
      const double t = (double)(s_pdf[e] * ex2_approx_f(-fr) * scale);
      y += t;
#pragma unroll
      for (int m = 0; m < M; m++) D[m] = __fma_rn(t, s_mu[e * M + m], D[m]);
    }
  }
  const double kLn2 = 0.6931471805599453;
  const size_t si = (size_t)v * g.width + g.start + c;
  double f = 0.0;  // g_m = f * D_m (D_m still in log2 units)
  if (MODE == 0) {
    const double p = (double)meas[si];
    if (p > 0.0 && y > 0.0) {
      const double wgt = wts ? (double)wts[si] : p;
      const double rres = log(y / ynorm) - log(p);
      loss = 0.5 * wgt * rres * rres;
      f = -wgt * rres / y * kLn2;
    }
  } else {
    f = -(double)meas[si] / ynorm * kLn2;
  }
  float gm = 0.0f;
#pragma unroll
  for (int m = 0; m < M; m++) {
    const float gv = (float)(f * D[m]);
    gout[ray * M + m] = gv;
    gm = fmaxf(gm, fabsf(gv));
  }
  if (kind == kAdjRayExact) atomicMax(gmax_special, __float_as_uint(gm));
  return loss;
}

template <int M, int MODE>
__global__ void __launch_bounds__(kAdjFwdThreads)
adj_forward_kernel(DevGeom g, const PixelRec* __restrict__ maps, const double* __restrict__ mu_l2,
                   const float* __restrict__ pdf, int NE, double ynorm, const double* __restrict__ cos_t,
                   const double* __restrict__ sin_t, const double* __restrict__ det_px0,
                   const double* __restrict__ det_py0, const int4* __restrict__ rec, const double* __restrict__ lsp,
                   const float* __restrict__ meas, const float* __restrict__ wts, float* __restrict__ gout,
                   double* __restrict__ loss_part, unsigned int* __restrict__ gmax_special) {
  extern __shared__ double smem[];
  double* s_mu = smem;                                             // [NE][M]
  float* s_pdf = reinterpret_cast<float*>(smem + (size_t)NE * M);  // [NE]
  __shared__ double s_loss[kAdjFwdThreads / 32];
  for (int i = threadIdx.x; i < NE * M; i += blockDim.x) s_mu[i] = mu_l2[i];
  for (int i = threadIdx.x; i < NE; i += blockDim.x) s_pdf[i] = pdf[i];
  __syncthreads();

  const long long nrays = (long long)g.views_used * g.C;
  const long long ray = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double loss = 0.0;
  if (ray < nrays)
    loss = adj_forward_ray<M, MODE>(g, maps, s_mu, s_pdf, NE, ynorm, cos_t, sin_t, det_px0, det_py0, rec, lsp, meas,
                                    wts, gout, gmax_special, ray);
  if (MODE == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if ((threadIdx.x & 31) == 0) s_loss[threadIdx.x >> 5] = loss;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kAdjFwdThreads / 32; w++) t += s_loss[w];
      loss_part[blockIdx.x] = t;
    }
  }
}

template <int M>
static int launch_adj_forward_m(const DevGeom& g, const PixelRec* d_maps, const double* d_mu_l2, const float* d_pdf,
                                int NE, double ynorm, const double* d_cos, const double* d_sin, const double* d_px0,
                                const double* d_py0, const int4* d_rec, const double* d_lsp, int mode,
                                const float* d_meas, const float* d_wts, float* d_g, double* d_loss_part,
                                unsigned int* d_gmax, cudaStream_t st) {
  const long long nrays = (long long)g.views_used * g.C;
  const int blocks = (int)((nrays + kAdjFwdThreads - 1) / kAdjFwdThreads);
  const size_t smem = (size_t)NE * M * sizeof(double) + (size_t)NE * sizeof(float);
  if (blocks == 0) return VCT_OK;
  auto k = mode == 0 ? adj_forward_kernel<M, 0> : adj_forward_kernel<M, 1>;
  VCT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<blocks, kAdjFwdThreads, smem, st>>>(g, d_maps, d_mu_l2, d_pdf, NE, ynorm, d_cos, d_sin, d_px0, d_py0, d_rec,
                                          d_lsp, d_meas, d_wts, d_g, d_loss_part, d_gmax);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int adj_forward_blocks(const DevGeom& g) {
  const long long nrays = (long long)g.views_used * g.C;
  return (int)((nrays + kAdjFwdThreads - 1) / kAdjFwdThreads);
}

int launch_adj_forward(const DevGeom& g, const PixelRec* d_maps, int M, const double* d_mu_l2, const float* d_pdf,
                       int NE, double ynorm, const double* d_cos, const double* d_sin, const double* d_px0,
                       const double* d_py0, const int4* d_rec, const double* d_lsp, int mode, const float* d_meas,
                       const float* d_wts, float* d_g, double* d_loss_part, unsigned int* d_gmax, cudaStream_t st) {
  switch (M) {
#define VCT_CASE(mm)                                                                                              \
  case mm:                                                                                                        \
    return launch_adj_forward_m<mm>(g, d_maps, d_mu_l2, d_pdf, NE, ynorm, d_cos, d_sin, d_px0, d_py0, d_rec, d_lsp, \
                                    mode, d_meas, d_wts, d_g, d_loss_part, d_gmax, st);
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default: return fail(VCT_E_ARG, "adjoint: 1..8 materials");
  }
}

// ------------------------------------------- exact-walk rays: line integrals
// One warp per listed ray (exact_lines_warp).
template <int M>
__device__ __forceinline__ void adj_lines_ray(const DevGeom& g, const PixelRec* __restrict__ maps,
                                              const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                                              const double* __restrict__ det_px0, const double* __restrict__ det_py0,
                                              int ray, double* __restrict__ out, int lane) {
  double L[8];
  int nseg;
  exact_lines_warp<M>(g, maps, cos_t, sin_t, det_px0, det_py0, ray, L, &nseg, lane);
  if (lane == 0) {
#pragma unroll
    for (int m = 0; m < M; m++) out[m] = L[m];
  }
}

template <int M>
__global__ void adj_lines_kernel(DevGeom g, const PixelRec* __restrict__ maps, const double* __restrict__ cos_t,
                                 const double* __restrict__ sin_t, const double* __restrict__ det_px0,
                                 const double* __restrict__ det_py0, const int* __restrict__ special, int n,
                                 double* __restrict__ lsp) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= n) return;  // warp-uniform
  adj_lines_ray<M>(g, maps, cos_t, sin_t, det_px0, det_py0, special[i], lsp + (size_t)i * M, threadIdx.x & 31);
}

int launch_adj_lines(const DevGeom& g, int M, const PixelRec* d_maps, const double* d_cos, const double* d_sin,
                     const double* d_px0, const double* d_py0, const int* d_special, int nspecial_host, double* d_lsp,
                     cudaStream_t st) {
  if (nspecial_host <= 0) return VCT_OK;
  const int blocks = (nspecial_host + 3) / 4;  // 4 warps of 32, one ray each
  switch (M) {
#define VCT_CASE(mm)                                                                                         \
  case mm:                                                                                                   \
    adj_lines_kernel<mm><<<blocks, 128, 0, st>>>(g, d_maps, d_cos, d_sin, d_px0, d_py0, d_special, nspecial_host, \
                                                 d_lsp);                                                     \
    break;
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default: return fail(VCT_E_ARG, "adjoint: 1..8 materials");
  }
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// Fixed-order sum of the per-block loss partials.
__global__ void adj_loss_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double s[256];
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) t += part[i];
  s[threadIdx.x] = t;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

int launch_adj_loss(const double* d_part, int n, double* d_out, cudaStream_t st) {
  adj_loss_kernel<<<1, 256, 0, st>>>(d_part, n, d_out);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------- exact-walk rays: fixed point
template <int M>
struct ScatterSink {
  const float* gr;
  double scale;
  unsigned long long* acc;
  int N;
  VCT_HD void operator()(int pix, double rr) const {
#if defined(__CUDA_ARCH__)
    const int P = N + 2 * kPad;
    const int col = pix % P - kPad, row = pix / P - kPad;
    const size_t idx = (size_t)row * N + col;
    const size_t n2 = (size_t)N * N;
#pragma unroll
    for (int m = 0; m < M; m++) {
      const long long q = __double2ll_rn((double)gr[m] * rr * scale);
      if (q) atomicAdd(acc + m * n2 + idx, (unsigned long long)q);
    }
#endif
  }
};

template <int M>
__global__ void adj_special_kernel(DevGeom g, const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                                   const double* __restrict__ det_px0, const double* __restrict__ det_py0,
                                   const int* __restrict__ special, const int* __restrict__ nspecial,
                                   const float* __restrict__ gr, const unsigned int* __restrict__ gmax,
                                   double lmax, int log2_terms, unsigned long long* __restrict__ acc) {
  // one warp per ray (the walk's steps across the lanes)
  const int n = *nspecial;
  const double scale = special_scale(*gmax, lmax, log2_terms);
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nw) {
    const int ray = special[i];
    const int v = ray / g.C, c = ray - (ray / g.C) * g.C;
    Ray r;
    if (!ray_setup(g, cos_t[v], sin_t[v], det_px0[c], det_py0[c], r)) continue;
    walk_exact_warp(g, r, ScatterSink<M>{gr + (size_t)ray * M, scale, acc, g.N}, lane);
  }
}

int launch_adj_special(const DevGeom& g, int M, const double* d_cos, const double* d_sin, const double* d_px0,
                       const double* d_py0, const int* d_special, const int* d_nspecial, int nspecial_host,
                       const float* d_g, const unsigned int* d_gmax, double lmax, int log2_terms,
                       unsigned long long* d_acc, cudaStream_t st) {
  if (nspecial_host <= 0) return VCT_OK;
  const int blocks = (nspecial_host + 3) / 4;  // 4 warps of 32, one ray each
  switch (M) {
#define VCT_CASE(mm)                                                                                        \
  case mm:                                                                                                  \
    adj_special_kernel<mm><<<blocks, 128, 0, st>>>(g, d_cos, d_sin, d_px0, d_py0, d_special, d_nspecial, d_g, \
                                                   d_gmax, lmax, log2_terms, d_acc);                        \
    break;
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default: return fail(VCT_E_ARG, "adjoint: 1..8 materials");
  }
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// Largest |g| over the exact-walk rays, for caller-given ray weights.
__global__ void adj_gmax_kernel(int M, const int* __restrict__ special, const int* __restrict__ nspecial,
                                const float* __restrict__ gr, unsigned int* __restrict__ gmax) {
  const int n = *nspecial;
  float gm = 0.0f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int m = 0; m < M; m++) gm = fmaxf(gm, fabsf(gr[(size_t)special[i] * M + m]));
  if (gm > 0.0f) atomicMax(gmax, __float_as_uint(gm));
}

int launch_adj_gmax(int M, const int* d_special, const int* d_nspecial, int nspecial_host, const float* d_g,
                    unsigned int* d_gmax, cudaStream_t st) {
  if (nspecial_host <= 0) return VCT_OK;
  adj_gmax_kernel<<<(nspecial_host + 255) / 256, 256, 0, st>>>(M, d_special, d_nspecial, d_g, d_gmax);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------------------ pixel-driven gather
// Staged rays per view (the channel window of one tile; the host picks the
// tile so the window fits).
constexpr int kAdjW = 64;

// Per (tile, view), computed once per context from the geometry and the walk
// plans (adj_tiles_kernel):
//   a = (J0, Jx, Jy, Jxx), b = (Jxy, Jyy, dj, bits of kmax | jn << 8 |
//   cplx << 16), c = (kmax, jlo, jn, cplx).
// The channel coordinate of a cell centre at offset (lx, ly) from the tile
// centre is modelled as jc = J0 + Jx lx + Jy ly + Jxx lx^2 + Jxy lx ly +
// Jyy ly^2 (second-order Taylor expansion of the fan angle at the tile
// centre, FP64, channels counted from jlo), and dj bounds a cell's angular
// half-width in channels with the expansion's third-order remainder as
// margin: every ray whose chord through the cell can be positive lies among
// the integers in (jc - dj, jc + dj), at most kmax = floor(2 dj) + 1 of
// them, inside the window of jn channels from jlo.  cplx = 1 when some ray of the window
// ends its walk or lumps inside the tile (else every cell takes the plain
// chord path for the view).
struct AdjTileView {
  float4 a, b;
  int4 c;
};

template <int TX, int TY>
__global__ void adj_tiles_kernel(AdjGeom a, const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                                 const int4* __restrict__ rec, AdjTileView* __restrict__ out,
                                 int* __restrict__ status) {
  const int NE1 = a.N + 1;
  const int nbx = (NE1 + TX - 1) / TX, nby = (NE1 + TY - 1) / TY;
  const int V = a.views_used;
  const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // one warp per (tile, view)
  const int lane = threadIdx.x & 31;
  if (item >= (long long)nbx * nby * V) return;
  const int tile = (int)(item / V), v = (int)(item - (long long)tile * V);
  const int e0 = (tile % nbx) * TX, f0 = (tile / nbx) * TY;
  const double s = a.s, h = 0.5 * s;
  const double Tx = (e0 - 1 + 0.5 * TX - a.nxm) * s;
  const double Ty = (a.nxm - (f0 - 1) - 0.5 * TY) * s;
  const double Lx = 0.5 * (TX - 1) * s, Ly = 0.5 * (TY - 1) * s;
  const double lmax = sqrt(Lx * Lx + Ly * Ly);
  int jlo = 0, jn = 0;
  AdjTileView o;
  if (lane == 0) {
    const double cb = cos_t[v], sb = sin_t[v];
    const double qx = Tx - a.sid * sb, qy = Ty - a.sid * cb;
    const double U = qx * cb - qy * sb, W = -(qx * sb + qy * cb);  // W > 0: the grid is below the source
    const double r2 = U * U + W * W, r4 = r2 * r2;
    const double phi = atan2(U, W);
    const double pU = W / r2, pW = -U / r2;
    const double pUU = -2.0 * U * W / r4, pWW = 2.0 * U * W / r4, pUW = (U * U - W * W) / r4;
    // dU/dx = cb, dU/dy = -sb, dW/dx = -sb, dW/dy = -cb
    const double px = pU * cb - pW * sb, py = -pU * sb - pW * cb;
    const double pxx = pUU * cb * cb - 2.0 * pUW * cb * sb + pWW * sb * sb;
    const double pyy = pUU * sb * sb + 2.0 * pUW * sb * cb + pWW * cb * cb;
    const double pxy = -pUU * cb * sb + pUW * (sb * sb - cb * cb) + pWW * sb * cb;
    const double ida = a.inv_dalpha;
    const double D = sqrt(r2), Dmin = D - lmax - h * 1.4142135623730951;
    // third-order remainder of the expansion (its bound doubled) plus rounding
    const double rem = 2.0 * (lmax / Dmin) * (lmax / Dmin) * (lmax / Dmin) * ida + 0.02;
    // A ray through the tile leaves the source within delta of the direction
    // to the tile centre, so h(|dx| + |dy|), the half-width of a cell across
    // the ray, is at most h(|qx| + |qy|)/D + h sqrt(2) delta.
    const double delta = asin(fmin(1.0, (lmax + h * 1.4142135623730951) / D));
    const double hw = h * fmin(1.4142135623730951, (fabs(qx) + fabs(qy)) / D + 1.4142135623730951 * delta);
    const double dj = asin(fmin(1.0, hw / Dmin)) * ida + rem;
    const double jcT = a.iso - phi * ida - a.start;  // 0-based channel at the tile centre
    const double Jx = -px * ida, Jy = -py * ida, Jxx = -0.5 * pxx * ida, Jxy = -pxy * ida, Jyy = -0.5 * pyy * ida;
    const double span = fabs(Jx) * Lx + fabs(Jy) * Ly + fabs(Jxx) * Lx * Lx + fabs(Jxy) * Lx * Ly +
                        fabs(Jyy) * Ly * Ly + dj + 1.0;
    int lo = (int)floor(jcT - span), hi = (int)ceil(jcT + span);
    lo = max(lo, 0);
    hi = min(hi, a.C - 1);
    jlo = lo;
    jn = max(hi - lo + 1, 0);
    if (jn > kAdjW) {
      jn = kAdjW;
      atomicOr(status, 1);
    }
    o.a = make_float4((float)(jcT - lo), (float)Jx, (float)Jy, (float)Jxx);
    o.b = make_float4((float)Jxy, (float)Jyy, (float)dj, 0.0f);
    o.c = make_int4(jn > 0 ? min((int)floor(2.0 * dj) + 1, 255) : 0, jlo, jn, 0);
  }
  jlo = __shfl_sync(0xffffffffu, jlo, 0);
  jn = __shfl_sync(0xffffffffu, jn, 0);
  int cplx = 0;
  for (int j = lane; j < jn; j += 32) {
    const int4 r = rec[(long long)v * a.C + jlo + j];
    if ((r.x & 3) != kAdjRayFast) continue;
    const int lo = (r.y & 0xffff) - 1, hi = (r.y >> 16) - 1;
    const int c0 = (r.x >> 2) ? e0 - 1 : f0 - 1;  // the tile's first cell on the ray's major axis
    const int c1 = c0 + ((r.x >> 2) ? TX : TY) - 1;
    bool cx = c0 < lo || c1 > hi;
    if (r.z >= 0) {
      const int lc = r.z & 0xffff, lr = r.z >> 16;
      cx = cx || (lc >= e0 - 1 && lc <= e0 + TX - 2 && lr >= f0 - 1 && lr <= f0 + TY - 2);
    }
    cplx |= cx;
  }
  cplx = __any_sync(0xffffffffu, cplx);
  if (lane == 0) {
    o.c.w = cplx;
    // what the gather's cell loop reads, in b.w: kmax | jn << 8 | cplx << 16
    o.b.w = __int_as_float(o.c.x | (o.c.z << 8) | (cplx << 16));
    out[item] = o;
  }
}

// Staged rays of one round in shared memory, ST slots.  Per slot, for a ray
// of direction (dx, dy) and offset bt of its line from the tile centre, with
// a = max(|dx|, |dy|), c = min(...) (each at least 1e-12) and h half a pixel:
//   q[0]  = (sign(dx)/|dy|, sign(dy)/|dx|, bt/(h |dx| |dy|), g0)
//   q[1]  = (g1, g2, g3, g4)                     (5 to 8 elements)
//   t     = the remaining 1-3 factors (float, float2 or float4)
//   x     = (xmaj, major-index range, lumped pixel, lumped length / h)
// A cell at offset (lx, ly) = h (lx', ly') from the tile centre then has
// b = q0.x ly' - q0.y lx' + q0.z = (offset of the line from the cell centre)
// / (h a c), and its chord in units of h is min(2/a, (a+c)/(a c) - |b|)
// clipped at 0, with 1/a = min(|q0.x|, |q0.y|) and (a+c)/(a c) = |q0.x| +
// |q0.y|: three floats of geometry per ray.  A ray the fast walk does not
// take has q0.z = +inf (no chord) and no lumped pixel.
template <int M, int ST>
struct AdjStage {
  static constexpr int NQ4 = 1 + (M - 1) / 4;
  static constexpr int R = (M - 1) % 4;
  static constexpr int TW = R == 0 ? 0 : (R == 1 ? 1 : (R == 2 ? 2 : 4));  // tail floats per slot
  static constexpr int MT = 1 + 4 * (NQ4 - 1);                           // first factor in the tail
  float4 q[NQ4][ST];
  alignas(16) float t[TW > 0 ? TW * ST : 4];
  int4 x[ST];
  float4 v[ST / kAdjW][2];  // a, b of each staged view's AdjTileView
};

// K candidate rays k0.. of one view for one cell, unrolled; candidate i
// counts when 0 <= j0 + i < jlim.  Chords in units of h (above), and with
// cplx the walk's major-index range and lumped piece.
template <int M, int K, int ST>
__device__ __forceinline__ void adj_cells(const AdjStage<M, ST>& S, int cplx, int k0, int j0, int jlim, float lxh,
                                          float lyh, int colx, int rowx, int pix, float* acc) {
  using St = AdjStage<M, ST>;
#pragma unroll
  for (int i = 0; i < K; i++) {
    if ((unsigned)(j0 + i) < (unsigned)jlim) {
      const int k = k0 + i;
      if (!VCT_INDEX_OK(k >= 0 && k < ST)) continue;
      const float4 q0 = S.q[0][k];
      const float b = fmaf(q0.x, lyh, fmaf(-q0.y, lxh, q0.z));
      // min(2/a, 1/a + 1/c - |b|) = 1/a + 1/c - max(1/c - 1/a, |b|)
      const float ax = fabsf(q0.x), ay = fabsf(q0.y);
      float len = fmaxf((ax + ay) - fmaxf(fabsf(ax - ay), fabsf(b)), 0.0f);
      if (cplx) {
        const int4 x = S.x[k];
        const int mi = x.x ? colx : rowx;
        if (mi < (x.y & 0xffff) || mi > (x.y >> 16)) len = 0.0f;
        if (x.z == pix) len += __int_as_float(x.w);
      }
#define VCT_ACC(m, val) \
  if ((m) < M) acc[(m) % M] = fmaf(len, (val), acc[(m) % M])
      VCT_ACC(0, q0.w);
      if (St::NQ4 > 1) {
        const float4 q1 = S.q[St::NQ4 - 1][k];
        VCT_ACC(1, q1.x);
        VCT_ACC(2, q1.y);
        VCT_ACC(3, q1.z);
        VCT_ACC(4, q1.w);
      }
      if (St::TW == 1) {
        VCT_ACC(St::MT, S.t[k]);
      } else if (St::TW == 2) {
        const float2 t = reinterpret_cast<const float2*>(S.t)[k];
        VCT_ACC(St::MT, t.x);
        VCT_ACC(St::MT + 1, t.y);
      } else if (St::TW == 4) {
        const float4 t = reinterpret_cast<const float4*>(S.t)[k];
        VCT_ACC(St::MT, t.x);
        VCT_ACC(St::MT + 1, t.y);
        VCT_ACC(St::MT + 2, t.z);
      }
#undef VCT_ACC
    }
  }
}

// The gather runs over the (N+1) x (N+1) cells with indices -1..N-1: cells
// at index -1 lie outside the grid, but the walk's truncating cast puts their
// pieces on index 0 (adj_fold_kernel adds them there).  One thread per cell
// of a TX x TY tile; blocks loop over the tiles.  Per round every warp stages
// one view's rays of the tile's channel window (from its AdjTileView) into an
// AdjStage slot row.  The chord of a line at offset b from the centre of a
// square of half-size h, direction with components a >= c: 2h/a while
// |b| <= h(a-c), then (h(a+c) - |b|)/(a c) down to 0.
// Resident blocks per SM the registers are held to (4 for the 256-thread
// tiles, in proportion for smaller ones: 64 registers; for 8 elements at
// 1024^2, 1440 x 1600 the gather 10.80 -> 10.61 ms against the compiler's 80
// registers, 3 blocks 11.41 ms; 7 elements then also lose the spills the
// compiler's own choice had), and how far the loop over a round's views is unrolled
// (measured on the 512^2, 800 x 609 gradient: 3 blocks per SM 1.27 ms and
// unrolling by 2 1.15 ms, against 1.14 ms at 4; later, 5 blocks per SM (48
// registers, small spills) 1.16 ms against 1.02 ms).
#ifndef VCT_ADJ_MINBLOCKS
#define VCT_ADJ_MINBLOCKS 4
#endif
#ifndef VCT_ADJ_CAP_MAXM
#define VCT_ADJ_CAP_MAXM 8
#endif
constexpr int adj_min_blocks(int M, int threads) {
  return M <= VCT_ADJ_CAP_MAXM ? VCT_ADJ_MINBLOCKS * 256 / threads : 0;
}
// The batch's gather (its job lookup costs registers) is left to the compiler
// (held to 64 registers at 7-8 elements it spills 72-88 bytes: the 8-slice
// 1024^2 dual-energy descent 285 -> 307 ms per iteration).
#ifndef VCT_ADJ_BATCH_MINBLOCKS
#define VCT_ADJ_BATCH_MINBLOCKS 0
#endif
#ifndef VCT_ADJ_BATCH_CAP_MINM
#define VCT_ADJ_BATCH_CAP_MINM 9
#endif
constexpr int adj_batch_min_blocks(int M, int threads) {
  return M >= VCT_ADJ_BATCH_CAP_MINM ? VCT_ADJ_MINBLOCKS * 256 / threads : VCT_ADJ_BATCH_MINBLOCKS;
}
// The loop over a round's views unrolled by 2: 0.989 -> 0.969 ms at 512^2 /
// 800 x 609 (gradient bit-identical; 1024^2, 8 elements and the 64-slice
// batch unchanged within 0.6%).
#ifndef VCT_ADJ_VUNROLL
#define VCT_ADJ_VUNROLL 2
#endif
#ifndef VCT_ADJ_LANEMAP
#define VCT_ADJ_LANEMAP 1
#endif
// One tile of the gather (all views), by a block of TX * TY threads; shared
// staging space from the caller.
// NCH: the number of view ranges the tile's views are split into (chunk is
// this item's); partial sums go to slot `chunk` of ext.
template <int M, int TX, int TY, int NCH>
__device__ __forceinline__ void adj_gather_tile(const AdjGeom& a, int tile, int chunk, const double* __restrict__ cos_t,
                                                const double* __restrict__ sin_t, const double2* __restrict__ dir,
                                                const int4* __restrict__ rec, const float* __restrict__ gr,
                                                const AdjTileView* __restrict__ tv, float* __restrict__ ext,
                                                AdjStage<M, TX * TY / 32 * kAdjW>& S) {
  constexpr int NW = TX * TY / 32, VB = NW;  // views per round: one per warp
  constexpr int ST = VB * kAdjW;
  using St = AdjStage<M, ST>;
  constexpr int kVUnroll = VCT_ADJ_VUNROLL;
  const int N = a.N, NE1 = N + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // Each warp covers a patch of PX x (32/PX) cells, as square as the tile
  // allows: the rays its lanes read then span the fewest channels, so its
  // shared-memory loads touch the fewest distinct lines.
  constexpr int PX = TX >= 8 ? 8 : TX, PY = 32 / PX, WPR = TX / PX;  // warps per tile row of patches
  static_assert(TX % PX == 0 && TY % PY == 0, "the tile must split into whole warp patches");
#if VCT_ADJ_LANEMAP
  // Within the 8 x 4 patch, each quarter of the warp (8 lanes, one phase of
  // a 16-byte shared load) covers a 4 x 2 block of cells rather than a row
  // of 8, so its candidate rays span fewer channels.
  static_assert(PX == 8, "the quarter-warp blocks assume 8 x 4 patches");
  const int px_ = (lane & 3) | (((lane >> 3) & 1) << 2), py_ = ((lane >> 2) & 1) | ((lane >> 4) << 1);
  const int tx = (warp % WPR) * PX + px_, ty = (warp / WPR) * PY + py_;
#else
  const int tx = (warp % WPR) * PX + lane % PX, ty = (warp / WPR) * PY + lane / PX;
#endif
  const double s = a.s, hd = 0.5 * s;
  const float ihf = (float)(1.0 / hd);
  // Cell-centre offsets from the tile centre, and the quadratic's terms.
  const float lx = (float)((tx + 0.5 - 0.5 * TX) * s);
  const float ly = (float)((0.5 * TY - ty - 0.5) * s);
  const float lxx = lx * lx, lxy = lx * ly, lyy = ly * ly;
  const float lxh = (float)(2 * tx + 1 - TX), lyh = (float)(TY - 2 * ty - 1);  // (lx, ly) / h
  const int nbx = (NE1 + TX - 1) / TX;
  const int V = a.views_used;
  const int e0 = (tile % nbx) * TX, f0 = (tile / nbx) * TY;  // first extended column / row
  const int col = e0 + tx - 1, row = f0 + ty - 1;              // cell indices, -1..N-1
  // Tile centre (world cm; x right, y up; row r spans y in ((n-r-1)s, (n-r)s]).
  const double Tx = (e0 - 1 + 0.5 * TX - a.nxm) * s;
  const double Ty = (a.nxm - (f0 - 1) - 0.5 * TY) * s;
  const int pix = (col >= 0 && row >= 0) ? (col | (row << 16)) : -2;  // -2: never a lumped pixel
  const int colx = col + 1, rowx = row + 1;
  const AdjTileView* __restrict__ tvt = tv + (size_t)tile * V;
  // this item's views [vb, ve)
  const int vb = NCH == 1 ? 0 : (int)((long long)V * chunk / NCH);
  const int ve = NCH == 1 ? V : (int)((long long)V * (chunk + 1) / NCH);

  double dacc[M];
#pragma unroll
  for (int m = 0; m < M; m++) dacc[m] = 0.0;

  for (int v0 = vb; v0 < ve; v0 += VB) {
    // ---- staging: warp `warp` takes view v0 + warp
    {
      const int vs = warp;  // slot
      const int v = v0 + vs;
      int4 vc = make_int4(0, 0, 0, 0);
      if (v < ve) {
        vc = tvt[v].c;
        if (lane < 2) S.v[vs][lane] = lane ? tvt[v].b : tvt[v].a;
      } else if (lane == 1) {
        S.v[vs][1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // kmax 0: nothing to gather
      }
      const int jlo = vc.y, jn = vc.z;
      const double cb = v < ve ? cos_t[v] : 0.0, sb = v < ve ? sin_t[v] : 0.0;
      const double Sx = a.sid * sb, Sy = a.sid * cb;
      for (int j = lane; j < jn; j += 32) {
        const int c = jlo + j;
        const int k = vs * kAdjW + j;
        const long long ray = (long long)v * a.C + c;
        if (!VCT_INDEX_OK(v < a.views_used && c >= 0 && c < a.C && j < kAdjW)) continue;
        const double2 e = dir[c];
        const double dx = e.x * cb + e.y * sb, dy = -e.x * sb + e.y * cb;
        const double bt = dx * (Ty - Sy) - dy * (Tx - Sx);
        const float rx = __frcp_rn(fmaxf(fabsf((float)dx), 1e-12f)), ry = __frcp_rn(fmaxf(fabsf((float)dy), 1e-12f));
        const int4 r = rec[ray];
        const bool fast = (r.x & 3) == kAdjRayFast;
        const float* gp = gr + ray * M;
        float g[8];
#pragma unroll
        for (int m = 0; m < 8; m++) g[m] = m < M ? gp[m] : 0.0f;
        S.q[0][k] = make_float4(copysignf(ry, (float)dx), copysignf(rx, (float)dy),
                                fast ? (float)bt * ihf * rx * ry : INFINITY, g[0]);
        if (St::NQ4 > 1) S.q[St::NQ4 - 1][k] = make_float4(g[1], g[2], g[3], g[4]);
        if (St::TW == 1) S.t[k] = g[St::MT];
        if (St::TW == 2) reinterpret_cast<float2*>(S.t)[k] = make_float2(g[St::MT], g[(St::MT + 1) & 7]);
        if (St::TW == 4)
          reinterpret_cast<float4*>(S.t)[k] = make_float4(g[St::MT], g[(St::MT + 1) & 7], g[(St::MT + 2) & 7], 0.0f);
        S.x[k] = make_int4(r.x >> 2, r.y, fast ? r.z : -1,
                           fast ? __float_as_int(__int_as_float(r.w) * ihf) : 0);
      }
    }
    __syncthreads();

    // ---- gather: every cell over the round's views
    float acc[M];
#pragma unroll
    for (int m = 0; m < M; m++) acc[m] = 0.0f;
#pragma unroll kVUnroll
    for (int vb = 0; vb < VB; vb++) {
      const float4 fb = S.v[vb][1];
      const int bits = __float_as_int(fb.w);
      const int4 vi = make_int4(bits & 0xff, 0, (bits >> 8) & 0xff, bits >> 16);  // kmax, -, jn, cplx
      if (vi.x == 0) continue;
      const float4 fa = S.v[vb][0];
      const float jc = fmaf(fb.y, lyy, fmaf(fb.x, lxy, fmaf(fa.w, lxx, fmaf(fa.z, ly, fmaf(fa.y, lx, fa.x)))));
      // this cell's candidates: the integers in (jc - dj, jc + dj) that lie
      // in the window, j0 <= j < jlim; at most kmax of them
      const int j0 = (int)floorf(jc - fb.z) + 1;
      const int jlim = max(min((int)ceilf(jc + fb.z), vi.z), 0);  // >= 0: the test below is unsigned
      const int k0 = vb * kAdjW + j0;
      switch (vi.x) {  // block-uniform
        case 1: adj_cells<M, 1, ST>(S, vi.w, k0, j0, jlim, lxh, lyh, colx, rowx, pix, acc); break;
        case 2: adj_cells<M, 2, ST>(S, vi.w, k0, j0, jlim, lxh, lyh, colx, rowx, pix, acc); break;
        case 3: adj_cells<M, 3, ST>(S, vi.w, k0, j0, jlim, lxh, lyh, colx, rowx, pix, acc); break;
        default:
          for (int i = 0; i < vi.x; i += 4)
            adj_cells<M, 4, ST>(S, vi.w, k0 + i, j0 + i, jlim, lxh, lyh, colx, rowx, pix, acc);
          break;
      }
    }
#pragma unroll
    for (int m = 0; m < M; m++) dacc[m] += (double)acc[m];
    __syncthreads();
  }
  if (col < N && row < N) {
    const size_t n2 = (size_t)NE1 * NE1;
    const size_t o = (NCH == 1 ? 0 : (size_t)chunk * M * n2) + (size_t)(row + 1) * NE1 + (col + 1);
#pragma unroll
    for (int m = 0; m < M; m++) ext[m * n2 + o] = (float)(dacc[m] * hd);  // chords were in units of h
  }
}

template <int M, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, adj_min_blocks(M, TX * TY))
adj_gather_kernel(AdjGeom a, const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                  const double2* __restrict__ dir, const int4* __restrict__ rec, const float* __restrict__ gr,
                  const AdjTileView* __restrict__ tv, float* __restrict__ ext) {
  __shared__ AdjStage<M, TX * TY / 32 * kAdjW> S;
  const int NE1 = a.N + 1;
  const int ntiles = ((NE1 + TX - 1) / TX) * ((NE1 + TY - 1) / TY);
  for (int item = blockIdx.x; item < ntiles * adj_chunks(M); item += gridDim.x)
    adj_gather_tile<M, TX, TY, adj_chunks(M)>(a, item % ntiles, item / ntiles, cos_t, sin_t, dir, rec, gr, tv, ext, S);
}

// grad[m][r][c] = ext at (r, c), plus the folded cells at index -1 (row -1
// onto row 0, column -1 onto column 0), summed over the view chunks, plus
// the exact-walk rays' fixed-point sums; fixed order, so the result is
// deterministic.
__device__ __forceinline__ void adj_fold_elem(long long i, int M, int N, const float* __restrict__ ext,
                                              const unsigned long long* __restrict__ sacc,
                                              const unsigned int* __restrict__ gmax, double lmax, int log2_terms,
                                              float* __restrict__ grad) {
  const size_t n2 = (size_t)N * N, e2 = (size_t)(N + 1) * (N + 1);
  if (i >= (long long)M * n2) return;
  const int m = (int)(i / n2);
  const int p = (int)(i - (long long)m * n2);
  const int r = p / N, c = p - (p / N) * N;
  const int N1 = N + 1;
  double v = 0.0;
  for (int k = 0; k < adj_chunks(M); k++) {
    const float* e = ext + ((size_t)k * M + m) * e2;
    v += e[(r + 1) * N1 + (c + 1)];
    if (c == 0) v += e[(r + 1) * N1];
    if (r == 0) v += e[c + 1];
    if (r == 0 && c == 0) v += e[0];
  }
  if (sacc) v += (double)(long long)sacc[i] / special_scale(*gmax, lmax, log2_terms);
  grad[i] = (float)v;
}

__global__ void adj_fold_kernel(int M, int N, const float* __restrict__ ext, const unsigned long long* __restrict__ sacc,
                                const unsigned int* __restrict__ gmax, double lmax, int log2_terms,
                                float* __restrict__ grad) {
  adj_fold_elem((long long)blockIdx.x * blockDim.x + threadIdx.x, M, N, ext, sacc, gmax, lmax, log2_terms, grad);
}

// Tile shapes, largest first; the channel window of a tile grows with its
// size and shrinks with the source distance.
static const int kTiles[][2] = {{16, 16}, {16, 8}, {8, 8}, {8, 4}};

int adj_pick_tile(const AdjGeom& a, double lim) {
  // Nearest approach of a tile's cells to the source, and its half-diagonal.
  const double dmin = a.sid - (lim + 2.0 * a.s) * sqrt(2.0);
  if (!(dmin > 0)) return -1;
  for (int t = 0; t < 4; t++) {
    const double hd = 0.5 * sqrt((double)(kTiles[t][0] + 2) * (kTiles[t][0] + 2) +
                                 (double)(kTiles[t][1] + 2) * (kTiles[t][1] + 2)) * a.s;
    if (hd >= dmin) continue;
    // the tile's angular extent, twice the widest cell half-width, and the
    // window's margins (the kernel's span adds one channel each side)
    const double ang = 2.0 * asin(hd / dmin);
    const double dj = asin(fmin(1.0, 0.5 * a.s * sqrt(2.0) / (dmin - hd))) * a.inv_dalpha + 0.1;
    const double jn = ang * a.inv_dalpha + 2.0 * dj + 5.0;
    if (jn <= kAdjW) return t;
  }
  return -1;
}

// Tiles of the gather for tile shape t (adj_pick_tile).
static int tiles_of(const AdjGeom& a, int t) {
  return ((a.N + 1 + kTiles[t][0] - 1) / kTiles[t][0]) * ((a.N + 1 + kTiles[t][1] - 1) / kTiles[t][1]);
}

size_t adj_tileview_bytes(const AdjGeom& a, int tile) {
  if (tile < 0 || tile > 3) return 0;
  return (size_t)tiles_of(a, tile) * a.views_used * sizeof(AdjTileView);
}

int launch_adj_tiles(const AdjGeom& a, int tile, const double* d_cos, const double* d_sin, const int4* d_rec,
                     void* d_tv, int* d_status, cudaStream_t st) {
  if (tile < 0 || tile > 3) return fail(VCT_E_UNSUPPORTED, "adjoint: no tile fits the channel window");
  const long long items = (long long)tiles_of(a, tile) * a.views_used;
  if (items == 0) return VCT_OK;
  const unsigned blocks = (unsigned)((items * 32 + 127) / 128);
  AdjTileView* tv = reinterpret_cast<AdjTileView*>(d_tv);
  switch (tile) {
    case 0: adj_tiles_kernel<16, 16><<<blocks, 128, 0, st>>>(a, d_cos, d_sin, d_rec, tv, d_status); break;
    case 1: adj_tiles_kernel<16, 8><<<blocks, 128, 0, st>>>(a, d_cos, d_sin, d_rec, tv, d_status); break;
    case 2: adj_tiles_kernel<8, 8><<<blocks, 128, 0, st>>>(a, d_cos, d_sin, d_rec, tv, d_status); break;
    default: adj_tiles_kernel<8, 4><<<blocks, 128, 0, st>>>(a, d_cos, d_sin, d_rec, tv, d_status); break;
  }
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

template <int M, int TX, int TY>
static int launch_adj_gather_t(const AdjGeom& a, const double* d_cos, const double* d_sin, const double2* d_dir,
                               const int4* d_rec, const float* d_g, const AdjTileView* d_tv, float* d_ext,
                               cudaStream_t st) {
  const int ntiles = ((a.N + 1 + TX - 1) / TX) * ((a.N + 1 + TY - 1) / TY);
  int dev = 0, sms = 0, per_sm = 0;
  VCT_CUDA(cudaGetDevice(&dev));
  VCT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  VCT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adj_gather_kernel<M, TX, TY>, TX * TY, 0));
  const int grid = min(ntiles, max(1, per_sm) * sms);
  adj_gather_kernel<M, TX, TY><<<grid, TX * TY, 0, st>>>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_tv, d_ext);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

template <int M>
static int launch_adj_gather_m(const AdjGeom& a, int tile, const double* d_cos, const double* d_sin,
                               const double2* d_dir, const int4* d_rec, const float* d_g, const AdjTileView* d_tv,
                               float* d_ext, cudaStream_t st) {
  switch (tile) {
    case 0: return launch_adj_gather_t<M, 16, 16>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_tv, d_ext, st);
    case 1: return launch_adj_gather_t<M, 16, 8>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_tv, d_ext, st);
    case 2: return launch_adj_gather_t<M, 8, 8>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_tv, d_ext, st);
    default: return launch_adj_gather_t<M, 8, 4>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_tv, d_ext, st);
  }
}

int launch_adj_gather(const AdjGeom& a, int M, int tile, const double* d_cos, const double* d_sin,
                      const double2* d_dir, const int4* d_rec, const float* d_g, const void* d_tv, float* d_ext,
                      cudaStream_t st) {
  if (tile < 0 || tile > 3) return fail(VCT_E_UNSUPPORTED, "adjoint: no tile fits the channel window");
  const AdjTileView* tv = reinterpret_cast<const AdjTileView*>(d_tv);
  switch (M) {
#define VCT_CASE(mm) \
  case mm: return launch_adj_gather_m<mm>(a, tile, d_cos, d_sin, d_dir, d_rec, d_g, tv, d_ext, st);
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default: return fail(VCT_E_ARG, "adjoint: 1..8 materials");
  }
}

int launch_adj_fold(const AdjGeom& a, int M, const unsigned long long* d_sacc, const unsigned int* d_gmax,
                    const float* d_ext, float* d_grad, cudaStream_t st) {
  const long long n = (long long)M * a.N * a.N;
  adj_fold_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(M, a.N, d_ext, d_sacc, d_gmax, a.lmax, a.log2_terms,
                                                                d_grad);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// ------------------------------------------------------------------ batch
// The batched stages of many slices' loss and gradient (vct_batch.cpp).
__device__ __forceinline__ int adj_job_of(const unsigned int* __restrict__ first, int n, unsigned int b) {
  int lo = 0, hi = n - 1;  // the last job whose first block is <= b
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__host__ __device__ unsigned int adj_job_ray_tiles(const DevGeom& g) {
  const long long nrays = (long long)g.views_used * g.C;
  return (unsigned int)((nrays + kAdjFwdThreads - 1) / kAdjFwdThreads);
}

void adj_job_blocks(const AdjJob& j, int M, int tile, unsigned int blocks[kAdjStages]) {
  const long long n2 = (long long)j.a.N * j.a.N;
  blocks[kAdjStReset] = j.sacc ? (unsigned int)((M * n2 + 255) / 256) : 1u;
  blocks[kAdjStLines] = (unsigned int)((j.nspecial + 3) / 4);  // 128 threads, a warp per ray
  blocks[kAdjStLoss] = 1u;
  blocks[kAdjStSpecial] = (unsigned int)((j.nspecial + 3) / 4);  // 128 threads, a warp per ray
  for (int t = 0; t < 4; t++)
    blocks[kAdjStGather + t] = t == tile ? (unsigned int)(tiles_of(j.a, tile) * adj_chunks(M)) : 0u;
  blocks[kAdjStFold] = (unsigned int)((M * n2 + 255) / 256);
}

// gmax and the exact-walk accumulators of every job back to zero.
__global__ void adj_reset_batch_kernel(const AdjJob* __restrict__ jobs, const unsigned int* __restrict__ first, int n,
                                       int M) {
  const int jx = adj_job_of(first, n, blockIdx.x);
  const AdjJob& J = jobs[jx];
  const unsigned int b = blockIdx.x - first[jx];
  if (b == 0 && threadIdx.x == 0) *J.gmax = 0u;
  if (!J.sacc) return;
  const long long i = (long long)b * blockDim.x + threadIdx.x;
  if (i < (long long)M * J.a.N * J.a.N) J.sacc[i] = 0ull;
}

// The persistent adjoint forward: every warp takes 128-ray tiles (the plain
// kernel's blocks) in job order from a counter and walks them in four
// chunks of 32 rays (the plain kernel's warps), reducing each chunk's loss
// as the plain kernel does and summing the chunks in warp order: the tile's
// loss partial equals the plain block's.
constexpr int kAdjBatchWarps = kAdjFwdThreads / 32;

template <int M>
__global__ void __launch_bounds__(kAdjFwdThreads)
adj_forward_batch_kernel(const AdjJob* __restrict__ jobs, int njobs, unsigned int ntiles, int ne_max,
                         unsigned int* __restrict__ counter) {
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slot = (size_t)ne_max * M + (size_t)(ne_max + 1) / 2;
  double* s_mu = smem + (size_t)warp * slot;                           // [ne_max][M]
  float* s_pdf = reinterpret_cast<float*>(s_mu + (size_t)ne_max * M);  // [ne_max]
  int cur = -1;
  for (;;) {
    unsigned int t = 0;
    int j = 0;
    if (lane == 0) {
      t = atomicAdd(counter, 1u);
      if (t < ntiles) {
        int lo = 0, hi = njobs - 1;  // last job whose first tile is <= t
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (jobs[mid].tile0 <= t) lo = mid;
          else hi = mid - 1;
        }
        j = lo;
      }
    }
    t = __shfl_sync(0xffffffffu, t, 0);
    j = __shfl_sync(0xffffffffu, j, 0);
    if (t >= ntiles) break;
    const AdjJob& J = jobs[j];
    if (j != cur) {
      __syncwarp();  // every lane is done with the previous job's slot
      for (int i = lane; i < J.NE * M; i += 32) s_mu[i] = J.mu[i];
      for (int i = lane; i < J.NE; i += 32) s_pdf[i] = J.pdf[i];
      __syncwarp();
      cur = j;
    }
    const long long nrays = (long long)J.g.views_used * J.g.C;
    const long long base = (long long)(t - J.tile0) * kAdjFwdThreads;
    double part = 0.0;
    for (int k = 0; k < kAdjFwdThreads / 32; k++) {
      const long long ray = base + k * 32 + lane;
      double loss = 0.0;
      if (ray < nrays)
        loss = adj_forward_ray<M, 0>(J.g, J.maps, s_mu, s_pdf, J.NE, J.ynorm, J.cos_t, J.sin_t, J.px0, J.py0, J.rec,
                                     J.lsp, J.meas, J.wts, J.gr, J.gmax, ray);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
      part += loss;
    }
    if (lane == 0) J.part[t - J.tile0] = part;
  }
}

// Fixed-order sum of one job's loss partials (adj_loss_kernel's order).
__global__ void adj_loss_batch_kernel(const AdjJob* __restrict__ jobs) {
  __shared__ double s[256];
  const AdjJob& J = jobs[blockIdx.x];
  const int n = (int)adj_job_ray_tiles(J.g);
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) t += J.part[i];
  s[threadIdx.x] = t;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *J.loss = s[0];
}

template <int M>
__global__ void adj_lines_batch_kernel(const AdjJob* __restrict__ jobs, const unsigned int* __restrict__ first,
                                       int n) {
  const int jx = adj_job_of(first, n, blockIdx.x);
  const AdjJob& J = jobs[jx];
  const int i = (int)(blockIdx.x - first[jx]) * (blockDim.x >> 5) + (threadIdx.x >> 5);  // one warp per ray
  if (i >= J.nspecial) return;
  adj_lines_ray<M>(J.g, J.maps, J.cos_t, J.sin_t, J.px0, J.py0, J.special[i], J.lsp + (size_t)i * M,
                   threadIdx.x & 31);
}

template <int M>
__global__ void adj_special_batch_kernel(const AdjJob* __restrict__ jobs, const unsigned int* __restrict__ first,
                                         int n) {
  const int jx = adj_job_of(first, n, blockIdx.x);
  const AdjJob& J = jobs[jx];
  const int i = (int)(blockIdx.x - first[jx]) * (blockDim.x >> 5) + (threadIdx.x >> 5);  // one warp per ray
  if (i >= J.nspecial) return;
  const double scale = special_scale(*J.gmax, J.lmax, J.log2_terms);
  const DevGeom& g = J.g;
  const int ray = J.special[i];
  const int v = ray / g.C, c = ray - (ray / g.C) * g.C;
  Ray r;
  if (!ray_setup(g, J.cos_t[v], J.sin_t[v], J.px0[c], J.py0[c], r)) return;
  walk_exact_warp(g, r, ScatterSink<M>{J.gr + (size_t)ray * M, scale, J.sacc, g.N}, threadIdx.x & 31);
}

template <int M, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, adj_batch_min_blocks(M, TX * TY))
adj_gather_batch_kernel(const AdjJob* __restrict__ jobs, const unsigned int* __restrict__ first, int n) {
  __shared__ AdjStage<M, TX * TY / 32 * kAdjW> S;
  // The job's geometry in shared memory, read where it is used (as the
  // single-slice kernel reads its parameters) rather than held in registers:
  // 96 -> 80 registers at 6 elements, the 64-slice batched gradient 59.9 ->
  // 58.6 ms.
  __shared__ AdjGeom sa;
  const unsigned int total = first[n];
  for (unsigned int b = blockIdx.x; b < total; b += gridDim.x) {
    // the same view ranges as the single-slice gather, so the sums (and the
    // gradient) are bit-identical to it
    const int jx = adj_job_of(first, n, b);
    const AdjJob& J = jobs[jx];
    __syncthreads();  // every thread is done with the previous item's copy
    if (threadIdx.x == 0) sa = J.a;
    __syncthreads();
    const AdjGeom& a = sa;
    const int ntiles = ((a.N + TX) / TX) * ((a.N + TY) / TY);  // tiles of the (N+1)^2 cells
    const int item = (int)(b - first[jx]);
    adj_gather_tile<M, TX, TY, adj_chunks(M)>(a, item % ntiles, item / ntiles, J.cos_t, J.sin_t, J.dir, J.rec, J.gr,
                                           reinterpret_cast<const AdjTileView*>(J.tv), J.ext, S);
  }
}

__global__ void adj_fold_batch_kernel(const AdjJob* __restrict__ jobs, const unsigned int* __restrict__ first, int n,
                                      int M) {
  const int jx = adj_job_of(first, n, blockIdx.x);
  const AdjJob& J = jobs[jx];
  const long long i = (long long)(blockIdx.x - first[jx]) * blockDim.x + threadIdx.x;
  adj_fold_elem(i, M, J.a.N, J.ext, J.sacc, J.gmax, J.lmax, J.log2_terms, J.grad);
}

template <int M, int TX, int TY>
static int launch_adj_gather_batch_t(const AdjJob* d_jobs, const unsigned int* d_first, int n, unsigned int blocks,
                                     cudaStream_t st) {
  int dev = 0, sms = 0, per_sm = 0;
  VCT_CUDA(cudaGetDevice(&dev));
  VCT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  VCT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adj_gather_batch_kernel<M, TX, TY>, TX * TY, 0));
  const unsigned int grid = min(blocks, (unsigned int)(max(1, per_sm) * sms));
  adj_gather_batch_kernel<M, TX, TY><<<grid, TX * TY, 0, st>>>(d_jobs, d_first, n);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

template <int M>
static int launch_adj_batch_m(const AdjJob* d_jobs, const unsigned int* d_first, int n, int ne_max,
                              unsigned int ntiles_ray, const unsigned int nb[kAdjStages], unsigned int* d_counter,
                              cudaStream_t st, cudaStream_t side, cudaEvent_t ev_fork, cudaEvent_t ev_join) {
  const unsigned int* f = d_first;
  adj_reset_batch_kernel<<<nb[kAdjStReset], 256, 0, st>>>(d_jobs, f + kAdjStReset * (n + 1), n, M);
  VCT_CUDA(cudaGetLastError());
  VCT_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned int), st));
  if (nb[kAdjStLines]) {
    adj_lines_batch_kernel<M><<<nb[kAdjStLines], 128, 0, st>>>(d_jobs, f + kAdjStLines * (n + 1), n);
    VCT_CUDA(cudaGetLastError());
  }
  {
    const size_t smem = kAdjBatchWarps * ((size_t)ne_max * M + (size_t)(ne_max + 1) / 2) * sizeof(double);
    int dev = 0, sms = 0, per_sm = 0;
    VCT_CUDA(cudaGetDevice(&dev));
    VCT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    auto k = adj_forward_batch_kernel<M>;
    VCT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    VCT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kAdjFwdThreads, smem));
    const unsigned int grid = min(ntiles_ray, (unsigned int)(max(1, per_sm) * sms));
    if (grid) k<<<grid, kAdjFwdThreads, smem, st>>>(d_jobs, n, ntiles_ray, ne_max, d_counter);
    VCT_CUDA(cudaGetLastError());
  }
  adj_loss_batch_kernel<<<n, 256, 0, st>>>(d_jobs);
  VCT_CUDA(cudaGetLastError());
  const bool fork = nb[kAdjStSpecial] && side && side != st && ev_fork && ev_join;
  if (nb[kAdjStSpecial]) {
    if (fork) {
      VCT_CUDA(cudaEventRecord(ev_fork, st));
      VCT_CUDA(cudaStreamWaitEvent(side, ev_fork, 0));
    }
    adj_special_batch_kernel<M><<<nb[kAdjStSpecial], 128, 0, fork ? side : st>>>(d_jobs, f + kAdjStSpecial * (n + 1), n);
    VCT_CUDA(cudaGetLastError());
    if (fork) VCT_CUDA(cudaEventRecord(ev_join, side));
  }
  // one gather launch per tile shape present (each job in its own shape)
  for (int t = 0; t < 4; t++) {
    const unsigned int blocks = nb[kAdjStGather + t];
    if (!blocks) continue;
    const unsigned int* fg = f + (kAdjStGather + t) * (n + 1);
    int rc;
    switch (t) {
      case 0: rc = launch_adj_gather_batch_t<M, 16, 16>(d_jobs, fg, n, blocks, st); break;
      case 1: rc = launch_adj_gather_batch_t<M, 16, 8>(d_jobs, fg, n, blocks, st); break;
      case 2: rc = launch_adj_gather_batch_t<M, 8, 8>(d_jobs, fg, n, blocks, st); break;
      default: rc = launch_adj_gather_batch_t<M, 8, 4>(d_jobs, fg, n, blocks, st); break;
    }
    if (rc) return rc;
  }
  if (fork) VCT_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
  adj_fold_batch_kernel<<<nb[kAdjStFold], 256, 0, st>>>(d_jobs, f + kAdjStFold * (n + 1), n, M);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int launch_adj_batch(const AdjJob* d_jobs, const unsigned int* d_first, int n, int M, int ne_max,
                     unsigned int ntiles_ray, const unsigned int nblocks[kAdjStages], unsigned int* d_counter,
                     cudaStream_t st, cudaStream_t side, cudaEvent_t ev_fork, cudaEvent_t ev_join) {
  switch (M) {
#define VCT_CASE(mm)                                                                                          \
  case mm:                                                                                                    \
    return launch_adj_batch_m<mm>(d_jobs, d_first, n, ne_max, ntiles_ray, nblocks, d_counter, st, side, ev_fork, \
                                  ev_join);
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default: return fail(VCT_E_ARG, "adjoint: 1..8 materials");
  }
}

VCT_BOUNDS_READER(bounds_adjoint)

}  // namespace vct
