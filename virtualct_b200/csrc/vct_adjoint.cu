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

#include "vct_fastmath.cuh"
#include "vct_internal.h"
#include "vct_walk.cuh"

namespace vct {

// ------------------------------------------------------------- walk plans
// Per-ray record: x = kind | xmaj << 2; y = (maj_lo + 1) | (maj_hi + 1) << 16;
// z = lumped pixel (col + row * N) or -1; w = lumped length (float bits, cm).
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
      o.x = kAdjRayExact;
      special[atomicAdd(nspecial, 1)] = (int)ray;
    } else if (p.status == kPlanWalk) {
      const int lo = min(p.maj0, p.majK), hi = max(p.maj0, p.majK);
      o.x = kAdjRayFast | (p.xmaj << 2);
      o.y = (lo + 1) | ((hi + 1) << 16);
      if (p.pix_lumped >= 0) {
        const int P = g.N + 2 * kPad;
        const int col = p.pix_lumped % P - kPad, row = p.pix_lumped / P - kPad;
        o.z = col + row * g.N;
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
template <int M, int MODE>
__global__ void __launch_bounds__(kAdjFwdThreads)
adj_forward_kernel(DevGeom g, const PixelRec* __restrict__ maps, const double* __restrict__ mu_l2,
                   const float* __restrict__ pdf, int NE, double ynorm, const double* __restrict__ cos_t,
                   const double* __restrict__ sin_t, const double* __restrict__ det_px0,
                   const double* __restrict__ det_py0, const int4* __restrict__ rec,
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
  if (ray < nrays) {
    const int v = (int)(ray / g.C);
    const int c = (int)(ray - (long long)v * g.C);
    const int kind = rec[ray].x & 3;
    RayAcc a;
    acc_init(a);
    if (kind != kAdjRayNone) {
      Ray r;
      ray_setup(g, cos_t[v], sin_t[v], det_px0[c], det_py0[c], r);
      if (kind == kAdjRayFast)
        walk_fast<M>(g, maps, r, a);
      else
        walk_exact<M>(g, maps, r, a);
    }
    double L[8];
    finish_lines<M>(a, L, g.dens_div);
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
  }
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
                                const double* d_py0, const int4* d_rec, int mode, const float* d_meas,
                                const float* d_wts, float* d_g, double* d_loss_part, unsigned int* d_gmax,
                                cudaStream_t st) {
  const long long nrays = (long long)g.views_used * g.C;
  const int blocks = (int)((nrays + kAdjFwdThreads - 1) / kAdjFwdThreads);
  const size_t smem = (size_t)NE * M * sizeof(double) + (size_t)NE * sizeof(float);
  if (blocks == 0) return VCT_OK;
  auto k = mode == 0 ? adj_forward_kernel<M, 0> : adj_forward_kernel<M, 1>;
  VCT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<blocks, kAdjFwdThreads, smem, st>>>(g, d_maps, d_mu_l2, d_pdf, NE, ynorm, d_cos, d_sin, d_px0, d_py0, d_rec,
                                          d_meas, d_wts, d_g, d_loss_part, d_gmax);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int adj_forward_blocks(const DevGeom& g) {
  const long long nrays = (long long)g.views_used * g.C;
  return (int)((nrays + kAdjFwdThreads - 1) / kAdjFwdThreads);
}

int launch_adj_forward(const DevGeom& g, const PixelRec* d_maps, int M, const double* d_mu_l2, const float* d_pdf,
                       int NE, double ynorm, const double* d_cos, const double* d_sin, const double* d_px0,
                       const double* d_py0, const int4* d_rec, int mode, const float* d_meas, const float* d_wts,
                       float* d_g, double* d_loss_part, unsigned int* d_gmax, cudaStream_t st) {
  switch (M) {
#define VCT_CASE(mm)                                                                                             \
  case mm:                                                                                                       \
    return launch_adj_forward_m<mm>(g, d_maps, d_mu_l2, d_pdf, NE, ynorm, d_cos, d_sin, d_px0, d_py0, d_rec, mode, \
                                    d_meas, d_wts, d_g, d_loss_part, d_gmax, st);
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default: return fail(VCT_E_ARG, "adjoint: 1..8 materials");
  }
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
  const int n = *nspecial;
  const double scale = special_scale(*gmax, lmax, log2_terms);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ray = special[i];
    const int v = ray / g.C, c = ray - (ray / g.C) * g.C;
    Ray r;
    if (!ray_setup(g, cos_t[v], sin_t[v], det_px0[c], det_py0[c], r)) continue;
    walk_exact_to(g, r, ScatterSink<M>{gr + (size_t)ray * M, scale, acc, g.N});
  }
}

int launch_adj_special(const DevGeom& g, int M, const double* d_cos, const double* d_sin, const double* d_px0,
                       const double* d_py0, const int* d_special, const int* d_nspecial, int nspecial_host,
                       const float* d_g, const unsigned int* d_gmax, double lmax, int log2_terms,
                       unsigned long long* d_acc, cudaStream_t st) {
  if (nspecial_host <= 0) return VCT_OK;
  const int blocks = (nspecial_host + 127) / 128;
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
// Largest channel window one tile needs per view (the host picks the tile so
// the window fits; see adj_pick_tile), rays staged per round, and the views a
// round considers: it takes as many as fit in the staging space (at least
// kAdjCap / kAdjWMax), so each barrier serves more views when windows are
// narrow.
constexpr int kAdjWMax = 128;
constexpr int kAdjCap = 4 * kAdjWMax;
constexpr int kAdjVB = 8;

// Angle of the direction (u, v) from the source, measured like the channel
// angle theta = (iso - jj) * dalpha: (sin theta, -cos theta) is channel jj's
// unrotated direction.  Only v < 0 occurs (the grid lies below the source).
// It only picks candidate channels, whose ranges carry a margin.
__device__ __forceinline__ float fan_angle(float u, float v) {
  const float t = u * rcp_approx(-v);
  return fabsf(t) <= 0.5f ? atan_small(t) : atanf(t);
}

// The gather runs over the (N+1) x (N+1) cells with indices -1..N-1: cells
// at index -1 lie outside the grid, but the walk's truncating cast puts their
// pieces on index 0 (adj_fold_kernel adds them there).  One thread per cell.
// Staged per ray (shared memory, vector loads):
//   A = (dx, dy, offset of the ray from the tile centre, h*(|dx|+|dy|))
//   B = (2h/max(|dx|,|dy|), 1/(|dx||dy|), lumped length, lumped pixel bits)
//   K = (xmaj, (maj_lo+1) | (maj_hi+1) << 16), G = the ray's M factors.
// A ray that the fast walk does not take gets h*(|dx|+|dy|) = -inf (no
// chord) and no lumped pixel.  The chord of a line at offset b from the
// centre of a square of half-size h, direction with components a >= c:
// 2h/a while |b| <= h(a-c), then (h(a+c) - |b|)/(a c) down to 0.
template <int M, int TX, int TY>
__global__ void __launch_bounds__(TX * TY)
adj_gather_kernel(AdjGeom a, const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                  const double2* __restrict__ dir, const int4* __restrict__ rec, const float* __restrict__ gr,
                  float* __restrict__ ext, int* __restrict__ status) {
  constexpr int MG = (M + 3) / 4 * 4;
  __shared__ float4 s_A[kAdjCap];
  __shared__ float4 s_B[kAdjCap];
  __shared__ int2 s_K[kAdjCap];
  __shared__ float4 s_g4[(MG / 4) * kAdjCap];  // ray factors, quad q of ray k at q * kAdjCap + k
  __shared__ int s_jlo[kAdjVB], s_jn[kAdjVB], s_base[kAdjVB + 1], s_cplx[kAdjVB], s_nvb;
  __shared__ float s_cb[kAdjVB], s_sb[kAdjVB], s_dtx[kAdjVB], s_dty[kAdjVB];

  const int N = a.N, NE1 = N + 1;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int e0 = blockIdx.x * TX, f0 = blockIdx.y * TY;  // first extended column / row
  const int col = e0 + tx - 1, row = f0 + ty - 1;         // cell indices, -1..N-1
  const bool live = col < N && row < N;
  const double s = a.s;
  const float h = (float)(0.5 * s);
  // Tile centre (world cm; x right, y up; row r spans y in ((n-r-1)s, (n-r)s]).
  const double Tx = (e0 - 1 + 0.5 * TX - a.nxm) * s;
  const double Ty = (a.nxm - (f0 - 1) - 0.5 * TY) * s;
  const float lx = (float)((tx + 0.5 - 0.5 * TX) * s);
  const float ly = (float)((0.5 * TY - ty - 0.5) * s);
  const int pix = (col >= 0 && row >= 0) ? row * N + col : -2;  // -2: never a lumped pixel
  const int colx = col + 1, rowx = row + 1;
  const float iso = (float)a.iso, ida = (float)a.inv_dalpha;
  const float kdj = h * ida * 1.05f;

  double dacc[M];
#pragma unroll
  for (int m = 0; m < M; m++) dacc[m] = 0.0;

  const int V = a.views_used;
  for (int v0 = 0; v0 < V;) {
    const int nvc = min(kAdjVB, V - v0);  // views considered this round
    // Channel window of the tile for each view: the angles of the tile's
    // corners grown by one cell, plus two channels.
    if (threadIdx.x < nvc) {
      const int v = v0 + threadIdx.x;
      const double cb = cos_t[v], sb = sin_t[v];
      const double Sx = a.sid * sb, Sy = a.sid * cb;
      const double x0 = (e0 - 2 - a.nxm) * s, x1 = (e0 + TX - a.nxm) * s;
      const double y0 = (a.nxm - f0 - TY) * s, y1 = (a.nxm - f0 + 2) * s;
      float tmin = 1e30f, tmax = -1e30f;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const double qx = ((k & 1) ? x1 : x0) - Sx, qy = ((k & 2) ? y1 : y0) - Sy;
        const float u = (float)(qx * cb - qy * sb), w = (float)(qx * sb + qy * cb);
        const float t = fan_angle(u, w);
        tmin = fminf(tmin, t);
        tmax = fmaxf(tmax, t);
      }
      int jlo = (int)floorf(iso - tmax * ida) - 2 - a.start;
      int jhi = (int)ceilf(iso - tmin * ida) + 2 - a.start;
      jlo = max(jlo, 0);
      jhi = min(jhi, a.C - 1);
      int jn = jhi - jlo + 1;
      if (jn < 0) jn = 0;
      if (jn > kAdjWMax) {
        jn = kAdjWMax;
        atomicOr(status, 1);
      }
      s_jlo[threadIdx.x] = jlo;
      s_jn[threadIdx.x] = jn;
      s_cplx[threadIdx.x] = 0;
      s_cb[threadIdx.x] = (float)cb;
      s_sb[threadIdx.x] = (float)sb;
      s_dtx[threadIdx.x] = (float)(Tx - Sx);
      s_dty[threadIdx.x] = (float)(Ty - Sy);
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the views whose windows fit the staging space
      int b = 0, k = 0;
      for (; k < nvc && b + s_jn[k] <= kAdjCap; k++) {
        s_base[k] = b;
        b += s_jn[k];
      }
      s_base[k] = b;
      s_nvb = k;
    }
    __syncthreads();
    const int nvb = s_nvb;
    // Stage the window's rays: direction and offset from the tile centre in
    // FP64, then float (small for every ray that can reach the tile).
    const int total = s_base[nvb];
    for (int k = threadIdx.x; k < total; k += TX * TY) {
      int vb = 0;
      while (vb + 1 < nvb && k >= s_base[vb + 1]) vb++;
      const int v = v0 + vb;
      const int c = s_jlo[vb] + (k - s_base[vb]);
      const long long ray = (long long)v * a.C + c;
      if (!VCT_INDEX_OK(v < a.views_used && c >= 0 && c < a.C && k < kAdjCap)) continue;
      const double cb = cos_t[v], sb = sin_t[v];
      const double2 e = dir[c];
      const double dx = e.x * cb + e.y * sb, dy = -e.x * sb + e.y * cb;
      const double Sx = a.sid * sb, Sy = a.sid * cb;
      const double bt = dx * (Ty - Sy) - dy * (Tx - Sx);
      const float ax = fabsf((float)dx), ay = fabsf((float)dy);
      const int4 r = rec[ray];
      const bool fast = (r.x & 3) == kAdjRayFast;
      s_A[k] = make_float4((float)dx, (float)dy, (float)bt, fast ? h * (ax + ay) : -INFINITY);
      s_B[k] = make_float4(2.0f * h / fmaxf(ax, ay), 1.0f / (ax * ay), fast ? __int_as_float(r.w) : 0.0f,
                           __int_as_float(fast ? r.z : -1));
      s_K[k] = make_int2(r.x >> 2, r.y);
#pragma unroll
      for (int q = 0; q < MG / 4; q++) {
        float4 gq;
        gq.x = 4 * q + 0 < M ? gr[ray * M + 4 * q + 0] : 0.0f;
        gq.y = 4 * q + 1 < M ? gr[ray * M + 4 * q + 1] : 0.0f;
        gq.z = 4 * q + 2 < M ? gr[ray * M + 4 * q + 2] : 0.0f;
        gq.w = 4 * q + 3 < M ? gr[ray * M + 4 * q + 3] : 0.0f;
        s_g4[q * kAdjCap + k] = gq;
      }
      // Does the ray's walk end or lump inside this tile?  If no staged ray
      // of the view does, the whole block takes the plain chord path.
      if (fast) {
        const int lo = (r.y & 0xffff) - 1, hi = (r.y >> 16) - 1;
        const int c0 = (r.x >> 2) ? e0 - 1 : f0 - 1;  // the tile's first cell on the ray's major axis
        const int c1 = c0 + ((r.x >> 2) ? TX : TY) - 1;
        bool cplx = c0 < lo || c1 > hi;
        if (r.z >= 0) {
          const int lc = r.z % a.N, lr = r.z / a.N;
          cplx = cplx || (lc >= e0 - 1 && lc <= e0 + TX - 2 && lr >= f0 - 1 && lr <= f0 + TY - 2);
        }
        if (cplx) atomicOr(&s_cplx[vb], 1);
      }
    }
    __syncthreads();

    float acc[M];
#pragma unroll
    for (int m = 0; m < M; m++) acc[m] = 0.0f;
    for (int vb = 0; vb < nvb; vb++) {
      const float cb = s_cb[vb], sb = s_sb[vb];
      const int jlo = s_jlo[vb], jn = s_jn[vb], base = s_base[vb];
      // Cell centre relative to the source, its fan angle and angular
      // half-width in channels (with a margin).
      const float qx = s_dtx[vb] + lx, qy = s_dty[vb] + ly;
      const float u = qx * cb - qy * sb, w = qx * sb + qy * cb;
      const float jc = iso - fan_angle(u, w) * ida;
      const float iq = rsqrtf(fmaf(qx, qx, qy * qy));
      const float dj = fmaf((fabsf(qx) + fabsf(qy)) * iq * iq, kdj, 0.05f);
      const int j0 = max((int)ceilf(jc - dj) - a.start - jlo, 0);
      const int j1 = min((int)floorf(jc + dj) - a.start - jlo, jn - 1);
      if (!s_cplx[vb]) {
        // every candidate's walk covers the whole tile: chord only
        for (int j = j0; j <= j1; j++) {
          const int k = base + j;
          if (!VCT_INDEX_OK(k >= 0 && k < kAdjCap)) continue;
          const float4 A = s_A[k];
          const float4 B = s_B[k];
          const float b = fmaf(A.x, ly, fmaf(-A.y, lx, A.z));
          const float num = A.w - fabsf(b);
          const float len = num > 0.0f ? fminf(B.x, num * B.y) : 0.0f;
#pragma unroll
          for (int q = 0; q < MG / 4; q++) {
            const float4 g = s_g4[q * kAdjCap + k];
            if (4 * q + 0 < M) acc[4 * q + 0] = fmaf(len, g.x, acc[4 * q + 0]);
            if (4 * q + 1 < M) acc[4 * q + 1] = fmaf(len, g.y, acc[4 * q + 1]);
            if (4 * q + 2 < M) acc[4 * q + 2] = fmaf(len, g.z, acc[4 * q + 2]);
            if (4 * q + 3 < M) acc[4 * q + 3] = fmaf(len, g.w, acc[4 * q + 3]);
          }
        }
      } else {
        for (int j = j0; j <= j1; j++) {
          const int k = base + j;
          if (!VCT_INDEX_OK(k >= 0 && k < kAdjCap)) continue;
          const float4 A = s_A[k];
          const float4 B = s_B[k];
          const int2 K = s_K[k];
          const float b = fmaf(A.x, ly, fmaf(-A.y, lx, A.z));
          const float num = A.w - fabsf(b);
          float len = num > 0.0f ? fminf(B.x, num * B.y) : 0.0f;
          const int mi = K.x ? colx : rowx;
          if (mi < (K.y & 0xffff) || mi > (K.y >> 16)) len = 0.0f;
          if (__float_as_int(B.w) == pix) len += B.z;
#pragma unroll
          for (int q = 0; q < MG / 4; q++) {
            const float4 g = s_g4[q * kAdjCap + k];
            if (4 * q + 0 < M) acc[4 * q + 0] = fmaf(len, g.x, acc[4 * q + 0]);
            if (4 * q + 1 < M) acc[4 * q + 1] = fmaf(len, g.y, acc[4 * q + 1]);
            if (4 * q + 2 < M) acc[4 * q + 2] = fmaf(len, g.z, acc[4 * q + 2]);
            if (4 * q + 3 < M) acc[4 * q + 3] = fmaf(len, g.w, acc[4 * q + 3]);
          }
        }
      }
    }
#pragma unroll
    for (int m = 0; m < M; m++) dacc[m] += (double)acc[m];
    __syncthreads();
    v0 += nvb;
  }
  if (!live) return;
  const size_t n2 = (size_t)NE1 * NE1;
  const size_t o = (size_t)(row + 1) * NE1 + (col + 1);
#pragma unroll
  for (int m = 0; m < M; m++) ext[m * n2 + o] = (float)dacc[m];
}

// grad[m][r][c] = ext at (r, c), plus the folded cells at index -1 (row -1
// onto row 0, column -1 onto column 0), plus the exact-walk rays'
// fixed-point sums; fixed order, so the result is deterministic.
__global__ void adj_fold_kernel(int M, int N, const float* __restrict__ ext, const unsigned long long* __restrict__ sacc,
                                const unsigned int* __restrict__ gmax, double lmax, int log2_terms,
                                float* __restrict__ grad) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n2 = (size_t)N * N, e2 = (size_t)(N + 1) * (N + 1);
  if (i >= (long long)M * n2) return;
  const int m = (int)(i / n2);
  const int p = (int)(i - (long long)m * n2);
  const int r = p / N, c = p - (p / N) * N;
  const float* e = ext + m * e2;
  const int N1 = N + 1;
  double v = e[(r + 1) * N1 + (c + 1)];
  if (c == 0) v += e[(r + 1) * N1];
  if (r == 0) v += e[c + 1];
  if (r == 0 && c == 0) v += e[0];
  if (sacc) v += (double)(long long)sacc[i] / special_scale(*gmax, lmax, log2_terms);
  grad[i] = (float)v;
}

// Tile shapes, largest first; the channel window of a tile grows with its
// size and shrinks with the source distance.
static const int kTiles[][2] = {{32, 8}, {16, 8}, {8, 8}, {8, 4}};

int adj_pick_tile(const AdjGeom& a, double lim) {
  // Nearest approach of the grown tile to the source, and its half-diagonal.
  const double dmin = a.sid - (lim + 2.0 * a.s) * sqrt(2.0);
  if (!(dmin > 0)) return -1;
  for (int t = 0; t < 4; t++) {
    const double hd = 0.5 * sqrt((double)(kTiles[t][0] + 2) * (kTiles[t][0] + 2) +
                                 (double)(kTiles[t][1] + 2) * (kTiles[t][1] + 2)) * a.s;
    if (hd >= dmin) continue;
    const double ang = 2.0 * asin(hd / dmin);
    const double jn = ang * a.inv_dalpha + 6.0;
    if (jn <= kAdjWMax) return t;
  }
  return -1;
}

template <int M>
static int launch_adj_gather_m(const AdjGeom& a, int tile, const double* d_cos, const double* d_sin,
                               const double2* d_dir, const int4* d_rec, const float* d_g, float* d_ext, int* d_status,
                               cudaStream_t st) {
  const int TX = kTiles[tile][0], TY = kTiles[tile][1];
  dim3 grid((a.N + 1 + TX - 1) / TX, (a.N + 1 + TY - 1) / TY);
  switch (tile) {
    case 0: adj_gather_kernel<M, 32, 8><<<grid, 256, 0, st>>>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_ext, d_status); break;
    case 1: adj_gather_kernel<M, 16, 8><<<grid, 128, 0, st>>>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_ext, d_status); break;
    case 2: adj_gather_kernel<M, 8, 8><<<grid, 64, 0, st>>>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_ext, d_status); break;
    default: adj_gather_kernel<M, 8, 4><<<grid, 32, 0, st>>>(a, d_cos, d_sin, d_dir, d_rec, d_g, d_ext, d_status); break;
  }
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int launch_adj_gather(const AdjGeom& a, int M, int tile, const double* d_cos, const double* d_sin,
                      const double2* d_dir, const int4* d_rec, const float* d_g, float* d_ext, int* d_status,
                      cudaStream_t st) {
  if (tile < 0 || tile > 3) return fail(VCT_E_UNSUPPORTED, "adjoint: no tile fits the channel window");
  switch (M) {
#define VCT_CASE(mm) \
  case mm: return launch_adj_gather_m<mm>(a, tile, d_cos, d_sin, d_dir, d_rec, d_g, d_ext, d_status, st);
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

VCT_BOUNDS_READER(bounds_adjoint)

}  // namespace vct
