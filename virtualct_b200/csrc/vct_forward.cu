// MBFPA forward projection on sm_100a.
//
// One thread walks one ray (view v, channel c) through the N x N grid along
// the reference's path (MB/reprojection_TOMO.cpp:53-283) and accumulates the
// per-element line integrals L_m = sum_seg (s_m/1000) * len, s_m the stored
// int16 density x 1000.  The walk is done once per ray for all energy bins
// (the reference repeats it for every bin, MB/main.cpp:492-506); the
// polyenergetic epilogue then evaluates sum_E pdf(E) exp(-sum_m mu_m(E) L_m)
// with the mu table in shared memory.
//
// Two walks:
//   walk_exact  the reference's expressions, operation for operation
//               (compiled with --fmad=false, IEEE division and square root),
//               so segment boundaries match it bit for bit;
//   walk_fast   the same segments found by a Siddon-style event loop (major
//               gridline / minor gridline, whichever comes first) with event
//               times in integer fixed point, one segment per iteration,
//               weights in 2^-31 steps and integer multiply-add
//               accumulation; no per-step division or FP64 arithmetic.
//
// Maps are one 16-byte record (8 x int16) per pixel in a padded
// (N+4) x (N+4) layout whose border reproduces the reference's truncating
// pixel index: row/column -1 repeats row/column 0 (a midpoint in (-1, 0)
// truncates to 0), the other border cells are zero (rejected).  At 512^2 the
// record array is 4.3 MB and stays L2-resident.
#include <cuda_runtime.h>
#include <string.h>

#include "vct_internal.h"
#include "vct_philox.h"
#include "vct_walk.cuh"

namespace vct {

// ---------------------------------------------------------------- map packing
// out_t, when given, receives the transposed copy.
VCT_HD void pack_maps_elem(int p, const int16_t* __restrict__ maps, int M, int N, PixelRec* __restrict__ out,
                           PixelRec* __restrict__ out_t) {
  const int P = N + 2 * kPad;
  const int r = p / P - kPad, c = p % P - kPad;  // padded row/column in [-kPad, N+kPad)
  PixelRec rec;
  const bool inside = r >= -1 && c >= -1 && r < N && c < N;
  const size_t src = (size_t)(r < 0 ? 0 : r) * N + (c < 0 ? 0 : c);
  const size_t n2 = (size_t)N * N;
#pragma unroll
  for (int m = 0; m < 8; m++) {
    int16_t v = (inside && m < M) ? maps[(size_t)m * n2 + src] : (int16_t)0;
    rec.m[m] = v < 0 ? (int16_t)0 : v;  // negative densities weigh 0 (:151-155)
  }
  out[p] = rec;
  // Transposed copy (column-major): walks whose major axis is x step along
  // a column of it, so a warp's rays read neighbouring records.
  if (out_t) out_t[(c + kPad) * P + (r + kPad)] = rec;
}

__global__ void pack_maps_kernel(const int16_t* __restrict__ maps, int M, int N,
                                 PixelRec* __restrict__ out, PixelRec* __restrict__ out_t) {
  const int P = N + 2 * kPad;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P * P) return;
  pack_maps_elem(p, maps, M, N, out, out_t);
}

unsigned int pack_maps_blocks(int N) {
  const int P = N + 2 * kPad;
  return (unsigned int)((P * P + 255) / 256);
}

// Job of block b in a batched launch: the last j with first[j] <= b.
__device__ __forceinline__ int batch_job_of(const unsigned int* __restrict__ first, int n, unsigned int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void pack_maps_batch_kernel(const PackJob* __restrict__ jobs, const unsigned int* __restrict__ first,
                                       int n, int M) {
  const int jx = batch_job_of(first, n, blockIdx.x);
  const PackJob J = jobs[jx];
  const int P = J.N + 2 * kPad;
  const int p = (int)(blockIdx.x - first[jx]) * blockDim.x + threadIdx.x;
  if (p >= P * P) return;
  pack_maps_elem(p, J.maps, M, J.N, J.out, VCT_FWD_DUAL_LAYOUT ? J.out + (size_t)P * P : nullptr);
}

int launch_pack_maps_batch(const PackJob* d_jobs, const unsigned int* d_first, int n, int M, unsigned int nblocks,
                           cudaStream_t st) {
  if (nblocks == 0) return VCT_OK;
  pack_maps_batch_kernel<<<nblocks, 256, 0, st>>>(d_jobs, d_first, n, M);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int launch_pack_maps(const int16_t* d_maps, int M, int N, PixelRec* d_packed, cudaStream_t st) {
  const int P = N + 2 * kPad;
  PixelRec* d_t = VCT_FWD_DUAL_LAYOUT ? d_packed + padded_pixels(N) : nullptr;
  pack_maps_kernel<<<(P * P + 255) / 256, 256, 0, st>>>(d_maps, M, N, d_packed, d_t);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}



// ------------------------------------------------------------- reductions
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

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr int kFwdThreads = 128;

// 2^-y with y = transp*log2(e) in FP64, split y = n + f: the fraction goes
// through the SFU exponential, the integer part into the float exponent; bins
// below 2^-126 contribute nothing.  FP64 sum.  mu: [NE][M] mu*log2(e)/xfactor.
template <int M>
__device__ __forceinline__ float spectral_compensated(const double L[8], const double* __restrict__ s_mu,
                                                      const float* __restrict__ s_pdf, int NE) {
  double accd = 0.0;
  for (int e = 0; e < NE; e++) {
    double y = 0.0;
#pragma unroll
    for (int m = 0; m < M; m++) y = __fma_rn(s_mu[e * M + m], L[m], y);
    const int nI = __double2int_rd(y);
    if (nI <= 125) {
      const float fr = (float)(y - (double)nI);
      const float scale = __int_as_float((127 - nI) << 23);
      accd += (double)(s_pdf[e] * ex2_approx(-fr) * scale);
    }
  }
  return (float)accd;
}

// The polyenergetic value of a ray from its line integrals: the reference's
// float sum in bin order (MB/reprojection_TOMO.cpp:196-197, MB/main.cpp:504)
// or the compensated FP64 sum.
template <int M, int SUM_MODE>
__device__ __forceinline__ float ray_value(const double L[8], const double* __restrict__ mu,
                                           const float* __restrict__ pdf, int NE) {
  if (SUM_MODE == VCT_SUM_REFERENCE) {
    float accf = 0.0f;
    for (int e = 0; e < NE; e++) {
      double t = 0.0;
#pragma unroll
      for (int m = 0; m < M; m++) t = __fma_rn(mu[e * M + m], L[m], t);
      accf = __fadd_rn(accf, (float)((double)pdf[e] * exp(-t)));
    }
    return accf;
  }
  return spectral_compensated<M>(L, mu, pdf, NE);
}

// One thread per ray (view v, channel c), rays numbered view-major so a warp
// holds 32 neighbouring channels of one view (similar paths and lengths).
// mu: [NE][M] in shared memory -- mu/xfactor for the reference summation,
// mu*log2(e)/xfactor for the compensated one.  Each warp publishes its
// max/min/segment count with atomics, so no warp waits for the block.
template <int M, int SUM_MODE>
__global__ void __launch_bounds__(kFwdThreads, VCT_FWD_MINBLOCKS)
forward_kernel(DevGeom g, const PixelRec* __restrict__ maps, const double* __restrict__ mu_tab,
               const float* __restrict__ pdf, int NE, const double* __restrict__ cos_t,
               const double* __restrict__ sin_t, const double* __restrict__ det_px0,
               const double* __restrict__ det_py0, int fast, int defer, float* __restrict__ out,
               double* __restrict__ lint, FwdStats* __restrict__ stats, long long ray0, long long ray1) {
  extern __shared__ double smem[];
  double* s_mu = smem;                                             // [NE][M]
  float* s_pdf = reinterpret_cast<float*>(smem + (size_t)NE * M);  // [NE]
  for (int i = threadIdx.x; i < NE * M; i += blockDim.x) s_mu[i] = mu_tab[i];
  for (int i = threadIdx.x; i < NE; i += blockDim.x) s_pdf[i] = pdf[i];
  __syncthreads();

  // rays [ray0, ray1) of the views_used * C
  const long long ray = ray0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool active = ray < ray1;
  float val = 0.0f;
  int nseg = 0;
  if (active) {
    const int v = (int)(ray / g.C);
    const int c = (int)(ray - (long long)v * g.C);
    RayAcc a;
    acc_init(a);
    Ray r;
    if (ray_setup(g, cos_t[v], sin_t[v], det_px0[c], det_py0[c], r)) {
      bool done = false;
      if (fast) done = walk_fast<M>(g, maps, r, a);
      // with defer, a ray the fast walk hands back is left to
      // forward_lines_kernel (a warp per ray) and counts nowhere here
      if (!done) {
        if (defer) active = false;
        else walk_exact<M>(g, maps, r, a);
      }
    }
    if (active) {
      nseg = a.nseg;
      double L[8];
      finish_lines<M>(a, L, g.dens_div);
      if (lint) {
#pragma unroll
        for (int m = 0; m < M; m++) lint[ray * M + m] = L[m];
      }
      if (out) {
        val = ray_value<M, SUM_MODE>(L, s_mu, s_pdf, NE);
        out[(size_t)v * g.width + g.start + c] = val;
      }
    }
  }
  float vmax = warp_max(active ? val : 0.0f);
  float vmin = warp_min(active ? val : 3.0e38f);
  unsigned long long ns = warp_sum_ull((unsigned long long)nseg);
  if ((threadIdx.x & 31) == 0) {
    // Non-negative floats order like their bit patterns.
    atomicMax(&stats->max_bits, __float_as_uint(vmax));
    atomicMin(&stats->min_bits, __float_as_uint(vmin));
    atomicAdd(&stats->segments, ns);
  }
}

// The rays the fast walk hands back (rays through the grid origin at even
// channel counts: the central channel of every view), listed once per
// context, walked by a whole warp each (exact_lines_warp) after the main
// kernel has skipped them: walked there in one thread each they held their
// blocks several times longer than the rest (512^2, 800 x 608 rays: 1.33
// against 0.53 ms for 609 channels).  Lane 0 does the ray's epilogue and its
// share of the statistics.
template <int M, int SUM_MODE>
__global__ void forward_lines_kernel(DevGeom g, const PixelRec* __restrict__ maps, const double* __restrict__ mu_tab,
                                     const float* __restrict__ pdf, int NE, const double* __restrict__ cos_t,
                                     const double* __restrict__ sin_t, const double* __restrict__ det_px0,
                                     const double* __restrict__ det_py0, const int* __restrict__ exact, int nexact,
                                     float* __restrict__ out, double* __restrict__ lint,
                                     FwdStats* __restrict__ stats, long long ray0, long long ray1) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= nexact) return;  // warp-uniform
  const int ray = exact[i];
  if (ray < ray0 || ray >= ray1) return;
  const int lane = threadIdx.x & 31;
  double L[8];
  int nseg;
  exact_lines_warp<M>(g, maps, cos_t, sin_t, det_px0, det_py0, ray, L, &nseg, lane);
  if (lane != 0) return;
  if (lint) {
#pragma unroll
    for (int m = 0; m < M; m++) lint[(size_t)ray * M + m] = L[m];
  }
  float val = 0.0f;
  if (out) {
    const int v = ray / g.C, c = ray - (ray / g.C) * g.C;
    val = ray_value<M, SUM_MODE>(L, mu_tab, pdf, NE);
    out[(size_t)v * g.width + g.start + c] = val;
  }
  atomicMax(&stats->max_bits, __float_as_uint(val));
  atomicMin(&stats->min_bits, __float_as_uint(val));
  atomicAdd(&stats->segments, (unsigned long long)nseg);
}

// Lists the rays of [0, views_used * C) whose fast-walk plan is the exact
// walk: count first (list == nullptr), then fill (any order).
__global__ void exact_list_kernel(DevGeom g, const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                                  const double* __restrict__ det_px0, const double* __restrict__ det_py0,
                                  int* __restrict__ list, int cap, int* __restrict__ count) {
  const long long nrays = (long long)g.views_used * g.C;
  const long long ray = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (ray >= nrays) return;
  const int v = (int)(ray / g.C), c = (int)(ray - (long long)v * g.C);
  Ray r;
  if (!ray_setup(g, cos_t[v], sin_t[v], det_px0[c], det_py0[c], r)) return;
  FastPlan p;
  fast_plan(g, r, p);
  if (p.status != kPlanExact) return;
  const int k = atomicAdd(count, 1);
  if (list && k < cap) list[k] = (int)ray;
}

int launch_exact_list(const DevGeom& g, const double* d_cos, const double* d_sin, const double* d_px0,
                      const double* d_py0, int* d_list, int cap, int* d_count, cudaStream_t st) {
  const long long nrays = (long long)g.views_used * g.C;
  VCT_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int), st));
  if (nrays == 0) return VCT_OK;
  exact_list_kernel<<<(unsigned)((nrays + 255) / 256), 256, 0, st>>>(g, d_cos, d_sin, d_px0, d_py0, d_list, cap,
                                                                     d_count);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

template <int M>
static int launch_forward_m(const DevGeom& g, const PixelRec* d_maps, const double* d_mu,
                            const float* d_pdf, int NE, const double* d_cos, const double* d_sin,
                            const double* d_px0, const double* d_py0, int sum_mode, int fast,
                            float* d_out, double* d_lint, FwdStats* d_stats, cudaStream_t st, int v0, int v1,
                            const int* d_exact, int nexact) {
  const long long ray0 = (long long)v0 * g.C, ray1 = (long long)v1 * g.C;
  const int blocks = (int)((ray1 - ray0 + kFwdThreads - 1) / kFwdThreads);
  const size_t smem = (size_t)NE * M * sizeof(double) + (size_t)NE * sizeof(float);
  if (blocks == 0) return VCT_OK;
  const int defer = fast && d_exact && nexact > 0;
  if (sum_mode == VCT_SUM_REFERENCE) {
    auto k = forward_kernel<M, VCT_SUM_REFERENCE>;
    VCT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<blocks, kFwdThreads, smem, st>>>(g, d_maps, d_mu, d_pdf, NE, d_cos, d_sin, d_px0, d_py0, fast, defer,
                                          d_out, d_lint, d_stats, ray0, ray1);
    VCT_CUDA(cudaGetLastError());
    if (defer)
      forward_lines_kernel<M, VCT_SUM_REFERENCE><<<(nexact + 3) / 4, 128, 0, st>>>(
          g, d_maps, d_mu, d_pdf, NE, d_cos, d_sin, d_px0, d_py0, d_exact, nexact, d_out, d_lint, d_stats, ray0, ray1);
  } else {
    auto k = forward_kernel<M, VCT_SUM_COMPENSATED>;
    VCT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<blocks, kFwdThreads, smem, st>>>(g, d_maps, d_mu, d_pdf, NE, d_cos, d_sin, d_px0, d_py0, fast, defer,
                                          d_out, d_lint, d_stats, ray0, ray1);
    VCT_CUDA(cudaGetLastError());
    if (defer)
      forward_lines_kernel<M, VCT_SUM_COMPENSATED><<<(nexact + 3) / 4, 128, 0, st>>>(
          g, d_maps, d_mu, d_pdf, NE, d_cos, d_sin, d_px0, d_py0, d_exact, nexact, d_out, d_lint, d_stats, ray0, ray1);
  }
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int launch_forward(const DevGeom& g, const PixelRec* d_maps, int M, const double* d_mu_tab,
                   const float* d_pdf, int NE, const double* d_cos, const double* d_sin,
                   const double* d_det_ox, const double* d_det_oy, int sum_mode, int fast, float* d_out,
                   double* d_lint, FwdStats* d_stats, cudaStream_t st, int v0, int v1, const int* d_exact,
                   int nexact) {
  fast = fast && !g.rmax_active;
  if (v1 < 0) v1 = g.views_used;
  if (v0 < 0 || v0 > v1 || v1 > g.views_used) return fail(VCT_E_ARG, "forward: view range outside the views used");
  switch (M) {
#define VCT_CASE(mm)                                                                                               \
  case mm:                                                                                                         \
    return launch_forward_m<mm>(g, d_maps, d_mu_tab, d_pdf, NE, d_cos, d_sin, d_det_ox, d_det_oy, sum_mode, fast, \
                                d_out, d_lint, d_stats, st, v0, v1, d_exact, nexact);
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default:
      return fail(VCT_E_ARG, "number of materials must be 1..8");
  }
}

// --------------------------------------------------------- batched forward
// Many slices (jobs) with one element count in one persistent launch.  The
// rays of every job are cut into tiles of `tile_rays` rays (view-major, as
// the plain kernel numbers them); every resident WARP takes tiles from a
// global counter in job order, so jobs of uneven size share the GPU without a
// tail per job and no warp waits for another's rays.  At a job change a warp
// copies the job's descriptor and mu/pdf tables into its own shared-memory
// slot.  Per ray the work and the outputs are the plain kernel's (compensated
// summation; statistics per job).
constexpr int kBatchWarps = kFwdThreads / 32;
#ifndef VCT_BATCH_MINBLOCKS
#define VCT_BATCH_MINBLOCKS 5
#endif

__host__ __device__ inline size_t batch_slot_doubles(int ne_max, int M) {
  return (size_t)ne_max * M + (size_t)(ne_max + 1) / 2;  // mu [ne_max][M] + pdf [ne_max] floats
}

template <int M>
__global__ void __launch_bounds__(kFwdThreads, VCT_BATCH_MINBLOCKS)
forward_batch_kernel(const FwdJob* __restrict__ jobs, int njobs, int tile_rays, unsigned int ntiles, int ne_max,
                     unsigned int* __restrict__ counter) {
  extern __shared__ double smem[];
  __shared__ FwdJob s_job[kBatchWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* s_mu = smem + (size_t)warp * batch_slot_doubles(ne_max, M);  // [ne_max][M]
  float* s_pdf = reinterpret_cast<float*>(s_mu + (size_t)ne_max * M);  // [ne_max]
  FwdJob& J = s_job[warp];
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
    if (j != cur) {
      __syncwarp();  // every lane is done with the previous job's slot
      if (lane == 0) J = jobs[j];
      const FwdJob& G = jobs[j];
      for (int i = lane; i < G.NE * M; i += 32) s_mu[i] = G.mu[i];
      for (int i = lane; i < G.NE; i += 32) s_pdf[i] = G.pdf[i];
      __syncwarp();
      cur = j;
    }
    const DevGeom& g = J.g;
    const long long nrays = (long long)g.views_used * g.C;
    const long long base = (long long)(t - J.tile0) * tile_rays;
    for (int r = lane; r < tile_rays; r += 32) {
      const long long ray = base + r;
      bool active = ray < nrays;
      float val = 0.0f;
      int nseg = 0;
      if (active) {
        const int v = (int)(ray / g.C);
        const int c = (int)(ray - (long long)v * g.C);
        RayAcc a;
        acc_init(a);
        Ray rr;
        if (ray_setup(g, J.cos_t[v], J.sin_t[v], J.px0[c], J.py0[c], rr)) {
          bool done = false;
          if (J.fast) done = walk_fast<M>(g, J.maps, rr, a);
          if (!done) {
            if (J.nexact > 0) active = false;  // listed: forward_lines_batch_kernel walks it
            else walk_exact<M>(g, J.maps, rr, a);
          }
        }
        if (active) {
          nseg = a.nseg;
          double L[8];
          finish_lines<M>(a, L, g.dens_div);
          val = spectral_compensated<M>(L, s_mu, s_pdf, J.NE);
          J.out[(size_t)v * g.width + g.start + c] = val;
        }
      }
      float vmax = warp_max(active ? val : 0.0f);
      float vmin = warp_min(active ? val : 3.0e38f);
      unsigned long long ns = warp_sum_ull((unsigned long long)nseg);
      if (lane == 0) {
        atomicMax(&J.stats->max_bits, __float_as_uint(vmax));
        atomicMin(&J.stats->min_bits, __float_as_uint(vmin));
        atomicAdd(&J.stats->segments, ns);
      }
    }
  }
}

// Statistics of every job back to their initial values.
__global__ void reset_stats_kernel(const FwdJob* __restrict__ jobs, int njobs) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  FwdStats* st = jobs[j].stats;
  st->max_bits = 0u;           // 0.0f
  st->min_bits = 0x7f7fffffu;  // FLT_MAX
  st->segments = 0ull;
}

template <int M>
static int launch_forward_batch_m(const FwdJob* d_jobs, int njobs, int tile_rays, unsigned int ntiles, int ne_max,
                                  int grid, unsigned int* d_counter, cudaStream_t st) {
  const size_t smem = kBatchWarps * batch_slot_doubles(ne_max, M) * sizeof(double);
  auto k = forward_batch_kernel<M>;
  VCT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<grid, kFwdThreads, smem, st>>>(d_jobs, njobs, tile_rays, ntiles, ne_max, d_counter);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

// The jobs' listed exact-walk rays (xfirst: prefix sums of their counts),
// a warp per ray, as forward_lines_kernel does for one slice.
template <int M>
__global__ void forward_lines_batch_kernel(const FwdJob* __restrict__ jobs, const unsigned int* __restrict__ xfirst,
                                           int n) {
  const unsigned int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= xfirst[n]) return;  // warp-uniform
  const int jx = batch_job_of(xfirst, n, w);
  const FwdJob& J = jobs[jx];
  const int lane = threadIdx.x & 31;
  const int ray = J.exact[w - xfirst[jx]];
  double L[8];
  int nseg;
  exact_lines_warp<M>(J.g, J.maps, J.cos_t, J.sin_t, J.px0, J.py0, ray, L, &nseg, lane);
  if (lane != 0) return;
  const int v = ray / J.g.C, c = ray - (ray / J.g.C) * J.g.C;
  const float val = spectral_compensated<M>(L, J.mu, J.pdf, J.NE);
  J.out[(size_t)v * J.g.width + J.g.start + c] = val;
  atomicMax(&J.stats->max_bits, __float_as_uint(val));
  atomicMin(&J.stats->min_bits, __float_as_uint(val));
  atomicAdd(&J.stats->segments, (unsigned long long)nseg);
}

int launch_forward_batch(const FwdJob* d_jobs, int njobs, int M, int tile_rays, unsigned int ntiles, int ne_max,
                         int grid, unsigned int* d_counter, const unsigned int* d_xfirst, unsigned int nexact_total,
                         cudaStream_t st) {
  if (tile_rays < 32 || tile_rays % 32) return fail(VCT_E_ARG, "batch: tile size must be a multiple of 32 rays");
  reset_stats_kernel<<<(njobs + 127) / 128, 128, 0, st>>>(d_jobs, njobs);
  VCT_CUDA(cudaGetLastError());
  VCT_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned int), st));
  int rc;
  switch (M) {
#define VCT_CASE(mm)                                                                                      \
  case mm:                                                                                                \
    if ((rc = launch_forward_batch_m<mm>(d_jobs, njobs, tile_rays, ntiles, ne_max, grid, d_counter, st))) \
      return rc;                                                                                          \
    if (nexact_total > 0) {                                                                               \
      forward_lines_batch_kernel<mm><<<(nexact_total + 3) / 4, 128, 0, st>>>(d_jobs, d_xfirst, njobs);    \
      VCT_CUDA(cudaGetLastError());                                                                       \
    }                                                                                                     \
    return VCT_OK;
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default: return fail(VCT_E_ARG, "number of materials must be 1..8");
  }
}

int forward_batch_occupancy(int M, int ne_max, int* blocks_per_sm) {
  const size_t smem = kBatchWarps * batch_slot_doubles(ne_max, M) * sizeof(double);
  cudaError_t e = cudaSuccess;
  switch (M) {
#define VCT_CASE(mm)                                                                                      \
  case mm:                                                                                                \
    e = cudaFuncSetAttribute(forward_batch_kernel<mm>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
    if (e == cudaSuccess)                                                                                 \
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, forward_batch_kernel<mm>, kFwdThreads, smem); \
    break;
    VCT_CASE(1) VCT_CASE(2) VCT_CASE(3) VCT_CASE(4) VCT_CASE(5) VCT_CASE(6) VCT_CASE(7) VCT_CASE(8)
#undef VCT_CASE
    default: return fail(VCT_E_ARG, "number of materials must be 1..8");
  }
  if (e != cudaSuccess) return cuda_fail(e, "forward_batch_occupancy");
  return VCT_OK;
}

// -------------------------------------------------- normalisation and noise
// MB/main.cpp:511-522 (divide by the float maximum) and gaussiannoise0
// (:51-76): p += sigma*z, p < 0 -> projection_min/10, p > 1 -> 1, with
// z = sqrt(-2 ln u1) sin(2 pi u2) (:46-49).  u1, u2 come from Philox4x32-10
// keyed by the 64-bit seed, counter (channel, view, 0, 0).
__device__ __forceinline__ void normalize_noise_elem(const float* __restrict__ in, float* __restrict__ out,
                                                     long long i, int W, const FwdStats* __restrict__ stats,
                                                     int pad_zero, double sigma, uint32_t k0, uint32_t k1) {
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

__global__ void normalize_noise_kernel(const float* __restrict__ in, float* __restrict__ out, int V,
                                       int W, const FwdStats* __restrict__ stats, int pad_zero,
                                       double sigma, uint32_t k0, uint32_t k1, long long i0, long long i1) {
  const long long i = i0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= i1) return;
  normalize_noise_elem(in, out, i, W, stats, pad_zero, sigma, k0, k1);
}

__global__ void normalize_noise_batch_kernel(const PostJob* __restrict__ jobs, const unsigned int* __restrict__ first,
                                             int n) {
  const int jx = batch_job_of(first, n, blockIdx.x);
  const PostJob& J = jobs[jx];
  const long long i = (long long)(blockIdx.x - first[jx]) * blockDim.x + threadIdx.x;
  if (i >= (long long)J.V * J.W) return;
  normalize_noise_elem(J.sino, J.sino, i, J.W, J.stats, J.pad_zero, J.sigma, J.key0, J.key1);
}

int launch_normalize_noise_batch(const PostJob* d_jobs, const unsigned int* d_first, int n, unsigned int nblocks,
                                 cudaStream_t st) {
  if (nblocks == 0) return VCT_OK;
  normalize_noise_batch_kernel<<<nblocks, 256, 0, st>>>(d_jobs, d_first, n);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

int launch_normalize_noise(const DevGeom& g, const float* d_in, float* d_out, const FwdStats* d_stats,
                           int pad_zero, double sigma, uint64_t seed, cudaStream_t st, int r0, int r1) {
  if (r1 < 0) r1 = g.views;
  if (r0 < 0 || r0 > r1 || r1 > g.views) return fail(VCT_E_ARG, "normalise: row range outside the sinogram");
  const long long i0 = (long long)r0 * g.width, i1 = (long long)r1 * g.width;
  const int threads = 256;
  const int blocks = (int)((i1 - i0 + threads - 1) / threads);
  if (blocks == 0) return VCT_OK;
  normalize_noise_kernel<<<blocks, threads, 0, st>>>(d_in, d_out, g.views, g.width, d_stats, pad_zero,
                                                     sigma, (uint32_t)seed, (uint32_t)(seed >> 32), i0, i1);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

VCT_BOUNDS_READER(bounds_forward)

}  // namespace vct
