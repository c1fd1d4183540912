// Ray walk of MB/reprojection_TOMO.cpp shared by the forward projector
// (vct_forward.cu) and its adjoint (vct_adjoint.cu).  Every translation unit
// that includes it is compiled with --fmad=false so both see the same
// floating-point decisions (segment boundaries, step counts, pixels).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "vct_internal.h"
#include "vct_philox.h"

namespace vct {

// Padded map: kMapPad cells on every side of the N x N grid.  Row/column -1
// repeats row/column 0 (the reference's (int) cast truncates a midpoint in
// (-1, 0) to pixel 0); every other border cell is 0 (rejected).
constexpr int kPad = kMapPad;
VCT_HD int pad_index(int col, int row, int N) { return (col + kPad) + (row + kPad) * (N + 2 * kPad); }

// Resident blocks per SM the register allocation is held to, and the number
// of walk segments whose gathers are issued together (chosen by measurement
// on the 512^2 slice with 800 x 609 rays: 2 / 4 / 5 / 6 / 8 / 12 segments gave
// 0.85 / 0.77 / 0.75 / 0.73 / 0.76 / 0.75 ms, with no spills).  Capping
// registers for 6 / 7 / 8 blocks per SM (small spills) gave 0.734 / 0.738 /
// 0.800 ms against 0.738 ms at 5: more resident warps do not help.  The cap
// of 5 blocks matters for 8 elements, where the compiler would otherwise take
// 102 registers, which the 256-register allocation unit rounds to 4 blocks
// (the 8-element 6 MV slice: 0.601 ms against 0.575 ms at 5).
#ifndef VCT_FWD_MINBLOCKS
#define VCT_FWD_MINBLOCKS 5
#endif
#ifndef VCT_FWD_UNROLL
#define VCT_FWD_UNROLL 6
#endif
// 1: a transposed copy of the padded map follows the row-major one; walks
// with x as the major axis read it.
#ifndef VCT_FWD_DUAL_LAYOUT
#define VCT_FWD_DUAL_LAYOUT 1
#endif

// ------------------------------------------------------------ host/device shims
// The walks are __host__ __device__ so the same code can run on the CPU
// (tests/host/walk_check.cu); these wrappers pick the device intrinsic or its
// host equivalent.
VCT_HD int4 ldg4(const int4* p) {
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}
VCT_HD double fma_rn(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}
VCT_HD int d2i_rz(double d) {
#if defined(__CUDA_ARCH__)
  return __double2int_rz(d);
#else
  return (int)d;
#endif
}
VCT_HD double dmul_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}

// (int)d as the reference's x86-64 build evaluates it (cvttsd2si): NaN and
// out-of-range values give INT_MIN, whereas the PTX conversion saturates and
// maps NaN to 0.  Only degenerate rays reach it, but it keeps the rejection of
// NaN segments identical.
VCT_HD int trunc_i32(double d) {
  return (d >= -2147483648.0 && d < 2147483648.0) ? d2i_rz(d) : (int)0x80000000;
}

VCT_HD unsigned int mat_of(const int4& w, int m) {
  const unsigned int u = (m >> 1) == 0 ? (unsigned)w.x : (m >> 1) == 1 ? (unsigned)w.y
                       : (m >> 1) == 2 ? (unsigned)w.z : (unsigned)w.w;
  return (m & 1) ? (u >> 16) : (u & 0xffffu);
}



// ----------------------------------------------------------------- accumulators
// Ld: sum s*len (cm) of segments emitted one by one (the exact walk, and the
// fast walk's first segment).  Lq: sum s*w_q of the fast walk's segments, w_q
// the segment's share of one major step in units of 2^-31; one major step is
// `sec` cm long.
struct RayAcc {
  double Ld[8];
  unsigned long long Lq[8];
  double sec;
  int nseg;
};

VCT_HD void acc_init(RayAcc& a) {
#pragma unroll
  for (int m = 0; m < 8; m++) {
    a.Ld[m] = 0.0;
    a.Lq[m] = 0ull;
  }
  a.sec = 0.0;
  a.nseg = 0;
}

// L_m in g/cm^2: densities are the stored values divided by `div` (1000, the
// reference's density x 1000, unless the context sets another scale).
template <int M>
VCT_HD void finish_lines(const RayAcc& a, double L[8], double div) {
#pragma unroll
  for (int m = 0; m < M; m++) {
    const double steps = (double)a.Lq[m] * (1.0 / 2147483648.0);
    L[m] = (a.Ld[m] + steps * a.sec) / div;
  }
}
template <int M>
VCT_HD void finish_lines(const RayAcc& a, double L[8]) {
  finish_lines<M>(a, L, 1000.0);
}

template <int M>
VCT_HD void gather_add_exact(const PixelRec* __restrict__ maps, int pix, double rr, RayAcc& a) {
  const int4 w = ldg4(reinterpret_cast<const int4*>(maps) + pix);
#pragma unroll
  for (int m = 0; m < M; m++) a.Ld[m] = fma_rn((double)mat_of(w, m), rr, a.Ld[m]);
  a.nseg++;
}

// Where the exact walk sends a segment: GatherSink adds it to a ray's line
// integrals (the forward projector); the adjoint passes a sink that scatters
// instead.  `pix` is the padded map index.
template <int M>
struct GatherSink {
  const PixelRec* __restrict__ maps;
  RayAcc* a;
  VCT_HD void operator()(int pix, double rr) const { gather_add_exact<M>(maps, pix, rr, *a); }
};

// Segment emission of MB/reprojection_TOMO.cpp:145-163 / :171-189: length,
// midpoint pixel (truncating casts), bounds test, then the sink.
template <class Sink>
VCT_HD void emit(const DevGeom& g, double xb0, double yb0, double xb1, double yb1, const Sink& sink) {
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
    sink(pad_index(xmc, ymc, g.N), rr);
  }
}

// The pixel (padded index, or -1 when rejected) and length of one segment
// under the emit() rule, without the gather; for geometries where the rmax
// test cannot fire.
VCT_HD int segment_pixel(const DevGeom& g, double xb0, double yb0, double xb1, double yb1, double* rr) {
  *rr = sqrt((xb0 - xb1) * (xb0 - xb1) + (yb0 - yb1) * (yb0 - yb1));
  const int xmc = trunc_i32((xb0 + xb1) * 0.5 / g.s + g.nxm);
  const int ymc = trunc_i32((-yb0 - yb1) * 0.5 / g.s + g.nxm);
  if (xmc >= 0 && ymc >= 0 && xmc <= g.N - 1 && ymc <= g.N - 1) return pad_index(xmc, ymc, g.N);
  return -1;
}

// -------------------------------------------------------------------- set-up
// Shared by both walks, MB/reprojection_TOMO.cpp:53-108: source, rotated
// detector point, intersections with the grid square, entry (xi,yi) and exit
// (xf,yf).  Returns false when the ray misses the square (the reference's walk
// loop is then never entered).
struct Ray {
  double sx, sy, px, py, xi, yi, xf, yf;
};

VCT_HD bool ray_setup(const DevGeom& g, double cb, double sb, double px0, double py0, Ray& r) {
  r.sx = g.sid * sb;            // :53
  r.sy = g.sid * cb;            // :54
  r.px = +px0 * cb + py0 * sb;  // :73
  r.py = -px0 * sb + py0 * cb;  // :74
  const double sx = r.sx, sy = r.sy, px = r.px, py = r.py, lim = g.lim;
  double xx0 = 0, yy0 = 0, xx1 = 0, yy1 = 0;
  int m = 0;
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
  if (m < 2) return false;
  if ((xx0 - sx) * (xx0 - sx) + (yy0 - sy) * (yy0 - sy) + 0.0 <
      (xx1 - sx) * (xx1 - sx) + (yy1 - sy) * (yy1 - sy) + 0.0) {
    r.xi = xx0; r.yi = yy0; r.xf = xx1; r.yf = yy1;
  } else {
    r.xi = xx1; r.yi = yy1; r.xf = xx0; r.yf = yy0;
  }
  return true;
}

// ---------------------------------------------------------------- exact walk
// The reference walk, operation for operation (:113-283).
template <class Sink>
VCT_HD void walk_exact_to(const DevGeom& g, const Ray& r, const Sink& sink) {
  const double sx = r.sx, sy = r.sy, px = r.px, py = r.py;
  const double xi = r.xi, yi = r.yi, xf = r.xf, yf = r.yf, lim = g.lim;
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
          emit(g, xb0, yb0, xiii, yiii, sink);
          xb0 = xiii;
          yb0 = yiii;
        }
      }
      emit(g, xb0, yb0, xii, yii, sink);
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
          emit(g, xb0, yb0, xiii, yiii, sink);
          xb0 = xiii;
          yb0 = yiii;
        }
      }
      emit(g, xb0, yb0, xii, yii, sink);
      xb0 = xii;
      yb0 = yii;
    }
  }
}

#if defined(__CUDACC__)
// walk_exact_to by a whole warp, for sinks whose result does not depend on
// the order of the segments (the adjoint's fixed-point scatter).  Step ik of
// the walk depends only on ik and on step ik - 1's point, so lane l takes the
// steps ik = 32 c + l of chunk c, gets step ik - 1's point from lane l - 1
// (or from the previous chunk), and emits the segments of its step exactly as
// the sequential loop does, with the same expressions.  A step runs while
// the points of all earlier steps are inside the square (a ballot per
// chunk), which is the sequential loop's test.  The major / minor roles of
// x and y are swapped for y-major rays; every expression keeps the
// reference's order of operations (:113-283).
template <class Sink>
__device__ void walk_exact_warp(const DevGeom& g, const Ray& r, const Sink& sink, int lane) {
  const double lim = g.lim, s = g.s;
  const bool xmaj = fabs(r.xi - r.xf) > fabs(r.yi - r.yf);
  const double su = xmaj ? r.sx : r.sy, sw = xmaj ? r.sy : r.sx;
  const double pu = xmaj ? r.px : r.py, pw = xmaj ? r.py : r.px;
  const double ui = xmaj ? r.xi : r.yi, uf = xmaj ? r.xf : r.yf;
  const double wi = xmaj ? r.yi : r.xi, wf = xmaj ? r.yf : r.xf;
  const double pha = (uf - ui) / fabs(ui - uf);
  int uin;
  if ((ui < 0 && (uf - ui) < 0) || (ui > 0 && (uf - ui) > 0))
    uin = trunc_i32((double)trunc_i32(ui) + (uf - ui) / fabs(uf - ui));
  else
    uin = trunc_i32(ui);
  const double wdir = (wf - wi) / fabs(wf - wi);
  const int max_steps = 4 * g.N + 64;
  auto emit_uw = [&](double u0, double w0, double u1, double w1) {
    if (xmaj) emit(g, u0, w0, u1, w1, sink);
    else emit(g, w0, u0, w1, u1, sink);
  };
  double cu = 0.0, cw = 0.0;  // step ik - 1's point for lane 0 (previous chunk's lane 31)
  int cwm = 0;
  for (int base = 0; base < max_steps; base += 32) {
    const int ik = base + lane;
    const double u = uin + pha * ik * s;
    const double w = (u - su) / (pu - su) * (pw - sw) + sw;
    const int wm = trunc_i32(w / s);
    double up = __shfl_up_sync(0xffffffffu, u, 1), wp = __shfl_up_sync(0xffffffffu, w, 1);
    int wmp = __shfl_up_sync(0xffffffffu, wm, 1);
    if (lane == 0) {
      up = cu;
      wp = cw;
      wmp = cwm;
    }
    // the state the loop tests before step ik: step ik - 1's point, or for
    // ik = 0 the first point, which equals step 0's
    const bool in = ik == 0 ? (u <= lim && u >= -lim && w <= lim && w >= -lim)
                            : (up <= lim && up >= -lim && wp <= lim && wp >= -lim);
    const unsigned int stop = __ballot_sync(0xffffffffu, !(in && ik < max_steps));
    const int nrun = stop ? __ffs(stop) - 1 : 32;
    if (lane < nrun) {
      double ub = ik == 0 ? ui : up, wb = ik == 0 ? wi : wp;  // segment start
      if (ik != 0 && (wm != wmp || (w / fabs(w) != wp / fabs(wp)))) {
        double wiii;
        if ((w < 0 && (wf - wi) < 0) || (w > 0 && (wf - wi) > 0))
          wiii = (double)(wm * s);
        else
          wiii = (double)(wm * s) - wdir * s;
        const double uiii = (wiii - sw) / (pw - sw) * (pu - su) + su;
        const double chy = (u - uiii) * (u - uiii) + (w - wiii) * (w - wiii);
        if (chy != 0) {
          emit_uw(ub, wb, uiii, wiii);
          ub = uiii;
          wb = wiii;
        }
      }
      emit_uw(ub, wb, u, w);
    }
    if (nrun < 32) break;
    cu = __shfl_sync(0xffffffffu, u, 31);
    cw = __shfl_sync(0xffffffffu, w, 31);
    cwm = __shfl_sync(0xffffffffu, wm, 31);
  }
}
#endif

#if defined(__CUDACC__)
// The line integrals L[0..M) (g/cm^2) and segment count of one ray of the
// exact walk, by a whole warp: walk_exact_warp with the gather sink, each
// lane's segment sums then added over the warp in a fixed order.  The same
// segments as walk_exact in one thread, the FP64 sum in another order;
// deterministic.  Every lane gets the result; every lane must call this.
template <int M>
__device__ void exact_lines_warp(const DevGeom& g, const PixelRec* __restrict__ maps, const double* __restrict__ cos_t,
                                 const double* __restrict__ sin_t, const double* __restrict__ det_px0,
                                 const double* __restrict__ det_py0, int ray, double L[8], int* nseg, int lane) {
  const int v = ray / g.C, c = ray - (ray / g.C) * g.C;
  RayAcc t;
  acc_init(t);
  Ray r;
  if (ray_setup(g, cos_t[v], sin_t[v], det_px0[c], det_py0[c], r))  // the same for every lane
    walk_exact_warp(g, r, GatherSink<M>{maps, &t}, lane);
#pragma unroll
  for (int m = 0; m < M; m++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t.Ld[m] += __shfl_xor_sync(0xffffffffu, t.Ld[m], o);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t.nseg += __shfl_xor_sync(0xffffffffu, t.nseg, o);
  finish_lines<M>(t, L, g.dens_div);
  *nseg = t.nseg;
}
#endif

template <int M>
VCT_HD void walk_exact(const DevGeom& g, const PixelRec* __restrict__ maps, const Ray& r, RayAcc& a) {
  walk_exact_to(g, r, GatherSink<M>{maps, &a});
}

// ------------------------------------------------------------------ fast walk
// The same segments as walk_exact:
//   - the first, lumped segment (entry point to the first major gridline,
//     :118-121 / :206-209) is emitted exactly;
//   - the reference then walks whole major steps u_k = uin + pha*k*s until a
//     step ends outside the square (:125 / :212), splitting a step where the
//     minor coordinate crosses a gridline (:134 / :221).  Here the number of
//     steps K is found once, with the reference's own expressions, and the
//     steps are walked as a Siddon event loop in units of major steps t:
//     major events at integer t, minor events at t_min, t_min + dt, ...;
//     every iteration closes one segment [t, min(next events)] and adds
//     s * w_q, w_q = its length in 2^-31 steps (event times in integer
//     fixed point).
// When uin/s is an integer, every major step spans exactly one pixel column
// and every piece between events lies inside one pixel, so the reference's
// midpoint rule picks the same pixel as the event bookkeeping.  Rays it does
// not cover return false and take walk_exact: uin/s not an integer (pixel
// sizes that do not divide 1 cm), a minor direction with no slope, and rays
// through the grid origin (the central channel of an even channel count):
// there the minor coordinate can be exactly 0 at a major step, the
// reference's sign test divides 0/0 and its crossing rule adds a backward
// piece, which walk_exact reproduces.
// The plan of a fast walk: everything the event loop needs, found from the
// ray alone (no map access).  The adjoint reads the same plan to know which
// cells a ray's walk covers.
struct FastPlan {
  int status;       // kPlanWalk, kPlanEmpty (no segment at all) or kPlanExact
  int xmaj;         // 1: x is the major axis
  int K;            // major steps walked (1..K)
  int maj0, majK;   // major cell index of step 1 and of step K (-1..N)
  int min0;         // minor cell index at step 1
  int dirw;         // minor index direction of travel in map-row/column terms
  int pha_pos;      // 1: the major coordinate increases along the ray
  int pix_lumped;   // padded index of the lumped first segment, -1 if rejected
  double rr_first;  // its length (cm)
  double sec;       // length of one major step (cm)
  double tmin0, dt; // first minor event and event spacing, in steps
};
constexpr int kPlanWalk = 0;
constexpr int kPlanEmpty = 1;
constexpr int kPlanExact = -1;

VCT_HD void fast_plan(const DevGeom& g, const Ray& r, FastPlan& p) {
  p.status = kPlanExact;
  const double orig = r.sx * r.py - r.sy * r.px;
  if (fabs(orig) < 1e-9 * (fabs(r.px - r.sx) + fabs(r.py - r.sy))) return;
  const bool xmaj = fabs(r.xi - r.xf) > fabs(r.yi - r.yf);
  const double ui = xmaj ? r.xi : r.yi, uf = xmaj ? r.xf : r.yf;
  const double su = xmaj ? r.sx : r.sy, sw = xmaj ? r.sy : r.sx;
  const double pu = xmaj ? r.px : r.py, pw = xmaj ? r.py : r.px;
  const double pha = (uf - ui) / fabs(ui - uf);
  int uin;
  if ((ui < 0 && (uf - ui) < 0) || (ui > 0 && (uf - ui) > 0))
    uin = trunc_i32((double)trunc_i32(ui) + (uf - ui) / fabs(uf - ui));
  else
    uin = trunc_i32(ui);
  const double s = g.s, lim = g.lim;
  const double Ua_d = (double)uin / s;
  const double Ua_r = rint(Ua_d);
  const double Wb = pha * ((pw - sw) / (pu - su));  // minor advance per step, pixels
  if (fabs(Ua_d - Ua_r) > 1e-6 || !(Wb != 0.0)) return;
  const int N = g.N, n = g.nxm;
  // First point (:120-121 / :208-209) and the loop's entry test (:125).
  const double u0 = (double)uin;
  const double w0 = (u0 - su) / (pu - su) * (pw - sw) + sw;
  if (!(u0 <= lim && u0 >= -lim && w0 <= lim && w0 >= -lim)) {
    p.status = kPlanEmpty;
    return;
  }

  // K: the first step whose end point is outside the square, evaluated with
  // the reference's expressions near the estimated exit (the walk processes
  // steps 1..K).
  const double W0 = w0 / s;
  int K = -1;
  {
    const double ku = (pha > 0 ? (lim - u0) : (u0 + lim)) / s;  // steps until |u| = lim
    const double kw = (Wb > 0 ? ((double)n - W0) : (W0 + (double)n)) / fabs(Wb);
    int k = (int)fmin(fmin(ku, kw), (double)(4 * N + 64)) - 1;
    if (k < 1) k = 1;
    for (int it = 0; it < 8; it++, k++) {
      const double u = uin + pha * k * s;
      const double w = (u - su) / (pu - su) * (pw - sw) + sw;
      if (!(u <= lim && u >= -lim && w <= lim && w >= -lim)) {
        K = k;
        break;
      }
    }
  }
  if (K < 1) return;

  const int Ua = (int)Ua_r;
  // Pixel of step 1: major floor index (midpoint at Ua + pha/2 pixels), minor
  // cell (lo, lo+1) holding W0 in the direction of travel.
  const int dirw = Wb > 0 ? 1 : -1;
  const double gd = dirw > 0 ? floor(W0) + 1.0 : ceil(W0) - 1.0;  // first minor gridline ahead
  const int lo = (int)(dirw > 0 ? gd - 1.0 : gd);
  const double dt = 1.0 / fabs(Wb);  // steps between minor gridlines
  const double tmin0 = (gd - W0) / Wb;
  // Index range check: the major index moves K-1 times, the minor index once
  // per minor event before K; both must end within one cell of the grid
  // (the padded border), else the exact walk takes the ray.
  const int nmin = tmin0 < (double)K ? (int)(((double)K - tmin0) / dt) + 1 : 0;
  int maj0, majK, min0, minK;
  if (xmaj) {
    maj0 = Ua + n + (pha > 0 ? 0 : -1);  // column: floor(Ua + pha/2 + n)
    majK = maj0 + (pha > 0 ? 1 : -1) * (K - 1);
    min0 = n - lo - 1;                   // row: floor(n - Wmid)
    minK = min0 - dirw * nmin;
  } else {
    maj0 = n - Ua + (pha > 0 ? -1 : 0);  // row: floor(n - (Ua + pha/2))
    majK = maj0 + (pha > 0 ? -1 : 1) * (K - 1);
    min0 = lo + n;                       // column: floor(Wmid + n)
    minK = min0 + dirw * nmin;
  }
  if (maj0 < -1 || maj0 > N || majK < -1 || majK > N || min0 < -1 || min0 > N || minK < -1 || minK > N)
    return;

  // The lumped first segment (entry point to the first major gridline).
  p.pix_lumped = xmaj ? segment_pixel(g, r.xi, r.yi, u0, w0, &p.rr_first)
                      : segment_pixel(g, r.xi, r.yi, w0, u0, &p.rr_first);
  p.status = kPlanWalk;
  p.xmaj = xmaj;
  p.K = K;
  p.maj0 = maj0;
  p.majK = majK;
  p.min0 = min0;
  p.dirw = dirw;
  p.pha_pos = pha > 0;
  p.sec = s * sqrt(1.0 + Wb * Wb);
  p.tmin0 = tmin0;
  p.dt = dt;
}

// Fixed-point accumulation of one segment, two elements per 32-bit record
// word u = s_lo | s_hi << 16: P += u * w adds s_lo * w + 2^16 * s_hi * w and
// H += s_hi * w, so sum(s_lo * w) = P - 2^16 * H modulo 2^64, which is exact
// because that sum itself fits in 64 bits (three integer instructions per
// pair instead of four).  A word with one element in use takes its low half.
template <int M>
VCT_HD void acc_words(const int4& w, unsigned int q, unsigned long long* P, unsigned long long* H) {
#pragma unroll
  for (int i = 0; i < (M + 1) / 2; i++) {
    const unsigned int u = i == 0 ? (unsigned)w.x : i == 1 ? (unsigned)w.y : i == 2 ? (unsigned)w.z : (unsigned)w.w;
    if (2 * i + 1 < M) {
      P[i] += (unsigned long long)u * q;
      H[i] += (unsigned long long)(u >> 16) * q;
    } else {
      P[i] += (unsigned long long)(u & 0xffffu) * q;
    }
  }
}

// State of one ray's fast walk from fast_begin to fast_end.  Event times are
// in fixed point, so the loop runs on the integer pipes:
//   kh  = k << 12, k the next major event (an integer step, 1..K);
//   T   = the next minor event in units of 2^-44 steps, 64 bits (its high
//         word is in units of 2^-12 steps, so k is due first iff kh <= T.hi);
//   t31 = the current time in units of 2^-31 steps, modulo 2^32.
// A segment's weight is the difference of its end and start times in 2^-31
// steps (0..2^31), so the weights of a ray add up to exactly K steps.  Minor
// events advance by DT = dt * 2^44 rounded (2^-45 steps per event at most;
// the reference's own crossing points are found afresh per step).
template <int M>
struct FastWalk {
  static constexpr int kWords = (M + 1) / 2;
  const int4* m4;         // the layout walked (row-major, or transposed for x-major rays)
  int P2;                 // P * P: padded indices are below it
  int pix, dpix_maj, dpix_min, pix_first;
  unsigned long long T, DT;
  unsigned int kh, kend, t31;
  int it, it_max, nseg;
  int pix_lumped;         // the lumped first segment (entry to the first major gridline)
  double rr_first;
  unsigned long long accP[kWords], accH[kWords];
};

// Every iteration closes kFastUnroll segments.  The event logic does not
// depend on the map, so the segments are laid out first and their gathers
// issued together before any is consumed.
constexpr int kFastUnroll = VCT_FWD_UNROLL;

// Sets up the event loop of a ray whose plan is kPlanWalk.
template <int M>
VCT_HD void fast_begin(const DevGeom& g, const PixelRec* __restrict__ maps, const FastPlan& pl, FastWalk<M>& w) {
  const int N = g.N;
  const int xmaj = pl.xmaj, maj0 = pl.maj0, min0 = pl.min0, dirw = pl.dirw;
  const int P = N + 2 * kPad;
  const PixelRec* __restrict__ mp = maps;
  if (xmaj && VCT_FWD_DUAL_LAYOUT) {
    // transposed copy: (col, row) at (col + kPad) * P + (row + kPad)
    mp = maps + (size_t)P * P;
    w.pix = (maj0 + kPad) * P + (min0 + kPad);
    w.dpix_maj = (pl.pha_pos ? 1 : -1) * P;
    w.dpix_min = -dirw;
  } else if (xmaj) {
    w.pix = pad_index(maj0, min0, N);
    w.dpix_maj = pl.pha_pos ? 1 : -1;
    w.dpix_min = -dirw * P;
  } else {
    w.pix = pad_index(min0, maj0, N);
    w.dpix_maj = (pl.pha_pos ? -1 : 1) * P;
    w.dpix_min = dirw;
  }
  w.pix_first = w.pix;
  w.P2 = P * P;
  w.m4 = reinterpret_cast<const int4*>(mp);
  // Times beyond 2^18 steps (past every walk's end) are clamped there.
  const double kTcap = 262144.0;  // 2^18 steps
  w.T = (unsigned long long)dmul_rn(fmin(pl.tmin0, kTcap), 17592186044416.0);  // 2^44
  w.DT = (unsigned long long)dmul_rn(fmin(pl.dt, kTcap), 17592186044416.0);
  w.kh = 1u << 12;                          // next major event: step 1
  w.kend = (unsigned int)pl.K << 12;        // the last major event, step K
  w.t31 = 0u;
  w.it = 0;
  w.it_max = (8 * N + 128) / kFastUnroll;
  w.nseg = 0;
  w.pix_lumped = pl.pix_lumped;
  w.rr_first = pl.rr_first;
#pragma unroll
  for (int i = 0; i < FastWalk<M>::kWords; i++) w.accP[i] = w.accH[i] = 0ull;
}

// Bulk iterations carry no per-slot end test.  A segment ends at the next
// major event at the latest, so the next major event advances by at most one
// step per segment: while k + kFastUnroll - 1 <= K every slot of the
// iteration starts before step K.  The integer sums do not depend on how the
// segments are grouped, so the result is the same as the checked loop's.
template <int M>
VCT_HD bool fast_bulk_ok(const FastWalk<M>& w) {
  constexpr unsigned int kSpan = (unsigned int)(kFastUnroll - 1) << 12;
  return w.it < w.it_max && w.kend >= kSpan && w.kh <= w.kend - kSpan;
}

template <int M>
VCT_HD void fast_layout_bulk(FastWalk<M>& w, int px[kFastUnroll], unsigned int wq[kFastUnroll]) {
#pragma unroll
  for (int u = 0; u < kFastUnroll; u++) {
    const bool mj = w.kh <= (unsigned int)(w.T >> 32);
    const unsigned int e31 = mj ? w.kh << 19 : (unsigned int)(w.T >> 13);
    wq[u] = e31 - w.t31;
    px[u] = w.pix;
    w.t31 = e31;
    if (mj) w.kh += 1u << 12;
    else w.T += w.DT;
    w.pix += mj ? w.dpix_maj : w.dpix_min;
  }
  w.nseg += kFastUnroll;
  w.it++;
}

// The last iterations, each slot tested against the end: a slot is live
// while major event K has not been passed.  Past the end, slots repeat the
// first segment's pixel with weight 0; the indices stay inside the padded
// border because the walk ends within one step of the square.
template <int M>
VCT_HD void fast_layout_checked(FastWalk<M>& w, int px[kFastUnroll], unsigned int wq[kFastUnroll]) {
#pragma unroll
  for (int u = 0; u < kFastUnroll; u++) {
    const bool live = w.kh <= w.kend;
    const bool mj = w.kh <= (unsigned int)(w.T >> 32);
    const unsigned int e31 = mj ? w.kh << 19 : (unsigned int)(w.T >> 13);
    wq[u] = live ? e31 - w.t31 : 0u;
    px[u] = live ? w.pix : w.pix_first;
    w.nseg += live;
    if (live) {
      w.t31 = e31;
      if (mj) w.kh += 1u << 12;
      else w.T += w.DT;
      w.pix += mj ? w.dpix_maj : w.dpix_min;
    }
  }
  w.it++;
}

// The records of the laid-out segments, all loads issued before any is used.
template <int M>
VCT_HD void fast_load(const FastWalk<M>& w, const int px[kFastUnroll], int4 wv[kFastUnroll]) {
#pragma unroll
  for (int u = 0; u < kFastUnroll; u++)
    wv[u] = VCT_INDEX_OK(px[u] >= 0 && px[u] < w.P2) ? ldg4(w.m4 + px[u]) : make_int4(0, 0, 0, 0);
}

template <int M>
VCT_HD void fast_acc(FastWalk<M>& w, const int4 wv[kFastUnroll], const unsigned int wq[kFastUnroll]) {
#pragma unroll
  for (int u = 0; u < kFastUnroll; u++) acc_words<M>(wv[u], wq[u], w.accP, w.accH);
}

// Walks what is left of the ray and adds its sums and the lumped first
// segment to the ray's accumulator.
template <int M>
VCT_HD void fast_end(const PixelRec* __restrict__ maps, FastWalk<M>& w, RayAcc& a) {
  while (fast_bulk_ok(w)) {
    int px[kFastUnroll];
    unsigned int wq[kFastUnroll];
    int4 wv[kFastUnroll];
    fast_layout_bulk(w, px, wq);
    fast_load(w, px, wv);
    fast_acc(w, wv, wq);
  }
  while (w.it < w.it_max && w.kh <= w.kend) {
    int px[kFastUnroll];
    unsigned int wq[kFastUnroll];
    int4 wv[kFastUnroll];
    fast_layout_checked(w, px, wq);
    fast_load(w, px, wv);
    fast_acc(w, wv, wq);
  }
#pragma unroll
  for (int i = 0; i < FastWalk<M>::kWords; i++) {
    a.Lq[2 * i] += w.accP[i] - (w.accH[i] << 16);
    if (2 * i + 1 < M) a.Lq[2 * i + 1] += w.accH[i];
  }
  a.nseg += w.nseg;
  if (w.pix_lumped >= 0 && VCT_INDEX_OK(w.pix_lumped < w.P2)) gather_add_exact<M>(maps, w.pix_lumped, w.rr_first, a);
}

// Returns false when the ray needs the exact walk.
template <int M>
VCT_HD bool walk_fast(const DevGeom& g, const PixelRec* __restrict__ maps, const Ray& r, RayAcc& a) {
  FastPlan pl;
  fast_plan(g, r, pl);
  if (pl.status == kPlanExact) return false;
  if (pl.status == kPlanEmpty) return true;
  a.sec = pl.sec;
  FastWalk<M> w;
  fast_begin(g, maps, pl, w);
  fast_end(maps, w, a);
  return true;
}

}  // namespace vct
