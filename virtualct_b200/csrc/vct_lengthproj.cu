// lengthproj_TOMO (MB/lengthproj_TOMO.cpp:14-185) on sm_100a: for every pixel
// of the reconstruction mask, npf = sum over the views used of
// (float)(lerp(proj, dj) * rr), accumulated in float in view order, where rr
// is the pixel-width chord of the line from the source to the pixel centre
// and dj the channel where that line meets the curved detector.  One thread
// per pixel, the views in order; the geometry in FP64 (compiled with
// --fmad=false, as the reference's x86-64 build rounds every operation), so
// the per-view terms follow the reference's expressions.  The side tables
// the reference writes (chord and detector position per pixel and view,
// [N][N][V] floats each) are not kept: every term is recomputed.
// lengthproj_TOMO_2 (:188-276, the iterative step) reads those tables back
// for every `stride`-th view from `first` on; with round_tables the chord and
// the channel are rounded to float, as the tables store them.
#include <cuda_runtime.h>
#include <math.h>

#include "vct_internal.h"

namespace vct {

__global__ void lengthproj_kernel(LpGeom q, const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                                  const float* __restrict__ proj, float* __restrict__ npf) {
  const int jx = blockIdx.x * blockDim.x + threadIdx.x;
  const int jy = blockIdx.y;
  const int N = q.N;
  if (jx >= N) return;
  // reconstruction mask, MB/misc_TOMO.cpp:10-39
  const double r = (double)(N - 1) / 2.0;
  if (!(((double)jy - r) * ((double)jy - r) + ((double)jx - r) * ((double)jx - r) <= r * r)) {
    npf[(size_t)jy * N + jx] = 0.0f;
    return;
  }
  const double s = q.s;
  const double ry = N * s * 0.5 - (jy + 0.5) * s;
  const double rx = -N * s * 0.5 + (jx + 0.5) * s;
  float acc = 0.0f;
  for (int k = 0; k < q.count; k++) {
    const int row_k = q.first + k * q.stride;  // sinogram row (j_one)
    int v = q.start + row_k - q.nrot * q.V;
    if (v >= q.V) v -= q.V;
    if (v < 0) v += q.V;  // the reference reads its tables out of range here
    if (!VCT_INDEX_OK(v >= 0 && v < q.V)) continue;
    const double cb = cos_t[v], sb = sin_t[v];
    const double sx = q.sid * sb, sy = q.sid * cb;
    double len;
    if (fabs(rx - sx) > fabs(ry - sy)) {
      const double x0 = rx - 0.5 * s, x1 = rx + 0.5 * s;
      const double y0 = (x0 - sx) / (rx - sx) * (ry - sy) + sy;
      const double y1 = (x1 - sx) / (rx - sx) * (ry - sy) + sy;
      len = sqrt((x0 - x1) * (x0 - x1) + (y0 - y1) * (y0 - y1));
    } else {
      // y-major: the reference evaluates both ends of x at y0, leaving only
      // the pixel's y extent (:95-101)
      const double y0 = ry - 0.5 * s, y1 = ry + 0.5 * s;
      len = sqrt((y0 - y1) * (y0 - y1));
    }
    // the line meets the detector circle (centre on the source, radius R):
    // the root nearer the origin (:110-134)
    const double dx = q.dsrc * sb, dy = q.dsrc * cb;
    const double a = (sy - ry) / (sx - rx);
    const double b = -sx * (sy - ry) / (sx - rx) + sy;
    const double qa = 1.0 + a * a;
    const double qb = 2.0 * a * b - 2.0 * a * dy - 2.0 * dx;
    const double qc = dx * dx + b * b + dy * dy - 2.0 * b * dy - q.R * q.R;
    const double disc = sqrt(qb * qb - 4.0 * qa * qc);
    const double x1 = (-qb + disc) / (2.0 * qa), y1 = a * x1 + b;
    const double x2 = (-qb - disc) / (2.0 * qa), y2 = a * x2 + b;
    double px, py;
    if (x1 * x1 + y1 * y1 > x2 * x2 + y2 * y2) {
      px = x2;
      py = y2;
    } else {
      px = x1;
      py = y1;
    }
    // angle along the detector from its centre point (:136-150)
    const double ox = -q.diso * sb, oy = -q.diso * cb;
    const double d2 = (px - ox) * (px - ox) + (py - oy) * (py - oy);
    const double ang = acos(1.0 - d2 / (2.0 * q.R * q.R));
    const double rpx = px * cb - py * sb;
    double dj = rpx > 0.0 ? q.iso - ang / q.dalpha : q.iso + ang / q.dalpha;
    if (q.round_tables) {
      len = (double)(float)len;
      dj = (double)(float)dj;
    }
    const float* row = proj + (size_t)row_k * q.W;
    // three explicit tests, as :158-172 (a NaN channel adds nothing)
    if (q.start_ch <= dj && dj < q.end_ch - 1) {
      const int ij = (int)dj;
      if (!VCT_INDEX_OK(ij >= 0 && ij + 1 < q.W)) continue;
      const double f = dj - (double)ij;
      acc += (float)(((1.0 - f) * row[ij] + f * row[ij + 1]) * len);
    } else if (q.start_ch > dj) {
      acc += (float)(row[q.start_ch] * len);
    } else if (dj >= q.end_ch - 1) {
      acc += (float)(row[q.end_ch - 1] * len);
    }
  }
  npf[(size_t)jy * N + jx] = acc;
}

// The same sum for the square grid's quarter-turn orbits (N even, every view
// used, V % 4 == 0): pixel (x, y) in view v sees the geometry of pixel
// (N-1-y, x) in view v + V/4 (and so on round the orbit), so the line's
// detector channel dj -- the divisions, square roots and arccosine -- is
// computed once per (orbit, view) and serves four (pixel, view) terms.  The
// chord is not invariant: the reference takes the pixel's x extent along the
// line when |dx| > |dy| and its bare y extent otherwise (:95-101), and a
// quarter turn swaps dx and dy, so each term's chord is evaluated with its
// own pixel and view, as the reference does (near |dx| = |dy| the rounding
// decides, and the two chords differ by up to sqrt(2)).  Each pixel's float
// sum runs over its views from a different first view (a cyclic shift of the
// reference's order).
__global__ void lengthproj_sym_kernel(LpGeom q, const double* __restrict__ cos_t, const double* __restrict__ sin_t,
                                      const float* __restrict__ proj, float* __restrict__ npf) {
  const int N = q.N, H = N / 2, V = q.V, V4 = V / 4;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= H) return;
  const int px[4] = {x, N - 1 - y, N - 1 - x, y};
  const int py[4] = {y, x, N - 1 - y, N - 1 - x};
  // reconstruction mask, MB/misc_TOMO.cpp:10-39 (invariant under the turn)
  const double r = (double)(N - 1) / 2.0;
  if (!(((double)y - r) * ((double)y - r) + ((double)x - r) * ((double)x - r) <= r * r)) {
#pragma unroll
    for (int k = 0; k < 4; k++) npf[(size_t)py[k] * N + px[k]] = 0.0f;
    return;
  }
  const double s = q.s;
  double rxt[4], ryt[4];
#pragma unroll
  for (int t = 0; t < 4; t++) {
    ryt[t] = N * s * 0.5 - (py[t] + 0.5) * s;
    rxt[t] = -N * s * 0.5 + (px[t] + 0.5) * s;
  }
  const double rx = rxt[0], ry = ryt[0];
  const double inv_2r2 = 1.0 / (2.0 * q.R * q.R), inv_dalpha = 1.0 / q.dalpha;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int k = 0; k < V; k++) {  // row k of the base pixel; rows k + j V/4 of the turned ones
    int v = q.start + k - q.nrot * V;
    if (v >= V) v -= V;
    if (v < 0) v += V;
    if (!VCT_INDEX_OK(v >= 0 && v < V)) continue;
    const double cb = cos_t[v], sb = sin_t[v];
    const double sx = q.sid * sb, sy = q.sid * cb;
    // the reference's intersection (:110-134), its divisions taken as
    // reciprocals (the sum's 1e-5 budget is far above the rounding this moves)
    const double dx = q.dsrc * sb, dy = q.dsrc * cb;
    const double a = (sy - ry) / (sx - rx);
    const double b = -sx * a + sy;
    const double qa = 1.0 + a * a;
    const double qb = 2.0 * a * b - 2.0 * a * dy - 2.0 * dx;
    const double qc = dx * dx + b * b + dy * dy - 2.0 * b * dy - q.R * q.R;
    const double disc = sqrt(qb * qb - 4.0 * qa * qc);
    const double i2qa = 0.5 / qa;
    const double x1 = (-qb + disc) * i2qa, y1 = a * x1 + b;
    const double x2 = (-qb - disc) * i2qa, y2 = a * x2 + b;
    double pxd, pyd;
    if (x1 * x1 + y1 * y1 > x2 * x2 + y2 * y2) {
      pxd = x2;
      pyd = y2;
    } else {
      pxd = x1;
      pyd = y1;
    }
    const double ox = -q.diso * sb, oy = -q.diso * cb;
    const double d2 = (pxd - ox) * (pxd - ox) + (pyd - oy) * (pyd - oy);
    const double ang = acos(1.0 - d2 * inv_2r2);
    const double rpx = pxd * cb - pyd * sb;
    const double dj = rpx > 0.0 ? q.iso - ang * inv_dalpha : q.iso + ang * inv_dalpha;
    // the interpolation at dj, as lengthproj_kernel (:158-172)
    int ij = -1;
    double f = 0.0;
    int edge = -1;
    if (q.start_ch <= dj && dj < q.end_ch - 1) {
      ij = (int)dj;
      f = dj - (double)ij;
    } else if (q.start_ch > dj) {
      edge = q.start_ch;
    } else if (dj >= q.end_ch - 1) {
      edge = q.end_ch - 1;
    } else {
      continue;  // a NaN channel adds nothing
    }
#pragma unroll
    for (int t = 0; t < 4; t++) {
      int row = k + t * V4;
      if (row >= V) row -= V;
      int vt = v + t * V4;
      if (vt >= V) vt -= V;
      // the chord of pixel t in its own view: the reference's branch test
      // with its own coordinates (:85-101), then s sqrt(1 + slope^2) for the
      // x extent along the line, or the bare y extent s
      double len = s;
      {
        const double ax = rxt[t] - q.sid * sin_t[vt], ay = ryt[t] - q.sid * cos_t[vt];
        if (fabs(ax) > fabs(ay)) {
          const double m = ay / ax;
          len = s * sqrt(1.0 + m * m);
        }
      }
      const float* pr = proj + (size_t)row * q.W;
      if (ij >= 0) {
        if (!VCT_INDEX_OK(ij + 1 < q.W)) continue;
        acc[t] += (float)(((1.0 - f) * pr[ij] + f * pr[ij + 1]) * len);
      } else {
        acc[t] += (float)(pr[edge] * len);
      }
    }
  }
#pragma unroll
  for (int t = 0; t < 4; t++) npf[(size_t)py[t] * N + px[t]] = acc[t];
}

int launch_lengthproj(const LpGeom& q, const double* d_cos, const double* d_sin, const float* d_proj, float* d_npf,
                      cudaStream_t st) {
  const bool sym = !q.round_tables && q.first == 0 && q.stride == 1 && q.count == q.V && q.V % 4 == 0 &&
                   q.N % 2 == 0 && q.N > 0;
  if (sym) {
    const int H = q.N / 2;
    dim3 grid((H + 127) / 128, H);
    lengthproj_sym_kernel<<<grid, 128, 0, st>>>(q, d_cos, d_sin, d_proj, d_npf);
  } else {
    dim3 grid((q.N + 127) / 128, q.N);
    lengthproj_kernel<<<grid, 128, 0, st>>>(q, d_cos, d_sin, d_proj, d_npf);
  }
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

VCT_BOUNDS_READER(bounds_lengthproj)

}  // namespace vct
