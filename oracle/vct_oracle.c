/*
 * vct_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of the reference's MBFPA forward projector, noise model and
 * fan-beam FBP (hagaakihiro/VirtualCT), used only to check the CUDA path.
 * See vct_oracle.h for the contract.  Reference citations are
 * "<dir>/<file>:<line>" with MB = Release_MBFPA_CPU_human and
 * FBP = Release_FBP_CPU.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include "vct_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* PI as the reference spells it (MB/physParamsTOMO.h:1): rounds to M_PI. */
#define ORC_PI 3.141592653589793238462643383279

void orc_geom_default(orc_geom* g) {
  g->start_channel = 0;
  g->end_channel = 609;
  g->iso_channel = 304.5;
  g->max_alpha = 0.326086956;
  g->max_beta = 0.326086956;
  g->sid = 85.0;
  g->det_radius = 142.6;
  g->det_src_iso = 85.0;
  g->views = 800;
  g->width = 609;
  g->recon_size = 512;
  g->pixel_cm = 0.1;
  g->xfactor = 1;
}

/* MB/projectionDataTOMO.cpp:362-368 and MB/misc_TOMO.cpp:93-97. */
void orc_trig_tables(int views, double start_view_deg, double* cos_t, double* sin_t) {
  for (int i = 0; i < views; i++) {
    double angle = (double)(360.0 / views * i);
    double rad = (start_view_deg + angle) * ORC_PI / 180.0;
    cos_t[i] = cos(rad);
    sin_t[i] = sin(rad);
  }
}

/* MB/prior_weight_production.cpp:191-244.  energy_mev receives the bin
 * centres as the reference stores them (a float, widened to double). */
int orc_spectrum(const char* path, int nthin, float* pdf, double* energy_mev, int cap) {
  FILE* fp = fopen(path, "r");
  if (!fp) return -1;
  char row[1024];
  float d0 = 0, d1 = 0, d2 = 0;
  double* pe = (double*)malloc(sizeof(double) * cap);
  float* raw = (float*)malloc(sizeof(float) * cap);
  int n = 0;
  if (fgets(row, sizeof(row), fp) == NULL) { /* header line (:196) */ }
  while (fgets(row, sizeof(row), fp) != NULL && n < cap) {
    /* A line sscanf cannot parse keeps the previous values, as at :202. */
    sscanf(row, "%f %f %f", &d0, &d1, &d2);
    pe[n] = (d1 + d0) * 0.5;
    raw[n] = d2;
    n++;
  }
  fclose(fp);
  /* Thinning (:210-235). */
  double psum = 0.0, esum = 0.0, sum_thin = 0.0;
  int nthin_out = 0;
  for (int i = 0; i < n; i++) {
    psum += raw[i];
    esum += pe[i];
    if (i - nthin + 1 == (i - nthin + 1) / nthin * nthin) {
      int k = (i - nthin + 1) / nthin;
      pdf[k] = (float)psum;
      energy_mev[k] = (double)(float)(esum / nthin);
      sum_thin += psum;
      psum = 0.0;
      esum = 0.0;
      nthin_out = k + 1;
    }
  }
  /* Normalisation in float (:229-244). */
  float sum = (float)sum_thin;
  for (int i = 0; i < nthin_out; i++) pdf[i] = pdf[i] / sum;
  free(pe);
  free(raw);
  return nthin_out;
}

/* MB/prior_weight_production.cpp:249-295 (photoelectric Z^3/E^3 term,
 * Klein-Nishina Compton term, pair term clamped at 0; Ek = 0). */
void orc_attenuation(const double* energy_mev, int NE, const double* ZZ, const double* AA, int M,
                     float* mu) {
  const double Avogadro = 6.0221; /* MB/physParamsTOMO.h:89 */
  double Ek = 0;
  for (int iz = 0; iz < M; iz++) {
    double Z = ZZ[iz], A = AA[iz];
    double fact = Avogadro * Z / A * (2.81794 * 2.81794) * 0.001;
    for (int i = 0; i < NE; i++) {
      double E = energy_mev[i] / 0.511;
      double photo = fact * 0.00000345 * (1.0 + 0.008 * Z) * (Z * Z * Z) / (E * E * E) *
                     (1.0 - Ek / (4.0 * E) - Ek * Ek / (1.21 * E));
      double compton = fact * 2 * ORC_PI *
                       ((1.0 + E) / (E * E) * (2.0 * (1.0 + E) / (1.0 + 2 * E) - log(1.0 + 2 * E) / E) +
                        log(1.0 + 2 * E) / (2 * E) - (1.0 + 3 * E) / ((1.0 + 2 * E) * (1.0 + 2 * E)));
      double pair = fact * 0.2545 * (E - 2.332) * Z / 137;
      if (pair < 0) pair = 0;
      mu[NE * iz + i] = (float)(photo + compton + pair);
    }
  }
}

/* One ray: MB/reprojection_TOMO.cpp:53-283, segment emission order kept. */
int orc_walk(const orc_geom* g, double cb, double sb, int jj, double* seg_len, int* seg_pix,
             double* seg_r, int cap) {
  const int N = g->recon_size;
  const double s = g->pixel_cm;
  const int nxm = (int)(N * 0.5); /* :25-26 */
  const int nym = (int)(N * 0.5);
  const int half = (g->end_channel - g->start_channel - 1) / 2; /* macro :57 */
  double sx = g->sid * sb;                                      /* :53 */
  double sy = g->sid * cb;                                      /* :54 */
  double theta = (g->iso_channel - jj) * g->max_alpha / half;   /* :61 */
  double ox0 = g->det_radius * sin(theta);                      /* :67 */
  double oy0 = -g->det_radius * cos(theta);                     /* :68 */
  double px0 = ox0;
  double py0 = oy0 + g->det_src_iso;      /* :71 */
  double px = +px0 * cb + py0 * sb;       /* :73 */
  double py = -px0 * sb + py0 * cb;       /* :74 */
  const double limx = (double)nxm * s, limy = (double)nym * s;
  double xx[4] = {0, 0, 0, 0}, yy[4] = {0, 0, 0, 0};
  int m = 0; /* grid-square intersections, :76-101 */
  yy[m] = (double)nym * s;
  if (fabs((yy[m] - sy) / (py - sy) * (px - sx) + sx) < limx) {
    xx[m] = (yy[m] - sy) / (py - sy) * (px - sx) + sx;
    m++;
  }
  yy[m] = -(double)nym * s;
  if (fabs((yy[m] - sy) / (py - sy) * (px - sx) + sx) < limx) {
    xx[m] = (yy[m] - sy) / (py - sy) * (px - sx) + sx;
    m++;
  }
  xx[m] = (double)nxm * s;
  if (fabs((xx[m] - sx) / (px - sx) * (py - sy) + sy) < limy) {
    yy[m] = (xx[m] - sx) / (px - sx) * (py - sy) + sy;
    m++;
  }
  xx[m] = -(double)nxm * s;
  if (fabs((xx[m] - sx) / (px - sx) * (py - sy) + sy) < limy) {
    yy[m] = (xx[m] - sx) / (px - sx) * (py - sy) + sy;
    m++;
  }
  /* A ray that misses the square leaves xx/yy[1] unset in the reference; its
   * walk loop is then never entered (no point of the line lies in the square),
   * so transp stays 0.  Reported here as zero segments. */
  if (m < 2) return 0;
  double xi, yi, xf, yf; /* :102-108 */
  if ((xx[0] - sx) * (xx[0] - sx) + (yy[0] - sy) * (yy[0] - sy) + 0.0 <
      (xx[1] - sx) * (xx[1] - sx) + (yy[1] - sy) * (yy[1] - sy) + 0.0) {
    xi = xx[0]; yi = yy[0]; xf = xx[1]; yf = yy[1];
  } else {
    xi = xx[1]; yi = yy[1]; xf = xx[0]; yf = yy[0];
  }
  double xb0 = xi, yb0 = yi, xb1, yb1, rr;
  double xii, yii, xiii = 0, yiii = 0, yj, xj;
  int n = 0;
#define ORC_EMIT()                                                                      \
  do {                                                                                  \
    rr = sqrt((xb0 - xb1) * (xb0 - xb1) + (yb0 - yb1) * (yb0 - yb1));                   \
    int xmc = (int)((xb0 + xb1) * 0.5 / s + nxm);                                      \
    int ymc = (int)((-yb0 - yb1) * 0.5 / s + nym);                                     \
    if (xmc >= 0 && ymc >= 0 && xmc <= N - 1 && ymc <= N - 1) {                         \
      if (n >= cap) return -1;                                                          \
      seg_len[n] = rr;                                                                  \
      seg_pix[n] = xmc + ymc * N;                                                       \
      seg_r[n] = sqrt((xb0 + xb1) * (xb0 + xb1) + (-yb0 - yb1) * (-yb0 - yb1)) * 0.5;    \
      n++;                                                                              \
    }                                                                                   \
  } while (0)

  if (fabs(xi - xf) > fabs(yi - yf)) { /* x-major walk, :113-200 */
    double pha = (xf - xi) / fabs(xi - xf);
    int xin, ik = 0, yma = 0, ymb;
    if ((xi < 0 && (xf - xi) < 0) || (xi > 0 && (xf - xi) > 0))
      xin = (int)((int)xi + (xf - xi) / fabs(xf - xi));
    else
      xin = (int)xi;
    xii = xin;
    yii = (xii - sx) / (px - sx) * (py - sy) + sy;
    while (xii <= limx && xii >= -limx && yii <= limy && yii >= -limy) {
      xii = xin + pha * ik * s;
      ymb = yma;
      yj = yii;
      yii = (xii - sx) / (px - sx) * (py - sy) + sy;
      yma = (int)(yii / s);
      int icheck = 0;
      double chy = 0;
      if ((ik != 0 && yma != ymb) || (ik != 0 && (yii / fabs(yii) != yj / fabs(yj)))) {
        if ((yii < 0 && (yf - yi) < 0) || (yii > 0 && (yf - yi) > 0))
          yiii = (double)(yma * s);
        else
          yiii = (double)(yma * s) - (yf - yi) / fabs(yf - yi) * s;
        xiii = (yiii - sy) / (py - sy) * (px - sx) + sx;
        chy = (xii - xiii) * (xii - xiii) + (yii - yiii) * (yii - yiii);
        icheck++;
      }
      if (icheck == 1 && chy != 0) {
        xb1 = xiii;
        yb1 = yiii;
        ORC_EMIT();
        xb0 = xb1;
        yb0 = yb1;
      }
      xb1 = xii;
      yb1 = yii;
      ORC_EMIT();
      xb0 = xb1;
      yb0 = yb1;
      ik++;
    }
  } else { /* y-major walk, :201-283 */
    double pha = (yf - yi) / fabs(yi - yf);
    int yin, ik = 0, xma = 0, xmb;
    if ((yi < 0 && (yf - yi) < 0) || (yi > 0 && (yf - yi) > 0))
      yin = (int)((int)yi + (yf - yi) / fabs(yf - yi));
    else
      yin = (int)yi;
    yii = yin;
    xii = (yii - sy) / (py - sy) * (px - sx) + sx;
    while (xii <= limx && xii >= -limx && yii <= limy && yii >= -limy) {
      yii = yin + pha * ik * s;
      xmb = xma;
      xj = xii;
      xii = (yii - sy) / (py - sy) * (px - sx) + sx;
      xma = (int)(xii / s);
      int icheck = 0;
      double chy = 0;
      if ((ik != 0 && xma != xmb) || (ik != 0 && (xii / fabs(xii) != xj / fabs(xj)))) {
        if ((xii < 0 && (xf - xi) < 0) || (xii > 0 && (xf - xi) > 0))
          xiii = (double)(xma * s);
        else
          xiii = (double)(xma * s) - (xf - xi) / fabs(xf - xi) * s;
        yiii = (xiii - sx) / (px - sx) * (py - sy) + sy;
        chy = (xii - xiii) * (xii - xiii) + (yii - yiii) * (yii - yiii);
        icheck++;
      }
      if (icheck == 1 && chy != 0) {
        xb1 = xiii;
        yb1 = yiii;
        ORC_EMIT();
        xb0 = xb1;
        yb0 = yb1;
      }
      xb1 = xii;
      yb1 = yii;
      ORC_EMIT();
      xb0 = xb1;
      yb0 = yb1;
      ik++;
    }
  }
#undef ORC_EMIT
  return n;
}

static int orc_seg_cap(const orc_geom* g) { return 4 * g->recon_size + 64; }

/* Density seen by one segment for material mat: the reference zeroes
 * material 0 in place and sets ph = 0 for other materials when the value is
 * negative or the midpoint radius (cm) reaches rmax = N/2 (a pixel count),
 * MB/reprojection_TOMO.cpp:150-156.  The in-place write only changes later
 * rays when r >= rmax can occur (pixel >= 0.707 cm); it is not reproduced. */
static inline float orc_rho_seen(const float* rho, size_t n2, int mat, int pix, double r,
                                 double rmax, double* ph) {
  float v = rho[(size_t)mat * n2 + pix];
  *ph = 1.0;
  if (mat == 0) {
    if (v < 0 || r >= rmax) v = 0;
  }
  if (v < 0 || r >= rmax) *ph = 0.0;
  return v;
}

void orc_forward_exact(const orc_geom* g, const double* cos_t, const double* sin_t, const float* rho,
                       int M, const float* mu, const float* pdf, int NE, float* full_out,
                       int* nseg_out, int nthreads) {
  const int V = g->views, W = g->width, N = g->recon_size;
  const int nviews = V / 2 * 2; /* end_angle_num, MB/reprojection_TOMO.cpp:35 */
  const size_t n2 = (size_t)N * N;
  const double rmax = N * 0.5 * 1.0; /* :37 */
  const int cap = orc_seg_cap(g);
  memset(full_out, 0, sizeof(float) * (size_t)V * W);
  if (nseg_out) memset(nseg_out, 0, sizeof(int) * (size_t)V * W);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    double* len = (double*)malloc(sizeof(double) * cap);
    double* rad = (double*)malloc(sizeof(double) * cap);
    int* pix = (int*)malloc(sizeof(int) * cap);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
    for (int j = 0; j < nviews; j++) {
      for (int jj = g->start_channel; jj < g->end_channel; jj++) {
        int ns = orc_walk(g, cos_t[j], sin_t[j], jj, len, pix, rad, cap);
        if (ns < 0) ns = 0;
        size_t o = (size_t)j * W + jj;
        if (nseg_out) nseg_out[o] = ns;
        float acc = 0.0f;
        for (int ke = 0; ke < NE; ke++) {
          double transp = 0.0;
          for (int q = 0; q < ns; q++) {
            for (int mat = 0; mat < M; mat++) {
              double ph;
              float v = orc_rho_seen(rho, n2, mat, pix[q], rad[q], rmax, &ph);
              transp += (double)(v * mu[mat * NE + ke]) * len[q] * ph;
            }
          }
          double intens = pdf[ke] * exp(-transp / (double)g->xfactor);
          acc += (float)intens;
        }
        full_out[o] = acc;
      }
    }
    free(len);
    free(rad);
    free(pix);
  }
}

void orc_forward_fp64(const orc_geom* g, const double* cos_t, const double* sin_t, const float* rho,
                      int M, const float* mu, const float* pdf, int NE, double* full_out,
                      double* lint_out, int nthreads) {
  const int V = g->views, W = g->width, N = g->recon_size;
  const int nviews = V / 2 * 2;
  const size_t n2 = (size_t)N * N;
  const double rmax = N * 0.5 * 1.0;
  const int cap = orc_seg_cap(g);
  memset(full_out, 0, sizeof(double) * (size_t)V * W);
  if (lint_out) memset(lint_out, 0, sizeof(double) * (size_t)V * W * M);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    double* len = (double*)malloc(sizeof(double) * cap);
    double* rad = (double*)malloc(sizeof(double) * cap);
    int* pix = (int*)malloc(sizeof(int) * cap);
    double L[16];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
    for (int j = 0; j < nviews; j++) {
      for (int jj = g->start_channel; jj < g->end_channel; jj++) {
        int ns = orc_walk(g, cos_t[j], sin_t[j], jj, len, pix, rad, cap);
        if (ns < 0) ns = 0;
        for (int mat = 0; mat < M; mat++) L[mat] = 0.0;
        for (int q = 0; q < ns; q++) {
          for (int mat = 0; mat < M; mat++) {
            double ph;
            float v = orc_rho_seen(rho, n2, mat, pix[q], rad[q], rmax, &ph);
            L[mat] += (double)v * len[q] * ph;
          }
        }
        size_t o = (size_t)j * W + jj;
        if (lint_out)
          for (int mat = 0; mat < M; mat++) lint_out[o * M + mat] = L[mat];
        double acc = 0.0;
        for (int ke = 0; ke < NE; ke++) {
          double t = 0.0;
          for (int mat = 0; mat < M; mat++) t += (double)mu[mat * NE + ke] * L[mat];
          acc += (double)pdf[ke] * exp(-t / (double)g->xfactor);
        }
        full_out[o] = acc;
      }
    }
    free(len);
    free(rad);
    free(pix);
  }
}

void orc_forward_fp64_maps(const orc_geom* g, const double* cos_t, const double* sin_t,
                           const short* maps, int M, const float* mu, const float* pdf, int NE,
                           double* full_out, double* lint_out, int nthreads) {
  const int V = g->views, W = g->width, N = g->recon_size;
  const int nviews = V / 2 * 2;
  const size_t n2 = (size_t)N * N;
  const double rmax = N * 0.5 * 1.0;
  const int cap = orc_seg_cap(g);
  memset(full_out, 0, sizeof(double) * (size_t)V * W);
  if (lint_out) memset(lint_out, 0, sizeof(double) * (size_t)V * W * M);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    double* len = (double*)malloc(sizeof(double) * cap);
    double* rad = (double*)malloc(sizeof(double) * cap);
    int* pix = (int*)malloc(sizeof(int) * cap);
    double L[16];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
    for (int j = 0; j < nviews; j++) {
      for (int jj = g->start_channel; jj < g->end_channel; jj++) {
        int ns = orc_walk(g, cos_t[j], sin_t[j], jj, len, pix, rad, cap);
        if (ns < 0) ns = 0;
        for (int mat = 0; mat < M; mat++) L[mat] = 0.0;
        for (int q = 0; q < ns; q++) {
          if (rad[q] >= rmax) continue;
          for (int mat = 0; mat < M; mat++) {
            short v = maps[(size_t)mat * n2 + pix[q]];
            if (v > 0) L[mat] += (double)v * len[q];
          }
        }
        for (int mat = 0; mat < M; mat++) L[mat] /= 1000.0;
        size_t o = (size_t)j * W + jj;
        if (lint_out)
          for (int mat = 0; mat < M; mat++) lint_out[o * M + mat] = L[mat];
        double acc = 0.0;
        for (int ke = 0; ke < NE; ke++) {
          double t = 0.0;
          for (int mat = 0; mat < M; mat++) t += (double)mu[mat * NE + ke] * L[mat];
          acc += (double)pdf[ke] * exp(-t / (double)g->xfactor);
        }
        full_out[o] = acc;
      }
    }
    free(len);
    free(rad);
    free(pix);
  }
}

/* MB/main.cpp:42-49 */
static double orc_uniform0(void) { return ((double)rand() + 1.0) / ((double)RAND_MAX + 2.0); }

double orc_normalize_noise(float* sino, int nn, double sigma, unsigned seed, int order) {
  /* MB/main.cpp:511-522 */
  float pmax = 0;
  for (int i = 0; i < nn; i++)
    if (pmax < sino[i]) pmax = sino[i];
  for (int i = 0; i < nn; i++) sino[i] = sino[i] / pmax;
  /* gaussiannoise0, MB/main.cpp:51-76 */
  double pmin = 10000000;
  for (int i = 0; i < nn; i++)
    if (pmin > sino[i]) pmin = sino[i];
  if (sigma <= 0) return pmin;
  srand(seed);
  for (int i = 0; i < nn; i++) {
    double nstar = sino[i];
    double u1, u2;
    if (order == 0) {
      u1 = orc_uniform0();
      u2 = orc_uniform0();
    } else {
      u2 = orc_uniform0();
      u1 = orc_uniform0();
    }
    double z = sqrt(-2.0 * log(u1)) * sin(2.0 * ORC_PI * u2);
    double psn = 0 + sigma * z;
    nstar = nstar + psn;
    sino[i] = (float)nstar;
    if (nstar < 0) sino[i] = (float)(pmin / 10);
    if (nstar > 1.0) sino[i] = 1.0f;
  }
  return pmin;
}

/* FBP/filterSinogramTOMO.cpp:9-123.  h is [C][C], C = end-start. */
void orc_fbp_constmap(const orc_geom* g, int filter, double* h) {
  const int C = g->end_channel - g->start_channel;
  const int half = (C - 1) / 2;
  double arc = g->max_beta / half; /* :30, parenthesised macro */
  double* sum = (double*)calloc(C, sizeof(double));
  for (int m = 0; m < C; m++) {
    sum[m] = 0.0;
    for (int n = 0; n < C; n++) {
      int MN = m - n;
      double v = 0.0;
      if (m == n) {
        if (filter == 1) {
          v = 0.125 / (arc * arc);
        } else if (filter == 2) {
          double oddterm = ORC_PI * ORC_PI * (arc);
          v = 0.25 / oddterm * (1.0 / tan((0.5) * arc) - 1.0 / tan((-0.5) * arc));
        }
      } else if (MN % 2 != 0) {
        if (filter == 1) {
          double oddterm = ORC_PI * sin(MN * arc);
          v = -0.5 / oddterm / oddterm;
        } else if (filter == 2) {
          double oddterm = ORC_PI * ORC_PI * arc;
          v = 0.25 / oddterm * (1.0 / tan((MN + 0.5) * arc) - 1.0 / tan((MN - 0.5) * arc));
        }
      } else {
        if (filter == 1) {
          v = 0.0;
        } else if (filter == 2) {
          double oddterm = ORC_PI * ORC_PI * arc;
          v = 0.25 / oddterm * (1.0 / tan((MN + 0.5) * arc) - 1.0 / tan((MN - 0.5) * arc));
        }
      }
      h[(size_t)m * C + n] = v;
      sum[m] += v;
    }
  }
  /* Edge-row renormalisation (:114-123); rows 0..20 and C-20..C-1. */
  for (int m = 0; m < C; m++)
    for (int n = 0; n < C; n++)
      if ((0 <= m && m <= 20) || (C - 20 <= m && m <= C))
        h[(size_t)m * C + n] = h[(size_t)m * C + n] * sum[21] / sum[m];
  free(sum);
}

/* FBP/filterSinogramTOMO.cpp:225-260.  sino is [V][width]; fltd is [V][C]. */
void orc_fbp_filter(const orc_geom* g, const float* sino, const double* h, int in_mode,
                    float* fltd) {
  const int C = g->end_channel - g->start_channel;
  const int half = (C - 1) / 2;
  const int cw = C / 2; /* centWidth, :227 */
  const int V = g->views, W = g->width;
  double* coeff = (double*)malloc(sizeof(double) * C);
  for (int k = 0; k < C; k++) coeff[k] = g->sid * cos((k - cw) * (g->max_beta / half));
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int n = 0; n < V; n++) {
    for (int m = 0; m < C; m++) {
      float acc = 0.0f;
      for (int k = 0; k < C; k++) {
        double projdat = sino[(size_t)n * W + k + g->start_channel];
        acc += h[(size_t)m * C + k] * (-log(projdat) * coeff[k]) * g->max_beta / half;
      }
      if (in_mode && (acc < 1000.0 || acc > 300000.0)) acc = 0.0f;
      fltd[(size_t)n * C + m] = acc;
    }
  }
  free(coeff);
}

void orc_mask(int N, unsigned char* mask) {
  double r = (double)(N - 1) / 2.0;
  double r2 = r * r;
  for (int j = 0; j < N; j++)
    for (int i = 0; i < N; i++)
      mask[j * N + i] = (((double)j - r) * ((double)j - r) + ((double)i - r) * ((double)i - r) <= r2);
}

/* FBP/reconstructImageTOMO.cpp:21-103 for one slice. */
void orc_fbp_backproject(const orc_geom* g, const float* fltd, const double* cos_t,
                         const double* sin_t, float* img) {
  const int N = g->recon_size, V = g->views;
  const int C = g->end_channel - g->start_channel;
  const int half = (C - 1) / 2;
  const int cw = C / 2;
  const double scale = g->pixel_cm;
  const double centerPos = (double)N / 2.0 - 0.5;
  const int use = V / 2 * 2; /* usesinogram, :30 */
  const double xfactor = (double)g->xfactor;
  unsigned char* mask = (unsigned char*)malloc((size_t)N * N);
  orc_mask(N, mask);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int y = 0; y < N; y++) {
    for (int x = 0; x < N; x++) {
      float acc = 0.0f;
      if (mask[y * N + x]) {
        double xx = -(x - centerPos) * scale;
        double yy = -(y - centerPos) * scale;
        for (int th = 0; th < use; th++) {
          double dbeta = 2.0 * ORC_PI / (V);
          double c = cos_t[th], s = sin_t[th];
          double X = xx * c + yy * s;
          double Y = -xx * s + yy * c;
          double L2 = (-Y + g->sid) * (-Y + g->sid) + X * X;
          double fGAM = atan(X / (g->sid - Y)) / (g->max_beta / half) + cw;
          int GAM = (int)(fGAM);
          double w = fGAM - GAM;
          if (GAM >= 0 && GAM < C - 1) {
            double sum1 = (1 - w) * fltd[(size_t)th * C + GAM] + w * fltd[(size_t)th * C + GAM + 1];
            double zw = 0.0, sum2 = 0;
            double sum = (1.0 - zw) * sum1 + zw * sum2;
            acc += (float)(1.0 / L2 * sum * dbeta * xfactor);
          }
        }
      }
      img[(size_t)y * N + x] = acc;
    }
  }
  free(mask);
}

/* The FBP of orc_fbp_filter + orc_fbp_backproject with every accumulation
 * and intermediate in double (the "error against FP64" denominator; the
 * reference accumulates both sums in float, FBP/filterSinogramTOMO.cpp:233-242
 * and FBP/reconstructImageTOMO.cpp:93).  img is [N][N]. */
void orc_fbp_fp64(const orc_geom* g, const float* sino, const double* h, const double* cos_t,
                  const double* sin_t, double* img) {
  const int C = g->end_channel - g->start_channel;
  const int half = (C - 1) / 2;
  const int cw = C / 2;
  const int V = g->views, W = g->width, N = g->recon_size;
  double* coeff = (double*)malloc(sizeof(double) * C);
  double* q = (double*)malloc(sizeof(double) * (size_t)V * C);
  for (int k = 0; k < C; k++) coeff[k] = g->sid * cos((k - cw) * (g->max_beta / half));
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int n = 0; n < V; n++) {
    for (int m = 0; m < C; m++) {
      double acc = 0.0;
      for (int k = 0; k < C; k++) {
        double projdat = sino[(size_t)n * W + k + g->start_channel];
        acc += h[(size_t)m * C + k] * (-log(projdat) * coeff[k]) * g->max_beta / half;
      }
      q[(size_t)n * C + m] = acc;
    }
  }
  const double scale = g->pixel_cm;
  const double centerPos = (double)N / 2.0 - 0.5;
  const int use = V / 2 * 2;
  const double xfactor = (double)g->xfactor;
  unsigned char* mask = (unsigned char*)malloc((size_t)N * N);
  orc_mask(N, mask);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int y = 0; y < N; y++) {
    for (int x = 0; x < N; x++) {
      double acc = 0.0;
      if (mask[y * N + x]) {
        double xx = -(x - centerPos) * scale;
        double yy = -(y - centerPos) * scale;
        for (int th = 0; th < use; th++) {
          double dbeta = 2.0 * ORC_PI / (V);
          double c = cos_t[th], s = sin_t[th];
          double X = xx * c + yy * s;
          double Y = -xx * s + yy * c;
          double L2 = (-Y + g->sid) * (-Y + g->sid) + X * X;
          double fGAM = atan(X / (g->sid - Y)) / (g->max_beta / half) + cw;
          int GAM = (int)(fGAM);
          double w = fGAM - GAM;
          if (GAM >= 0 && GAM < C - 1) {
            double sum = (1 - w) * q[(size_t)th * C + GAM] + w * q[(size_t)th * C + GAM + 1];
            acc += 1.0 / L2 * sum * dbeta * xfactor;
          }
        }
      }
      img[(size_t)y * N + x] = acc;
    }
  }
  free(mask);
  free(q);
  free(coeff);
}

void orc_fbp_transpose(const orc_geom* g, const double* h, const double* cos_t, const double* sin_t,
                       const double* u, double* out) {
  const int N = g->recon_size, V = g->views, W = g->width;
  const int C = g->end_channel - g->start_channel;
  const int half = (C - 1) / 2;
  const int cw = C / 2;
  const double scale = g->pixel_cm;
  const double centerPos = (double)N / 2.0 - 0.5;
  const int use = V / 2 * 2;
  const double xfactor = (double)g->xfactor;
  const double dbeta = 2.0 * ORC_PI / (V);
  unsigned char* mask = (unsigned char*)malloc((size_t)N * N);
  orc_mask(N, mask);
  double* qb = (double*)calloc((size_t)V * C, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int th = 0; th < use; th++) {
    const double c = cos_t[th], s = sin_t[th];
    double* q = qb + (size_t)th * C;
    for (int y = 0; y < N; y++)
      for (int x = 0; x < N; x++) {
        if (!mask[y * N + x]) continue;
        const double xx = -(x - centerPos) * scale, yy = -(y - centerPos) * scale;
        const double X = xx * c + yy * s;
        const double Y = -xx * s + yy * c;
        const double L2 = (-Y + g->sid) * (-Y + g->sid) + X * X;
        const double fGAM = atan(X / (g->sid - Y)) / (g->max_beta / half) + cw;
        const int GAM = (int)(fGAM);
        const double w = fGAM - GAM;
        if (GAM >= 0 && GAM < C - 1) {
          const double a = u[(size_t)y * N + x] / L2 * dbeta * xfactor;
          q[GAM] += (1 - w) * a;
          q[GAM + 1] += w * a;
        }
      }
  }
  memset(out, 0, sizeof(double) * (size_t)V * W);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int n = 0; n < V; n++)
    for (int k = 0; k < C; k++) {
      double acc = 0.0;
      for (int m = 0; m < C; m++) acc += h[(size_t)m * C + k] * qb[(size_t)n * C + m];
      out[(size_t)n * W + g->start_channel + k] = acc * g->sid * cos((k - cw) * (g->max_beta / half)) * g->max_beta / half;
    }
  free(qb);
  free(mask);
}

/* ---------------------------------------------------------------- adjoint */
static void orc_ray_points(const orc_geom* g, double cb, double sb, int jj, double* sx, double* sy,
                           double* px, double* py) {
  const int half = (g->end_channel - g->start_channel - 1) / 2;
  double theta = (g->iso_channel - jj) * g->max_alpha / half;
  double px0 = g->det_radius * sin(theta);
  double py0 = -g->det_radius * cos(theta) + g->det_src_iso;
  *sx = g->sid * sb;
  *sy = g->sid * cb;
  *px = +px0 * cb + py0 * sb;
  *py = -px0 * sb + py0 * cb;
}

static int orc_cmp_double(const void* a, const void* b) {
  double x = *(const double*)a, y = *(const double*)b;
  return x < y ? -1 : x > y;
}

int orc_siddon(const orc_geom* g, double cb, double sb, int jj, double* seg_len, int* seg_pix, int cap) {
  const int N = g->recon_size;
  const double s = g->pixel_cm;
  const double n = (double)(int)(N * 0.5);
  double sx, sy, px, py;
  orc_ray_points(g, cb, sb, jj, &sx, &sy, &px, &py);
  const double dx = px - sx, dy = py - sy;
  const double len = sqrt(dx * dx + dy * dy);
  const double lo = -n * s, hi = (N - n) * s;
  /* Clip the line (parameter t along S->P) to the grid square. */
  double t0 = -1e300, t1 = 1e300;
  if (dx != 0) {
    double a = (lo - sx) / dx, b = (hi - sx) / dx;
    if (a > b) { double t = a; a = b; b = t; }
    if (a > t0) t0 = a;
    if (b < t1) t1 = b;
  } else if (sx < lo || sx > hi) return 0;
  if (dy != 0) {
    double a = (lo - sy) / dy, b = (hi - sy) / dy;
    if (a > b) { double t = a; a = b; b = t; }
    if (a > t0) t0 = a;
    if (b < t1) t1 = b;
  } else if (sy < lo || sy > hi) return 0;
  if (!(t1 > t0)) return 0;
  /* All gridline crossings inside (t0, t1), sorted. */
  int cnt = 0;
  double* ts = (double*)malloc(sizeof(double) * (2 * N + 8));
  ts[cnt++] = t0;
  for (int k = 0; k <= N; k++) {
    double gx = lo + k * s;
    if (dx != 0) {
      double t = (gx - sx) / dx;
      if (t > t0 && t < t1) ts[cnt++] = t;
    }
    if (dy != 0) {
      double t = (gx - sy) / dy;
      if (t > t0 && t < t1) ts[cnt++] = t;
    }
  }
  ts[cnt++] = t1;
  qsort(ts, cnt, sizeof(double), orc_cmp_double);
  int ns = 0;
  for (int q = 0; q + 1 < cnt; q++) {
    double ta = ts[q], tb = ts[q + 1];
    if (!(tb > ta)) continue;
    double tm = 0.5 * (ta + tb);
    double xm = sx + tm * dx, ym = sy + tm * dy;
    int col = (int)floor(xm / s + n), row = (int)floor(n - ym / s);
    if (col < 0 || col >= N || row < 0 || row >= N) continue;
    if (ns >= cap) { free(ts); return -1; }
    seg_len[ns] = (tb - ta) * len;
    seg_pix[ns] = col + row * N;
    ns++;
  }
  free(ts);
  return ns;
}

void orc_siddon_project(const orc_geom* g, const double* cos_t, const double* sin_t, const double* x, int M,
                        double* out, int nthreads) {
  const int V = g->views, W = g->width, N = g->recon_size;
  const int nviews = V / 2 * 2;
  const size_t n2 = (size_t)N * N;
  const int cap = 4 * N + 64;
  memset(out, 0, sizeof(double) * (size_t)V * W * M);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    double* len = (double*)malloc(sizeof(double) * cap);
    int* pix = (int*)malloc(sizeof(int) * cap);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
    for (int j = 0; j < nviews; j++)
      for (int jj = g->start_channel; jj < g->end_channel; jj++) {
        int ns = orc_siddon(g, cos_t[j], sin_t[j], jj, len, pix, cap);
        double* o = out + ((size_t)j * W + jj) * M;
        for (int q = 0; q < ns; q++)
          for (int m = 0; m < M; m++) o[m] += x[(size_t)m * n2 + pix[q]] * len[q];
      }
    free(len);
    free(pix);
  }
}

void orc_walk_project(const orc_geom* g, const double* cos_t, const double* sin_t, const double* rho, int M,
                      double* out, int nthreads) {
  const int V = g->views, W = g->width, N = g->recon_size;
  const int nviews = V / 2 * 2;
  const size_t n2 = (size_t)N * N;
  const double rmax = N * 0.5 * 1.0;
  const int cap = orc_seg_cap(g);
  memset(out, 0, sizeof(double) * (size_t)V * W * M);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    double* len = (double*)malloc(sizeof(double) * cap);
    double* rad = (double*)malloc(sizeof(double) * cap);
    int* pix = (int*)malloc(sizeof(int) * cap);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
    for (int j = 0; j < nviews; j++)
      for (int jj = g->start_channel; jj < g->end_channel; jj++) {
        int ns = orc_walk(g, cos_t[j], sin_t[j], jj, len, pix, rad, cap);
        double* o = out + ((size_t)j * W + jj) * M;
        for (int q = 0; q < ns; q++) {
          if (rad[q] >= rmax) continue;
          for (int m = 0; m < M; m++) o[m] += rho[(size_t)m * n2 + pix[q]] * len[q];
        }
      }
    free(len);
    free(rad);
    free(pix);
  }
}

/* Views are split statically over the threads; each thread scatters into its
 * own image and the images are summed in thread order, so the result does not
 * depend on scheduling. */
void orc_walk_backproject(const orc_geom* g, const double* cos_t, const double* sin_t, const double* w, int M,
                          double* out, int nthreads) {
  const int V = g->views, W = g->width, N = g->recon_size;
  const int nviews = V / 2 * 2;
  const size_t n2 = (size_t)N * N;
  const double rmax = N * 0.5 * 1.0;
  const int cap = orc_seg_cap(g);
  int nt = 1;
#ifdef _OPENMP
  nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
  double* part = (double*)calloc((size_t)nt * M * n2, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* img = part + (size_t)tid * M * n2;
    double* len = (double*)malloc(sizeof(double) * cap);
    double* rad = (double*)malloc(sizeof(double) * cap);
    int* pix = (int*)malloc(sizeof(int) * cap);
    const int per = (nviews + nt - 1) / nt;
    for (int j = tid * per; j < nviews && j < (tid + 1) * per; j++)
      for (int jj = g->start_channel; jj < g->end_channel; jj++) {
        const double* wr = w + ((size_t)j * W + jj) * M;
        int any = 0;
        for (int m = 0; m < M; m++) any |= wr[m] != 0.0;
        if (!any) continue;
        int ns = orc_walk(g, cos_t[j], sin_t[j], jj, len, pix, rad, cap);
        for (int q = 0; q < ns; q++) {
          if (rad[q] >= rmax) continue;
          for (int m = 0; m < M; m++) img[(size_t)m * n2 + pix[q]] += wr[m] * len[q];
        }
      }
    free(len);
    free(rad);
    free(pix);
  }
  memset(out, 0, sizeof(double) * M * n2);
  for (int t = 0; t < nt; t++)
    for (size_t i = 0; i < (size_t)M * n2; i++) out[i] += part[(size_t)t * M * n2 + i];
  free(part);
}

void orc_walk_project_rays(const orc_geom* g, const double* cos_t, const double* sin_t, const double* rho, int M,
                           const int* rays, int nrays, double* out, int nthreads) {
  const int W = g->width, N = g->recon_size;
  const size_t n2 = (size_t)N * N;
  const double rmax = N * 0.5 * 1.0;
  const int cap = orc_seg_cap(g);
  memset(out, 0, sizeof(double) * (size_t)nrays * M);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    double* len = (double*)malloc(sizeof(double) * cap);
    double* rad = (double*)malloc(sizeof(double) * cap);
    int* pix = (int*)malloc(sizeof(int) * cap);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
    for (int i = 0; i < nrays; i++) {
      const int j = rays[i] / W, jj = rays[i] % W;
      int ns = orc_walk(g, cos_t[j], sin_t[j], jj, len, pix, rad, cap);
      double* o = out + (size_t)i * M;
      for (int q = 0; q < ns; q++) {
        if (rad[q] >= rmax) continue;
        for (int m = 0; m < M; m++) o[m] += rho[(size_t)m * n2 + pix[q]] * len[q];
      }
    }
    free(len);
    free(rad);
    free(pix);
  }
}

/* ------------------------------------------------------------ lengthproj */
/* First view of the slice and view count, MB/lengthproj_TOMO.cpp:36-47. */
static void orc_lp_views(const orc_geom* g, double z, double couch_speed, int* start, int* count, int* nrot) {
  const int V = g->views;
  const int used = V / 2 * 2; /* sngrmHeight/UsedReconAngle*2 with UsedReconAngle 2 */
  int s0 = 0;
  if (couch_speed != 0.0) {
    const double pitch = (double)(couch_speed / V);
    s0 = (int)(z / pitch - V / 2 + 0.00000001);
  }
  *start = s0;
  *count = used;
  *nrot = s0 / V;
}

static void orc_lengthproj_rows(const orc_geom* g, const double* cos_t, const double* sin_t, const float* proj,
                                double z, double couch_speed, int first, int stride, int tables, float* npf) {
  const int N = g->recon_size, V = g->views, W = g->width;
  const double s = g->pixel_cm;
  const int C = g->end_channel - g->start_channel;
  const int half = (C - 1) / 2;
  const double dalpha = g->max_alpha / half;
  const double R = g->det_radius;            /* DETECTOR_RADIUS_CURVATURE_CM */
  const double dsrc = g->det_src_iso;        /* DIST_BTWN_DETERCTORSRC_AND_ISOCENT_CM */
  const double diso = g->det_radius - g->sid; /* DIST_BTWN_ISO_AND_DETECTOR_CM (142.6 - 85) */
  int start, count, nrot;
  orc_lp_views(g, z, couch_speed, &start, &count, &nrot);
  count /= stride;
  unsigned char* mask = (unsigned char*)malloc((size_t)N * N);
  orc_mask(N, mask);
  memset(npf, 0, sizeof(float) * (size_t)N * N);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int jy = 0; jy < N; jy++) {
    const double ry = N * s * 0.5 - (jy + 0.5) * s;
    for (int jx = 0; jx < N; jx++) {
      if (!mask[jy * N + jx]) continue;
      const double rx = -N * s * 0.5 + (jx + 0.5) * s;
      float acc = 0.0f;
      for (int k = 0; k < count; k++) {
        const int rk = first + k * stride; /* sinogram row j_one */
        int v = start + rk - nrot * V;
        if (v >= V) v -= V;
        if (v < 0) v += V; /* the reference reads its tables out of range here */
        const double cb = cos_t[v], sb = sin_t[v];
        const double sx = g->sid * sb, sy = g->sid * cb;
        double len;
        if (fabs(rx - sx) > fabs(ry - sy)) {
          /* chord across the pixel column, x-major */
          const double x0 = rx - 0.5 * s, x1 = rx + 0.5 * s;
          const double y0 = (x0 - sx) / (rx - sx) * (ry - sy) + sy;
          const double y1 = (x1 - sx) / (rx - sx) * (ry - sy) + sy;
          len = sqrt((x0 - x1) * (x0 - x1) + (y0 - y1) * (y0 - y1));
        } else {
          /* y-major: the reference evaluates both ends at y0, so only the
           * y extent remains (:95-101) */
          const double y0 = ry - 0.5 * s, y1 = ry + 0.5 * s;
          len = sqrt((y0 - y1) * (y0 - y1));
        }
        /* the source-pixel line meets the detector circle (centre dsrc on
         * the source side, radius R); the hit nearer the origin (:110-134) */
        const double dx = dsrc * sb, dy = dsrc * cb;
        const double a = (sy - ry) / (sx - rx);
        const double b = -sx * (sy - ry) / (sx - rx) + sy;
        const double qa = 1.0 + a * a;
        const double qb = 2.0 * a * b - 2.0 * a * dy - 2.0 * dx;
        const double qc = dx * dx + b * b + dy * dy - 2.0 * b * dy - R * R;
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
        /* detector angle from the detector's centre point (:136-150) */
        const double ox = -diso * sb, oy = -diso * cb;
        const double d2 = (px - ox) * (px - ox) + (py - oy) * (py - oy);
        const double ang = acos(1.0 - d2 / (2.0 * R * R));
        const double rpx = px * cb - py * sb;
        double dj = rpx > 0.0 ? g->iso_channel - ang / dalpha : g->iso_channel + ang / dalpha;
        if (tables) { /* the side tables hold float (:76, :153) */
          len = (double)(float)len;
          dj = (double)(float)dj;
        }
        const int ij = dj == dj ? (int)dj : 0;
        const double f = dj - (double)ij;
        const float* row = proj + (size_t)rk * W;
        /* three explicit tests, as :158-172: a NaN channel (a source on the
         * pixel's vertical, 0/0 in the line slope) matches none and adds
         * nothing */
        if (g->start_channel <= dj && dj < g->end_channel - 1)
          acc += (float)(((1.0 - f) * row[ij] + f * row[ij + 1]) * len);
        else if (g->start_channel > dj)
          acc += (float)(row[g->start_channel] * len);
        else if (dj >= g->end_channel - 1)
          acc += (float)(row[g->end_channel - 1] * len);
      }
      npf[jy * N + jx] = acc;
    }
  }
  free(mask);
}

/* ------------------------------------------------- beam-hardening correction */
/* MB/beam_hardening_correction.cpp:49-56, elementwise: y = -ln p,
 * y' = |y| + alpha |y|^beta, p' = (float)exp(-y'); mins[0], mins[1] receive
 * the minima before and after, as the program prints them.  The reference is
 * C++: log() of its float sample resolves to the float overload, so the
 * logarithm is taken in single precision (logf) and widened. */
void orc_beam_hardening(float* p, long long n, double alpha, double beta, double* mins) {
  double min_org = 1000000, min_new = 1000000;
  for (long long i = 0; i < n; i++) {
    if (min_org > p[i]) min_org = p[i];
    double y = -(double)logf(p[i]);
    y = fabs(y) + (alpha * pow(fabs(y), beta));
    p[i] = (float)exp(-y);
    if (min_new > p[i]) min_new = p[i];
  }
  if (mins) {
    mins[0] = min_org;
    mins[1] = min_new;
  }
}

void orc_lengthproj(const orc_geom* g, const double* cos_t, const double* sin_t, const float* proj, double z,
                    double couch_speed, float* npf) {
  orc_lengthproj_rows(g, cos_t, sin_t, proj, z, couch_speed, 0, 1, 0, npf);
}

void orc_lengthproj2(const orc_geom* g, const double* cos_t, const double* sin_t, const float* proj, double z,
                     double couch_speed, int ite, int thinout, float* npf) {
  orc_lengthproj_rows(g, cos_t, sin_t, proj, z, couch_speed, (ite - 1) % thinout, thinout, 1, npf);
}

/* ------------------------------------------------------ IR image update */
/* The total-variation derivative of MB/IR_ImageTOMO.cpp:10-17: differences
 * and squares in float, roots and the quotients in double. */
static double orc_tv(float a, float a1, float a2, float a3, float a4, float a7, float a8) {
  const float s1 = (a - a2) * (a - a2) + (a - a4) * (a - a4);
  const float s2 = (a - a1) * (a - a1) + (a1 - a7) * (a1 - a7);
  const float s3 = (a3 - a8) * (a3 - a8) + (a - a3) * (a - a3);
  const double d1 = sqrt((double)s1) + 0.00000001;
  const double d2 = sqrt((double)s2) + 0.00000001;
  const double d3 = sqrt((double)s3) + 0.00000001;
  const float t1 = (a - a2) + (a - a4);
  return t1 / d1 + (a - a1) / d2 + (a - a3) / d3;
}

void orc_ir_update(int N, const float* before, const float* prior, const float* npf, const float* npf_re,
                   double wbefore, double w_tv, double w_prior, int ite, int thinout, float* after) {
  unsigned char* mask = (unsigned char*)malloc((size_t)N * N);
  orc_mask(N, mask);
  for (int y = 0; y < N; y++)
    for (int x = 0; x < N; x++) {
      const int k = y * N + x;
      if (!mask[k]) continue;
      double cost_tv = 0.0, cost_prior = 0.0;
      if (y < N - 1 && x < N - 1 && x > 0 && y > 0) {
        const int k1 = k - 1, k2 = k + 1, k3 = k - N, k4 = k + N, k7 = k + N - 1, k8 = k - N + 1;
        cost_tv = -orc_tv(before[k], before[k1], before[k2], before[k3], before[k4], before[k7], before[k8]);
#define ORC_PR(i) (prior ? prior[i] : 0.0f)
        cost_prior = -orc_tv(before[k] - ORC_PR(k), before[k1] - ORC_PR(k1), before[k2] - ORC_PR(k2),
                             before[k3] - ORC_PR(k3), before[k4] - ORC_PR(k4), before[k7] - ORC_PR(k7),
                             before[k8] - ORC_PR(k8));
#undef ORC_PR
      }
      const double lambda = w_tv * cost_tv + w_prior * cost_prior + 0.000001;
      const double del_F = (float)(npf_re[k] - npf[k] / (float)thinout) + lambda;
      double w = wbefore;
      if (ite > 300) w = before[k] / (npf[k] / (float)thinout - lambda);
      float v = (float)(before[k] + w * del_F);
      if (v < 0.0f) v = 0.0f;
      after[k] = v;
    }
  free(mask);
}


/* ------------------------------------------------- measured-data ingestion */
/* MB/projectionDataTOMO.cpp:324-508.  Each fread below fills the same
 * buffer the reference fills, with the same byte count, so a short read
 * leaves the previous contents in the tail just as it does there. */
int orc_load_measured(const char* proj_file, const char* air_file, int in_mode, int width, int views, int nskip,
                      int rotations, int rows_per_view, int ch, int skip, int air_rows, int air_blocks,
                      int start_ch, int end_ch, float* vol, unsigned char* mask, double* maxv) {
  *maxv = 0.0;
  const long long plane = (long long)ch * air_rows;
  if (in_mode) {
    if ((long long)(views - 1) * ch + skip + width > plane) return -3;  /* air rows read past a block */
  } else {
    if ((long long)(air_rows - 1) * ch + skip + width > plane) return -3;
    if ((air_rows + nskip - 1) / nskip != views) return -3;  /* kept rows per rotation != views */
  }
  FILE* fp = fopen(proj_file, "rb");
  if (!fp) return -1;
  FILE* fa = fopen(air_file, "rb");
  if (!fa) {
    fclose(fp);
    return -1;
  }
  float* air = (float*)calloc((size_t)plane, sizeof(float));
  float* sum_air = (float*)calloc((size_t)plane, sizeof(float));
  float* proj = (float*)calloc((size_t)plane, sizeof(float));
  size_t got;
  /* the first air block is read and not used (:385, :401) */
  got = fread(air, 1, (size_t)plane * sizeof(float), fa);
  for (int b = 0; b < air_blocks; b++) {
    got = fread(air, 1, (size_t)plane * sizeof(float), fa);
    if (!in_mode) {
      for (long long k = 0; k < plane; k++) sum_air[k] += air[k] / air_blocks;  /* :389-393 */
    } else {
      long long k = 0; /* :404-412 */
      for (int k1 = 0; k1 < views; k1++)
        for (int k2 = skip; k2 < skip + width; k2++) sum_air[k++] += air[(long long)k1 * ch + k2] / air_blocks;
    }
  }
  (void)got;
  fclose(fa);
  int ret = rotations;
  if (!in_mode) {
    long long out = 0; /* :435-455 */
    for (int t = 0; t < rotations; t++) {
      got = fread(proj, 1, (size_t)plane * sizeof(float), fp);
      for (int k1 = 0; k1 < air_rows; k1++)
        for (int k2 = skip; k2 < skip + width; k2++) {
          const long long kk = (long long)k1 * ch + k2;
          const float d = proj[kk] / sum_air[kk];
          if (k1 / nskip * nskip == k1) {
            vol[out] = d;
            mask[out] = 1;
            out++;
          }
        }
    }
  } else {
    double pmax = 0.0; /* :458-500 */
    for (int t = 0; t < rotations && ret >= 0; t++)
      for (int j = 0; j < views && ret >= 0; j++) {
        got = fread(proj, 1, (size_t)ch * sizeof(float), fp);
        int k = 0;
        for (int i = skip; i < skip + width; i++) {
          const long long kk = (long long)j * ch + i;
          float d = proj[kk] / (sum_air[k] * 2);
          if (pmax < d && i >= start_ch && i < end_ch) {
            pmax = d;
            if (pmax > 1.0) {
              ret = -2;
              break;
            }
          }
          const long long o = ((long long)t * views + j) * width + k;
          mask[o] = 1;
          if (d < 0.1) {
            d = 0.0f;
            mask[o] = 0;
          }
          vol[o] = d;
          k++;
        }
        for (int r = 1; r < rows_per_view && ret >= 0; r++) got = fread(proj, 1, (size_t)ch * sizeof(float), fp);
      }
    *maxv = pmax;
  }
  fclose(fp);
  free(air);
  free(sum_air);
  free(proj);
  return ret;
}

/* MB/main.cpp:347-371 with start_angle_num = 0 and UsedReconAngle = 2. */
void orc_helical(const float* vol, int rotations, int views, int width, float* out) {
  const int use = views / 2 * 2;
  for (int j = 0; j < use; j++) {
    const int num_pro = j;
    int iphase = 0;
    if (num_pro < use / 2) iphase = 1;
    else if (num_pro > use / 2) iphase = -1;
    if (j + iphase * views < views) iphase = 0;
    if (j + iphase * views > (rotations - 1) * views) iphase = 0;
    const double zw = 0.5 * fabs(num_pro - (views / 2.0)) / (views / 2.0);
    for (int c = 0; c < width; c++)
      out[(long long)num_pro * width + c] =
          (float)((1.0 - zw) * vol[(long long)j * width + c] + zw * vol[(long long)(j + iphase * views) * width + c]);
  }
}
