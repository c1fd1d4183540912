// Test-infrastructure harness: exposes the reference's own MBFPA kernels,
// compiled from Release_MBFPA_CPU_human/*.cpp by oracle/Makefile, through a
// plain C ABI so that tests and bench.py (reference arm, cpu_baseline leg) can
// call them with ctypes.  This file contains no reference code: it only
// allocates the buffers the reference functions expect and calls them.
//
//   attenuation_coefficient  Release_MBFPA_CPU_human/prior_weight_production.cpp:180
//   reprojection_TOMO        Release_MBFPA_CPU_human/reprojection_TOMO.cpp:13
//   energy loop + sum        Release_MBFPA_CPU_human/main.cpp:492-506
//   lengthproj_TOMO          Release_MBFPA_CPU_human/lengthproj_TOMO.cpp:14
//   prepareMaskData          Release_MBFPA_CPU_human/misc_TOMO.cpp:10
//   lengthproj_TOMO_2        Release_MBFPA_CPU_human/lengthproj_TOMO.cpp:188
//   IR_ImageTOMO             Release_MBFPA_CPU_human/IR_ImageTOMO.cpp:19
//   loadProjectionData       Release_MBFPA_CPU_human/projectionDataTOMO.cpp:324
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>
#include <fcntl.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "physParamsTOMO.h"
#include "mallocMD.h"
#include "reprojection_TOMO.h"
#include "lengthproj_TOMO.h"
#include "misc_TOMO.h"
#include "IR_ImageTOMO.h"
#include "projectionDataTOMO.h"
#include "virtual_projection.h"

static double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// attenuation_coefficient prints its whole table to stdout; keep the caller's
// stdout clean by pointing fd 1 at /dev/null for the duration of the call.
struct QuietStdout {
  int saved = -1;
  QuietStdout() {
    fflush(stdout);
    saved = dup(1);
    int nul = open("/dev/null", O_WRONLY);
    if (nul >= 0) { dup2(nul, 1); close(nul); }
  }
  ~QuietStdout() {
    fflush(stdout);
    if (saved >= 0) { dup2(saved, 1); close(saved); }
  }
};

extern "C" {

int vctref_mb_channels(void) { return End_Channel - Start_Channel; }

// Fills att[num_material*NE] (bin index fastest) and pdf[NE]; both buffers must
// hold 1024*num_material and 1024 floats as main.cpp:338-339 allocates them.
int vctref_attenuation(const char* spectrum, int num_material, float* att, float* pdf, int* NE) {
  QuietStdout q;
  *NE = 0;
  attenuation_coefficient((char*)spectrum, num_material, att, pdf, NE, 1);
  return *NE > 0 ? 0 : -1;
}

int vctref_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// Runs reprojection_TOMO for energy bins [ke0, ke1) and accumulates each bin's
// sinogram into full[] in float, in bin order, as main.cpp:492-506 does.
// rho is the float density stack [6][N][N] (main.cpp:93-109); it is copied
// because the reference clamps material 0 in place.  cos/sin hold V entries.
// Returns the wall time of the reprojection_TOMO calls in *seconds.
int vctref_reprojection_bins(int N, double pixel_cm, const float* rho, int V, int W,
                             const double* cosT, const double* sinT, int xfactor,
                             const float* att, const float* pdf, int NE, int ke0, int ke1,
                             float* full, float* last_bin, int* nseg, double* seconds) {
  if (W < End_Channel) return -1;
  const int M = 6;
  size_t n2 = (size_t)N * N;
  float* work = (float*)malloc(sizeof(float) * M * n2);
  float* proj = (float*)calloc((size_t)V * W, sizeof(float));
  // Segment side tables written by the walk (never read on this path).  The
  // reference sizes them W*V*N*2 (main.cpp:261-262); a ray has at most about
  // 2N+4 segments, so the margin keeps small grids in bounds too.  They are
  // kept between calls, as the reference's main allocates them once, so only
  // the first call pays for faulting their pages in.
  static float* sysmat = nullptr;
  static int* vnum = nullptr;
  static size_t cap = 0;
  size_t slots = (size_t)W * V * (size_t)(2 * N + 16);
  if (slots > cap) {
    free(sysmat);
    free(vnum);
    sysmat = (float*)malloc(sizeof(float) * slots);
    vnum = (int*)malloc(sizeof(int) * slots);
    cap = (sysmat && vnum) ? slots : 0;
  }
  int* rsum = (int*)calloc((size_t)V * W, sizeof(int));
  char* mask = (char*)calloc(n2, 1);
  if (!work || !proj || !sysmat || !vnum || !rsum || !mask) {
    free(work); free(proj); free(rsum); free(mask);
    return -2;
  }
  memcpy(work, rho, sizeof(float) * M * n2);
  double xalpha[1] = {0.0};
  double t0 = now_s();
  for (int ke = ke0; ke < ke1; ke++) {
    reprojection_TOMO(1, N, work, proj, pixel_cm, W, V, (double*)cosT, (double*)sinT, 0.0, 0.0,
                      (double)xfactor, xalpha, mask, sysmat, vnum, rsum, 1, (float*)att, (float*)pdf,
                      M, NE, ke);
    if (full)
      for (size_t i = 0; i < (size_t)V * W; i++) full[i] += proj[i];
  }
  double t1 = now_s();
  if (seconds) *seconds = t1 - t0;
  if (last_bin) memcpy(last_bin, proj, sizeof(float) * V * W);
  if (nseg) memcpy(nseg, rsum, sizeof(int) * V * W);
  free(work); free(proj); free(rsum); free(mask);
  return 0;
}

// Runs lengthproj_TOMO on one slice: proj is the sinogram the reference's
// main passes (rows j_one = 0.. of the views used, W floats each), cos/sin
// the V-entry trig tables, z and couch_speed the txt's values.  The system
// matrix and detector-position side tables it writes ([N][N][V] floats each)
// are allocated here and dropped.
int vctref_lengthproj(int N, double pixel_cm, const float* proj, int W, int V, const double* cosT,
                      const double* sinT, double z, double couch_speed, float* npf, double* seconds) {
  if (W < End_Channel) return -1;
  size_t n2 = (size_t)N * N;
  float* sysmat = (float*)malloc(sizeof(float) * n2 * V);
  float* tracedet = (float*)malloc(sizeof(float) * n2 * V);
  char* mask = prepareMaskData(N);
  if (!sysmat || !tracedet || !mask) {
    free(sysmat); free(tracedet);
    return -2;
  }
  memset(npf, 0, sizeof(float) * n2);
  double t0 = now_s();
  lengthproj_TOMO(0, N, npf, (float*)proj, pixel_cm, W, V, (double*)cosT, (double*)sinT, z, couch_speed, mask,
                  sysmat, tracedet, 1);
  if (seconds) *seconds = now_s() - t0;
  free(sysmat); free(tracedet);
  delete1DArray(mask);
  return 0;
}

// The iterative step's backprojection: lengthproj_TOMO (ite 0) fills the side
// tables as the reference's main does, then lengthproj_TOMO_2 reads them for
// iteration `ite` with `thinout` on the sinogram proj.
int vctref_lengthproj2(int N, double pixel_cm, const float* proj0, const float* proj, int W, int V,
                       const double* cosT, const double* sinT, double z, double couch_speed, int ite, int thinout,
                       float* npf) {
  if (W < End_Channel) return -1;
  size_t n2 = (size_t)N * N;
  float* sysmat = (float*)malloc(sizeof(float) * n2 * V);
  float* tracedet = (float*)malloc(sizeof(float) * n2 * V);
  float* npf0 = (float*)calloc(n2, sizeof(float));
  char* mask = prepareMaskData(N);
  if (!sysmat || !tracedet || !mask || !npf0) {
    free(sysmat); free(tracedet); free(npf0);
    return -2;
  }
  lengthproj_TOMO(0, N, npf0, (float*)proj0, pixel_cm, W, V, (double*)cosT, (double*)sinT, z, couch_speed, mask,
                  sysmat, tracedet, 1);
  memset(npf, 0, sizeof(float) * n2);
  lengthproj_TOMO_2(ite, N, npf, (float*)proj, pixel_cm, W, V, z, couch_speed, mask, sysmat, tracedet, thinout);
  free(sysmat); free(tracedet); free(npf0);
  delete1DArray(mask);
  return 0;
}

// IR_ImageTOMO on one N x N map; `after` keeps its values outside the mask.
int vctref_ir_update(int N, const float* before, const float* prior, const float* npf, const float* npf_re,
                     double wbefore, double w_tv, double w_prior, int ite, int thinout, float* after) {
  char* mask = prepareMaskData(N);
  if (!mask) return -2;
  IR_ImageTOMO(ite, N, (float*)before, after, (float*)prior, (float*)npf, (float*)npf_re, wbefore, w_tv, w_prior,
               mask, thinout);
  delete1DArray(mask);
  return 0;
}

}  // extern "C"

extern "C" {
// loadProjectionData on a PROJECTION_DATA holding the fields it reads.  It
// writes projections.raw into the current directory (the caller picks it).
// height_raw is projImgHeight before the sino_fact thinning.  Returns what
// loadProjectionData returns; vol/mask receive projVolume/mask_projVolume
// ([rotations][height_raw/nskip][width]) when it returned >= 0.
int vctref_load_measured(const char* proj_file, const char* air_file, const char* in_pr, int width, int height_raw,
                         int nskip, int rotations, double rate_orig, float* vol, unsigned char* mask) {
  PROJECTION_DATA* pd = newProjectionData();
  memset(pd, 0, sizeof *pd);
  snprintf(pd->projImgFileName, sizeof pd->projImgFileName, "%s", proj_file);
  snprintf(pd->AirScanImgFileName, sizeof pd->AirScanImgFileName, "%s", air_file);
  snprintf(pd->InPrClassString, sizeof pd->InPrClassString, "%s", in_pr);
  pd->projImgWidth = width;
  pd->projImgHeight = height_raw;
  pd->sino_fact = nskip;
  pd->totalProjNumber = rotations;
  pd->datatype = UNIT_FLOAT32;
  pd->datasize = 4;
  pd->DataSamplingRateOrig = rate_orig;
  const int ret = loadProjectionData(pd);
  if (ret >= 0) {
    const size_t n = (size_t)width * pd->projImgHeight * pd->usedProjNumber;
    memcpy(vol, pd->projVolume, n * sizeof(float));
    memcpy(mask, pd->mask_projVolume, n);
  }
  deleteProjectionData(pd);
  return ret;
}
}  // extern "C"
