// Test-infrastructure harness: exposes the reference's own FBP kernels,
// compiled from Release_FBP_CPU/*.cpp by oracle/Makefile, through a plain C
// ABI.  No reference code lives here; it allocates the reference's row-pointer
// arrays and calls, in the order Release_FBP_CPU/main.cpp:66-167 does:
//   prepareConstMap                      filterSinogramTOMO.cpp:9
//   prepareCorrectedDetectorInterpolation filterSinogramTOMO.cpp:140
//   prepareMaskData                      misc.cpp:10
//   filterSinogram                       filterSinogramTOMO.cpp:205
//   reconstructImage                     reconstructImageTOMO.cpp:11
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>
#include <fcntl.h>

#include "physParamsTOMO.h"
#include "mallocMD.h"
#include "misc.h"
#include "filterSinogramTOMO.h"
#include "reconstructImageTOMO.h"

static double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

struct QuietStd {
  int s1 = -1, s2 = -1;
  QuietStd() {
    fflush(stdout); fflush(stderr);
    s1 = dup(1); s2 = dup(2);
    int nul = open("/dev/null", O_WRONLY);
    if (nul >= 0) { dup2(nul, 1); dup2(nul, 2); close(nul); }
  }
  ~QuietStd() {
    fflush(stdout); fflush(stderr);
    if (s1 >= 0) { dup2(s1, 1); close(s1); }
    if (s2 >= 0) { dup2(s2, 2); close(s2); }
  }
};

extern "C" {

int vctref_fbp_channels(void) { return End_Channel - Start_Channel; }

// sino: [V][W] float as read in "PR" mode (projectionDataTOMO.cpp:250-273).
// img_out: [N][N] float (one slice).  filtered_out (optional): [V][W].
// filter: 1 Ram-Lak, 2 Shepp-Logan.  t_filter/t_bp receive the wall times of
// filterSinogram and reconstructImage.
int vctref_fbp(int filter, int V, int W, const float* sino, int N, double pixel_cm, int xfactor,
               const double* cosT, const double* sinT, float* img_out, float* filtered_out,
               double* t_filter, double* t_bp) {
  if (W != End_Channel - Start_Channel) return -1;
  QuietStd q;
  float** proj = (float**)new2DArray(W, V, UNIT_FLOAT32);
  float** fltd = (float**)new2DArray(W, V, UNIT_FLOAT32);
  float*** img = (float***)new3DArray(N, N, 1, UNIT_FLOAT32);
  if (!proj || !fltd || !img) return -2;
  memcpy(get1DArrayOf2DArray((void**)proj, UNIT_FLOAT32), sino, sizeof(float) * V * W);
  double** constMap = prepareConstMap(W, filter);
  double* w0 = (double*)new1DArray(W, UNIT_FLOAT64);
  double* w1 = (double*)new1DArray(W, UNIT_FLOAT64);
  double* w2 = (double*)new1DArray(W, UNIT_FLOAT64);
  prepareCorrectedDetectorInterpolation(W, w0, w1, w2);
  char** mask = prepareMaskData(N);
  double* xs = (double*)new1DArray(V, UNIT_FLOAT64);
  double* ys = (double*)new1DArray(V, UNIT_FLOAT64);
  char cls[16] = "PR";
  double t0 = now_s();
  filterSinogram(V, 1, 1, proj, fltd, constMap, w0, w1, w2, xs, ys, cls);
  double t1 = now_s();
  reconstructImage(N, img, mask, W, V, fltd, (double*)cosT, (double*)sinT, 0.0, 0.2, 1, 0.0, 0.0, 1,
                   (double)xfactor, pixel_cm, cls);
  double t2 = now_s();
  if (t_filter) *t_filter = t1 - t0;
  if (t_bp) *t_bp = t2 - t1;
  memcpy(img_out, get1DArrayOf3DArray((void***)img, UNIT_FLOAT32), sizeof(float) * N * N);
  if (filtered_out)
    memcpy(filtered_out, get1DArrayOf2DArray((void**)fltd, UNIT_FLOAT32), sizeof(float) * V * W);
  delete2DArray((void**)proj, W, V, UNIT_FLOAT32);
  delete2DArray((void**)fltd, W, V, UNIT_FLOAT32);
  delete3DArray((void***)img, N, N, 1, UNIT_FLOAT32);
  delete2DArray((void**)constMap, W, W, UNIT_FLOAT64);
  delete2DArray((void**)mask, N, N, UNIT_UINT8);
  delete1DArray(w0); delete1DArray(w1); delete1DArray(w2);
  delete1DArray(xs); delete1DArray(ys);
  return 0;
}

}  // extern "C"
