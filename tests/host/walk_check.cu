// CPU check of the device ray walks: compiles the product's walk code
// (virtualct_b200/csrc/vct_forward.cu, __host__ __device__) for the host and
// compares the fast walk with the reference-exact walk on every ray.
//   walk_check <maps.raw int16 [6][N][N]> <N> <pixel_cm> <views> <channels> <out.bin>
// out.bin: double L_exact[views][channels][6] then L_fast[...]; stdout: counts.
#include "../../virtualct_b200/csrc/vct_forward.cu"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace vct {
void set_error(const std::string&) {}
int fail(int code, const std::string&) { return code; }
int cuda_fail(cudaError_t, const char*) { return VCT_E_CUDA; }
}  // namespace vct
using namespace vct;

int main(int argc, char** argv) {
  if (argc != 7) return 2;
  const int N = atoi(argv[2]), V = atoi(argv[4]), C = atoi(argv[5]);
  const double s = atof(argv[3]);
  const int M = 6;
  std::vector<int16_t> maps((size_t)M * N * N);
  FILE* f = fopen(argv[1], "rb");
  if (!f || fread(maps.data(), 2, maps.size(), f) != maps.size()) return 3;
  fclose(f);
  // The device layout, packed by the product's own per-pixel routine: both
  // 16-byte layouts and the split copy.
  std::vector<PixelRec> packed(map_records(N));
  const int P = N + 2 * kMapPad;
  for (int p = 0; p < P * P; p++) pack_maps_elem(p, maps.data(), M, N, packed.data(), packed.data() + (size_t)P * P);
  // Geometry exactly as vct_create derives it (defaults of physParamsTOMO.h).
  DevGeom dg;
  dg.N = N;
  dg.nxm = (int)(N * 0.5);
  dg.s = s;
  dg.lim = (double)dg.nxm * s;
  dg.rmax = N * 0.5 * 1.0;
  dg.rmax_active = (dg.lim * sqrt(2.0) + 2.0 * s) >= dg.rmax;
  dg.sid = 85.0;
  dg.views = V;
  dg.views_used = V / 2 * 2;
  dg.width = C;
  dg.C = C;
  dg.start = 0;
  const double kPI = 3.141592653589793238462643383279;
  const double iso = C / 2.0, max_alpha = 0.326086956;
  const int half = (C - 1) / 2;
  std::vector<double> ct(V), st(V), px0(C), py0(C);
  for (int i = 0; i < V; i++) {
    double angle = (double)(360.0 / V * i);
    double rad = (0.0 + angle) * kPI / 180.0;
    ct[i] = cos(rad);
    st[i] = sin(rad);
  }
  for (int c = 0; c < C; c++) {
    double theta = (iso - c) * max_alpha / half;
    px0[c] = 142.6 * sin(theta);
    py0[c] = -142.6 * cos(theta) + 85.0;
  }
  std::vector<double> Le((size_t)V * C * M, 0), Lf((size_t)V * C * M, 0);
  long long nse = 0, nsf = 0, fallback = 0, miss = 0;
  for (int v = 0; v < dg.views_used; v++)
    for (int c = 0; c < C; c++) {
      Ray r;
      RayAcc ae, af;
      acc_init(ae);
      acc_init(af);
      if (!ray_setup(dg, ct[v], st[v], px0[c], py0[c], r)) {
        miss++;
        continue;
      }
      walk_exact<M>(dg, packed.data(), r, ae);
      if (dg.rmax_active || !walk_fast<M>(dg, packed.data(), r, af)) {
        fallback++;
        acc_init(af);
        walk_exact<M>(dg, packed.data(), r, af);
      }
      double le[8], lf[8];
      finish_lines<M>(ae, le);
      finish_lines<M>(af, lf);
      nse += ae.nseg;
      nsf += af.nseg;
      for (int m = 0; m < M; m++) {
        size_t o = ((size_t)v * C + c) * M + m;
        Le[o] = le[m];
        Lf[o] = lf[m];
      }
    }
  printf("%lld %lld %lld %lld\n", miss, fallback, nse, nsf);
  FILE* o = fopen(argv[6], "wb");
  fwrite(Le.data(), 8, Le.size(), o);
  fwrite(Lf.data(), 8, Lf.size(), o);
  fclose(o);
  return 0;
}
