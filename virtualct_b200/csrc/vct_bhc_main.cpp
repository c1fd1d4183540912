// vct_bhc -- drop-in for the reference's beam-hardening correction program
// (Release_MBFPA_CPU_human/beam_hardening_correction.cpp):
//
//   vct_bhc <alpha> <beta> [--views V --width W] [--device N]
//
// Reads reprojection_float.raw (float32 [800][609] unless --views/--width)
// from the working directory, corrects every transmission on the GPU
// (vct_beam_hardening), prints the minimum before and after, and writes
// reprojection_float_cor.raw.  Like the reference: without two arguments it
// prints its usage and exits 0; a missing input file is an error.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "vct.h"
#include "vct_io.h"

int main(int argc, char** argv) {
  int views = 800, width = 609, device = 0;
  std::vector<const char*> pos;
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "--views") && i + 1 < argc) views = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--width") && i + 1 < argc) width = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--device") && i + 1 < argc) device = atoi(argv[++i]);
    else pos.push_back(argv[i]);
  }
  if (pos.size() != 2) {
    fprintf(stderr, "\n[usage]$ no alpha and beta \n\n");
    return 0;
  }
  const double alpha = atof(pos[0]), beta = atof(pos[1]);
  const size_t n = (size_t)views * width;
  std::vector<float> p(n), out(n);
  FILE* fp = fopen("reprojection_float.raw", "rb");
  if (!fp) {
    fprintf(stderr, "data file: %s not found\n", "reprojection_float.raw");
    return 255;
  }
  size_t got = fread(p.data(), sizeof(float), n, fp);
  fclose(fp);
  if (got != n) {
    fprintf(stderr, "reprojection_float.raw: %zu of %zu floats\n", got, n);
    return 1;
  }
  vct_geometry g;
  vct_geometry_default(&g);
  g.views = views;
  g.width = width;
  g.end_channel = width;
  g.iso_channel = width / 2.0;
  vct_ctx* ctx = nullptr;
  int rc = vct_create(&g, device, &ctx);
  if (rc == VCT_OK) rc = vct_beam_hardening(ctx, p.data(), alpha, beta, out.data());
  vct_destroy(ctx);
  if (rc != VCT_OK) {
    fprintf(stderr, "%s\n", vct_last_error());
    return 1;
  }
  double min_org = 1000000, min_new = 1000000;
  for (size_t i = 0; i < n; i++) {
    if (min_org > p[i]) min_org = p[i];
    if (min_new > out[i]) min_new = out[i];
  }
  printf("%lf %lf \n", min_org, min_new);
  if (vct_write_raw("reprojection_float_cor.raw", out.data(), n * sizeof(float)) != VCT_OK) {
    fprintf(stderr, "%s\n", vct_last_error());
    return 1;
  }
  return 0;
}
