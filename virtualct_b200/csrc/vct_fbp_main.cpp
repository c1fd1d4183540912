// vct_fbp -- drop-in for Release_FBP_CPU/mvct.exe.
//
//   vct_fbp <input.txt> [--device N]
//
// Reads the reference's 21-field FBP txt and the float32 sinogram it names,
// runs filterSinogram + reconstructImage (FBP/main.cpp:137-167) as one
// vct_fbp() call on the GPU and writes float32 [slices][N][N] to the output
// name of the txt, as FBP/main.cpp:187-190.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "vct.h"
#include "vct_io.h"

int main(int argc, char* argv[]) {
  if (argc < 2) {
    fprintf(stderr, "\n[usage]$ cbct <info filename>\n\n");
    return 0;
  }
  int device = 0;
  for (int i = 2; i < argc; i++) {
    std::string a = argv[i];
    if (a == "--device" && i + 1 < argc) device = atoi(argv[++i]);
    else {
      fprintf(stderr, "unknown option %s\n", a.c_str());
      return 1;
    }
  }
  vct_fbp_config cfg;
  if (vct_load_fbp_config(argv[1], &cfg) != VCT_OK) {
    fprintf(stderr, "%s\n", vct_last_error());
    return 0;  // FBP/main.cpp:44-48
  }
  if (strcmp(cfg.proj_data_type, "float") != 0) {
    fprintf(stderr, "data type %s: only float sinograms are supported\n", cfg.proj_data_type);
    return 1;
  }
  vct_geometry g;
  vct_fbp_geometry(&cfg, &g);
  const int V = g.views, W = g.width;
  // loadProjectionData (FBP/projectionDataTOMO.cpp:250-292): the first
  // rotation's [V][W] floats; a short file leaves the rest 0.
  std::vector<float> sino((size_t)V * W, 0.0f);
  size_t got = 0;
  if (vct_read_raw(cfg.proj_file, 0, sino.data(), sino.size() * sizeof(float), &got) == VCT_E_IO && got == 0) {
    fprintf(stderr, "data file: %s not found\n", cfg.proj_file);
  }
  if (strcmp(cfg.in_pr_class, "IN") == 0)
    for (auto& p : sino)
      if (p < 50000.0f) p = 1.0f;  // :285-288

  FILE* fp = fopen(cfg.output_file, "wb");
  if (!fp) {
    fprintf(stderr, "ERROR: output file NOT writable\n");
    return 0;
  }
  // Reconstruction range check, FBP/main.cpp:118-128.
  const double zstart = cfg.recon_offset;
  const double zend = cfg.recon_offset + (cfg.recon_slices - 1) * cfg.recon_step;
  const double s_start = cfg.start_couch_position + cfg.couch_speed / 2 + cfg.couch_speed - 0.0000001;
  const double s_end = cfg.start_couch_position + (cfg.total_proj_number) * cfg.couch_speed -
                       cfg.couch_speed / (2 + 0.0000001);
  fprintf(stderr, "Allowable reconstraction range = %lf to %lf \n", s_start, s_end);
  if (zstart < s_start || zend > s_end) {
    fprintf(stderr, "\n Wrong reconstruction range !!-- STOP\n\n");
    fclose(fp);
    return 0;
  }
  vct_ctx* ctx = nullptr;
  const size_t n2 = (size_t)g.recon_size * g.recon_size;
  std::vector<float> img(n2);
  int rc = vct_create(&g, device, &ctx);
  if (rc == VCT_OK) rc = vct_fbp(ctx, sino.data(), cfg.filter, strcmp(cfg.in_pr_class, "IN") == 0, img.data());
  vct_destroy(ctx);
  if (rc != VCT_OK) {
    fprintf(stderr, "vct_fbp failed: %s (%s)\n", vct_strerror(rc), vct_last_error());
    fclose(fp);
    return 1;
  }
  // Every slice reconstructs from the same first-rotation views (z_image = 0,
  // FBP/reconstructImageTOMO.cpp:36-41).
  for (int z = 0; z < cfg.recon_slices; z++) fwrite(img.data(), sizeof(float), n2, fp);
  fclose(fp);
  fprintf(stderr, "done.\n");
  return 0;
}
