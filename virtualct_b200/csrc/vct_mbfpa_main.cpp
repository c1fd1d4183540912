// vct_mbfpa -- drop-in for Release_MBFPA_CPU_human/mvct.exe.
//
//   vct_mbfpa <input.txt> [--weights FILE] [--elements H,C,N,O,P,Ca[,Mg,Si]]
//             [--seed N] [--device N] [--sum compensated|reference]
//
// Reads the reference's 31-field input txt, the int16 element maps (the
// reference hard-codes Weight_input_ICRU110.raw and six elements,
// MB/main.cpp:240,422) and the spectrum txt; writes reprojection_float.raw
// (float32 [views][width]) and npf_float.raw (lengthproj_TOMO of the measured
// sinogram, MB/main.cpp:407-419, on the GPU).
// The measured sinogram: when the txt names a sinogram and an air scan that
// exist, vct_load_measured normalises them (loadProjectionData,
// MB/projectionDataTOMO.cpp:324-508; the volume is also written to
// projections.raw, as there) and vct_helical_sinogram interpolates the
// slice's sinogram (MB/main.cpp:347-371).  The virtual path names none ("*"),
// so, as in the reference, the measured sinogram and npf are all zeros.
// The energy loop, spectral sum, normalisation and noise of
// MB/main.cpp:492-530 are one call to vct_mbfpa() on the GPU.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <string>
#include <vector>

#include "vct.h"
#include "vct_io.h"

static int element_z(const std::string& s) {
  if (s == "H") return 1;
  if (s == "C") return 6;
  if (s == "N") return 7;
  if (s == "O") return 8;
  if (s == "P") return 15;
  if (s == "Ca") return 20;
  if (s == "Mg") return 12;
  if (s == "Si") return 14;
  return -1;
}

int main(int argc, char* argv[]) {
  if (argc < 2) {
    fprintf(stderr, "\n[usage]$ mvct <info filename>\n\n");
    return 0;
  }
  std::string weights = "Weight_input_ICRU110.raw";
  std::vector<int> Z = {1, 6, 7, 8, 15, 20};
  unsigned long long seed = 1;
  int device = 0;
  int sum_mode = VCT_SUM_COMPENSATED;
  for (int i = 2; i < argc; i++) {
    std::string a = argv[i];
    if (a == "--weights" && i + 1 < argc) weights = argv[++i];
    else if (a == "--seed" && i + 1 < argc) seed = strtoull(argv[++i], nullptr, 10);
    else if (a == "--device" && i + 1 < argc) device = atoi(argv[++i]);
    else if (a == "--sum" && i + 1 < argc) {
      std::string m = argv[++i];
      sum_mode = m == "reference" ? VCT_SUM_REFERENCE : VCT_SUM_COMPENSATED;
    } else if (a == "--elements" && i + 1 < argc) {
      Z.clear();
      std::string list = argv[++i];
      size_t p = 0;
      while (p <= list.size()) {
        size_t q = list.find(',', p);
        if (q == std::string::npos) q = list.size();
        int z = element_z(list.substr(p, q - p));
        if (z < 0) {
          fprintf(stderr, "unknown element %s\n", list.substr(p, q - p).c_str());
          return 1;
        }
        Z.push_back(z);
        p = q + 1;
      }
    } else {
      fprintf(stderr, "unknown option %s\n", a.c_str());
      return 1;
    }
  }
  const int M = (int)Z.size();

  vct_mb_config cfg;
  if (vct_load_mb_config(argv[1], &cfg) != VCT_OK) {
    fprintf(stderr, "%s\n", vct_last_error());
    return 0;  // the reference exits 0 here (MB/main.cpp:225-228)
  }
  FILE* fp = fopen(cfg.recon_data_file, "rb");
  if (!fp) fprintf(stderr, "No prior image \n");
  else {
    fprintf(stderr, "Prior image: %s \n", cfg.recon_data_file);
    fclose(fp);
  }
  vct_geometry g;
  vct_mb_geometry(&cfg, &g);
  fprintf(stderr, "usedProj: %d SngrmH: %d SngrmW: %d\n", cfg.total_proj_number, g.views, g.width);
  struct stat st;
  if (stat("ReconImageRaw", &st) != 0) mkdir("ReconImageRaw", 0775);

  std::vector<float> mu((size_t)M * VCT_MAX_BINS), pdf(VCT_MAX_BINS);
  int NE = 0;
  if (vct_attenuation_coefficient(cfg.spectrum_file, 1, Z.data(), M, mu.data(), pdf.data(), &NE) != VCT_OK) {
    fprintf(stderr, "%s\n", vct_last_error());
    return 1;
  }
  printf("%d energy bins, %d elements\n", NE, M);

  const size_t n2 = (size_t)g.recon_size * g.recon_size;
  std::vector<int16_t> maps((size_t)M * n2);
  if (vct_read_raw(weights.c_str(), 0, maps.data(), maps.size() * sizeof(int16_t), nullptr) != VCT_OK) {
    fprintf(stderr, "%s\n", vct_last_error());
    return 1;
  }
  // loadProjectionData (MB/projectionDataTOMO.cpp:324-508), reached from
  // loadData before the prior-image message.
  const size_t proj2 = (size_t)g.views * g.width;
  std::vector<float> measured(proj2, 0.0f);  // projection_float of MB/main.cpp:248
  {
    fprintf(stderr, strcmp(cfg.in_pr_class, "PR") == 0 ? "Pre-treatment CT \n" : "In-treatment CT \n");
    vct_raw_layout lay;
    vct_raw_layout_default(&lay);
    const int R = cfg.total_proj_number;
    std::vector<float> volume((size_t)(R > 0 ? R : 0) * proj2);
    std::vector<unsigned char> vmask(volume.size());
    int got = 0;
    double pmax = 0.0;
    const int rc = vct_load_measured(&cfg, &lay, device, volume.data(), vmask.data(), &got, &pmax);
    if (rc == VCT_E_IO) {
      fprintf(stderr, "%s\n", vct_last_error());  // the reference goes on with a zero volume
    } else if (rc == VCT_E_RANGE) {
      fprintf(stderr, "%s \n", vct_last_error());
      return 0;  // :474-477
    } else if (rc != VCT_OK) {
      fprintf(stderr, "%s\n", vct_last_error());
      return 1;
    } else {
      fprintf(stderr, "Maximum projection: %lf \n", pmax);
      if (vct_write_raw("projections.raw", volume.data(), volume.size() * sizeof(float)) != VCT_OK)
        fprintf(stderr, "%s\n", vct_last_error());
      if (got == 0) return 0;  // loadData returned 0: main exits (MB/main.cpp:225-228)
      if (vct_helical_sinogram(volume.data(), got, g.views, g.width, measured.data(), device) != VCT_OK) {
        fprintf(stderr, "%s\n", vct_last_error());
        return 1;
      }
    }
  }
  vct_ctx* ctx = nullptr;
  int rc = vct_create(&g, device, &ctx);
  if (rc == VCT_OK) rc = vct_set_sum_mode(ctx, sum_mode);
  if (rc == VCT_OK) rc = vct_set_maps(ctx, maps.data(), M);
  if (rc == VCT_OK) rc = vct_set_spectrum(ctx, mu.data(), pdf.data(), M, NE);
  if (rc == VCT_OK) {
    // lengthproj_TOMO at the first slice's z with the measured sinogram
    // (MB/main.cpp:346-370, zeros on the virtual path).
    std::vector<float> npf(n2, 0.0f);
    rc = vct_lengthproj(ctx, measured.data(), cfg.recon_offset, cfg.couch_speed, npf.data());
    if (rc == VCT_OK) rc = vct_write_raw("npf_float.raw", npf.data(), n2 * sizeof(float));
  }
  std::vector<float> sino((size_t)g.views * g.width);
  float stats[3] = {0, 0, 0};
  if (rc == VCT_OK) rc = vct_mbfpa(ctx, cfg.photon_noise, seed, sino.data(), stats);
  if (rc != VCT_OK) {
    fprintf(stderr, "vct_mbfpa failed: %s (%s)\n", vct_strerror(rc), vct_last_error());
    vct_destroy(ctx);
    return 1;
  }
  printf("projection_min = %lf, used noise = %lf\n", (double)stats[1], cfg.photon_noise);
  rc = vct_write_raw("reprojection_float.raw", sino.data(), sino.size() * sizeof(float));
  // The iterative step (MB/main.cpp:432-600 at ite 1, after the energy loop):
  // first element's map updated by IR_ImageTOMO, written as
  // ReconImageRaw/Reconstruction_ite0001_z0000.raw, and as int16
  // 1024*(x - 0.0716)/0.0716 of the best image to Reconstruction_512x512x<slices>.raw.
  // The reference's slice loop runs for slice 0 only, whatever the txt's
  // slice count (MB/main.cpp:322-323).
  if (rc == VCT_OK) {
    char name[256];
    snprintf(name, sizeof name, "ReconImageRaw/Reconstruction_512x512x%d.raw", cfg.recon_slices);
    FILE* fprecon = fopen(name, "wb");
    const int thinout = cfg.osemset > 0 ? cfg.osemset : 1;
    std::vector<float> npf(n2, 0.0f), before(n2), after(n2), best(n2, 0.0f);
    std::vector<int16_t> img16(n2);
    for (int rz = 0; rz < 1 && rc == VCT_OK; rz++) {
      const double zpos = cfg.recon_offset + rz * cfg.recon_step;
      rc = vct_lengthproj(ctx, measured.data(), zpos, cfg.couch_speed, npf.data());
      for (size_t i = 0; i < n2; i++) before[i] = (float)maps[i] / 1000;  // initial_image_def
      std::fill(after.begin(), after.end(), 0.0f);
      double wbefore = cfg.gradient_decent_const + 0.0005, objective = 10000000.0, quadratic = 0.0;
      double min_squdiff = 10000000.0;
      if (rc == VCT_OK)
        rc = vct_ir_step(ctx, measured.data(), npf.data(), before.data(), nullptr, zpos, cfg.couch_speed, 1, thinout,
                         cfg.num_ite, cfg.total_variation, cfg.prior_const, &wbefore, &objective, &quadratic,
                         after.data());
      if (rc != VCT_OK) break;
      snprintf(name, sizeof name, "ReconImageRaw/Reconstruction_ite%04d_z%04d.raw", 1, rz);
      rc = vct_write_raw(name, after.data(), n2 * sizeof(float));
      if (min_squdiff > objective) best = after;  // calc_reconImagefloat_min
      else std::fill(best.begin(), best.end(), 0.0f);
      for (size_t i = 0; i < n2; i++) img16[i] = (short)(1024 * (best[i] - 0.0716) / 0.0716);
      if (fprecon) fwrite(img16.data(), sizeof(int16_t), n2, fprecon);
    }
    if (fprecon) fclose(fprecon);
  }
  vct_destroy(ctx);
  if (rc != VCT_OK) {
    fprintf(stderr, "%s\n", vct_last_error());
    return 1;
  }
  fprintf(stderr, "done.\n");
  return 0;
}
