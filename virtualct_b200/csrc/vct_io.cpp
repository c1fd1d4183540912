// Input-txt parsers and raw file helpers (include/vct_io.h).
#include "../../include/vct_io.h"

#include <stdio.h>
#include <string.h>

#include <string>

#include "vct_internal.h"

using vct::fail;

namespace {
constexpr int kLineBuf = 512;  // LINEBUF_SIZE, MB/projectionDataTOMO.cpp:11

struct TxtReader {
  FILE* fp;
  char line[kLineBuf];
  int field = 0;     // fields read so far
  int missing = -1;  // the first field whose value line is past the end of the file
  void skip(int n) {
    for (int i = 0; i < n; i++)
      if (!fgets(line, kLineBuf, fp)) line[0] = 0;
  }
  // One field = two skipped lines + one value line (:24-64).  A value line
  // that sscanf cannot parse leaves the field unchanged, as in the reference;
  // a file that ends before a value line is refused (the reference would read
  // on with the field uninitialised).
  void next() {
    skip(2);
    if (!fgets(line, kLineBuf, fp)) {
      line[0] = 0;
      if (missing < 0) missing = field;
    }
    field++;
  }
  int check(const char* path) const {
    if (missing < 0) return VCT_OK;
    return fail(VCT_E_IO, std::string("info file: ") + path + " ends before field " + std::to_string(missing + 1));
  }
  void i(int* v) { next(); sscanf(line, "%d", v); }
  void d(double* v) { next(); sscanf(line, "%lf", v); }
  void d3(double* a, double* b, double* c) { next(); sscanf(line, "%lf %lf %lf", a, b, c); }
  void s(char* v, size_t cap) {
    next();
    char tmp[kLineBuf];
    tmp[0] = 0;
    if (sscanf(line, "%511s", tmp) == 1) {
      strncpy(v, tmp, cap - 1);
      v[cap - 1] = 0;
    }
  }
};
}  // namespace

extern "C" {

int vct_load_mb_config(const char* path, vct_mb_config* c) {
  if (!path || !c) return fail(VCT_E_ARG, "null argument");
  memset(c, 0, sizeof(*c));
  FILE* fp = fopen(path, "r");
  if (!fp) return fail(VCT_E_IO, std::string("info file: ") + path + " not found");
  TxtReader r{fp, {0}};
  r.skip(6);
  r.s(c->in_pr_class, sizeof c->in_pr_class);
  r.i(&c->prior_image_onoff);
  r.i(&c->proj_width);
  r.i(&c->proj_height);
  r.s(c->proj_data_type, sizeof c->proj_data_type);
  r.i(&c->proj_file_offset);
  r.s(c->proj_file, sizeof c->proj_file);
  r.s(c->air_scan_file, sizeof c->air_scan_file);
  r.d(&c->gantry_rotation_period);
  r.d(&c->data_sampling_rate);
  r.d(&c->start_view_angle);
  r.d(&c->couch_speed);
  r.d(&c->start_couch_position);
  r.i(&c->recon_size);
  r.d(&c->recon_pix_size);
  r.s(c->recon_tgt_class, sizeof c->recon_tgt_class);
  r.d(&c->recon_offset);
  r.d(&c->recon_step);
  r.i(&c->recon_slices);
  r.i(&c->xfactor);
  r.s(c->recon_data_file, sizeof c->recon_data_file);
  r.i(&c->fbp_slice);
  r.d3(&c->x_reg, &c->y_reg, &c->z_reg);
  r.d(&c->scan_list_z);
  c->z_reg = c->scan_list_z - c->couch_speed * 1.5 + c->recon_offset + c->z_reg;  // :109
  r.i(&c->osemset);
  r.d3(&c->total_variation, &c->prior_const, &c->markov_const);
  r.d(&c->gradient_decent_const);
  r.i(&c->num_ite);
  r.i(&c->sino_fact);
  r.s(c->spectrum_file, sizeof c->spectrum_file);
  r.d(&c->photon_noise);
  fclose(fp);
  if (int rc = r.check(path)) return rc;
  // :125-134
  c->data_sampling_rate_orig = c->data_sampling_rate;
  if (c->data_sampling_rate >= 200) c->data_sampling_rate = c->data_sampling_rate / 5;
  c->total_proj_number = (int)(c->proj_height / (c->gantry_rotation_period * c->data_sampling_rate_orig));
  c->proj_height = (int)(c->gantry_rotation_period * c->data_sampling_rate);
  // loadProjectionData :332-333 (sino_fact thins the views).
  if (c->sino_fact > 0) c->proj_height = c->proj_height / c->sino_fact;
  return VCT_OK;
}

int vct_load_fbp_config(const char* path, vct_fbp_config* c) {
  if (!path || !c) return fail(VCT_E_ARG, "null argument");
  memset(c, 0, sizeof(*c));
  FILE* fp = fopen(path, "r");
  if (!fp) return fail(VCT_E_IO, std::string("info file: ") + path + " not found");
  TxtReader r{fp, {0}};
  r.skip(6);
  r.s(c->in_pr_class, sizeof c->in_pr_class);
  r.i(&c->filter);
  r.i(&c->proj_width);
  r.i(&c->proj_height);
  r.s(c->proj_data_type, sizeof c->proj_data_type);
  r.i(&c->proj_file_offset);
  r.s(c->proj_file, sizeof c->proj_file);
  r.s(c->air_scan_file, sizeof c->air_scan_file);
  r.d(&c->gantry_rotation_period);
  r.d(&c->data_sampling_rate);
  r.d(&c->start_view_angle);
  r.d(&c->couch_speed);
  r.d(&c->start_couch_position);
  r.i(&c->recon_size);
  r.d(&c->recon_pix_size);
  r.s(c->recon_tgt_class, sizeof c->recon_tgt_class);
  r.d(&c->recon_offset);
  r.d(&c->recon_step);
  r.i(&c->recon_slices);
  r.i(&c->xfactor);
  r.s(c->output_file, sizeof c->output_file);
  fclose(fp);
  if (int rc = r.check(path)) return rc;
  // FBP/projectionDataTOMO.cpp:94-96
  c->total_proj_number = (int)(c->proj_height / (c->gantry_rotation_period * c->data_sampling_rate));
  c->proj_height = (int)(c->gantry_rotation_period * c->data_sampling_rate);
  return VCT_OK;
}

void vct_mb_geometry(const vct_mb_config* c, vct_geometry* g) {
  vct_geometry_default(g);
  g->views = c->proj_height;
  g->width = c->proj_width;
  g->start_view_deg = c->start_view_angle;
  g->recon_size = c->recon_size;
  g->pixel_cm = c->recon_pix_size;
  g->xfactor = c->xfactor;
}

void vct_fbp_geometry(const vct_fbp_config* c, vct_geometry* g) {
  vct_geometry_default(g);
  g->views = c->proj_height;
  g->width = c->proj_width;
  g->start_view_deg = c->start_view_angle;
  g->recon_size = c->recon_size;
  g->pixel_cm = c->recon_pix_size;
  g->xfactor = c->xfactor;
}

int vct_read_raw(const char* path, long offset, void* buf, size_t bytes, size_t* got) {
  if (got) *got = 0;
  if (!path || (!buf && bytes)) return fail(VCT_E_ARG, "null argument");
  FILE* fp = fopen(path, "rb");
  if (!fp) return fail(VCT_E_IO, std::string("data file: ") + path + " not found");
  if (offset > 0 && fseek(fp, offset, SEEK_SET) != 0) {
    fclose(fp);
    return fail(VCT_E_IO, std::string("cannot seek in ") + path);
  }
  size_t n = fread(buf, 1, bytes, fp);
  fclose(fp);
  if (got) *got = n;
  if (n != bytes) return fail(VCT_E_IO, std::string("WARNING: data size unmatch in ") + path);
  return VCT_OK;
}

int vct_write_raw(const char* path, const void* buf, size_t bytes) {
  if (!path || (!buf && bytes)) return fail(VCT_E_ARG, "null argument");
  FILE* fp = fopen(path, "wb");
  if (!fp) return fail(VCT_E_IO, std::string("ERROR: output file NOT writable: ") + path);
  size_t n = fwrite(buf, 1, bytes, fp);
  fclose(fp);
  if (n != bytes) return fail(VCT_E_IO, std::string("short write to ") + path);
  return VCT_OK;
}

}  // extern "C"
