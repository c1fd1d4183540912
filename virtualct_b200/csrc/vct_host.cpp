// Host side of libvct: context, geometry tables, spectrum model and the C ABI
// declared in include/vct.h.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "vct_internal.h"
#include "vct_philox.h"

namespace vct {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? VCT_E_NOMEM : VCT_E_CUDA;
}
int check_geometry(const vct_geometry* g, const char* who) {
  const int C = g->end_channel - g->start_channel;
  if (g->views < 2 || g->views > 100000 || C < 3 || g->start_channel < 0 || g->width < g->end_channel ||
      g->recon_size < 2 || g->recon_size > 8192 || !(g->pixel_cm > 0) || g->xfactor == 0)
    return fail(VCT_E_ARG, std::string(who) + ": geometry out of range");
  return VCT_OK;
}

// PI as the reference spells it (MB/physParamsTOMO.h:1); rounds to M_PI.
static const double kPI = 3.141592653589793238462643383279;

}  // namespace vct

using namespace vct;

#include "vct_ctx.h"

// An NVTX range over a host entry point (visible to ncu --nvtx and to any
// NVTX-aware profiler; free when none is attached).
struct NvtxScope {
  explicit NvtxScope(const char* name) { nvtxRangePushA(name); }
  ~NvtxScope() { nvtxRangePop(); }
};

static int check_ctx(vct_ctx* c) {
  if (!c) return fail(VCT_E_ARG, "null context");
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  return VCT_OK;
}

extern "C" {

int vct_version(void) { return 100; }

void vct_geometry_default(vct_geometry* g) {
  if (!g) return;
  g->sid_cm = 85.0;
  g->det_radius_cm = 142.6;
  g->det_src_iso_cm = 85.0;
  g->start_channel = 0;
  g->end_channel = 609;
  g->iso_channel = 304.5;
  g->max_alpha = 0.326086956;
  g->max_beta = 0.326086956;
  g->views = 800;
  g->width = 609;
  g->start_view_deg = 0.0;
  g->recon_size = 512;
  g->pixel_cm = 0.1;
  g->xfactor = 1;
}

const char* vct_strerror(int code) {
  switch (code) {
    case VCT_OK: return "ok";
    case VCT_E_ARG: return "invalid argument";
    case VCT_E_CUDA: return "CUDA error";
    case VCT_E_TIMEOUT: return "device wait timed out";
    case VCT_E_NOMEM: return "out of memory";
    case VCT_E_IO: return "I/O error";
    case VCT_E_STATE: return "invalid call order";
    case VCT_E_UNSUPPORTED: return "unsupported configuration";
    case VCT_E_RANGE: return "measured value out of range";
    default: return "unknown error";
  }
}

const char* vct_last_error(void) { return g_last_error.c_str(); }

int vct_bounds_violations(unsigned long long* hits, int* where) {
  if (!hits || !where) return fail(VCT_E_ARG, "vct_bounds_violations: null argument");
#if VCT_BOUNDS
  int (*readers[])(unsigned int*, int*) = {bounds_forward, bounds_adjoint, bounds_fbp, bounds_lengthproj,
                                          bounds_measured};
  *hits = 0;
  *where = 0;
  for (int u = 0; u < (int)(sizeof readers / sizeof readers[0]); u++) {
    unsigned int h = 0;
    int line = 0;
    const int rc = readers[u](&h, &line);
    if (rc) return rc;
    if (h && !*where) *where = (u + 1) * 100000 + line;
    *hits += h;
  }
  return VCT_OK;
#else
  *hits = 0;
  *where = 0;
  return fail(VCT_E_UNSUPPORTED, "this library has no index checks; libvct_bounds.so has");
#endif
}

int vct_create(const vct_geometry* g, int device, vct_ctx** out) {
  if (!g || !out) return fail(VCT_E_ARG, "vct_create: null argument");
  *out = nullptr;
  const int C = g->end_channel - g->start_channel;
  if (int rc = check_geometry(g, "vct_create")) return rc;
  if ((C - 1) / 2 == 0) return fail(VCT_E_ARG, "vct_create: too few channels");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(VCT_E_CUDA, "vct_create: no CUDA device");
  if (device < 0 || device >= ndev) return fail(VCT_E_ARG, "vct_create: bad device index");
  VCT_CUDA(cudaSetDevice(device));
  vct_ctx* c = new vct_ctx();
  c->device = device;
  c->geo = *g;
  DevGeom& dg = c->dg;
  dg.N = g->recon_size;
  dg.nxm = (int)(g->recon_size * 0.5);
  dg.s = g->pixel_cm;
  dg.lim = (double)dg.nxm * g->pixel_cm;
  dg.rmax = g->recon_size * 0.5 * 1.0;
  // Largest midpoint radius a kept segment can have: half-diagonal of the
  // square plus one (pixel-sized) poke-out step.
  dg.rmax_active = (dg.lim * sqrt(2.0) + 2.0 * g->pixel_cm) >= dg.rmax ? 1 : 0;
  dg.sid = g->sid_cm;
  dg.dens_div = 1000.0;
  dg.views = g->views;
  dg.views_used = g->views / 2 * 2;
  dg.width = g->width;
  dg.C = C;
  dg.start = g->start_channel;

  int rc = VCT_OK;
  auto bail = [&](int code) {
    vct_destroy(c);
    return code;
  };
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(VCT_E_CUDA, "cudaStreamCreate"));
  c->stream = c->own_stream;

  // View angles and trig tables: MB/projectionDataTOMO.cpp:362-368,
  // MB/misc_TOMO.cpp:93-97 (host libm, so the tables equal the reference's).
  const int V = g->views;
  std::vector<double> ct(V), st(V);
  std::vector<float> csf(2 * V);
  for (int i = 0; i < V; i++) {
    double angle = (double)(360.0 / V * i);
    double rad = (g->start_view_deg + angle) * kPI / 180.0;
    ct[i] = cos(rad);
    st[i] = sin(rad);
    csf[2 * i] = (float)ct[i];
    csf[2 * i + 1] = (float)st[i];
  }
  // Detector point of every channel before rotation (:61-71).
  const int half = (C - 1) / 2;
  std::vector<double> px0(C), py0(C);
  for (int c0 = 0; c0 < C; c0++) {
    int jj = g->start_channel + c0;
    double theta = (g->iso_channel - jj) * g->max_alpha / half;
    double ox0 = g->det_radius_cm * sin(theta);
    double oy0 = -g->det_radius_cm * cos(theta);
    px0[c0] = ox0;
    py0[c0] = oy0 + g->det_src_iso_cm;
  }
  // FBP weight: SID*cos((k-centWidth)*dbeta) (FBP/filterSinogramTOMO.cpp:236),
  // times dbeta, the constant factor of each filter term (:242).
  const int cw = C / 2;
  const double dbeta = g->max_beta / half;
  std::vector<double> coeff(C);
  for (int k = 0; k < C; k++) coeff[k] = g->sid_cm * cos((k - cw) * (g->max_beta / half)) * dbeta;

  if ((rc = c->cos_t.ensure(V)) || (rc = c->sin_t.ensure(V)) || (rc = c->cs_f.ensure(2 * V)) ||
      (rc = c->det_px0.ensure(C)) || (rc = c->det_py0.ensure(C)) || (rc = c->fbp_coeff.ensure(C)) ||
      (rc = c->stats.ensure(2)))
    return bail(rc);
  if (cudaMallocHost((void**)&c->h_stats, sizeof(FwdStats)) != cudaSuccess)
    return bail(fail(VCT_E_NOMEM, "cudaMallocHost"));
  FwdStats init{};
  init.max_bits = 0u;           // 0.0f
  init.min_bits = 0x7f7fffffu;  // FLT_MAX
  init.segments = 0ull;
  cudaError_t e;
  if ((e = cudaMemcpy(c->stats.p + 1, &init, sizeof(FwdStats), cudaMemcpyHostToDevice)))
    return bail(cuda_fail(e, "vct_create: stats init"));
  if ((e = cudaMemcpy(c->cos_t.p, ct.data(), V * sizeof(double), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(c->sin_t.p, st.data(), V * sizeof(double), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(c->cs_f.p, csf.data(), 2 * V * sizeof(float), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(c->det_px0.p, px0.data(), C * sizeof(double), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(c->det_py0.p, py0.data(), C * sizeof(double), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(c->fbp_coeff.p, coeff.data(), C * sizeof(double), cudaMemcpyHostToDevice)))
    return bail(cuda_fail(e, "vct_create: table upload"));
  // The rays the fast walk hands back to the exact walk (rays through the
  // grid origin at even channel counts): counted, then listed.
  if (!c->dg.rmax_active) {
    int n = 0;
    if ((rc = c->fwd_exact.ensure(1)) ||
        (rc = launch_exact_list(c->dg, c->cos_t.p, c->sin_t.p, c->det_px0.p, c->det_py0.p, nullptr, 0, c->fwd_exact.p,
                                c->stream)))
      return bail(rc);
    if ((e = cudaMemcpyAsync(&n, c->fwd_exact.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream)) ||
        (e = cudaStreamSynchronize(c->stream)))
      return bail(cuda_fail(e, "vct_create: exact-walk rays"));
    if (n > 0) {
      if ((rc = c->fwd_exact.ensure((size_t)n + 1)) ||
          (rc = launch_exact_list(c->dg, c->cos_t.p, c->sin_t.p, c->det_px0.p, c->det_py0.p, c->fwd_exact.p + 1, n,
                                  c->fwd_exact.p, c->stream)))
        return bail(rc);
      if ((e = cudaStreamSynchronize(c->stream))) return bail(cuda_fail(e, "vct_create: exact-walk rays"));
    }
    c->fwd_nexact = n;
  }
  *out = c;
  return VCT_OK;
}

void vct_destroy(vct_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->own_stream) cudaStreamSynchronize(c->own_stream);
  c->cos_t.release(); c->sin_t.release(); c->cs_f.release(); c->det_px0.release(); c->det_py0.release();
  c->maps_raw.release(); c->maps.release(); c->mu_scaled.release(); c->mu_log2.release(); c->pdf.release();
  c->full.release(); c->out.release(); c->stats.release(); c->fwd_exact.release();
  c->fbp_coeff.release();
  for (auto& h : c->fbp_h) h.release();
  c->fbp_g.release(); c->fbp_q.release(); c->fbp_sino.release(); c->fbp_img.release(); c->fbp_tacc.release();
  c->fbp_q2.release();
  c->adj_rec.release(); c->adj_special.release(); c->adj_ints.release(); c->adj_dir.release();
  c->adj_tv.release();
  c->adj_g.release(); c->adj_part.release(); c->adj_loss.release(); c->adj_gmax.release();
  c->adj_sacc.release(); c->adj_lsp.release(); c->adj_meas.release(); c->adj_wts.release(); c->adj_grad.release();
  c->adj_ext.release();
  c->sq_part.release();
  c->ir_proj.release(); c->ir_reproj.release(); c->ir_img.release(); c->ir_out.release();
  if (c->h_stats) cudaFreeHost(c->h_stats);
  if (c->pipe) {
    cudaStreamSynchronize(c->pipe->out);
    delete c->pipe;
  }
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

int vct_set_stream(vct_ctx* c, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return VCT_OK;
}

int vct_synchronize(vct_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  return VCT_OK;
}

long long vct_kernel_launches(vct_ctx* c) { return c ? c->launches : -1; }

static int fetch_stats(vct_ctx* c);

int vct_last_segment_count(vct_ctx* c, long long* segments) {
  if (!c || !segments) return fail(VCT_E_ARG, "null argument");
  int rc = check_ctx(c);
  if (rc) return rc;
  if ((rc = fetch_stats(c))) return rc;  // waits for the context's stream
  *segments = c->last_segments;
  return VCT_OK;
}

// ------------------------------------------------------------------ spectrum
// Restates attenuation_coefficient, MB/prior_weight_production.cpp:180-297.
int vct_attenuation_coefficient(const char* path, int nthin, const int* Zs, int M, float* mu, float* pdf,
                                int* NE) {
  if (!path || !Zs || !mu || !pdf || !NE || M < 1 || M > VCT_MAX_MATERIALS || nthin < 1)
    return fail(VCT_E_ARG, "vct_attenuation_coefficient: bad argument");
  *NE = 0;
  FILE* fp = fopen(path, "r");
  if (!fp) return fail(VCT_E_IO, std::string("ERROR: no photon energy file ") + path);
  char row[1024];
  float d0 = 0, d1 = 0, d2 = 0;
  std::vector<double> pe;
  std::vector<float> raw;
  if (fgets(row, sizeof(row), fp) == NULL) { /* header line, :196 */ }
  while (fgets(row, sizeof(row), fp) != NULL) {
    if ((int)pe.size() >= VCT_MAX_BINS) {
      fclose(fp);
      return fail(VCT_E_UNSUPPORTED, "spectrum has more than 1024 bins");
    }
    sscanf(row, "%f %f %f", &d0, &d1, &d2);  // unparsable lines keep the last values (:202)
    pe.push_back((d1 + d0) * 0.5);
    raw.push_back(d2);
  }
  fclose(fp);
  const int n = (int)pe.size();
  if (n == 0) return fail(VCT_E_IO, "spectrum file has no bins");
  // Thinning by nthin (:210-235).
  std::vector<float> pdf_thin;
  std::vector<double> e_thin;
  double psum = 0.0, esum = 0.0, sum_thin = 0.0;
  for (int i = 0; i < n; i++) {
    psum += raw[i];
    esum += pe[i];
    if (i - nthin + 1 == (i - nthin + 1) / nthin * nthin) {
      pdf_thin.push_back((float)psum);
      e_thin.push_back((double)(float)(esum / nthin));
      sum_thin += psum;
      psum = 0.0;
      esum = 0.0;
    }
  }
  const int ne = (int)pdf_thin.size();
  const float sum = (float)sum_thin;  // float normalisation (:236-244)
  for (int i = 0; i < ne; i++) pdf[i] = pdf_thin[i] / sum;
  // Element table: (Z, A) of :250-255 plus Mg and Si with A = 2Z.
  const double Avogadro = 6.0221;  // MB/physParamsTOMO.h:89
  for (int iz = 0; iz < M; iz++) {
    double Z = Zs[iz], A;
    switch (Zs[iz]) {
      case 1: A = 1; break;
      case 6: A = 12; break;
      case 7: A = 14; break;
      case 8: A = 16; break;
      case 15: A = 31; break;
      case 20: A = 40; break;
      case 12: A = 24; break;
      case 14: A = 28; break;
      default: return fail(VCT_E_ARG, "element Z not in the reference's table");
    }
    double Ek = 0;
    double fact = Avogadro * Z / A * (2.81794 * 2.81794) * 0.001;
    for (int i = 0; i < ne; i++) {
      double E = e_thin[i] / 0.511;
      double photo = fact * 0.00000345 * (1.0 + 0.008 * Z) * (Z * Z * Z) / (E * E * E) *
                     (1.0 - Ek / (4.0 * E) - Ek * Ek / (1.21 * E));
      double compton = fact * 2 * kPI *
                       ((1.0 + E) / (E * E) * (2.0 * (1.0 + E) / (1.0 + 2 * E) - log(1.0 + 2 * E) / E) +
                        log(1.0 + 2 * E) / (2 * E) - (1.0 + 3 * E) / ((1.0 + 2 * E) * (1.0 + 2 * E)));
      double pair = fact * 0.2545 * (E - 2.332) * Z / 137;
      if (pair < 0) pair = 0;
      mu[ne * iz + i] = (float)(photo + compton + pair);
    }
  }
  *NE = ne;
  return VCT_OK;
}

// ------------------------------------------------------------------- MBFPA
int vct_set_maps_dev(vct_ctx* c, const int16_t* d_maps, int M) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_maps || M < 1 || M > VCT_MAX_MATERIALS) return fail(VCT_E_ARG, "vct_set_maps: bad argument");
  if (c->spectrum_ready && M != c->M) return fail(VCT_E_ARG, "vct_set_maps: M differs from the spectrum's");
  if ((rc = c->maps.ensure(map_records(c->dg.N)))) return rc;
  if ((rc = launch_pack_maps(d_maps, M, c->dg.N, c->maps.p, c->stream))) return rc;
  c->launches++;
  c->M = M;
  c->maps_ready = 1;
  return VCT_OK;
}

int vct_set_maps(vct_ctx* c, const int16_t* maps, int M) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!maps || M < 1 || M > VCT_MAX_MATERIALS) return fail(VCT_E_ARG, "vct_set_maps: bad argument");
  const size_t n2 = (size_t)c->dg.N * c->dg.N;
  if ((rc = c->maps_raw.ensure(n2 * M))) return rc;
  VCT_CUDA(cudaMemcpyAsync(c->maps_raw.p, maps, n2 * M * sizeof(int16_t), cudaMemcpyHostToDevice, c->stream));
  return vct_set_maps_dev(c, c->maps_raw.p, M);
}

int vct_set_spectrum(vct_ctx* c, const float* mu, const float* pdf, int M, int NE) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!mu || !pdf || M < 1 || M > VCT_MAX_MATERIALS || NE < 1 || NE > VCT_MAX_BINS)
    return fail(VCT_E_ARG, "vct_set_spectrum: bad argument");
  if (c->maps_ready && M != c->M) return fail(VCT_E_ARG, "vct_set_spectrum: M differs from the maps'");
  // Transpose to [NE][M] and fold 1/xfactor (exp(-transp/xfactor), :196).
  std::vector<double> t((size_t)NE * M), t2((size_t)NE * M);
  const double log2e = 1.4426950408889634073599246810019;
  for (int e = 0; e < NE; e++)
    for (int m = 0; m < M; m++) {
      t[(size_t)e * M + m] = (double)mu[(size_t)m * NE + e] / (double)c->geo.xfactor;
      t2[(size_t)e * M + m] = t[(size_t)e * M + m] * log2e;
    }
  if ((rc = c->mu_scaled.ensure((size_t)NE * M)) || (rc = c->mu_log2.ensure((size_t)NE * M)) ||
      (rc = c->pdf.ensure(NE)))
    return rc;
  VCT_CUDA(cudaMemcpyAsync(c->mu_scaled.p, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  VCT_CUDA(cudaMemcpyAsync(c->mu_log2.p, t2.data(), t2.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  VCT_CUDA(cudaMemcpyAsync(c->pdf.p, pdf, NE * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));  // t is a host temporary
  c->M = M;
  c->NE = NE;
  c->ynorm = 0.0;
  for (int e = 0; e < NE; e++) c->ynorm += (double)pdf[e];
  c->spectrum_ready = 1;
  return VCT_OK;
}

int vct_set_density_scale(vct_ctx* c, double units_per_gcc) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!(units_per_gcc > 0) || !(units_per_gcc < 1e9)) return fail(VCT_E_ARG, "vct_set_density_scale: bad scale");
  c->dg.dens_div = units_per_gcc;
  return VCT_OK;
}

int vct_set_sum_mode(vct_ctx* c, int mode) {
  if (!c) return fail(VCT_E_ARG, "null context");
  if (mode != VCT_SUM_COMPENSATED && mode != VCT_SUM_REFERENCE) return fail(VCT_E_ARG, "bad sum mode");
  c->sum_mode = mode;
  return VCT_OK;
}

int vct_set_walk_mode(vct_ctx* c, int mode) {
  if (!c) return fail(VCT_E_ARG, "null context");
  if (mode != VCT_WALK_FAST && mode != VCT_WALK_EXACT) return fail(VCT_E_ARG, "bad walk mode");
  c->walk_mode = mode;
  return VCT_OK;
}

// The exact-walk ray list the forward defers (with the fast walk), and the
// launches one forward takes.
static const int* exact_list(const vct_ctx* c) { return c->fwd_nexact > 0 ? c->fwd_exact.p + 1 : nullptr; }
static int forward_launches(const vct_ctx* c) {
  return 1 + (c->fwd_nexact > 0 && c->walk_mode == VCT_WALK_FAST && !c->dg.rmax_active);
}

static int forward_into(vct_ctx* c, float* d_out, double* d_lint) {
  if (!c->maps_ready || !c->spectrum_ready) return fail(VCT_E_STATE, "forward: maps or spectrum not set");
  const size_t nsino = (size_t)c->geo.views * c->geo.width;
  VCT_CUDA(cudaMemcpyAsync(c->stats.p, c->stats.p + 1, sizeof(FwdStats), cudaMemcpyDeviceToDevice, c->stream));
  if (d_out) VCT_CUDA(cudaMemsetAsync(d_out, 0, nsino * sizeof(float), c->stream));
  const double* mu_tab = c->sum_mode == VCT_SUM_REFERENCE ? c->mu_scaled.p : c->mu_log2.p;
  c->timer.begin(c->stream);
  int rc = launch_forward(c->dg, c->maps.p, c->M, mu_tab, c->pdf.p, c->NE, c->cos_t.p, c->sin_t.p,
                          c->det_px0.p, c->det_py0.p, c->sum_mode, c->walk_mode == VCT_WALK_FAST, d_out,
                          d_lint, c->stats.p, c->stream, 0, -1, exact_list(c), c->fwd_nexact);
  if (rc) return rc;
  c->timer.mark("forward_kernel", c->stream);
  c->launches += forward_launches(c);
  return VCT_OK;
}

static int fetch_stats(vct_ctx* c) {
  VCT_CUDA(cudaMemcpyAsync(c->h_stats, c->stats.p, sizeof(FwdStats), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  c->last_segments = (long long)c->h_stats->segments;
  return VCT_OK;
}

int vct_forward_dev(vct_ctx* c, float* d_out) {
  NvtxScope nvtx_scope("vct_forward_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_out) return fail(VCT_E_ARG, "null output");
  return forward_into(c, d_out, nullptr);
}

int vct_forward(vct_ctx* c, float* out) {
  NvtxScope nvtx_scope("vct_forward");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out) return fail(VCT_E_ARG, "null output");
  const size_t nsino = (size_t)c->geo.views * c->geo.width;
  if ((rc = c->full.ensure(nsino))) return rc;
  if ((rc = forward_into(c, c->full.p, nullptr))) return rc;
  VCT_CUDA(cudaMemcpyAsync(out, c->full.p, nsino * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  return fetch_stats(c);
}

int vct_line_integrals_dev(vct_ctx* c, double* d_lint) {
  NvtxScope nvtx_scope("vct_line_integrals_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_lint) return fail(VCT_E_ARG, "null output");
  return forward_into(c, nullptr, d_lint);
}

static int pad_zero_of(const vct_ctx* c) {
  // The reference's min runs over the whole [views][width] array: rows past
  // views/2*2 and channels outside [start,end) hold 0.
  return (c->dg.views_used < c->dg.views || c->dg.C < c->dg.width) ? 1 : 0;
}

int vct_normalize_noise_dev(vct_ctx* c, float* d_sino, double sigma, uint64_t seed) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_sino) return fail(VCT_E_ARG, "null sinogram");
  rc = launch_normalize_noise(c->dg, d_sino, d_sino, c->stats.p, pad_zero_of(c), sigma, seed, c->stream);
  if (!rc) c->launches++;
  return rc;
}

int vct_mbfpa_dev(vct_ctx* c, double sigma, uint64_t seed, float* d_out) {
  NvtxScope nvtx_scope("vct_mbfpa_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_out) return fail(VCT_E_ARG, "null output");
  const size_t nsino = (size_t)c->geo.views * c->geo.width;
  if ((rc = c->full.ensure(nsino))) return rc;
  if ((rc = forward_into(c, c->full.p, nullptr))) return rc;
  rc = launch_normalize_noise(c->dg, c->full.p, d_out, c->stats.p, pad_zero_of(c), sigma, seed, c->stream);
  if (!rc) c->launches++;
  return rc;
}

int vct_mbfpa(vct_ctx* c, double sigma, uint64_t seed, float* out, float* stats3) {
  NvtxScope nvtx_scope("vct_mbfpa");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out) return fail(VCT_E_ARG, "null output");
  const size_t nsino = (size_t)c->geo.views * c->geo.width;
  if ((rc = c->out.ensure(nsino))) return rc;
  if ((rc = vct_mbfpa_dev(c, sigma, seed, c->out.p))) return rc;
  VCT_CUDA(cudaMemcpyAsync(out, c->out.p, nsino * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  if ((rc = fetch_stats(c))) return rc;
  if (stats3) {
    float mx = 0, mn = 0;
    memcpy(&mx, &c->h_stats->max_bits, 4);
    memcpy(&mn, &c->h_stats->min_bits, 4);
    if (pad_zero_of(c)) mn = fminf(mn, 0.0f);
    stats3[0] = mx;
    stats3[1] = mn / mx;
    stats3[2] = (float)c->h_stats->segments;
  }
  return VCT_OK;
}

// Many slices from host buffers: slice i's maps go host->device on pipe->in
// while slice i-1 projects on the context's stream and slice i-2's sinogram
// goes device->host on pipe->out.  Two staging and two sinogram buffers; the
// events order each buffer's reuse.
static int ensure_pipe(vct_ctx* c) {
  if (c->pipe) return VCT_OK;
  vct::Pipe* p = new vct::Pipe();
  c->pipe = p;
  VCT_CUDA(cudaStreamCreateWithFlags(&p->in, cudaStreamNonBlocking));
  VCT_CUDA(cudaStreamCreateWithFlags(&p->out, cudaStreamNonBlocking));
  VCT_CUDA(cudaEventCreateWithFlags(&p->start, cudaEventDisableTiming));
  for (int s = 0; s < 2; s++)
    for (cudaEvent_t* e : {&p->ev_in[s], &p->ev_packed[s], &p->ev_done[s], &p->ev_out[s]})
      VCT_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return VCT_OK;
}

int vct_mbfpa_many(vct_ctx* c, int n, const int16_t* const* maps, int M, double sigma, uint64_t seed,
                   float* const* out, float* stats3) {
  NvtxScope nvtx_scope("vct_mbfpa_many");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (n < 0 || (n > 0 && (!maps || !out)) || M < 1 || M > VCT_MAX_MATERIALS)
    return fail(VCT_E_ARG, "vct_mbfpa_many: bad argument");
  if (n == 0) return VCT_OK;
  if (!c->spectrum_ready) return fail(VCT_E_STATE, "vct_mbfpa_many: spectrum not set");
  if (M != c->M) return fail(VCT_E_ARG, "vct_mbfpa_many: M differs from the spectrum's");
  for (int i = 0; i < n; i++)
    if (!maps[i] || !out[i]) return fail(VCT_E_ARG, "vct_mbfpa_many: null slice buffer");
  const size_t n2 = (size_t)c->dg.N * c->dg.N, nsino = (size_t)c->geo.views * c->geo.width;
  if ((rc = ensure_pipe(c))) return rc;
  vct::Pipe* p = c->pipe;
  for (int s = 0; s < 2; s++)
    if ((rc = p->stage[s].ensure(n2 * M)) || (rc = p->sino[s].ensure(nsino))) return rc;
  if ((rc = c->maps.ensure(map_records(c->dg.N))) || (rc = c->full.ensure(nsino))) return rc;
  vct::FwdStats* h = nullptr;  // per-slice statistics, pinned
  if (stats3) VCT_CUDA(cudaMallocHost((void**)&h, (size_t)n * sizeof(vct::FwdStats)));
  struct FreeHost {
    void* p;
    ~FreeHost() {
      if (p) cudaFreeHost(p);
    }
  } free_h{h};
  // everything below comes after the work already queued on the context's stream
  VCT_CUDA(cudaEventRecord(p->start, c->stream));
  VCT_CUDA(cudaStreamWaitEvent(p->in, p->start, 0));
  VCT_CUDA(cudaStreamWaitEvent(p->out, p->start, 0));
  const int pad = pad_zero_of(c);
  for (int i = 0; i < n; i++) {
    const int s = i & 1;
    if (i >= 2) VCT_CUDA(cudaStreamWaitEvent(p->in, p->ev_packed[s], 0));  // slice i-2 left stage[s]
    VCT_CUDA(cudaMemcpyAsync(p->stage[s].p, maps[i], n2 * M * sizeof(int16_t), cudaMemcpyHostToDevice, p->in));
    VCT_CUDA(cudaEventRecord(p->ev_in[s], p->in));
    VCT_CUDA(cudaStreamWaitEvent(c->stream, p->ev_in[s], 0));
    if ((rc = launch_pack_maps(p->stage[s].p, M, c->dg.N, c->maps.p, c->stream))) return rc;
    c->launches++;
    VCT_CUDA(cudaEventRecord(p->ev_packed[s], c->stream));
    c->maps_ready = 1;
    if ((rc = forward_into(c, c->full.p, nullptr))) return rc;
    if (i >= 2) VCT_CUDA(cudaStreamWaitEvent(c->stream, p->ev_out[s], 0));  // slice i-2 left sino[s]
    if ((rc = launch_normalize_noise(c->dg, c->full.p, p->sino[s].p, c->stats.p, pad, sigma, seed + (uint64_t)i,
                                     c->stream)))
      return rc;
    c->launches++;
    if (h) VCT_CUDA(cudaMemcpyAsync(h + i, c->stats.p, sizeof(vct::FwdStats), cudaMemcpyDeviceToHost, c->stream));
    VCT_CUDA(cudaEventRecord(p->ev_done[s], c->stream));
    VCT_CUDA(cudaStreamWaitEvent(p->out, p->ev_done[s], 0));
    VCT_CUDA(cudaMemcpyAsync(out[i], p->sino[s].p, nsino * sizeof(float), cudaMemcpyDeviceToHost, p->out));
    VCT_CUDA(cudaEventRecord(p->ev_out[s], p->out));
  }
  VCT_CUDA(cudaStreamWaitEvent(c->stream, p->ev_out[(n - 1) & 1], 0));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  VCT_CUDA(cudaStreamSynchronize(p->out));
  if (h) {
    for (int i = 0; i < n; i++) {
      float mx = 0, mn = 0;
      memcpy(&mx, &h[i].max_bits, 4);
      memcpy(&mn, &h[i].min_bits, 4);
      if (pad) mn = fminf(mn, 0.0f);
      stats3[3 * i] = mx;
      stats3[3 * i + 1] = mn / mx;
      stats3[3 * i + 2] = (float)h[i].segments;
    }
    c->last_segments = (long long)h[n - 1].segments;
  }
  return VCT_OK;
}

// --------------------------------------------------------------------- FBP
// prepareConstMap, FBP/filterSinogramTOMO.cpp:9-123, in double on the host.
// Every row is the kernel h0(m-k); rows m <= 20 and m >= C-20 are scaled by
// sum[21]/sum[m] (:114-123).  Stored for the device as float
// [h0(-(C-1)) .. h0(C-1)] followed by the C row factors.
static int build_filter(vct_ctx* c, int filter) {
  if (c->fbp_h[filter].p) return VCT_OK;
  const int C = c->dg.C;
  const int half = (C - 1) / 2;
  const double arc = c->geo.max_beta / half;
  auto kernel = [&](int MN) -> double {
    if (MN == 0) {
      if (filter == 1) return 0.125 / (arc * arc);
      double oddterm = kPI * kPI * (arc);
      return 0.25 / oddterm * (1.0 / tan((0.5) * arc) - 1.0 / tan((-0.5) * arc));
    }
    if (MN % 2 != 0) {
      if (filter == 1) {
        double oddterm = kPI * sin(MN * arc);
        return -0.5 / oddterm / oddterm;
      }
      double oddterm = kPI * kPI * arc;
      return 0.25 / oddterm * (1.0 / tan((MN + 0.5) * arc) - 1.0 / tan((MN - 0.5) * arc));
    }
    if (filter == 1) return 0.0;
    double oddterm = kPI * kPI * arc;
    return 0.25 / oddterm * (1.0 / tan((MN + 0.5) * arc) - 1.0 / tan((MN - 0.5) * arc));
  };
  std::vector<double> h0(2 * C - 1), sum(C, 0.0);
  for (int d = -(C - 1); d <= C - 1; d++) h0[d + C - 1] = kernel(d);
  for (int m = 0; m < C; m++)
    for (int n = 0; n < C; n++) sum[m] += h0[(m - n) + C - 1];  // row sums in n order, as :35-108
  std::vector<float> buf(3 * C - 1);
  for (int i = 0; i < 2 * C - 1; i++) buf[i] = (float)h0[i];
  const int r21 = C > 21 ? 21 : C - 1;
  for (int m = 0; m < C; m++) {
    double f = 1.0;
    if ((0 <= m && m <= 20) || (C - 20 <= m && m <= C)) f = sum[r21] / sum[m];
    buf[2 * C - 1 + m] = (float)f;
  }
  int rc = c->fbp_h[filter].ensure(buf.size());
  if (rc) return rc;
  VCT_CUDA(cudaMemcpy(c->fbp_h[filter].p, buf.data(), buf.size() * sizeof(float), cudaMemcpyHostToDevice));
  return VCT_OK;
}

static int fbp_into(vct_ctx* c, const float* d_sino, int filter, int in_mode, float* d_img, int view_groups,
                    int band0 = 0, int band1 = -1) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_sino || !d_img) return fail(VCT_E_ARG, "null buffer");
  if (filter != 1 && filter != 2) return fail(VCT_E_ARG, "filter must be 1 (Ram-Lak) or 2 (Shepp-Logan)");
  const int V = c->geo.views, C = c->dg.C;
  if ((rc = build_filter(c, filter))) return rc;
  if ((rc = c->fbp_q.ensure((size_t)V * C))) return rc;
  // the quarter-turn backprojector reads the filtered rows as pairs
  const bool sym = V % 4 == 0 && c->dg.N % 2 == 0;
  if (sym && (rc = c->fbp_q2.ensure((size_t)V * C))) return rc;
  float2* q2 = sym ? c->fbp_q2.p : nullptr;
  c->timer.begin(c->stream);
  if ((rc = launch_fbp_weight_filter(d_sino, c->geo.width, c->geo.start_channel, c->fbp_coeff.p, c->bh_alpha,
                                     c->bh_beta, c->fbp_h[filter].p, c->fbp_h[filter].p + 2 * C - 1, V, C, in_mode,
                                     c->fbp_q.p, q2, c->stream)))
    return rc;
  c->timer.mark("fbp_weight_filter_kernel", c->stream);
  if ((rc = launch_fbp_backproject(c->fbp_q.p, V, C, c->dg.N, c->geo.pixel_cm, c->geo.sid_cm, c->geo.max_beta,
                                   c->geo.xfactor, c->cs_f.p, d_img, c->stream, view_groups, band0, band1, q2)))
    return rc;
  c->timer.mark("fbp_backproject", c->stream);
  c->launches += 2;
  return VCT_OK;
}

// ------------------------------------------------------ one slice, sharded
int vct_forward_views_dev(vct_ctx* c, int v0, int v1, float* d_out, float* d_maxmin) {
  NvtxScope nvtx_scope("vct_forward_views_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_out || !d_maxmin) return fail(VCT_E_ARG, "vct_forward_views_dev: null buffer");
  if (v0 < 0 || v0 > v1 || v1 > c->dg.views_used) return fail(VCT_E_ARG, "vct_forward_views_dev: bad view range");
  if (!c->maps_ready || !c->spectrum_ready) return fail(VCT_E_STATE, "forward: maps or spectrum not set");
  const size_t row = (size_t)c->geo.width;
  VCT_CUDA(cudaMemcpyAsync(c->stats.p, c->stats.p + 1, sizeof(FwdStats), cudaMemcpyDeviceToDevice, c->stream));
  if (v1 > v0) VCT_CUDA(cudaMemsetAsync(d_out + v0 * row, 0, (size_t)(v1 - v0) * row * sizeof(float), c->stream));
  const double* mu_tab = c->sum_mode == VCT_SUM_REFERENCE ? c->mu_scaled.p : c->mu_log2.p;
  if (v1 > v0) {
    rc = launch_forward(c->dg, c->maps.p, c->M, mu_tab, c->pdf.p, c->NE, c->cos_t.p, c->sin_t.p, c->det_px0.p,
                        c->det_py0.p, c->sum_mode, c->walk_mode == VCT_WALK_FAST, d_out, nullptr, c->stats.p,
                        c->stream, v0, v1, exact_list(c), c->fwd_nexact);
    if (rc) return rc;
    c->launches += forward_launches(c);
  }
  // (max, min) of the rows as two floats: FwdStats begins with their bits
  VCT_CUDA(cudaMemcpyAsync(d_maxmin, c->stats.p, 2 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
  return VCT_OK;
}

int vct_normalize_noise_rows_dev(vct_ctx* c, float* d_sino, int r0, int r1, const float* d_maxmin, double sigma,
                                 uint64_t seed) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_sino || !d_maxmin) return fail(VCT_E_ARG, "vct_normalize_noise_rows_dev: null buffer");
  if (((uintptr_t)d_maxmin & 7) != 0) return fail(VCT_E_ARG, "vct_normalize_noise_rows_dev: d_maxmin not 8-byte aligned");
  rc = launch_normalize_noise(c->dg, d_sino, d_sino, reinterpret_cast<const FwdStats*>(d_maxmin), pad_zero_of(c),
                              sigma, seed, c->stream, r0, r1);
  if (!rc) c->launches++;
  return rc;
}

int vct_fbp_band_count(vct_ctx* c, int* count) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!count) return fail(VCT_E_ARG, "vct_fbp_band_count: null argument");
  *count = fbp_band_count(c->geo.views, c->dg.N);
  return VCT_OK;
}

int vct_fbp_band_dev(vct_ctx* c, const float* d_sino, int filter, int in_mode, int band0, int band1, float* d_img) {
  NvtxScope nvtx_scope("vct_fbp_band_dev");
  return fbp_into(c, d_sino, filter, in_mode, d_img, 4, band0, band1);
}

int vct_fbp_dev(vct_ctx* c, const float* d_sino, int filter, int in_mode, float* d_img) {
  NvtxScope nvtx_scope("vct_fbp_dev");
  return fbp_into(c, d_sino, filter, in_mode, d_img, 4);
}

int vct_fbp(vct_ctx* c, const float* sino, int filter, int in_mode, float* img) {
  NvtxScope nvtx_scope("vct_fbp");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!sino || !img) return fail(VCT_E_ARG, "null buffer");
  const size_t nsino = (size_t)c->geo.views * c->geo.width;
  const size_t nimg = (size_t)c->dg.N * c->dg.N;
  if ((rc = c->fbp_sino.ensure(nsino)) || (rc = c->fbp_img.ensure(nimg))) return rc;
  VCT_CUDA(cudaMemcpyAsync(c->fbp_sino.p, sino, nsino * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if ((rc = vct_fbp_dev(c, c->fbp_sino.p, filter, in_mode, c->fbp_img.p))) return rc;
  VCT_CUDA(cudaMemcpyAsync(img, c->fbp_img.p, nimg * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  return VCT_OK;
}

int vct_lengthproj2(vct_ctx* c, const float* proj, double z, double couch_speed, int ite, int thinout, float* npf) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!proj || !npf) return fail(VCT_E_ARG, "vct_lengthproj2: null buffer");
  const size_t nproj = (size_t)(c->geo.views / 2 * 2) * c->geo.width;
  const size_t nimg = (size_t)c->dg.N * c->dg.N;
  if ((rc = c->fbp_sino.ensure(c->geo.views * (size_t)c->geo.width)) || (rc = c->fbp_img.ensure(nimg))) return rc;
  VCT_CUDA(cudaMemcpyAsync(c->fbp_sino.p, proj, nproj * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if ((rc = vct_lengthproj2_dev(c, c->fbp_sino.p, z, couch_speed, ite, thinout, c->fbp_img.p))) return rc;
  VCT_CUDA(cudaMemcpyAsync(npf, c->fbp_img.p, nimg * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  return VCT_OK;
}

// The image update of IR_ImageTOMO, MB/IR_ImageTOMO.cpp:19-72.
int vct_ir_update_dev(vct_ctx* c, const float* d_before, const float* d_prior, const float* d_npf,
                      const float* d_npf_re, double wbefore, double w_tv, double w_prior, int ite, int thinout,
                      float* d_after) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_before || !d_npf || !d_npf_re || !d_after || thinout < 1) return fail(VCT_E_ARG, "vct_ir_update_dev: bad argument");
  if ((rc = launch_ir_update(c->dg.N, d_before, d_prior, d_npf, d_npf_re, wbefore, w_tv, w_prior, ite, thinout, d_after,
                             c->stream)))
    return rc;
  c->launches++;
  return VCT_OK;
}

// calc_squdiff_quad, MB/main.cpp:111-134: objective (and, at ite == num_ite,
// the quadratic) over the rows of iteration `ite`; d_out2 is 2 device doubles.
int vct_squdiff_dev(vct_ctx* c, const float* d_proj, const float* d_reproj, int ite, int thinout, int num_ite,
                    double* d_out2) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_proj || !d_reproj || !d_out2 || thinout < 1 || ite < 1) return fail(VCT_E_ARG, "vct_squdiff_dev: bad argument");
  if ((rc = c->sq_part.ensure(squdiff_scratch_doubles()))) return rc;
  const int used = c->geo.views / 2 * 2;
  if ((rc = launch_squdiff(d_proj, d_reproj, c->geo.width, c->geo.start_channel, c->dg.C, (ite - 1) % thinout, thinout,
                           used / thinout, ite == num_ite, c->sq_part.p, d_out2, c->stream)))
    return rc;
  c->launches += 2;
  return VCT_OK;
}

// One pass of the iterative step, MB/main.cpp:432-600 for ite >= 1: the
// last energy bin's sinogram (the reprojection_float buffer the reference's
// step reads after its energy loop, un-normalised, float per bin), the
// squared difference to the measured sinogram, update_wbefore
// (MB/main.cpp:136-150), lengthproj_TOMO_2 of that sinogram and the
// IR_ImageTOMO update of the first element's map.
int vct_ir_step(vct_ctx* c, const float* proj, const float* npf, const float* before, const float* prior, double z,
                double couch_speed, int ite, int thinout, int num_ite, double w_tv, double w_prior, double* wbefore,
                double* objective, double* quadratic, float* after) {
  NvtxScope nvtx_scope("vct_ir_step");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!proj || !npf || !before || !wbefore || !objective || !after || ite < 1 || thinout < 1)
    return fail(VCT_E_ARG, "vct_ir_step: bad argument");
  if (!c->maps_ready || !c->spectrum_ready) return fail(VCT_E_STATE, "vct_ir_step: maps or spectrum not set");
  const size_t nsino = (size_t)c->geo.views * c->geo.width, n2 = (size_t)c->dg.N * c->dg.N;
  const size_t nused = (size_t)(c->geo.views / 2 * 2) * c->geo.width;
  if ((rc = c->ir_proj.ensure(nsino)) || (rc = c->ir_reproj.ensure(nsino)) || (rc = c->ir_img.ensure(5 * n2)) ||
      (rc = c->ir_out.ensure(2)))
    return rc;
  float* d_npf = c->ir_img.p;
  float* d_npf_re = d_npf + n2;
  float* d_before = d_npf + 2 * n2;
  float* d_prior = d_npf + 3 * n2;
  float* d_after = d_npf + 4 * n2;
  VCT_CUDA(cudaMemsetAsync(c->ir_proj.p, 0, nsino * sizeof(float), c->stream));
  VCT_CUDA(cudaMemcpyAsync(c->ir_proj.p, proj, nused * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  VCT_CUDA(cudaMemcpyAsync(d_npf, npf, n2 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  VCT_CUDA(cudaMemcpyAsync(d_before, before, n2 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if (prior) VCT_CUDA(cudaMemcpyAsync(d_prior, prior, n2 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  VCT_CUDA(cudaMemcpyAsync(d_after, after, n2 * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  // the last bin alone: its row of the reference-summation table, one bin
  VCT_CUDA(cudaMemsetAsync(c->ir_reproj.p, 0, nsino * sizeof(float), c->stream));
  VCT_CUDA(cudaMemcpyAsync(c->stats.p, c->stats.p + 1, sizeof(FwdStats), cudaMemcpyDeviceToDevice, c->stream));
  if ((rc = launch_forward(c->dg, c->maps.p, c->M, c->mu_scaled.p + (size_t)(c->NE - 1) * c->M, c->pdf.p + c->NE - 1,
                           1, c->cos_t.p, c->sin_t.p, c->det_px0.p, c->det_py0.p, VCT_SUM_REFERENCE,
                           c->walk_mode == VCT_WALK_FAST, c->ir_reproj.p, nullptr, c->stats.p, c->stream, 0, -1,
                           exact_list(c), c->fwd_nexact)))
    return rc;
  c->launches += forward_launches(c);
  // calc_squdiff_quad over the measured rows used (the measured sinogram
  // holds the views used, row k = view k).
  if ((rc = vct_squdiff_dev(c, c->ir_proj.p, c->ir_reproj.p, ite, thinout, num_ite, c->ir_out.p))) return rc;
  double h_out[2];
  VCT_CUDA(cudaMemcpyAsync(h_out, c->ir_out.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  const double obj_before = *objective;
  *objective = h_out[0];
  if (quadratic) *quadratic = h_out[1];
  // update_wbefore, MB/main.cpp:136-150
  if (*objective < obj_before) *wbefore += 0.0001;
  else if (ite > 1) *wbefore -= 0.0002;
  if (*wbefore <= 0.0) *wbefore = 0.0001;
  if ((rc = vct_lengthproj2_dev(c, c->ir_reproj.p, z, couch_speed, ite, thinout, d_npf_re))) return rc;
  if ((rc = vct_ir_update_dev(c, d_before, prior ? d_prior : nullptr, d_npf, d_npf_re, *wbefore, w_tv, w_prior, ite,
                              thinout, d_after)))
    return rc;
  VCT_CUDA(cudaMemcpyAsync(after, d_after, n2 * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  return VCT_OK;
}

// Beam-hardening correction, MB/beam_hardening_correction.cpp:21-69.
int vct_set_beam_hardening(vct_ctx* c, double alpha, double beta) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!(alpha == alpha) || !(beta == beta)) return fail(VCT_E_ARG, "vct_set_beam_hardening: NaN");
  c->bh_alpha = alpha;
  c->bh_beta = beta;
  return VCT_OK;
}

int vct_beam_hardening_dev(vct_ctx* c, float* d_sino, double alpha, double beta) {
  NvtxScope nvtx_scope("vct_beam_hardening_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_sino) return fail(VCT_E_ARG, "vct_beam_hardening_dev: null buffer");
  if ((rc = launch_beam_hardening(d_sino, (long long)c->geo.views * c->geo.width, alpha, beta, c->stream)))
    return rc;
  c->launches++;
  return VCT_OK;
}

int vct_beam_hardening(vct_ctx* c, const float* sino, double alpha, double beta, float* out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!sino || !out) return fail(VCT_E_ARG, "vct_beam_hardening: null buffer");
  const size_t n = (size_t)c->geo.views * c->geo.width;
  if ((rc = c->fbp_sino.ensure(n))) return rc;
  VCT_CUDA(cudaMemcpyAsync(c->fbp_sino.p, sino, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if ((rc = vct_beam_hardening_dev(c, c->fbp_sino.p, alpha, beta))) return rc;
  VCT_CUDA(cudaMemcpyAsync(out, c->fbp_sino.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  return VCT_OK;
}

// lengthproj_TOMO, MB/lengthproj_TOMO.cpp:14-185.  The first view follows the
// reference's formula (:36-47: z over the couch advance per view, minus half
// a rotation); with no couch motion the reference divides 0/0 there and reads
// its trig tables out of range, and this build starts at view 0, as the
// reference's main does for the sinogram it passes in (MB/main.cpp:350).
static int lengthproj_into(vct_ctx* c, const float* d_proj, double z, double couch_speed, int ite, int thinout,
                           int tables, float* d_npf) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_proj || !d_npf) return fail(VCT_E_ARG, "vct_lengthproj: null buffer");
  if (thinout < 1 || ite < 1 - (tables ? 0 : 1)) return fail(VCT_E_ARG, "vct_lengthproj: bad ite/thinout");
  const vct_geometry& g = c->geo;
  LpGeom q{};
  q.N = c->dg.N;
  q.V = g.views;
  q.W = g.width;
  q.start_ch = g.start_channel;
  q.end_ch = g.end_channel;
  q.count = g.views / 2 * 2;  // sngrmHeight/UsedReconAngle*2
  q.start = 0;
  if (couch_speed != 0.0) {
    const double pitch = (double)(couch_speed / g.views);
    const double sv = z / pitch - g.views / 2 + 0.00000001;
    if (!(sv > -2147483648.0 && sv < 2147483647.0)) return fail(VCT_E_ARG, "vct_lengthproj_dev: view index overflow");
    q.start = (int)sv;
  }
  q.nrot = q.start / g.views;
  q.first = tables ? (ite - 1) % thinout : 0;  // thinnumb, :195-196
  q.stride = thinout;
  q.count = tables ? q.count / thinout : q.count;
  q.round_tables = tables;
  q.s = g.pixel_cm;
  q.sid = g.sid_cm;
  q.dsrc = g.det_src_iso_cm;
  q.R = g.det_radius_cm;
  q.diso = g.det_radius_cm - g.sid_cm;  // DIST_BTWN_ISO_AND_DETECTOR_CM (57.6 = 142.6 - 85)
  q.iso = g.iso_channel;
  q.dalpha = g.max_alpha / ((g.end_channel - g.start_channel - 1) / 2);
  if ((rc = launch_lengthproj(q, c->cos_t.p, c->sin_t.p, d_proj, d_npf, c->stream))) return rc;
  c->launches++;
  return VCT_OK;
}

int vct_lengthproj_dev(vct_ctx* c, const float* d_proj, double z, double couch_speed, float* d_npf) {
  NvtxScope nvtx_scope("vct_lengthproj_dev");
  return lengthproj_into(c, d_proj, z, couch_speed, 0, 1, 0, d_npf);
}

int vct_lengthproj2_dev(vct_ctx* c, const float* d_proj, double z, double couch_speed, int ite, int thinout,
                        float* d_npf) {
  return lengthproj_into(c, d_proj, z, couch_speed, ite, thinout, 1, d_npf);
}

int vct_lengthproj(vct_ctx* c, const float* proj, double z, double couch_speed, float* npf) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!proj || !npf) return fail(VCT_E_ARG, "vct_lengthproj: null buffer");
  const size_t nproj = (size_t)(c->geo.views / 2 * 2) * c->geo.width;
  const size_t nimg = (size_t)c->dg.N * c->dg.N;
  if ((rc = c->fbp_sino.ensure(c->geo.views * (size_t)c->geo.width)) || (rc = c->fbp_img.ensure(nimg))) return rc;
  VCT_CUDA(cudaMemcpyAsync(c->fbp_sino.p, proj, nproj * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if ((rc = vct_lengthproj_dev(c, c->fbp_sino.p, z, couch_speed, c->fbp_img.p))) return rc;
  VCT_CUDA(cudaMemcpyAsync(npf, c->fbp_img.p, nimg * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  return VCT_OK;
}

// Transpose of the FBP's linear part (no counterpart in the reference):
// backprojection, filter and weight transposed, in reverse order.
int vct_fbp_transpose_dev(vct_ctx* c, const float* d_u, int filter, float* d_lam) {
  NvtxScope nvtx_scope("vct_fbp_transpose_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_u || !d_lam) return fail(VCT_E_ARG, "null buffer");
  if (filter != 1 && filter != 2) return fail(VCT_E_ARG, "filter must be 1 (Ram-Lak) or 2 (Shepp-Logan)");
  const int V = c->geo.views, C = c->dg.C;
  if ((rc = build_filter(c, filter))) return rc;
  if ((rc = c->fbp_g.ensure((size_t)V * C)) || (rc = c->fbp_q.ensure((size_t)V * C)) ||
      (rc = c->fbp_tacc.ensure(fbp_backproject_t_scratch(V, C, c->dg.N))))
    return rc;
  c->timer.begin(c->stream);
  if ((rc = launch_fbp_backproject_t(d_u, V, C, c->dg.N, c->geo.pixel_cm, c->geo.sid_cm, c->geo.max_beta,
                                     c->geo.xfactor, c->cs_f.p, c->fbp_tacc.p, c->fbp_q.p, c->stream)))
    return rc;
  c->timer.mark("fbp_backproject_t", c->stream);
  if ((rc = launch_fbp_filter_t(c->fbp_q.p, c->fbp_h[filter].p, c->fbp_h[filter].p + 2 * C - 1, V, C, c->fbp_g.p,
                                c->stream)))
    return rc;
  c->timer.mark("fbp_filter_t", c->stream);
  if ((rc = launch_fbp_weight_t(c->fbp_g.p, V, c->geo.width, c->geo.start_channel, C, c->fbp_coeff.p, d_lam,
                                c->stream)))
    return rc;
  c->timer.mark("fbp_weight_t", c->stream);
  c->launches += 3;
  return VCT_OK;
}

int vct_fbp_transpose(vct_ctx* c, const float* u, int filter, float* lam) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!u || !lam) return fail(VCT_E_ARG, "null buffer");
  const size_t nsino = (size_t)c->geo.views * c->geo.width;
  const size_t nimg = (size_t)c->dg.N * c->dg.N;
  if ((rc = c->fbp_sino.ensure(nsino)) || (rc = c->fbp_img.ensure(nimg))) return rc;
  VCT_CUDA(cudaMemcpyAsync(c->fbp_img.p, u, nimg * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if ((rc = vct_fbp_transpose_dev(c, c->fbp_img.p, filter, c->fbp_sino.p))) return rc;
  VCT_CUDA(cudaMemcpyAsync(lam, c->fbp_sino.p, nsino * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  return VCT_OK;
}

int vct_set_stage_timing(vct_ctx* c, int on) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (on && !c->timer.ev[0])
    for (cudaEvent_t& e : c->timer.ev) VCT_CUDA(cudaEventCreate(&e));
  c->timer.on = on != 0;
  c->timer.n = 0;
  return VCT_OK;
}

int vct_stage_times(vct_ctx* c, int cap, const char** names, float* ms, int* n) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!n || (cap > 0 && (!names || !ms))) return fail(VCT_E_ARG, "vct_stage_times: null argument");
  if (!c->timer.on) return fail(VCT_E_STATE, "vct_stage_times: stage timing is off (vct_set_stage_timing)");
  *n = c->timer.n;
  if (c->timer.n > 0) VCT_CUDA(cudaEventSynchronize(c->timer.ev[c->timer.n]));
  for (int i = 0; i < c->timer.n && i < cap; i++) {
    names[i] = c->timer.name[i];
    VCT_CUDA(cudaEventElapsedTime(&ms[i], c->timer.ev[i], c->timer.ev[i + 1]));
  }
  return VCT_OK;
}

int vct_fbp_filtered_dev(vct_ctx* c, const float** d_fltd) {
  if (!c || !d_fltd) return fail(VCT_E_ARG, "null argument");
  if (!c->fbp_q.p) return fail(VCT_E_STATE, "no FBP has run on this context");
  *d_fltd = c->fbp_q.p;
  return VCT_OK;
}

// Philox4x32-10 on the host, for known-answer checks of the noise generator.
void vct_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  Philox4 c;
  for (int i = 0; i < 4; i++) c.v[i] = ctr[i];
  Philox4 r = philox4x32_10(c, key[0], key[1]);
  for (int i = 0; i < 4; i++) out[i] = r.v[i];
}

}  // extern "C"

// ----------------------------------------------------------------- adjoint
// Plans every ray once per context (geometry only) and reads back how many
// rays need the exact walk, which sizes the fixed-point scatter.
static int adj_prepare(vct_ctx* c) {
  if (c->adj_ready) return VCT_OK;
  const vct_geometry& g = c->geo;
  if (fabs(g.det_src_iso_cm - g.sid_cm) > 1e-9)
    return fail(VCT_E_UNSUPPORTED, "adjoint: needs det_src_iso_cm == sid_cm (fan centred on the source)");
  const DevGeom& dg = c->dg;
  const int C = dg.C, half = (C - 1) / 2;
  const long long nrays = (long long)dg.views_used * C;
  AdjGeom& a = c->ag;
  a.N = dg.N;
  a.nxm = dg.nxm;
  a.C = C;
  a.start = dg.start;
  a.views_used = dg.views_used;
  a.s = dg.s;
  a.sid = g.sid_cm;
  a.iso = g.iso_channel;
  a.inv_dalpha = half / g.max_alpha;
  a.lmax = 2.0 * sqrt(2.0) * dg.lim + 4.0 * dg.s;
  c->adj_tile = adj_pick_tile(a, dg.lim);
  if (c->adj_tile < 0) return fail(VCT_E_UNSUPPORTED, "adjoint: pixel too large for the channel window");
  // Unit direction of every channel's ray before rotation (detector point
  // minus source, MB/reprojection_TOMO.cpp:61-71).
  std::vector<double2> dir(C);
  for (int c0 = 0; c0 < C; c0++) {
    const int jj = g.start_channel + c0;
    const double theta = (g.iso_channel - jj) * g.max_alpha / half;
    const double ex = g.det_radius_cm * sin(theta);
    const double ey = -g.det_radius_cm * cos(theta) + g.det_src_iso_cm - g.sid_cm;
    const double nrm = sqrt(ex * ex + ey * ey);
    dir[c0] = make_double2(ex / nrm, ey / nrm);
  }
  int rc;
  if ((rc = c->adj_rec.ensure(nrays)) || (rc = c->adj_special.ensure(nrays)) || (rc = c->adj_ints.ensure(2)) ||
      (rc = c->adj_dir.ensure(C)) || (rc = c->adj_part.ensure(adj_forward_blocks(dg))) ||
      (rc = c->adj_loss.ensure(1)) || (rc = c->adj_gmax.ensure(1)))
    return rc;
  VCT_CUDA(cudaMemcpyAsync(c->adj_dir.p, dir.data(), C * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  VCT_CUDA(cudaMemsetAsync(c->adj_ints.p, 0, 2 * sizeof(int), c->stream));
  if ((rc = launch_adj_plan(dg, c->cos_t.p, c->sin_t.p, c->det_px0.p, c->det_py0.p, c->adj_rec.p,
                            c->adj_special.p, c->adj_ints.p, c->stream)))
    return rc;
  c->launches++;
  // The gather's per (tile, view) records: geometry and walk plans only.
  if ((rc = c->adj_tv.ensure((adj_tileview_bytes(a, c->adj_tile) + 15) / 16))) return rc;
  if ((rc = launch_adj_tiles(a, c->adj_tile, c->cos_t.p, c->sin_t.p, c->adj_rec.p, c->adj_tv.p, c->adj_ints.p + 1,
                             c->stream)))
    return rc;
  c->launches++;
  int ns_status[2] = {0, 0};
  VCT_CUDA(cudaMemcpyAsync(ns_status, c->adj_ints.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  if (ns_status[1]) return fail(VCT_E_UNSUPPORTED, "adjoint: a tile's channel window overflowed");
  const int ns = ns_status[0];
  c->adj_nspecial = ns;
  // Terms per pixel of the scatter: at most a few segments per ray and pixel.
  a.log2_terms = (int)ceil(log2(4.0 * ns + 2.0));
  c->adj_ready = 1;
  return VCT_OK;
}

static int adj_run(vct_ctx* c, int mode, const float* d_meas, const float* d_wts, const float* d_g_in,
                   float* d_grad, double* d_loss) {
  int rc;
  if ((rc = adj_prepare(c))) return rc;
  const DevGeom& dg = c->dg;
  const int M = c->M;
  const long long nrays = (long long)dg.views_used * dg.C;
  const size_t n2 = (size_t)dg.N * dg.N;
  const float* d_g = d_g_in;
  c->timer.begin(c->stream);
  VCT_CUDA(cudaMemsetAsync(c->adj_gmax.p, 0, sizeof(unsigned int), c->stream));
  if (!d_g) {
    if (!c->maps_ready || !c->spectrum_ready) return fail(VCT_E_STATE, "adjoint: maps or spectrum not set");
    if ((rc = c->adj_g.ensure((size_t)nrays * M))) return rc;
    if (c->adj_nspecial > 0) {
      if ((rc = c->adj_lsp.ensure((size_t)c->adj_nspecial * M))) return rc;
      if ((rc = launch_adj_lines(dg, M, c->maps.p, c->cos_t.p, c->sin_t.p, c->det_px0.p, c->det_py0.p,
                                 c->adj_special.p, c->adj_nspecial, c->adj_lsp.p, c->stream)))
        return rc;
      c->timer.mark("adj_lines_kernel", c->stream);
      c->launches++;
    }
    if ((rc = launch_adj_forward(dg, c->maps.p, M, c->mu_log2.p, c->pdf.p, c->NE, c->ynorm, c->cos_t.p, c->sin_t.p,
                                 c->det_px0.p, c->det_py0.p, c->adj_rec.p, c->adj_lsp.p, mode, d_meas, d_wts,
                                 c->adj_g.p, c->adj_part.p, c->adj_gmax.p, c->stream)))
      return rc;
    c->timer.mark("adj_forward_kernel", c->stream);
    c->launches++;
    d_g = c->adj_g.p;
    if (mode == 0) {
      if ((rc = launch_adj_loss(c->adj_part.p, adj_forward_blocks(dg), d_loss ? d_loss : c->adj_loss.p,
                                c->stream)))
        return rc;
      c->timer.mark("adj_loss_kernel", c->stream);
      c->launches++;
    }
  } else if (c->adj_nspecial > 0) {
    // Caller-given ray weights: their maximum over the exact-walk rays sets
    // the fixed-point scale.
    if ((rc = launch_adj_gmax(M, c->adj_special.p, c->adj_ints.p, c->adj_nspecial, d_g, c->adj_gmax.p, c->stream)))
      return rc;
    c->launches++;
  }
  const unsigned long long* sacc = nullptr;
  if (c->adj_nspecial > 0) {
    if ((rc = c->adj_sacc.ensure(n2 * M))) return rc;
    VCT_CUDA(cudaMemsetAsync(c->adj_sacc.p, 0, n2 * M * sizeof(unsigned long long), c->stream));
    if ((rc = launch_adj_special(dg, M, c->cos_t.p, c->sin_t.p, c->det_px0.p, c->det_py0.p, c->adj_special.p,
                                 c->adj_ints.p, c->adj_nspecial, d_g, c->adj_gmax.p, c->ag.lmax, c->ag.log2_terms,
                                 c->adj_sacc.p, c->stream)))
      return rc;
    c->timer.mark("adj_special_kernel", c->stream);
    c->launches++;
    sacc = c->adj_sacc.p;
  }
  if ((rc = c->adj_ext.ensure((size_t)kAdjChunks * M * (dg.N + 1) * (dg.N + 1)))) return rc;
  if ((rc = launch_adj_gather(c->ag, M, c->adj_tile, c->cos_t.p, c->sin_t.p, c->adj_dir.p, c->adj_rec.p, d_g,
                              c->adj_tv.p, c->adj_ext.p, c->stream)))
    return rc;
  c->timer.mark("adj_gather_kernel", c->stream);
  if ((rc = launch_adj_fold(c->ag, M, sacc, c->adj_gmax.p, c->adj_ext.p, d_grad, c->stream))) return rc;
  c->timer.mark("adj_fold_kernel", c->stream);
  c->launches += 2;
  return VCT_OK;
}

extern "C" {

int vct_forward_adjoint_dev(vct_ctx* c, const float* d_meas, const float* d_weights, float* d_grad, double* d_loss) {
  NvtxScope nvtx_scope("vct_forward_adjoint_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_meas || !d_grad) return fail(VCT_E_ARG, "vct_forward_adjoint_dev: null buffer");
  return adj_run(c, 0, d_meas, d_weights, nullptr, d_grad, d_loss);
}

int vct_forward_vjp_dev(vct_ctx* c, const float* d_dy, float* d_grad) {
  NvtxScope nvtx_scope("vct_forward_vjp_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_dy || !d_grad) return fail(VCT_E_ARG, "vct_forward_vjp_dev: null buffer");
  return adj_run(c, 1, d_dy, nullptr, nullptr, d_grad, nullptr);
}

int vct_adjoint_rays_dev(vct_ctx* c, const float* d_g, float* d_out) {
  NvtxScope nvtx_scope("vct_adjoint_rays_dev");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d_g || !d_out) return fail(VCT_E_ARG, "vct_adjoint_rays_dev: null buffer");
  if (!c->maps_ready) return fail(VCT_E_STATE, "vct_adjoint_rays_dev: maps not set (M unknown)");
  return adj_run(c, 1, nullptr, nullptr, d_g, d_out, nullptr);
}

int vct_forward_adjoint(vct_ctx* c, const float* meas, const float* weights, float* grad, double* loss) {
  NvtxScope nvtx_scope("vct_forward_adjoint");
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!meas || !grad) return fail(VCT_E_ARG, "vct_forward_adjoint: null buffer");
  const size_t nsino = (size_t)c->geo.views * c->geo.width;
  const size_t ng = (size_t)c->dg.N * c->dg.N * (c->M > 0 ? c->M : 1);
  if ((rc = c->adj_meas.ensure(nsino)) || (rc = c->adj_grad.ensure(ng))) return rc;
  VCT_CUDA(cudaMemcpyAsync(c->adj_meas.p, meas, nsino * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if (weights) {
    if ((rc = c->adj_wts.ensure(nsino))) return rc;
    VCT_CUDA(cudaMemcpyAsync(c->adj_wts.p, weights, nsino * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  }
  if ((rc = adj_run(c, 0, c->adj_meas.p, weights ? c->adj_wts.p : nullptr, nullptr, c->adj_grad.p, c->adj_loss.p)))
    return rc;
  VCT_CUDA(cudaMemcpyAsync(grad, c->adj_grad.p, ng * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  double l = 0.0;
  int status = 0;
  VCT_CUDA(cudaMemcpyAsync(&l, c->adj_loss.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaMemcpyAsync(&status, c->adj_ints.p + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  VCT_CUDA(cudaStreamSynchronize(c->stream));
  if (status) return fail(VCT_E_UNSUPPORTED, "adjoint: a tile's channel window overflowed");
  if (loss) *loss = l;
  return VCT_OK;
}

}  // extern "C"

// Internal entry points for the batch engine (vct_batch.cpp).
namespace vct {
int ctx_check(vct_ctx* c) { return check_ctx(c); }
int ctx_build_filter(vct_ctx* c, int filter) { return build_filter(c, filter); }
int ctx_pad_zero(const vct_ctx* c) { return pad_zero_of(c); }
int ctx_fbp(vct_ctx* c, const float* d_sino, int filter, float* d_img, int view_groups) {
  return fbp_into(c, d_sino, filter, 0, d_img, view_groups);
}
int ctx_adj_prepare(vct_ctx* c) { return adj_prepare(c); }
int ctx_adj_run(vct_ctx* c, int mode, const float* d_meas, const float* d_wts, const float* d_g, float* d_grad,
                double* d_loss) {
  return adj_run(c, mode, d_meas, d_wts, d_g, d_grad, d_loss);
}
}  // namespace vct
