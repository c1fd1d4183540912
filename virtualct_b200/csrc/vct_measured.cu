// Measured-data ingestion and the helical z-interpolation on sm_100a.
//
//   vct_load_measured(_dev)  MB/projectionDataTOMO.cpp:324-508 (loadProjectionData):
//       air-scan mean and normalisation of a measured sinogram, "PR"
//       (pre-treatment CT) and "IN" (in-treatment) modes.
//   vct_helical_sinogram(_dev)  MB/main.cpp:347-371: the sinogram of one
//       reconstruction z, each view blended with the same view of the next
//       rotation.
//
// The files are read on the host exactly as the reference reads them -- the
// same byte counts into buffers that persist between reads, so a short file
// leaves the previous read's bytes in the tail -- and only what the
// reference's arithmetic then uses goes to the device:
//   PR: the air blocks and each rotation's [air_rows][ch] plane;
//   IN: the air blocks and, per rotation, the one raw row the reference's
//       loop reads: it fills only row 0 of its [air_rows][ch] buffer per view
//       but indexes row j for view j, so views j >= 1 see the buffer's
//       never-written (zero) rows and only view 0 of each rotation carries
//       data (:466-476).
// The kernels are elementwise and bound by HBM; --fmad=false keeps every
// product and sum rounded as the reference's x86-64 -O2 build rounds it.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/vct_io.h"
#include "vct_internal.h"

namespace vct {

// sum_air[k] += air_b[k] / blocks in block order (:389-393); PR uses every k
// of the plane, IN only row 0's channels skip.. (:404-412, of which the
// normalisation reads k < width, :468).
__global__ void air_mean_kernel(const float* __restrict__ blocks, int nblocks, long long plane, long long first,
                                long long n, float* __restrict__ out) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int b = 0; b < nblocks; b++) s += blocks[b * plane + first + k] / nblocks;
    out[k] = s;
  }
}

// PR (:438-452): vol[t][r][k] = raw_t[kk] / air[kk], kk = (r*nskip)*ch + skip + k.
__global__ void normalize_pr_kernel(const float* __restrict__ raw, const float* __restrict__ air, int rotations,
                                    int views, int width, int nskip, int ch, int skip, long long plane,
                                    float* __restrict__ vol, unsigned char* __restrict__ mask) {
  const long long total = (long long)rotations * views * width;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(o % width);
    const long long tr = o / width;
    const int r = (int)(tr % views);
    const int t = (int)(tr / views);
    const long long kk = (long long)r * nskip * ch + skip + k;
    if (!VCT_INDEX_OK(kk >= 0 && kk < plane)) continue;
    vol[o] = raw[t * plane + kk] / air[kk];
    mask[o] = 1;
  }
}

// IN (:462-492): d = row / (air[k] * 2) for view 0 (zero beyond the row's ch
// channels: the buffer's row 1 was never written), 0 / (air[k] * 2) for
// views >= 1; values below 0.1 become 0 with mask 0 (NaN stays, mask 1).
// The first value above 1 inside the channel window, in (t, j, k) order, is
// where the reference stops; its index goes to *first_over.
__global__ void normalize_in_kernel(const float* __restrict__ rows, const float* __restrict__ air, int rotations,
                                    int views, int width, int ch, int skip, int start_ch, int end_ch,
                                    float* __restrict__ vol, unsigned char* __restrict__ mask,
                                    unsigned long long* __restrict__ first_over, unsigned int* __restrict__ max_bits) {
  const long long total = (long long)rotations * views * width;
  unsigned int local_max = 0u;  // bits of a non-negative float
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(o % width);
    const long long tj = o / width;
    const int j = (int)(tj % views);
    const int t = (int)(tj / views);
    const int i = skip + k;
    const float num = (j == 0 && i < ch) ? rows[(long long)t * ch + i] : 0.0f;
    float d = num / (air[k] * 2);
    if (i >= start_ch && i < end_ch && d > 0.0f) {
      local_max = max(local_max, __float_as_uint(d));
      if (d > 1.0f) atomicMin(first_over, (unsigned long long)o);
    }
    unsigned char m = 1;
    if (d < 0.1f) {
      d = 0.0f;
      m = 0;
    }
    vol[o] = d;
    mask[o] = m;
  }
  if (local_max) atomicMax(max_bits, local_max);
}

// MB/main.cpp:347-371 with start_angle_num = 0 and UsedReconAngle = 2.
__global__ void helical_kernel(const float* __restrict__ vol, int rotations, int views, int width,
                               float* __restrict__ out) {
  const int use = views / 2 * 2;
  const long long total = (long long)use * width;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(o % width);
    const int j = (int)(o / width);
    int iphase = 0;
    if (j < use / 2) iphase = 1;
    else if (j > use / 2) iphase = -1;
    if (j + iphase * views < views) iphase = 0;
    if (j + iphase * views > (rotations - 1) * views) iphase = 0;
    const double zw = 0.5 * fabs(j - (views / 2.0)) / (views / 2.0);
    if (!VCT_INDEX_OK(j + iphase * views >= 0 && j + iphase * views < rotations * views)) continue;
    out[o] = (float)((1.0 - zw) * (double)vol[(long long)j * width + c] +
                     zw * (double)vol[(long long)(j + iphase * views) * width + c]);
  }
}

static unsigned grid_for(long long n) {
  const long long b = (n + 255) / 256;
  return (unsigned)(b < 148LL * 16 ? (b > 0 ? b : 1) : 148LL * 16);
}

namespace {

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t bytes) {
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 1);
    return e == cudaSuccess ? VCT_OK : cuda_fail(e, "cudaMalloc");
  }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace

// The reference's reader, on the host: returns VCT_OK with the arrays the
// device needs, VCT_E_IO when a file is missing (the reference's -1).
struct MeasuredRaw {
  std::vector<float> air;   // [air_blocks][plane] as each read left the buffer
  std::vector<float> data;  // PR: [rotations][plane]; IN: [rotations][ch]
};

static int read_measured(const vct_mb_config* cfg, const vct_raw_layout* l, int in_mode, int views, MeasuredRaw* out) {
  const long long plane = (long long)l->raw_channels * l->air_rows;
  const int R = cfg->total_proj_number;
  File fp, fa;
  fp.f = fopen(cfg->proj_file, "rb");
  if (!fp.f) return fail(VCT_E_IO, std::string("data file: ") + cfg->proj_file + " not found");
  fa.f = fopen(cfg->air_scan_file, "rb");
  if (!fa.f) return fail(VCT_E_IO, std::string("data file: ") + cfg->air_scan_file + " not found");
  std::vector<float> buf((size_t)plane, 0.0f);
  size_t got = fread(buf.data(), 1, (size_t)plane * sizeof(float), fa.f);  // first block: not used (:385, :401)
  out->air.resize((size_t)l->air_blocks * plane);
  for (int b = 0; b < l->air_blocks; b++) {
    got = fread(buf.data(), 1, (size_t)plane * sizeof(float), fa.f);
    memcpy(out->air.data() + (size_t)b * plane, buf.data(), (size_t)plane * sizeof(float));
  }
  std::fill(buf.begin(), buf.end(), 0.0f);
  if (!in_mode) {
    out->data.resize((size_t)R * plane);
    for (int t = 0; t < R; t++) {
      got = fread(buf.data(), 1, (size_t)plane * sizeof(float), fp.f);
      memcpy(out->data.data() + (size_t)t * plane, buf.data(), (size_t)plane * sizeof(float));
    }
  } else {
    const int rows_per_view = cfg->data_sampling_rate_orig >= 200 ? 5 : 1;  // :493-499
    const size_t row_bytes = (size_t)l->raw_channels * sizeof(float);
    out->data.resize((size_t)R * l->raw_channels);
    for (int t = 0; t < R; t++)
      for (int j = 0; j < views; j++) {
        got = fread(buf.data(), 1, row_bytes, fp.f);
        if (j == 0) memcpy(out->data.data() + (size_t)t * l->raw_channels, buf.data(), row_bytes);
        for (int r = 1; r < rows_per_view; r++) got = fread(buf.data(), 1, row_bytes, fp.f);
      }
  }
  (void)got;
  return VCT_OK;
}

static int check_measured(const vct_mb_config* cfg, const vct_raw_layout* l, int* in_mode) {
  if (!cfg || !l) return fail(VCT_E_ARG, "vct_load_measured: null argument");
  if (strcmp(cfg->in_pr_class, "PR") != 0 && strcmp(cfg->in_pr_class, "IN") != 0)
    return fail(VCT_E_ARG, std::string("vct_load_measured: energy label ") + cfg->in_pr_class + " is neither PR nor IN");
  *in_mode = strcmp(cfg->in_pr_class, "IN") == 0;
  const int W = cfg->proj_width, V = cfg->proj_height, nskip = cfg->sino_fact;
  if (W <= 0 || V <= 0 || nskip <= 0 || cfg->total_proj_number < 0 || l->raw_channels <= 0 || l->air_rows <= 0 ||
      l->air_blocks <= 0 || l->skip_channels < 0)
    return fail(VCT_E_ARG, "vct_load_measured: sizes must be positive");
  // The reference opens both files before it reads anything (:369-378):
  // a missing file ends the load there, whatever the layout.
  for (const char* path : {cfg->proj_file, cfg->air_scan_file}) {
    FILE* f = fopen(path, "rb");
    if (!f) return fail(VCT_E_IO, std::string("data file: ") + path + " not found");
    fclose(f);
  }
  const long long plane = (long long)l->raw_channels * l->air_rows;
  // Beyond these the reference reads or writes past its own buffers.
  if (*in_mode) {
    if ((long long)(V - 1) * l->raw_channels + l->skip_channels + W > plane)
      return fail(VCT_E_UNSUPPORTED, "vct_load_measured: IN-mode rows reach past the air-scan block");
  } else {
    if (l->skip_channels + W > l->raw_channels)
      return fail(VCT_E_UNSUPPORTED, "vct_load_measured: skipped + used channels exceed the raw row");
    if ((l->air_rows + nskip - 1) / nskip != V)
      return fail(VCT_E_UNSUPPORTED, "vct_load_measured: kept air-scan rows differ from the sinogram height");
  }
  return VCT_OK;
}

VCT_BOUNDS_READER(bounds_measured)

}  // namespace vct

using namespace vct;

extern "C" void vct_raw_layout_default(vct_raw_layout* l) {
  if (!l) return;
  l->raw_channels = 609;  // NumberOfChannels        MB/physParamsTOMO.h:32
  l->skip_channels = 27;  // NumberOfSkips           :33
  l->air_rows = 800;      // AirScn_Sinogram_Height  :64
  l->air_blocks = 5;      // AirScn_Sinogram_Number  :65
  l->start_channel = 0;   // Start_Channel           :43
  l->end_channel = 609;   // End_Channel             :46
}

extern "C" int vct_load_measured_dev(const vct_mb_config* cfg, const vct_raw_layout* l, float* d_volume,
                                     unsigned char* d_mask, int* rotations, double* max_value, void* stream) {
  int in_mode = 0;
  int rc = check_measured(cfg, l, &in_mode);
  if (rc) return rc;
  if (!d_volume || !d_mask) return fail(VCT_E_ARG, "vct_load_measured_dev: null output");
  const int R = cfg->total_proj_number, V = cfg->proj_height, W = cfg->proj_width;
  if (rotations) *rotations = 0;
  if (max_value) *max_value = 0.0;
  MeasuredRaw raw;
  if ((rc = read_measured(cfg, l, in_mode, V, &raw))) return rc;
  if (R == 0) return VCT_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const long long plane = (long long)l->raw_channels * l->air_rows;
  DevBuf d_air, d_raw, d_mean, d_flags;
  if ((rc = d_air.alloc(raw.air.size() * sizeof(float))) || (rc = d_raw.alloc(raw.data.size() * sizeof(float))) ||
      (rc = d_mean.alloc((size_t)plane * sizeof(float))) || (rc = d_flags.alloc(16)))
    return rc;
  VCT_CUDA(cudaMemcpyAsync(d_air.p, raw.air.data(), raw.air.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  VCT_CUDA(cudaMemcpyAsync(d_raw.p, raw.data.data(), raw.data.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  const long long total = (long long)R * V * W;
  if (!in_mode) {
    air_mean_kernel<<<grid_for(plane), 256, 0, st>>>(d_air.as<float>(), l->air_blocks, plane, 0, plane,
                                                     d_mean.as<float>());
    normalize_pr_kernel<<<grid_for(total), 256, 0, st>>>(d_raw.as<float>(), d_mean.as<float>(), R, V, W,
                                                         cfg->sino_fact, l->raw_channels, l->skip_channels, plane,
                                                         d_volume, d_mask);
    VCT_CUDA(cudaGetLastError());
    VCT_CUDA(cudaStreamSynchronize(st));  // the host buffers above are freed on return
  } else {
    air_mean_kernel<<<grid_for(W), 256, 0, st>>>(d_air.as<float>(), l->air_blocks, plane, l->skip_channels, W,
                                                 d_mean.as<float>());
    unsigned long long* first = d_flags.as<unsigned long long>();
    unsigned int* max_bits = (unsigned int*)(first + 1);
    const unsigned long long init[2] = {~0ull, 0ull};
    VCT_CUDA(cudaMemcpyAsync(first, init, sizeof init, cudaMemcpyHostToDevice, st));
    normalize_in_kernel<<<grid_for(total), 256, 0, st>>>(d_raw.as<float>(), d_mean.as<float>(), R, V, W,
                                                         l->raw_channels, l->skip_channels, l->start_channel,
                                                         l->end_channel, d_volume, d_mask, first, max_bits);
    VCT_CUDA(cudaGetLastError());
    unsigned long long flags[2];
    VCT_CUDA(cudaMemcpyAsync(flags, first, sizeof flags, cudaMemcpyDeviceToHost, st));
    VCT_CUDA(cudaStreamSynchronize(st));
    if (flags[0] != ~0ull) {
      float v = 0.0f;
      VCT_CUDA(cudaMemcpy(&v, d_volume + flags[0], sizeof v, cudaMemcpyDeviceToHost));
      if (max_value) *max_value = v;
      char msg[128];
      snprintf(msg, sizeof msg, "Maximum projection: %lf > 1.0... STOP", (double)v);
      return fail(VCT_E_RANGE, msg);
    }
    if (max_value) {
      const unsigned int bits = (unsigned int)flags[1];
      float m;
      memcpy(&m, &bits, sizeof m);
      *max_value = (double)m;
    }
  }
  if (rotations) *rotations = R;
  return VCT_OK;
}

extern "C" int vct_load_measured(const vct_mb_config* cfg, const vct_raw_layout* l, int device, float* volume,
                                 unsigned char* mask, int* rotations, double* max_value) {
  int in_mode = 0;
  int rc = check_measured(cfg, l, &in_mode);
  if (rc) return rc;
  if (!volume || !mask) return fail(VCT_E_ARG, "vct_load_measured: null output");
  VCT_CUDA(cudaSetDevice(device));
  const size_t n = (size_t)cfg->total_proj_number * cfg->proj_height * cfg->proj_width;
  DevBuf d_vol, d_mask;
  if ((rc = d_vol.alloc(n * sizeof(float))) || (rc = d_mask.alloc(n))) return rc;
  int got = 0;
  rc = vct_load_measured_dev(cfg, l, d_vol.as<float>(), d_mask.as<unsigned char>(), &got, max_value, nullptr);
  if (rotations) *rotations = got;
  if (rc) return rc;
  VCT_CUDA(cudaMemcpy(volume, d_vol.p, n * sizeof(float), cudaMemcpyDeviceToHost));
  VCT_CUDA(cudaMemcpy(mask, d_mask.p, n, cudaMemcpyDeviceToHost));
  return VCT_OK;
}

extern "C" int vct_helical_sinogram_dev(const float* d_volume, int rotations, int views, int width, float* d_out,
                                        void* stream) {
  if (!d_volume || !d_out || rotations < 1 || views <= 0 || width <= 0)
    return fail(VCT_E_ARG, "vct_helical_sinogram_dev: bad argument");
  const long long n = (long long)(views / 2 * 2) * width;
  if (n == 0) return VCT_OK;
  helical_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(d_volume, rotations, views, width, d_out);
  VCT_CUDA(cudaGetLastError());
  return VCT_OK;
}

extern "C" int vct_helical_sinogram(const float* volume, int rotations, int views, int width, float* out,
                                    int device) {
  if (!volume || !out || rotations < 1 || views <= 0 || width <= 0)
    return fail(VCT_E_ARG, "vct_helical_sinogram: bad argument");
  VCT_CUDA(cudaSetDevice(device));
  const size_t nin = (size_t)rotations * views * width, nout = (size_t)views * width;
  DevBuf d_in, d_out;
  int rc;
  if ((rc = d_in.alloc(nin * sizeof(float))) || (rc = d_out.alloc(nout * sizeof(float)))) return rc;
  VCT_CUDA(cudaMemcpy(d_in.p, volume, nin * sizeof(float), cudaMemcpyHostToDevice));
  VCT_CUDA(cudaMemcpy(d_out.p, out, nout * sizeof(float), cudaMemcpyHostToDevice));  // rows past views/2*2 kept
  if ((rc = vct_helical_sinogram_dev(d_in.as<float>(), rotations, views, width, d_out.as<float>(), nullptr))) return rc;
  VCT_CUDA(cudaMemcpy(out, d_out.p, nout * sizeof(float), cudaMemcpyDeviceToHost));
  return VCT_OK;
}
