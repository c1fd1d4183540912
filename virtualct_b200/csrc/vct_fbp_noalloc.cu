// vct_fbp_noalloc: FBP for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they reconstruct:
// code that runs under a device-memory budget owned by another allocator
// (a framework's memory pool, a fixed partition of the GPU), real-time loops
// that must not pay for an allocation's latency and implicit device
// synchronisation, or library code that is not allowed to fail on an
// allocation at run time.  This entry point gives them the FBP of
// vct_fbp_dev without any allocation: the caller passes the sinogram and the
// image (device pointers); the intermediate buffers (weighted and filtered
// sinograms) and the small per-call tables live in the file-scope device
// arrays below.  A device holds them from the first call on it until the
// process exits: with CUDA's lazy module loading (the default) the driver
// allocates them when that first call loads this file's module, so make it at
// start-up, where an allocation may still fail safely.  Every call shares
// the arrays, so calls that overlap on the GPU race.
#include <cuda.h>  // CUresult and CUcontext only: the driver call is looked up through the runtime
#include <cuda_runtime.h>
#include <math.h>

#include <mutex>

#include "vct_internal.h"

namespace vct {

// Limits of the static scratch (about 8.1 MB per device).
constexpr int kNoAllocMaxVC = 1 << 20;  // views * channels
constexpr int kNoAllocMaxC = 2048;      // channels
constexpr int kNoAllocMaxV = 4096;      // views

static __device__ __align__(256) float g_noalloc_weighted[kNoAllocMaxVC];  // g[v][k]
static __device__ __align__(256) float g_noalloc_filtered[kNoAllocMaxVC];  // q[v][m]
static __device__ __align__(256) float g_noalloc_kernel[3 * kNoAllocMaxC];  // h0[2C-1], row factors[C]
static __device__ __align__(256) double g_noalloc_coeff[kNoAllocMaxC];     // SID*cos((k-cw)*db)*db
static __device__ __align__(256) float g_noalloc_cs[2 * kNoAllocMaxV];     // (cos, sin) per view

// Device addresses of the arrays above on one device, valid in the CUDA
// context whose unique id is ctx_id.
struct NoAllocPtrs {
  float* weighted;
  float* filtered;
  float* kernel;
  double* coeff;
  float* cs;
  unsigned long long ctx_id;
  int ready;
};
static NoAllocPtrs g_ptrs[64];  // per device
static std::mutex g_ptrs_mutex;  // guards g_ptrs and g_ctx_get_id

// cuCtxGetId (CUDA 12.0+), reached through the runtime so that libvct needs
// no link against the driver library.
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
static CtxGetIdFn g_ctx_get_id = nullptr;

// Unique id of the calling thread's current CUDA context; 0 when none is
// current yet (the runtime creates the device's primary context at its first
// call that needs one).
static int current_context_id(unsigned long long* id) {
  *id = 0;
  if (!g_ctx_get_id) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess) return cuda_fail(e, "vct_fbp_noalloc: cudaGetDriverEntryPointByVersion(cuCtxGetId)");
    if (q != cudaDriverEntryPointSuccess || !fn)
      return fail(VCT_E_CUDA, "vct_fbp_noalloc: the driver has no cuCtxGetId");
    g_ctx_get_id = (CtxGetIdFn)fn;
  }
  if (g_ctx_get_id(nullptr, id) != CUDA_SUCCESS) *id = 0;
  return VCT_OK;
}

// Host code cannot use the arrays' names as device addresses; their device
// addresses come from cudaGetSymbolAddress, called with the device current.
// They are looked up at the first call on a device and again whenever the
// current context is not the one they were looked up in (after
// cudaDeviceReset, say, when the module is loaded anew at other addresses).
// The lookup also makes the runtime load this file's module on the device,
// which is when the driver allocates the arrays.  One lock serialises the
// set-up of all devices, so concurrent first calls cannot see a half-written
// entry.
static int noalloc_setup(int device, NoAllocPtrs* out) {
  if (device < 0 || device >= 64) return fail(VCT_E_ARG, "vct_fbp_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_ptrs_mutex);
  NoAllocPtrs& p = g_ptrs[device];
  unsigned long long id = 0;
  if (int rc = current_context_id(&id)) return rc;
  if (!p.ready || id == 0 || p.ctx_id != id) {
    NoAllocPtrs n = {};
    cudaError_t e;
    if ((e = cudaGetSymbolAddress((void**)&n.weighted, g_noalloc_weighted)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&n.filtered, g_noalloc_filtered)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&n.kernel, g_noalloc_kernel)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&n.coeff, g_noalloc_coeff)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&n.cs, g_noalloc_cs)) != cudaSuccess)
      return cuda_fail(e, "vct_fbp_noalloc: cudaGetSymbolAddress");
    // The lookups bound a context to this thread if none was.
    if (int rc = current_context_id(&n.ctx_id)) return rc;
    if (n.ctx_id == 0) return fail(VCT_E_CUDA, "vct_fbp_noalloc: no current CUDA context after set-up");
    n.ready = 1;
    p = n;
  }
  *out = p;
  return VCT_OK;
}

// The per-call tables, built on the device so the call needs no host buffer:
// view trig (MB/projectionDataTOMO.cpp:362-368), the filter weight of
// FBP/filterSinogramTOMO.cpp:236 times dbeta, and prepareConstMap's kernel
// and edge-row factors (FBP/filterSinogramTOMO.cpp:9-123), in double,
// stored as float where the device filter reads float.
__device__ double noalloc_h0(int MN, int filter, double arc) {
  const double PI = 3.141592653589793238462643383279;
  if (MN == 0) {
    if (filter == 1) return 0.125 / (arc * arc);
    const double oddterm = PI * PI * (arc);
    return 0.25 / oddterm * (1.0 / tan((0.5) * arc) - 1.0 / tan((-0.5) * arc));
  }
  if (MN % 2 != 0) {
    if (filter == 1) {
      const double oddterm = PI * sin(MN * arc);
      return -0.5 / oddterm / oddterm;
    }
    const double oddterm = PI * PI * arc;
    return 0.25 / oddterm * (1.0 / tan((MN + 0.5) * arc) - 1.0 / tan((MN - 0.5) * arc));
  }
  if (filter == 1) return 0.0;
  const double oddterm = PI * PI * arc;
  return 0.25 / oddterm * (1.0 / tan((MN + 0.5) * arc) - 1.0 / tan((MN - 0.5) * arc));
}

__global__ void noalloc_tables_kernel(int V, int C, double start_deg, double sid, double max_beta, int filter,
                                      float* __restrict__ kern, double* __restrict__ coeff,
                                      float* __restrict__ cs) {
  const double PI = 3.141592653589793238462643383279;
  const int half = (C - 1) / 2;
  const double arc = max_beta / half;
  const int cw = C / 2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 2 * C - 1) kern[i] = (float)noalloc_h0(i - (C - 1), filter, arc);
  if (i < C) {
    coeff[i] = sid * cos((i - cw) * (max_beta / half)) * (max_beta / half);
    // Row factor sum[21]/sum[m] for rows 0..20 and C-20..C-1; row sums in n
    // order as the reference accumulates them.
    double f = 1.0;
    if (i <= 20 || i >= C - 20) {
      const int r21 = C > 21 ? 21 : C - 1;
      double sm = 0.0, s21 = 0.0;
      for (int n = 0; n < C; n++) {
        sm += noalloc_h0(i - n, filter, arc);
        s21 += noalloc_h0(r21 - n, filter, arc);
      }
      f = s21 / sm;
    }
    kern[2 * C - 1 + i] = (float)f;
  }
  if (i < V) {
    const double rad = (start_deg + (double)(360.0 / V * i)) * PI / 180.0;
    cs[2 * i] = (float)cos(rad);
    cs[2 * i + 1] = (float)sin(rad);
  }
}

}  // namespace vct

using namespace vct;

// See include/vct.h.  The first call on a device (and the first after its
// context was reset) looks up the scratch arrays' device addresses there and
// may make the driver allocate them; make that call at start-up, before any
// stream capture.
extern "C" int vct_fbp_noalloc(const vct_geometry* g, const float* d_sino, int filter, int in_mode, float* d_img,
                               void* stream) {
  if (!g || !d_sino || !d_img) return fail(VCT_E_ARG, "vct_fbp_noalloc: null argument");
  if (filter != 1 && filter != 2) return fail(VCT_E_ARG, "vct_fbp_noalloc: filter must be 1 or 2");
  if (int rc = check_geometry(g, "vct_fbp_noalloc")) return rc;
  const int C = g->end_channel - g->start_channel, V = g->views, N = g->recon_size;
  if (C > kNoAllocMaxC || V > kNoAllocMaxV || (long long)V * C > kNoAllocMaxVC)
    return fail(VCT_E_ARG,
                "vct_fbp_noalloc: views*channels above the static scratch limit (views <= 4096, "
                "channels <= 2048, views*channels <= 1048576)");
  int device = 0;
  VCT_CUDA(cudaGetDevice(&device));
  NoAllocPtrs p;
  int rc = noalloc_setup(device, &p);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = 2 * C - 1 > V ? 2 * C - 1 : V;
  noalloc_tables_kernel<<<(n + 127) / 128, 128, 0, st>>>(V, C, g->start_view_deg, g->sid_cm, g->max_beta, filter,
                                                         p.kernel, p.coeff, p.cs);
  VCT_CUDA(cudaGetLastError());
  if ((rc = launch_fbp_weight(d_sino, V, g->width, g->start_channel, C, p.coeff, p.weighted, st))) return rc;
  if ((rc = launch_fbp_filter(p.weighted, p.kernel, p.kernel + 2 * C - 1, V, C, in_mode, p.filtered, st)))
    return rc;
  return launch_fbp_backproject(p.filtered, V, C, N, g->pixel_cm, g->sid_cm, g->max_beta, g->xfactor, p.cs, d_img,
                                st);
}
