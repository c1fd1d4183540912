// Peak probes used by bench.py as roofline denominators: the B200 figures
// this path is bound by (L2 read bandwidth for the map gathers, FP64 and FP32
// FMA issue) are not among the measured HBM and GEMM peaks, so they are
// measured live.  Built as its own library (lib/libvct_peaks.so), not part of
// the product libvct.so.
#include <cuda_runtime.h>
#include <stdio.h>

namespace {

thread_local char g_err[256];

int probe_fail(cudaError_t e, const char* what) {
  snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
  return -2;
}

#define PROBE_CUDA(call)                                  \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return probe_fail(e_, #call);  \
  } while (0)

// L2 read bandwidth: every block streams the same L2-resident buffer with
// ld.global.cg (cached in L2, not L1), 16 B per thread per load.
__global__ void probe_l2_kernel(const int4* __restrict__ buf, size_t n16, int reps,
                                unsigned int* __restrict__ sink) {
  unsigned int acc = 0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int r = 0; r < reps; r++) {
    // Each block starts at a different offset so blocks spread over slices.
    size_t start = ((size_t)blockIdx.x * 977 + (size_t)r * 131) * blockDim.x % n16;
    for (size_t i = start + threadIdx.x, k = 0; k < n16; i += stride, k += stride) {
      if (i >= n16) i -= n16;
      int4 v = __ldcg(buf + i);
      acc ^= (unsigned)(v.x ^ v.y ^ v.z ^ v.w);
    }
  }
  if (acc == 0x9e3779b9u) sink[0] = acc;  // keeps the loads alive
}

template <typename T>
__global__ void probe_fma_kernel(int iters, T seed, T* __restrict__ sink) {
  T a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
    a7 = a0 + 7;
  const T m = (T)0.999999, c = (T)1e-7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      a0 = a0 * m + c; a1 = a1 * m + c; a2 = a2 * m + c; a3 = a3 * m + c;
      a4 = a4 * m + c; a5 = a5 * m + c; a6 = a6 * m + c; a7 = a7 * m + c;
    }
  }
  T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == (T)-1.2345) sink[0] = s;
}

}  // namespace

extern "C" const char* vct_peaks_error(void) { return g_err; }

// Returns 0, or a negative code with the message in vct_peaks_error().
extern "C" int vct_probe_peaks(int device, double* l2_read_gbs, double* fp64_tflops, double* fp32_tflops) {
  PROBE_CUDA(cudaSetDevice(device));
  int sms = 0;
  PROBE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  cudaStream_t st;
  PROBE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const size_t bytes = 16u << 20;  // 16 MB: L2-resident, far above L1
  int4* buf = nullptr;
  unsigned int* sink = nullptr;
  double* dsink = nullptr;
  float* fsink = nullptr;
  int rc = 0;
  if (cudaMalloc((void**)&buf, bytes) != cudaSuccess || cudaMalloc((void**)&sink, 64) != cudaSuccess ||
      cudaMalloc((void**)&dsink, 64) != cudaSuccess || cudaMalloc((void**)&fsink, 64) != cudaSuccess) {
    rc = probe_fail(cudaErrorMemoryAllocation, "vct_probe_peaks: allocation");
  }
  float ms = 0;
  if (rc == 0) {
    cudaMemsetAsync(buf, 1, bytes, st);
    const int blocks = sms * 4, threads = 512, reps = 64;
    probe_l2_kernel<<<blocks, threads, 0, st>>>(buf, bytes / 16, 1, sink);  // warm L2
    cudaEventRecord(e0, st);
    probe_l2_kernel<<<blocks, threads, 0, st>>>(buf, bytes / 16, reps, sink);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    // Every rep reads the whole buffer once across the grid.
    if (l2_read_gbs) *l2_read_gbs = (double)bytes * reps / (ms * 1e-3) / 1e9;
    const int iters = 4096;
    const int fthreads = 256, fblocks = sms * 8;
    probe_fma_kernel<double><<<fblocks, fthreads, 0, st>>>(iters / 8, 1.0, dsink);
    cudaEventRecord(e0, st);
    probe_fma_kernel<double><<<fblocks, fthreads, 0, st>>>(iters, 1.0, dsink);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (fp64_tflops) *fp64_tflops = 2.0 * 32 * (double)iters * fthreads * fblocks / (ms * 1e-3) / 1e12;
    probe_fma_kernel<float><<<fblocks, fthreads, 0, st>>>(iters / 8, 1.0f, fsink);
    cudaEventRecord(e0, st);
    probe_fma_kernel<float><<<fblocks, fthreads, 0, st>>>(iters * 4, 1.0f, fsink);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (fp32_tflops) *fp32_tflops = 2.0 * 32 * (double)iters * 4 * fthreads * fblocks / (ms * 1e-3) / 1e12;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = probe_fail(e, "vct_probe_peaks");
  }
  cudaFree(buf);
  cudaFree(sink);
  cudaFree(dsink);
  cudaFree(fsink);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  return rc;
}
