// FP64 fused multiply-add throughput of the device: the denominator of the
// FP64-pipe fractions that bench.py reports beside the HBM roofline.  This is
// a measurement aid built into its own library (liblag2d_bench.so); it is not
// part of the time-step API in include/lag2d.h.
//
// Every thread runs kChains independent FMA chains a = a * b + c for `iters`
// rounds (b slightly below 1 keeps the values bounded), so the FP64 pipe sees
// kChains independent instructions per thread between dependent ones; the
// grid is 8 blocks of 256 threads per SM.  FLOPs = 2 * kChains * iters *
// threads.  The result of every thread is stored, so no chain is dead code.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_dfma_peak(int iters, double b, double c, double *out) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; k++) a[k] = 1.0 + 1e-3 * (threadIdx.x + k);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < kChains; k++) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; k++) s += a[k];
  out[blockIdx.x * (size_t)kThreads + threadIdx.x] = s;
}

}  // namespace

// Best of `repeats` timed launches after one warm-up launch, in TFLOP/s;
// a negative value is an error (no device, allocation or launch failure).
// The caller picks the device.
extern "C" double lag2d_bench_dfma_tflops(int iters, int repeats) {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1.0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1.0;
  const int nblk = 8 * nsm;
  double *out = nullptr;
  if (cudaMalloc(&out, (size_t)nblk * kThreads * sizeof(double)) != cudaSuccess) return -2.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 0.0;
  for (int r = 0; r <= repeats; r++) {
    cudaEventRecord(e0);
    k_dfma_peak<<<nblk, kThreads>>>(iters, 0.9999999, 1e-7, out);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * kChains * (double)iters * nblk * kThreads;
    if (r > 0 && ms > 0.0f) {
      const double tf = flops / (ms * 1e-3) / 1e12;
      if (tf > best) best = tf;
    }
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return err == cudaSuccess ? best : -3.0;
}
