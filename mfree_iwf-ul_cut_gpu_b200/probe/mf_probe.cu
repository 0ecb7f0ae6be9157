// Measurement aid for the benchmark only (no counterpart in the reference, not part of the
// product library): the FP64 FMA throughput of the device, which the step's FP64 kernels are
// compared against, and the latency of the double-precision calls on the return map's critical
// path (pow, log, division), measured with the SM clock. Built into lib/libmf_probe.so.
#include <cuda_runtime.h>

#include "mfree_b200.h"

namespace {

constexpr int PROBE_CHAINS = 8;
constexpr int PROBE_ITERS = 2048;

// 8 independent FMA chains per thread; the sum keeps them live
__global__ void k_probe_fma(double seed, double *out) {
  double a[PROBE_CHAINS];
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) a[k] = seed + 1e-3 * (threadIdx.x + k);
  const double b = 0.999999, c = 1e-7;
  for (int i = 0; i < PROBE_ITERS; ++i) {
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; ++k) a[k] = fma(a[k], b, c);
  }
  double s = 0.;
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) s += a[k];
  if (s == 12345.678) out[0] = s;  // practically never: the store only keeps the work alive
}

// one thread, a dependent chain of `n` calls; out = clock cycles per call
__global__ void k_probe_latency(int which, int n, double x0, double *out) {
  double x = x0;
  const long long t0 = clock64();
  for (int i = 0; i < n; ++i) {
    if (which == 0) x = pow(x, 0.93) + 0.5;
    else if (which == 1) x = log(x) + 2.5;
    else x = 3.0 / x + 0.7;
  }
  const long long t1 = clock64();
  out[0] = (double)(t1 - t0) / n;
  out[1] = x;
}

}  // namespace

extern "C" int mf_probe_fp64(int device, double *fma_tflops, double *pow_cycles, double *log_cycles,
                             double *div_cycles, double *sm_clock_mhz) {
  if (cudaSetDevice(device) != cudaSuccess) return MF_ERR_NO_DEVICE;
  int sms = 0, clk_khz = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, device);
  double *d = nullptr;
  if (cudaMalloc(&d, 4 * sizeof(double)) != cudaSuccess) return MF_ERR_NOMEM;
  int rc = MF_OK;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256;
  k_probe_fma<<<blocks, threads>>>(1.0, d);  // warm-up
  cudaEventRecord(e0);
  for (int r = 0; r < 5; ++r) k_probe_fma<<<blocks, threads>>>(1.0 + r, d);
  cudaEventRecord(e1);
  if (cudaEventSynchronize(e1) != cudaSuccess) rc = MF_ERR_CUDA;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  if (fma_tflops)
    *fma_tflops = 5.0 * 2.0 * (double)blocks * threads * PROBE_ITERS * PROBE_CHAINS / (ms * 1e-3) / 1e12;
  double h[2];
  double *outs[3] = {pow_cycles, log_cycles, div_cycles};
  const double x0[3] = {1.7, 3.0, 1.3};
  for (int w = 0; w < 3 && rc == MF_OK; ++w) {
    k_probe_latency<<<1, 1>>>(w, 8, x0[w], d);  // warm-up (instruction cache)
    k_probe_latency<<<1, 1>>>(w, 1024, x0[w], d);
    if (cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) rc = MF_ERR_CUDA;
    if (outs[w]) *outs[w] = h[0];
  }
  if (sm_clock_mhz) *sm_clock_mhz = clk_khz / 1000.0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  return rc == MF_OK && cudaGetLastError() == cudaSuccess ? MF_OK : MF_ERR_CUDA;
}
