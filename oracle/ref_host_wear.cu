// Test infrastructure: the reference's Usui wear evaluation (tool_wear.cu:20-64) compiled from
// its own source where it lies, with its device-to-host cudaMemcpy calls turned into host
// copies, so that it can be run on host arrays as a checker.
#include <cstring>

#include <cuda_runtime.h>

static cudaError_t harness_host_copy(void *dst, const void *src, size_t n, cudaMemcpyKind) {
  std::memcpy(dst, src, n);
  return cudaSuccess;
}
#define cudaMemcpy harness_host_copy
#include "tool_wear.cu"
#undef cudaMemcpy

// eval_usui on host arrays (interleaved x, y for the vectors); out = min, max, avg, accumulated
extern "C" int refh_usui(int N, const double *pos, const double *vel, const double *fc, const double *ft,
                         const double *h, const double *n, const double *T, double K, double alpha,
                         double tool_vx, double tool_vy, double dt, double out[4]) {
  phys_constants phys;
  std::memset(&phys, 0, sizeof(phys));
  tool_wear w(K, alpha, (unsigned)N, phys, vec2_t(tool_vx, tool_vy));
  std::vector<double> rho((size_t)N, 1.);
  particle_gpu p((float2_t *)pos, (float2_t *)vel, rho.data(), (float_t *)h, (unsigned)N);
  p.vel = (float2_t *)vel;
  p.fc = (float2_t *)fc;
  p.ft = (float2_t *)ft;
  p.h = (float_t *)h;
  p.n = (float2_t *)n;
  p.T = (float_t *)T;
  float_t mn = 0., mx = 0., avg = 0.;
  w.eval_usui(&p, dt, mn, mx, avg);
  out[0] = mn;
  out[1] = mx;
  out[2] = avg;
  out[3] = w.get_accum_wear();
  return 0;
}
