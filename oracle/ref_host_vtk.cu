// Test infrastructure: the reference's VTK writer (vtk_writer.cpp) compiled from its own source
// where it lies, its device-to-host copies made host copies, so that its tool output
// (vtk_writer.cpp:185-264) can be produced on the host as a checker.
#include <cstring>

#include <cuda_runtime.h>

static cudaError_t harness_vtk_copy(void *dst, const void *src, size_t n, cudaMemcpyKind) {
  std::memcpy(dst, src, n);
  return cudaSuccess;
}
#define cudaMemcpy harness_vtk_copy
#include "vtk_writer.cpp"
#undef cudaMemcpy
