// ORACLE recipe - test infrastructure only, never part of the product.
//
// Force-included (nvcc -include) ahead of every reference source of the GPU oracle build
// (oracle/build_oracle.py, build_ref_gpu), so that the reference's own CUDA files compile
// unchanged, where they lie, with CUDA 12.9. The reference fetches its neighbour data through
// the legacy texture-reference API (interactions_gpu.cu:38-76, 355-421), which CUDA 12
// removed. This header supplies that API's documented behaviour for 1D textures bound to
// linear device memory:
//   * a file-scope `texture<T, 1, mode> name;` becomes a __device__ variable holding the bound
//     pointer and its length in elements (the macro below; on a function parameter the
//     __device__ qualifier is ignored, with nvcc warning 1835, so by-value texture parameters
//     keep working);
//   * cudaBindTexture(offset, tex, ptr, bytes) stores (ptr, bytes / sizeof(T)) into that
//     variable (cudaMemcpyToSymbol, ordered on the legacy default stream like the kernels);
//   * tex1Dfetch(tex, i) returns element i, and zero for an index outside [0, length): the
//     reference relies on this where it binds tool_particle with sizeof(int) * N bytes for an
//     array of N doubles (interactions_gpu.cu:405), so that indices >= N/2 read 0.
#ifndef MF_REF_TEXTURE_SHIM_H
#define MF_REF_TEXTURE_SHIM_H

#include <cuda_runtime.h>

// every library header the reference includes, before the `texture` macro below exists
#include <thrust/device_vector.h>
#include <thrust/device_ptr.h>
#include <thrust/host_vector.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include <thrust/reduce.h>
#include <thrust/extrema.h>
#include <thrust/functional.h>
#include <thrust/transform.h>
#include <thrust/partition.h>
#include <thrust/gather.h>
#include <thrust/scan.h>
#include <thrust/unique.h>
#include <thrust/random.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/discard_iterator.h>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <vector>

template <class T, int dim = 1, enum cudaTextureReadMode mode = cudaReadModeElementType>
struct mf_ref_texref {
  const T *ptr;
  long long n;  // bound length in elements
};

template <class T, int D, enum cudaTextureReadMode M>
__device__ __forceinline__ T tex1Dfetch(const mf_ref_texref<T, D, M> &t, int i) {
  if (i < 0 || (long long)i >= t.n) return T{};
  return __ldg(t.ptr + i);
}

template <class T, int D, enum cudaTextureReadMode M>
static inline cudaError_t cudaBindTexture(size_t *offset, const mf_ref_texref<T, D, M> &tex, const void *ptr,
                                          size_t size) {
  mf_ref_texref<T, D, M> v;
  v.ptr = static_cast<const T *>(ptr);
  v.n = (long long)(size / sizeof(T));
  if (offset) *offset = 0;
  return cudaMemcpyToSymbol(tex, &v, sizeof(v));
}

template <class T, int D, enum cudaTextureReadMode M>
static inline cudaError_t cudaUnbindTexture(const mf_ref_texref<T, D, M> &tex) {
  (void)tex;
  return cudaSuccess;
}

#define texture __device__ mf_ref_texref

#endif
