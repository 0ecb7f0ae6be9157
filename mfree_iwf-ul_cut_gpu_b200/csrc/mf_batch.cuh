// Batched step kernels: many particle systems (cutting instances of uneven size) advanced
// together, one launch per phase of the step for all of them (mf_batch_*). The reference keeps
// its constants in __constant__ memory per translation unit (actions_gpu.cu:438-469,
// interactions_gpu.cu:423-459, tool_gpu.cu:20-27), one system per process; here every system's
// constants and buffers are one entry of a device array, and each block of a batched launch
// finds its system by the block's index and runs the same kernel body as the single-system
// kernel on that system's share of the grid. The arithmetic of every system is the
// single-system step's, bit for bit (same bodies, same force-sum tree per 256 particles).
#pragma once

#include "mf_mixed.cuh"

namespace mf {

// one system's step parameters, buffers (bound to one parity of its double buffer) and scan size
struct __align__(16) batch_entry {
  params P;
  dev_buffers D;
  int scan_tiles;
};

// one batched launch: entries of every system and first[k] = the first grid block of system k
// (n + 1 values, first[n] = the grid size)
struct batch_map {
  const batch_entry *e;
  const int *first;
  int n;
};

// The system of batched block vb (the largest k with first[k] <= vb), its entry copied into
// shared memory by the block's threads (16-byte words), and the block's index and count within
// it. A batched launch passes its own block index; the persistent kernel each phase block it
// takes.
__device__ __forceinline__ blk batch_block_at(const batch_map &M, batch_entry &s, int vb) {
  __shared__ int s_k;
  if (threadIdx.x == 0) {
    int lo = 0, hi = M.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(M.first + mid) <= vb) lo = mid;
      else hi = mid - 1;
    }
    s_k = lo;
  }
  __syncthreads();
  const int k = s_k;
  static_assert(sizeof(batch_entry) % 16 == 0, "entries are whole 16-byte words");
  const int4 *src = reinterpret_cast<const int4 *>(M.e + k);
  int4 *dst = reinterpret_cast<int4 *>(&s);
  for (int w = threadIdx.x; w < (int)(sizeof(batch_entry) / 16); w += blockDim.x) dst[w] = __ldg(src + w);
  __syncthreads();
  const int f0 = __ldg(M.first + k), f1 = __ldg(M.first + k + 1);
  return blk{vb - f0, f1 - f0};
}
__device__ __forceinline__ blk batch_block(const batch_map &M, batch_entry &s) {
  return batch_block_at(M, s, (int)blockIdx.x);
}

static __global__ void __launch_bounds__(SCAN_THREADS) kb_scan(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  scan_body(s.D, s.P.N, 0, b);
}

static __global__ void __launch_bounds__(BLOCK) kb_scatter(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  scatter_body(s.P.N, s.D, 0, b);
}

template <bool MIXED>
static __global__ void __launch_bounds__(BLOCK, 4) kb_reorder(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  reorder_body<true, MIXED>(s.P, s.D, b);
}

// The pair kernels for a block size chosen by the batch's tuner. A batched kernel reads its
// system's parameters from shared memory instead of the constant bank, which costs registers:
// its launch bounds leave more room per thread than the single-system kernel's, so that it
// does not spill.
template <int BS>
static __global__ void __launch_bounds__(BS) kb_pair_fp64(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  pair_fp64_body(s.P, s.D, b);
}

template <int BS>
static __global__ void __launch_bounds__(BS, 640 / BS) kb_pair_mixed(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  pair_mixed_body<false>(s.P, s.D, b);
}

template <int BS>
static __global__ void __launch_bounds__(BS) kb_pse(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  pse_body(s.P, s.D, b);
}

template <int BS>
static __global__ void __launch_bounds__(BS) kb_pse_mixed(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  pse_mixed_body(s.P, s.D, b);
}

static __global__ void __launch_bounds__(FINISH_BLOCK, 2) kb_finish(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  finish_flat_body<true, false>(s.P, s.D, s.scan_tiles, b);
}

template <bool PAIRED>
static __global__ void __launch_bounds__(BLOCK, 2) kb_plastic(batch_map M) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ batch_entry s;
  const blk b = batch_block(M, s);
  plastic_body<PAIRED>(s.P, s.D, b);
}

}  // namespace mf
