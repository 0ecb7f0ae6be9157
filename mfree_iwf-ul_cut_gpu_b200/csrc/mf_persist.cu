// Persistent batched step: one cooperative launch of a fixed grid (one or two 256-thread
// blocks per SM) runs K whole steps of every system of a mixed-precision batch. Each phase of a step (cell
// scan, scatter, reorder + predictor, pair sums, PSE, finish, return map) is the batched
// phase kernel's work (mf_batch.cuh): the phase's blocks, counted per system as the per-phase
// launch counts them, are taken by the resident blocks in turn (block b runs phase blocks b,
// b + grid, ...), each running the same kernel body on its system's share; a grid-wide
// barrier separates the phases. The per-system arithmetic is therefore the single-system
// step's, bit for bit. (An FP64 variant was built and measured: its pair sums, whose
// multiply-adds the compiler contracts, came out contracted differently inside this kernel -
// deterministic, ~1e-16 relative off the single-system step - so the persistent form serves the
// mixed form only, whose pair arithmetic spells out its fused multiply-adds.)
//
// Loads. Within one launch a phase reads what the phase before it wrote on other SMs. The
// read-only data path (ld.global.nc, which __ldg and const __restrict__ pointers select) is
// coherent only at kernel boundaries, so this translation unit compiles the shared kernel
// bodies with plain loads: __ldg becomes a plain dereference and __restrict__ is dropped
// (the CUDA headers are included before the two definitions, so only the bodies see them).
// Plain loads after the barrier's acquire see every write made before any block's arrival.
//
// The barrier waits with a limit (globaltimer, default 2 s): a block whose wait expires aborts
// that barrier, which then releases no block, and sets error bit 3 in every system's status;
// every block returns at that barrier, so the launch always ends. The cooperative launch attribute makes the driver refuse a grid that cannot be
// resident at once, instead of starting blocks that would wait on blocks never scheduled.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>

#define __ldg(p) (*(p))
#define __restrict__

#include "mf_batch.cuh"
#include "mf_persist.h"

namespace mf {

namespace {

__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The barrier is one 64-bit word changed only by atomics: arrivals in bits 0-30, an abort bit
// (31) and the generation in bits 32-63. A block publishes its writes (fence) and arrives; the
// last to arrive releases the next generation with a compare-and-swap from the full count. A
// waiter whose time runs out sets the abort bit with a compare-and-swap on the value it saw.
// Exactly one of the two swaps can succeed, so a barrier either releases every block or none:
// no block ever starts a phase whose inputs another block left unfinished.
constexpr unsigned long long BAR_COUNT = 0x7fffffffull, BAR_ABORT = 0x80000000ull;

__device__ void persist_report(const persist_args &A) {
  for (int k = 0; k < A.n; ++k) atomicOr(&A.e[k].D.st->error_flags, ERR_BATCH_WAIT);
}

// False when the barrier was aborted (a wait ran out here or in another block).
__device__ bool persist_sync(const persist_args &A) {
  __shared__ unsigned s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned ok = 1u;
    __threadfence();
    const unsigned long long old = atomicAdd(A.bar, 1ull);
    const unsigned long long gen = old >> 32;
    if (old & BAR_ABORT) {
      ok = 0u;
    } else if ((old & BAR_COUNT) == gridDim.x - 1u) {
      __threadfence();
      if (atomicCAS(A.bar, old + 1ull, (gen + 1ull) << 32) != old + 1ull) ok = 0u;  // aborted meanwhile
    } else {
      const unsigned long long t0 = global_ns();
      for (;;) {
        const unsigned long long v = ld_acquire_gpu(A.bar);
        if ((v >> 32) != gen) break;  // released
        if (v & BAR_ABORT) {
          ok = 0u;
          break;
        }
        if (global_ns() - t0 > A.wait_ns) {
          if (atomicCAS(A.bar, v, v | BAR_ABORT) == v) {
            persist_report(A);
            ok = 0u;
            break;
          }
          continue;  // the word changed: look again
        }
        __nanosleep(100);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0u;
}

// the blocks vb = blockIdx.x, blockIdx.x + gridDim.x, ... of one phase (nvb blocks over all
// systems), each with its system's entry in shared memory
template <class F>
__device__ __forceinline__ void persist_phase(const batch_map &m, int nvb, batch_entry &s, F body) {
  for (int vb = (int)blockIdx.x; vb < nvb; vb += (int)gridDim.x) {
    const blk b = batch_block_at(m, s, vb);
    body(b);
    __syncthreads();  // s and the body's shared memory are reused by the next block
  }
}

__global__ void __launch_bounds__(PERSIST_BLOCK, 2) kp_batch_mixed(persist_args A) {
  __shared__ batch_entry s;
  for (int st = 0; st < A.K; ++st) {
    const batch_entry *ent = A.e + (size_t)(st & 1) * A.n;
    const batch_map m_scan{ent, A.first, A.n}, m_256{ent, A.first + (A.n + 1), A.n},
        m_pair{ent, A.first + 2 * (A.n + 1), A.n}, m_pl{ent, A.first + 3 * (A.n + 1), A.n};
    persist_phase(m_scan, A.grid[0], s, [&](blk b) { scan_body(s.D, s.P.N, 0, b); });
    if (!persist_sync(A)) return;
    persist_phase(m_256, A.grid[1], s, [&](blk b) { scatter_body(s.P.N, s.D, 0, b); });
    if (!persist_sync(A)) return;
    persist_phase(m_256, A.grid[1], s, [&](blk b) { reorder_body<true, true>(s.P, s.D, b); });
    if (!persist_sync(A)) return;
    persist_phase(m_pair, A.grid[2], s, [&](blk b) { pair_mixed_body<false>(s.P, s.D, b); });
    if (!persist_sync(A)) return;
    if (A.pse) {
      persist_phase(m_pair, A.grid[2], s, [&](blk b) { pse_mixed_body(s.P, s.D, b); });
      if (!persist_sync(A)) return;
    }
    persist_phase(m_256, A.grid[1], s, [&](blk b) { finish_flat_body<true, false>(s.P, s.D, s.scan_tiles, b); });
    if (!persist_sync(A)) return;
    if (A.plastic) {
      if (A.paired) persist_phase(m_pl, A.grid[3], s, [&](blk b) { plastic_body<true>(s.P, s.D, b); });
      else persist_phase(m_pl, A.grid[3], s, [&](blk b) { plastic_body<false>(s.P, s.D, b); });
      if (st + 1 < A.K && !persist_sync(A)) return;
    }
  }
}

}  // namespace

int persist_blocks_per_sm(int *blocks) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kp_batch_mixed, PERSIST_BLOCK, 0) != cudaSuccess) return -1;
  *blocks = b;
  return 0;
}

int persist_launch(cudaStream_t stream, int grid, const persist_args &A) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)PERSIST_BLOCK);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kp_batch_mixed, A) == cudaSuccess ? 0 : -1;
}

}  // namespace mf
