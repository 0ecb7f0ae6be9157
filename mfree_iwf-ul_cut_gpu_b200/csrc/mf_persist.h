// The persistent batched step (mf_persist.cu): its launch arguments and host entry points.
#pragma once

#include "mf_batch.cuh"

namespace mf {

// threads per block of the persistent kernel: every phase body's block size
// (SCAN_THREADS, BLOCK, FINISH_BLOCK; the pair phase's block map is built for it)
constexpr int PERSIST_BLOCK = 256;
static_assert(PERSIST_BLOCK == SCAN_THREADS && PERSIST_BLOCK == BLOCK && PERSIST_BLOCK == FINISH_BLOCK,
              "the persistent kernel runs every phase body at its own block size");

struct persist_args {
  const batch_entry *e;  // [2][n] entries, by buffer parity
  const int *first;      // 4 block maps of n + 1 entries: scan, 256-thread phases, pair, plastic
  int n, K;              // systems, steps per launch
  int grid[4];           // blocks of each map's phase over all systems
  int pse, plastic, paired;
  unsigned long long *bar;     // barrier word: arrivals, abort bit, generation
  unsigned long long wait_ns;  // limit of one barrier wait
};

// resident blocks per SM of the persistent (mixed-precision) kernel (-1 on a CUDA error)
int persist_blocks_per_sm(int *blocks);
// one cooperative launch of the persistent kernel (-1 on a CUDA error)
int persist_launch(cudaStream_t stream, int grid, const persist_args &A);

}  // namespace mf
