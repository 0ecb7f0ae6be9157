// Cell-list build that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: a host application that reserves
// all of its device memory when it starts and forbids any driver allocation afterwards
// (so that a long cutting run cannot fail half-way on an allocation, or because another
// memory manager owns the device), or a foreign-language host whose binding hands over
// device pointers but gives no access to the CUDA allocator. For them,
// mf_cells_build_noalloc computes the same cell list as mf_grid_build (hash, stable
// permutation, cell start/end) with the caller's inputs and outputs only; its scratch
// memory is the file-scope device array below, of a fixed maximum size.
//
// The array is part of this file's module image: every GPU on which the module is loaded
// holds it (26 MiB) until the process exits. In host code its name is only a stand-in, not a
// device address, so the address is looked up once per device with cudaGetSymbolAddress,
// with that device current, during the first call on that device, and cached. A
// cudaDeviceReset unloads the module, so the cached address is stale afterwards: a process
// that resets a device must not call this entry point on that device again. All calls share
// the array and it keeps the last call's contents: each call clears what must start at
// zero. Calls that overlap on the GPU (other streams, other host threads) race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "mf_kernels.cuh"
#include "mfree_b200.h"

namespace {

using namespace mf;

constexpr int NA_MAX_PARTICLES = MF_NOALLOC_MAX_PARTICLES;
constexpr int NA_MAX_CELLS = MF_NOALLOC_MAX_CELLS;
constexpr int NA_SCAN_TILES = (NA_MAX_CELLS + SCAN_TILE - 1) / SCAN_TILE + 1;

struct noalloc_scratch {
  int4 perm_u[NA_MAX_PARTICLES];
  int count[NA_MAX_CELLS];
  int off[NA_MAX_CELLS + 1];
  int hash_new[NA_MAX_PARTICLES];
  int tsum[2][NA_SCAN_TILES];  // per-tile count totals: [0] counted into, [1] zeroed by the scan
  geom g;
  dev_status st;
};
static_assert(sizeof(noalloc_scratch) < (27u << 20), "the scratch array stays near 26 MiB");

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(noalloc_scratch)];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[NA_MAX_DEVICES] = {};

// device address of the scratch array on the current device (looked up once per device)
int scratch_for_current_device(noalloc_scratch **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return MF_ERR_NO_DEVICE;
  if (dev >= NA_MAX_DEVICES) return MF_ERR_RANGE;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return MF_ERR_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<noalloc_scratch *>(g_scratch_addr[dev]);
  return MF_OK;
}

// zero the counts, the scan's per-tile totals and the status; store the geometry
__global__ void k_na_clear(noalloc_scratch *S, geom g) {
  const int stride = gridDim.x * blockDim.x;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int c = gid; c < g.num_cell; c += stride) S->count[c] = 0;
  const int tiles = (g.num_cell + SCAN_TILE - 1) / SCAN_TILE + 1;
  for (int t = gid; t < tiles; t += stride) S->tsum[0][t] = 0;
  if (gid == 0) {
    S->g = g;
    dev_status z{};
    S->st = z;
  }
}

// cell hash (compute_hashes, grid.cu:34-51) and per-cell count; a particle outside the grid
// is clamped into the nearest cell and counted (the reference writes out of bounds there)
__global__ void k_na_hash(const double2 *__restrict__ pos, int N, noalloc_scratch *S) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned oog = 0;
  if (i < N) {
    const geom g = S->g;
    const double2 p = pos[i];
    const int ix = __double2int_rz((p.x - g.bbmin_x) / g.dx);
    const int iy = __double2int_rz((p.y - g.bbmin_y) / g.dx);
    long long hh = (long long)ix * (long long)g.ny + (long long)iy;
    if (hh < 0) { hh = 0; oog = 1; }
    else if (hh >= g.num_cell) { hh = g.num_cell - 1; oog = 1; }
    const int h = (int)hh;
    S->hash_new[i] = h;
    count_particle(S->count, S->tsum[0], h);
  }
  const unsigned any = __ballot_sync(0xffffffffu, oog);
  if (any && (threadIdx.x & 31u) == 0) atomicAdd(&S->st.out_of_grid, (unsigned long long)__popc(any));
}

// sorted outputs: permutation and hash per sorted position (each member moved to its stable
// slot in its cell); cell bounds in the grid_gpu_green format (-1 on empty cells)
__global__ void k_na_output(int N, const noalloc_scratch *__restrict__ S, int *__restrict__ hash_sorted,
                            int *__restrict__ idx, int *__restrict__ cell_start, int *__restrict__ cell_end,
                            int num_cell) {
  const int stride = gridDim.x * blockDim.x;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int t = gid; t < N; t += stride) {
    const int4 u = S->perm_u[t];
    const int q = u.z + stable_rank(S->perm_u, u);
    idx[q] = u.x;
    hash_sorted[q] = u.y;
  }
  for (int c = gid; c < num_cell; c += stride) {
    const int s = S->off[c], e = S->off[c + 1];
    cell_start[c] = e > s ? s : -1;
    cell_end[c] = e > s ? e : -1;
  }
}

// the call's status into the caller's memory, after every other kernel of the call
__global__ void k_na_status(const noalloc_scratch *__restrict__ S, mf_noalloc_status *out) {
  out->out_of_grid = S->st.out_of_grid;
  out->error_flags = S->st.error_flags;
  out->max_cell_occupancy = S->st.max_cell_occupancy;
}

// one launch; its own launch error is returned (an earlier error of the caller's work left
// in the runtime's last-error slot is neither read nor cleared)
template <typename... KArgs, typename... Args>
cudaError_t na_launch(void (*kernel)(KArgs...), int grid, int block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.stream = st;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

bool aligned(const void *p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

}  // namespace

extern "C" int mf_cells_build_noalloc(const double *d_pos, int N, double bbmin_x, double bbmin_y, double dx,
                                      int nx, int ny, int *d_hash_sorted, int *d_idx, int *d_cell_start,
                                      int *d_cell_end, mf_noalloc_status *d_status, void *stream) {
  if (N < 1 || nx < 1 || ny < 1 || !(dx > 0.)) return MF_ERR_INVALID;
  if (N > NA_MAX_PARTICLES || (long long)nx * ny > NA_MAX_CELLS) return MF_ERR_RANGE;
  if (!d_pos || !d_hash_sorted || !d_idx || !d_cell_start || !d_cell_end) return MF_ERR_INVALID;
  // the positions are read as 16-byte pairs, the outputs as 4-byte ints, the status as
  // 8-byte words: a pointer off those boundaries is refused before anything is launched
  if (!aligned(d_pos, 16) || !aligned(d_hash_sorted, 4) || !aligned(d_idx, 4) || !aligned(d_cell_start, 4) ||
      !aligned(d_cell_end, 4) || (d_status && !aligned(d_status, 8)))
    return MF_ERR_INVALID;
  noalloc_scratch *S = nullptr;
  int rc = scratch_for_current_device(&S);
  if (rc != MF_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  geom g{};
  g.nx = nx;
  g.ny = ny;
  g.num_cell = nx * ny;
  g.max_cell = g.num_cell;
  g.bbmin_x = bbmin_x;
  g.bbmin_y = bbmin_y;
  g.dx = dx;
  g.locked = 1;
  // the scan and the scatter of mf_grid_build, pointed at the scratch array
  dev_buffers D{};
  D.count = S->count;
  D.off = S->off;
  D.hash_new = S->hash_new;
  D.perm_u = S->perm_u;
  D.tsum_r = S->tsum[0];
  D.tsum_w = S->tsum[1];
  D.g = &S->g;
  D.st = &S->st;
  const int scan_tiles = (g.num_cell + SCAN_TILE - 1) / SCAN_TILE + 1;
  const int nb = (N + BLOCK - 1) / BLOCK;
  const int ob = (std::max(N, g.num_cell) + BLOCK - 1) / BLOCK;
  cudaError_t e = na_launch(k_na_clear, std::min(ob, 148 * 8), BLOCK, st, S, g);
  if (e == cudaSuccess) e = na_launch(k_na_hash, nb, BLOCK, st, reinterpret_cast<const double2 *>(d_pos), N, S);
  if (e == cudaSuccess) e = na_launch(k_scan, scan_tiles, SCAN_THREADS, st, D, N, 0);
  if (e == cudaSuccess) e = na_launch(k_scatter, nb, BLOCK, st, N, D, 0);
  if (e == cudaSuccess)
    e = na_launch(k_na_output, std::min(ob, 148 * 16), BLOCK, st, N, (const noalloc_scratch *)S, d_hash_sorted,
                  d_idx, d_cell_start, d_cell_end, g.num_cell);
  if (e == cudaSuccess && d_status) e = na_launch(k_na_status, 1, 1, st, (const noalloc_scratch *)S, d_status);
  return e == cudaSuccess ? MF_OK : MF_ERR_CUDA;
}
