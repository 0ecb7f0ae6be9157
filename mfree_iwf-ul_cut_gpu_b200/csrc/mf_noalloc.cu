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
// holds it (about 22 MB) until the process exits. In host code its name is only a stand-in, not a
// device address, so the address is looked up once per device with cudaGetSymbolAddress,
// with that device current, during the first call on that device. All calls share the
// array and it keeps the last call's contents: each call clears what must start at zero.
// Calls that overlap on the GPU (other streams, other host threads) race on it.
#include <cuda_runtime.h>

#include <algorithm>
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
  unsigned long long scan_status[NA_SCAN_TILES];
  geom g;
  dev_status st;
  unsigned scan_done;
};

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

// zero the counts, the scan's tile states and tickets; store the geometry
__global__ void k_na_clear(noalloc_scratch *S, geom g) {
  const int stride = gridDim.x * blockDim.x;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int c = gid; c < g.num_cell; c += stride) S->count[c] = 0;
  const int tiles = (g.num_cell + SCAN_TILE - 1) / SCAN_TILE + 1;
  for (int t = gid; t < tiles; t += stride) S->scan_status[t] = 0ull;
  if (gid == 0) {
    S->g = g;
    dev_status z{};
    S->st = z;
    S->scan_done = 0u;
  }
}
// cell hash (compute_hashes, grid.cu:34-51), clamped into the grid, and per-cell count
// cell hash (compute_hashes, grid.cu:34-51), clamped into the grid, and per-cell slot
__global__ void k_na_hash(const double2 *__restrict__ pos, int N, noalloc_scratch *S) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const geom g = S->g;
  const double2 p = pos[i];
  const int ix = __double2int_rz((p.x - g.bbmin_x) / g.dx);
  const int iy = __double2int_rz((p.y - g.bbmin_y) / g.dx);
  long long hh = (long long)ix * (long long)g.ny + (long long)iy;
  if (hh < 0) hh = 0;
  else if (hh >= g.num_cell) hh = g.num_cell - 1;
  const int h = (int)hh;
  S->hash_new[i] = h;
  atomicAdd(&S->count[h], 1);
}

// sorted outputs: permutation and hash per sorted position; cell bounds in the
// grid_gpu_green format (-1 on empty cells)
__global__ void k_na_output(int N, dev_buffers D, int *__restrict__ hash_sorted, int *__restrict__ idx,
                            int *__restrict__ cell_start, int *__restrict__ cell_end, int num_cell) {
  const int stride = gridDim.x * blockDim.x;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int q = gid; q < N; q += stride) {
    const int4 u = D.perm_u[q];
    idx[q] = stable_member(D, q, u);
    hash_sorted[q] = u.y;
  }
  for (int c = gid; c < num_cell; c += stride) {
    const int s = D.off[c], e = D.off[c + 1];
    cell_start[c] = e > s ? s : -1;
    cell_end[c] = e > s ? e : -1;
  }
}

}  // namespace

extern "C" int mf_cells_build_noalloc(const double *d_pos, int N, double bbmin_x, double bbmin_y, double dx,
                                      int nx, int ny, int *d_hash_sorted, int *d_idx, int *d_cell_start,
                                      int *d_cell_end, void *stream) {
  if (N < 1 || nx < 1 || ny < 1 || !(dx > 0.)) return MF_ERR_INVALID;
  if (N > NA_MAX_PARTICLES || (long long)nx * ny > NA_MAX_CELLS) return MF_ERR_RANGE;
  if (!d_pos || !d_hash_sorted || !d_idx || !d_cell_start || !d_cell_end) return MF_ERR_INVALID;
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
  // the scan and the stable fix-up of mf_grid_build, pointed at the scratch array
  dev_buffers D{};
  D.count = S->count;
  D.off = S->off;
  D.hash_new = S->hash_new;
  D.perm_u = S->perm_u;
  D.scan_status = S->scan_status;
  D.scan_done = &S->scan_done;
  D.g = &S->g;
  D.st = &S->st;
  const int scan_tiles = (g.num_cell + SCAN_TILE - 1) / SCAN_TILE + 1;
  const int nb = (N + BLOCK - 1) / BLOCK;
  const int ob = (std::max(N, g.num_cell) + BLOCK - 1) / BLOCK;
  k_na_clear<<<std::min(ob, 148 * 8), BLOCK, 0, st>>>(S, g);
  k_na_hash<<<nb, BLOCK, 0, st>>>(reinterpret_cast<const double2 *>(d_pos), N, S);
  k_scan<<<scan_tiles, SCAN_THREADS, 0, st>>>(D, N, 0);
  k_scatter<<<nb, BLOCK, 0, st>>>(N, D, 0);
  k_na_output<<<std::min(ob, 148 * 16), BLOCK, 0, st>>>(N, D, d_hash_sorted, d_idx, d_cell_start, d_cell_end,
                                                        g.num_cell);
  return cudaGetLastError() == cudaSuccess ? MF_OK : MF_ERR_CUDA;
}
