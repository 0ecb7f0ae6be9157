// C ABI of the B200 SPH step (include/mfree_b200.h): context, device buffers, launches and
// CUDA-graph replay of leap_frog::step (leap_frog.cu:94-155).
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "mf_kernels.cuh"
#include "mf_mixed.cuh"
#include "mf_batch.cuh"
#include "mf_persist.h"
#include "mfree_b200.h"

using namespace mf;

namespace {
// a named NVTX range for profilers (Nsight Compute --nvtx filters, timelines) over one entry
// point or stage; header-only NVTX, a no-op unless a tool is attached
struct nvtx_range {
  explicit nvtx_range(const char *name) { nvtxRangePushA(name); }
  ~nvtx_range() { nvtxRangePop(); }
  nvtx_range(const nvtx_range &) = delete;
  nvtx_range &operator=(const nvtx_range &) = delete;
};
}  // namespace

namespace mf {
// the differentiable step (csrc/mf_tangent.cu): one derivative direction (tg), all six (tg6);
// out_dmean holds d(mean Fc), d(mean Ff) per direction
namespace tg {
int run_mean_force(mf_ctx *ctx, int device, params P, const dev_buffers &Dctx, int skip_steps, int window_steps,
                   int param, double out_mean[2], double out_dmean[]);
}  // namespace tg
namespace tg6 {
int run_mean_force(mf_ctx *ctx, int device, params P, const dev_buffers &Dctx, int skip_steps, int window_steps,
                   int param, double out_mean[2], double out_dmean[]);
}  // namespace tg6
}  // namespace mf

// one asynchronous particle dump: a device snapshot of the fields, their copy into pinned
// host memory on a side stream, and a host thread that writes the file once it has landed
struct vtk_job {
  int n = 0;
  double *dev = nullptr;   // snapshot: pos 2n, vel 2n, rho n, p n, T n, eps n, S 4n
  unsigned *dev_flags = nullptr;
  double *host = nullptr;  // pinned copy of the same
  unsigned *host_flags = nullptr;
  cudaEvent_t snap = nullptr, landed = nullptr;
  std::thread writer;
  int rc = 0;
};

struct mf_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int last_cuda_err = 0;
  int flags = 0;
  // particles
  int N = 0;
  bool has_particles = false;
  // grid
  bool has_grid = false;
  int grid_kind = MF_GRID_GREEN;
  geom G{};
  // constants / options
  params P{};
  bool has_constants = false;
  mf_tool_state tool{};
  // device memory
  dev_buffers D{};
  state_set set[2]{};
  int cur = 0;          // set holding the current state
  bool mid_step = false; // stages 1-2 ran: reads see the step's buffer
  bool last_staged = false; // the last predictor ran staged (all intermediates stored)
  int scan_tiles = 0;   // tiles for max_cell + 1 entries
  int *tsum[2] = {nullptr, nullptr};  // per-tile count totals: written with one parity, read with the other
  int bbox_blocks = 0;
  int sm_count = 148;
  mf_tool_state *tool_buf[2] = {nullptr, nullptr};  // tool after the last step, by parity
  // k_finish_flat of the last step already hashed and counted the particles for the next one
  // (locked grid): the next step starts at the scan
  bool counts_ready = false;
  double skin = 0.;  // neighbour-list skin (mixed form); <= 0: a tenth of the cell size
  std::vector<void *> particle_allocs, grid_allocs, fixed_allocs;
  // graphs: one per parity of the double buffer
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  bool graph_valid = false;
  // bumped whenever captured work goes stale (buffers, constants, options, dt, flags)
  unsigned long long gen = 0;
  long long steps = 0;
  unsigned long long force_read_head = 0;
  unsigned long long status_newly_blanked_seen = 0;
  cudaStream_t io_stream = nullptr;  // device-to-host copies of asynchronous dumps
  std::vector<std::unique_ptr<vtk_job>> vtk_jobs;
};

namespace {

#define CK(call)                                    \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) {                        \
      ctx->last_cuda_err = (int)e_;                 \
      return MF_ERR_CUDA;                           \
    }                                               \
  } while (0)

int set_device(mf_ctx *ctx) {
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) { ctx->last_cuda_err = (int)e; return MF_ERR_CUDA; }
  return MF_OK;
}

template <class T>
int dalloc(mf_ctx *ctx, std::vector<void *> &list, T **ptr, size_t count) {
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, count ? count * sizeof(T) : sizeof(T));
  if (e != cudaSuccess) {
    ctx->last_cuda_err = (int)e;
    return e == cudaErrorMemoryAllocation ? MF_ERR_NOMEM : MF_ERR_CUDA;
  }
  e = cudaMemset(p, 0, count ? count * sizeof(T) : sizeof(T));
  if (e != cudaSuccess) { ctx->last_cuda_err = (int)e; return MF_ERR_CUDA; }
  list.push_back(p);
  *ptr = (T *)p;
  return MF_OK;
}

void free_list(std::vector<void *> &list) {
  for (void *p : list) cudaFree(p);
  list.clear();
}

int invalidate_counts(mf_ctx *ctx);

// Captured work is stale: buffers, constants, options, dt or flags changed. The next step also
// starts over from a sort (its counts primed again): with neighbour lists the last step may
// have run the next step's predictor with the old parameters.
void drop_graphs(mf_ctx *ctx) {
  ctx->gen++;
  for (int k = 0; k < 2; ++k)
    if (ctx->graph[k]) { cudaGraphExecDestroy(ctx->graph[k]); ctx->graph[k] = nullptr; }
  ctx->graph_valid = false;
  (void)invalidate_counts(ctx);  // (a failed memset surfaces at the next synchronizing call)
}

#define TRY(x)                 \
  do {                         \
    int r_ = (x);              \
    if (r_ != MF_OK) return r_; \
  } while (0)

int alloc_set(mf_ctx *ctx, state_set &s, int N) {
  auto &L = ctx->particle_allocs;
  TRY(dalloc(ctx, L, &s.pos, N)); TRY(dalloc(ctx, L, &s.vel, N)); TRY(dalloc(ctx, L, &s.fc, N));
  TRY(dalloc(ctx, L, &s.ft, N)); TRY(dalloc(ctx, L, &s.pos_t, N)); TRY(dalloc(ctx, L, &s.vel_t, N));
  TRY(dalloc(ctx, L, &s.rho, N)); TRY(dalloc(ctx, L, &s.T, N)); TRY(dalloc(ctx, L, &s.eps_pl, N));
  TRY(dalloc(ctx, L, &s.eps_pl_dot, N)); TRY(dalloc(ctx, L, &s.h, N)); TRY(dalloc(ctx, L, &s.rho_t, N));
  TRY(dalloc(ctx, L, &s.T_t, N)); TRY(dalloc(ctx, L, &s.S, N)); TRY(dalloc(ctx, L, &s.S_t, N));
  TRY(dalloc(ctx, L, &s.flags, N)); TRY(dalloc(ctx, L, &s.idx, N)); TRY(dalloc(ctx, L, &s.id, N));
  TRY(dalloc(ctx, L, &s.pp, N));
  return MF_OK;
}

// the counts the last step's k_finish_flat prepared are stale once the host changes the state
int invalidate_counts(mf_ctx *ctx) {
  if (ctx->counts_ready && ctx->D.count) {
    CK(cudaMemsetAsync(ctx->D.count, 0, sizeof(int) * (size_t)ctx->G.max_cell, ctx->stream));
    for (int k = 0; k < 2; ++k) CK(cudaMemsetAsync(ctx->tsum[k], 0, sizeof(int) * (size_t)ctx->scan_tiles, ctx->stream));
  }
  ctx->counts_ready = false;
  return MF_OK;
}

int alloc_particles(mf_ctx *ctx, int N) {
  drop_graphs(ctx);
  free_list(ctx->particle_allocs);
  auto &L = ctx->particle_allocs;
  TRY(alloc_set(ctx, ctx->set[0], N));
  TRY(alloc_set(ctx, ctx->set[1], N));
  dev_buffers &D = ctx->D;
  TRY(dalloc(ctx, L, &D.n, N));
  TRY(dalloc(ctx, L, &D.rec, (size_t)N * R_WIDTH));
  TRY(dalloc(ctx, L, &D.recf, (size_t)N * F_WIDTH));
  TRY(dalloc(ctx, L, &D.S_der, N));
  TRY(dalloc(ctx, L, &D.v_der, N));
  TRY(dalloc(ctx, L, &D.hash_cur, N));
  TRY(dalloc(ctx, L, &D.hash_new, N));
  TRY(dalloc(ctx, L, &D.perm_u, N));
  TRY(dalloc(ctx, L, &D.perm, N));
  TRY(dalloc(ctx, L, &D.plastic_list, N));
  TRY(dalloc(ctx, L, &D.nlist, (size_t)LIST_CAP * N));
  TRY(dalloc(ctx, L, &D.ncount, N));
  TRY(dalloc(ctx, L, &D.pos_build, N));
  ctx->bbox_blocks = std::min((N + BLOCK - 1) / BLOCK, ctx->sm_count * 4);
  // per-chunk force partials of the finish kernel and their group sums (or per-block partials of
  // the bbox pass), the force sum's group tickets
  const int finish_chunks = (N + FINISH_BLOCK - 1) / FINISH_BLOCK;
  const int force_groups = (finish_chunks + FORCE_GROUP - 1) / FORCE_GROUP;
  TRY(dalloc(ctx, L, &D.partials,
             (size_t)std::max(std::max(finish_chunks + force_groups, ctx->bbox_blocks), 1) * 8));
  TRY(dalloc(ctx, L, &D.gticket, (size_t)std::max(force_groups, 1)));
  TRY(invalidate_counts(ctx));
  ctx->N = N;
  return MF_OK;
}

int alloc_grid(mf_ctx *ctx, int max_cell) {
  drop_graphs(ctx);
  free_list(ctx->grid_allocs);
  auto &L = ctx->grid_allocs;
  TRY(dalloc(ctx, L, &ctx->D.count, (size_t)max_cell));
  TRY(dalloc(ctx, L, &ctx->D.off, (size_t)max_cell + 1));
  ctx->scan_tiles = (max_cell + SCAN_TILE - 1) / SCAN_TILE + 1;
  TRY(dalloc(ctx, L, &ctx->tsum[0], (size_t)ctx->scan_tiles));
  TRY(dalloc(ctx, L, &ctx->tsum[1], (size_t)ctx->scan_tiles));
  ctx->counts_ready = false;
  return MF_OK;
}


int upload_geom(mf_ctx *ctx) {
  CK(cudaMemcpyAsync(ctx->D.g, &ctx->G, sizeof(geom), cudaMemcpyHostToDevice, ctx->stream));
  return MF_OK;
}

void bind_sets(mf_ctx *ctx) {
  ctx->D.A = ctx->set[ctx->cur];
  ctx->D.B = ctx->set[ctx->cur ^ 1];
  ctx->D.tool_prev = ctx->tool_buf[ctx->cur];
  ctx->D.tool_next = ctx->tool_buf[ctx->cur ^ 1];
  // a step's scan reads the tile totals the previous step's finish kernel (or the priming
  // count) added to, and zeroes the ones this step's finish kernel adds to
  ctx->D.tsum_r = ctx->tsum[ctx->cur ^ 1];
  ctx->D.tsum_w = ctx->tsum[ctx->cur];
}

// the steady-state step of a locked grid starts at the scan: the previous step's k_finish_flat
// hashed and counted the particles
bool fused_step(const mf_ctx *ctx) { return ctx->G.locked && !ctx->P.staged; }

bool ready(const mf_ctx *ctx) { return ctx->has_particles && ctx->has_grid && ctx->has_constants; }

// Neighbour lists for the mixed form (steps on a locked grid), when asked for: its pair sums
// are not tied to the reference's summation order, so the cell list need not be sorted every
// step. Not with the PSE solver, whose window has no support cut-off, nor when asked to sort
// every step.
bool list_mode(const mf_ctx *ctx) {
  return ctx->P.precision == MF_PRECISION_MIXED && fused_step(ctx) && (ctx->flags & MF_OPT_NEIGHBOUR_LISTS) &&
         !(ctx->flags & MF_OPT_SORT_EVERY_STEP) &&
         !(ctx->P.thermal_solver == MF_THERMAL_PSE && ctx->P.thermal_wp) &&
         (long long)ctx->N <= (long long)LIST_INDEX_MASK + 1;
}

void set_list_mode(mf_ctx *ctx) {
  // the EOS sound speed of every particle: the device's float rounding of the same IEEE
  // operations, computed once
  ctx->P.eos_c0 = (double)sqrtf((float)(ctx->P.phys.K / ctx->P.phys.rho0));
  ctx->P.verlet = list_mode(ctx) ? 1 : 0;
  ctx->P.fuse = ctx->P.verlet && (ctx->flags & MF_OPT_FUSED_PREDICTOR) ? 1 : 0;
  // at most half a cell: the lists are built over the 7x7 cells around a particle, which hold
  // every candidate within 2 h + skin while h + skin / 2 is at most the cell size, and 64
  // entries hold the candidates of a lattice with h = 1.5 spacings up to that skin
  const double skin = ctx->skin > 0. ? ctx->skin : 0.1 * ctx->G.dx;
  ctx->P.skin = (float)std::min(skin, 0.5 * ctx->G.dx);
}

#ifndef MF_USE_PDL
#define MF_USE_PDL 1
#endif
// a step kernel, launched so that it may be scheduled while the previous kernel on the stream
// drains (programmatic dependent launch); the kernel waits for its predecessor before it
// touches memory (MF_PDL_WAIT)
template <typename... KArgs, typename... Args>
int launch_pdl_smem(mf_ctx *ctx, void (*kernel)(KArgs...), int grid, int block, size_t smem, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = MF_USE_PDL ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, args...);
  if (e != cudaSuccess) {
    ctx->last_cuda_err = (int)e;
    return MF_ERR_CUDA;
  }
  return MF_OK;
}

template <typename... KArgs, typename... Args>
int launch_pdl(mf_ctx *ctx, void (*kernel)(KArgs...), int grid, int block, Args... args) {
  return launch_pdl_smem(ctx, kernel, grid, block, 0, args...);
}

// cell-list build into the other buffer (k_hash_count .. k_reorder); PREDICT adds the
// predictor of the step
int launch_cells(mf_ctx *ctx, bool step_mode) {
  const int N = ctx->N;
  const int nb = (N + BLOCK - 1) / BLOCK;
  bind_sets(ctx);
  if (!ctx->G.locked)
    TRY(launch_pdl(ctx, k_bbox, ctx->bbox_blocks, BLOCK, N, (const double2 *)ctx->D.A.pos, (const double *)ctx->D.A.h, ctx->D));
  if (!(step_mode && fused_step(ctx))) {
    const int hash_blocks = std::max(nb, (ctx->scan_tiles + BLOCK - 1) / BLOCK);
    TRY(launch_pdl(ctx, k_hash_count, hash_blocks, BLOCK, N, ctx->D.A, ctx->D, ctx->scan_tiles));
  }
  const int verlet = step_mode ? ctx->P.verlet : 0;  // a sort outside a step always sorts
  TRY(launch_pdl(ctx, k_scan, ctx->scan_tiles, SCAN_THREADS, ctx->D, N, verlet));
  TRY(launch_pdl(ctx, k_scatter, nb, BLOCK, N, ctx->D, verlet));
  return MF_OK;
}

int launch_stage(mf_ctx *ctx, int stage) {
  static const char *const names[4] = {"mf stage 0: cell list", "mf stage 1: predictor",
                                       "mf stage 2: pair sums", "mf stage 3: finish + return map"};
  nvtx_range range(stage >= 0 && stage < 4 ? names[stage] : "mf stage");
  const int N = ctx->N;
  const int nb = (N + BLOCK - 1) / BLOCK;
  const int npb = (N + PAIR_BLOCK - 1) / PAIR_BLOCK;
  bind_sets(ctx);
  set_list_mode(ctx);
  const bool mixed = ctx->P.precision == MF_PRECISION_MIXED;
  switch (stage) {
    case 0:
      TRY(launch_cells(ctx, true));
      break;
    case 1:
      if (mixed) TRY(launch_pdl(ctx, k_reorder<true, true>, nb, BLOCK, ctx->P, ctx->D));
      else TRY(launch_pdl(ctx, k_reorder<true, false>, nb, BLOCK, ctx->P, ctx->D));
      break;
    case 2:
      if (mixed && ctx->P.verlet) TRY(launch_pdl(ctx, k_pair_mixed<true>, npb, PAIR_BLOCK, ctx->P, ctx->D));
      else if (mixed) TRY(launch_pdl(ctx, k_pair_mixed<false>, npb, PAIR_BLOCK, ctx->P, ctx->D));
      else TRY(launch_pdl(ctx, k_pair_fp64, (N + PAIR64_BLOCK - 1) / PAIR64_BLOCK, PAIR64_BLOCK, ctx->P, ctx->D));
      if (ctx->P.thermal_solver == MF_THERMAL_PSE && ctx->P.thermal_wp) {
        if (mixed) TRY(launch_pdl(ctx, k_pse_mixed, npb, PAIR_BLOCK, ctx->P, ctx->D));
        else TRY(launch_pdl(ctx, k_pse, npb, PAIR_BLOCK, ctx->P, ctx->D));
      }
      break;
    case 3:
      {
        const int fb = (N + FINISH_BLOCK - 1) / FINISH_BLOCK;
        const bool hash = fused_step(ctx);
        if (ctx->P.h_contact > 0.) {  // with contact conductance
          if (ctx->P.fuse && hash)
            TRY(launch_pdl(ctx, k_finish_flat<true, true, true>, fb, FINISH_BLOCK, ctx->P, ctx->D, ctx->scan_tiles));
          else if (ctx->P.fuse)
            TRY(launch_pdl(ctx, k_finish_flat<false, true, true>, fb, FINISH_BLOCK, ctx->P, ctx->D, ctx->scan_tiles));
          else if (hash)
            TRY(launch_pdl(ctx, k_finish_flat<true, false, true>, fb, FINISH_BLOCK, ctx->P, ctx->D, ctx->scan_tiles));
          else
            TRY(launch_pdl(ctx, k_finish_flat<false, false, true>, fb, FINISH_BLOCK, ctx->P, ctx->D, ctx->scan_tiles));
        } else if (ctx->P.fuse) {  // the next step's predictor runs here too
          if (hash)
            TRY(launch_pdl(ctx, k_finish_flat<true, true>, fb, FINISH_BLOCK, ctx->P, ctx->D, ctx->scan_tiles));
          else
            TRY(launch_pdl(ctx, k_finish_flat<false, true>, fb, FINISH_BLOCK, ctx->P, ctx->D, ctx->scan_tiles));
        } else if (hash) {
          TRY(launch_pdl(ctx, k_finish_flat<true, false>, fb, FINISH_BLOCK, ctx->P, ctx->D, ctx->scan_tiles));
        } else {
          TRY(launch_pdl(ctx, k_finish_flat<false, false>, fb, FINISH_BLOCK, ctx->P, ctx->D, ctx->scan_tiles));
        }
      }
      if (ctx->P.plastic) {
        if (ctx->P.jc_model == MF_JC_TANH)
          TRY(launch_pdl(ctx, k_plastic<false>, ctx->sm_count * PLASTIC_BLOCKS_PER_SM, BLOCK, ctx->P, ctx->D));
        else
          TRY(launch_pdl(ctx, k_plastic<true>, ctx->sm_count * PLASTIC_BLOCKS_PER_SM, BLOCK, ctx->P, ctx->D));
      }
      break;
    default:
      return MF_ERR_INVALID;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { ctx->last_cuda_err = (int)e; return MF_ERR_CUDA; }
  return MF_OK;
}

int launch_step(mf_ctx *ctx) {
  for (int s = 0; s < 4; ++s) TRY(launch_stage(ctx, s));
  return MF_OK;
}

// hash + count for the first fused step (afterwards each step's k_finish_flat prepares them)
int prime_counts(mf_ctx *ctx) {
  if (!fused_step(ctx) || ctx->counts_ready) return MF_OK;
  bind_sets(ctx);
  const int nb = (ctx->N + BLOCK - 1) / BLOCK;
  const int hash_blocks = std::max(nb, (ctx->scan_tiles + BLOCK - 1) / BLOCK);
  k_hash_count<<<hash_blocks, BLOCK, 0, ctx->stream>>>(ctx->N, ctx->D.A, ctx->D, ctx->scan_tiles);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { ctx->last_cuda_err = (int)e; return MF_ERR_CUDA; }
  // with neighbour lists the next step sorts (and builds the lists): any nonzero value
  CK(cudaMemsetAsync(&ctx->D.st->sort_now, 1, sizeof(unsigned), ctx->stream));
  ctx->counts_ready = true;
  return MF_OK;
}

int build_graphs(mf_ctx *ctx) {
  drop_graphs(ctx);
  const int saved = ctx->cur;
  for (int k = 0; k < 2; ++k) {
    ctx->cur = k;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = launch_step(ctx);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != MF_OK) { if (g) cudaGraphDestroy(g); ctx->cur = saved; return rc; }
    if (e != cudaSuccess) { ctx->last_cuda_err = (int)e; ctx->cur = saved; return MF_ERR_CUDA; }
    e = cudaGraphInstantiate(&ctx->graph[k], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { ctx->last_cuda_err = (int)e; ctx->cur = saved; return MF_ERR_CUDA; }
  }
  ctx->cur = saved;
  ctx->graph_valid = true;
  return MF_OK;
}

// field storage: 0 current set, 1 position-indexed array, 2 derived
struct field_desc {
  int width;
  bool is_int;
};
field_desc describe(int f) {
  switch (f) {
    case MF_FIELD_POS: case MF_FIELD_VEL: case MF_FIELD_FC: case MF_FIELD_FT: case MF_FIELD_N:
    case MF_FIELD_POS_T: case MF_FIELD_VEL_T:
      return {2, false};
    case MF_FIELD_S: case MF_FIELD_R: case MF_FIELD_S_T: case MF_FIELD_S_DER: case MF_FIELD_V_DER:
      return {4, false};
    case MF_FIELD_IDX: case MF_FIELD_HASH: case MF_FIELD_ID:
      return {1, true};
    default:
      return {1, false};
  }
}

int view_set(const mf_ctx *ctx) { return ctx->mid_step ? (ctx->cur ^ 1) : ctx->cur; }

void *field_ptr(mf_ctx *ctx, int f) {
  state_set &s = ctx->set[view_set(ctx)];
  switch (f) {
    case MF_FIELD_POS: return s.pos;
    case MF_FIELD_VEL: return s.vel;
    case MF_FIELD_H: return s.h;
    case MF_FIELD_RHO: return s.rho;
    case MF_FIELD_P: return s.pp;
    case MF_FIELD_S: return s.S;
    case MF_FIELD_FC: return s.fc;
    case MF_FIELD_FT: return s.ft;
    case MF_FIELD_N: return ctx->D.n;
    case MF_FIELD_EPS_PL: return s.eps_pl;
    case MF_FIELD_EPS_PL_DOT: return s.eps_pl_dot;
    case MF_FIELD_T: return s.T;
    case MF_FIELD_POS_T: return s.pos_t;
    case MF_FIELD_VEL_T: return s.vel_t;
    case MF_FIELD_RHO_T: return s.rho_t;
    case MF_FIELD_S_T: return s.S_t;
    case MF_FIELD_T_T: return s.T_t;
    case MF_FIELD_S_DER: return ctx->D.S_der;
    case MF_FIELD_V_DER: return ctx->D.v_der;
    case MF_FIELD_IDX: return s.idx;
    case MF_FIELD_HASH: return ctx->D.hash_cur;
    case MF_FIELD_ID: return s.id;
    default: return nullptr;
  }
}

unsigned flag_bit(int f) {
  return f == MF_FIELD_FIXED ? FLAG_FIXED : f == MF_FIELD_BLANKED ? FLAG_BLANKED : f == MF_FIELD_TOOL ? FLAG_TOOL : 0u;
}

}  // namespace

extern "C" {

int mf_version(void) { return MF_ABI_VERSION; }

const char *mf_error_string(int code) {
  switch (code) {
    case MF_OK: return "ok";
    case MF_ERR_INVALID: return "invalid argument";
    case MF_ERR_CUDA: return "CUDA runtime error";
    case MF_ERR_STATE: return "call out of order";
    case MF_ERR_RANGE: return "size out of range";
    case MF_ERR_NOMEM: return "out of memory";
    case MF_ERR_NO_DEVICE: return "no CUDA device";
    case MF_ERR_DEVICE_FAULT: return "a kernel reported an internal error";
    case MF_ERR_IO: return "state file input/output failed";
    case MF_ERR_CORRUPT: return "state file failed its checks";
    default: return "unknown error";
  }
}

int mf_last_cuda_error(const mf_ctx *ctx) { return ctx ? ctx->last_cuda_err : 0; }

int mf_ctx_create(int device, mf_ctx **out) {
  if (!out) return MF_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return MF_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return MF_ERR_INVALID;
  mf_ctx *ctx = new (std::nothrow) mf_ctx;
  if (!ctx) return MF_ERR_NOMEM;
  ctx->device = device;
  int rc = set_device(ctx);
  if (rc == MF_OK) {
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) rc = MF_ERR_CUDA;
  }
  if (rc == MF_OK) rc = dalloc(ctx, ctx->fixed_allocs, &ctx->D.g, 1);
  if (rc == MF_OK) rc = dalloc(ctx, ctx->fixed_allocs, &ctx->D.st, 1);
  if (rc == MF_OK) rc = dalloc(ctx, ctx->fixed_allocs, &ctx->D.plastic_count, 1);
  if (rc == MF_OK) rc = dalloc(ctx, ctx->fixed_allocs, &ctx->tool_buf[0], 1);
  if (rc == MF_OK) rc = dalloc(ctx, ctx->fixed_allocs, &ctx->tool_buf[1], 1);
  if (rc == MF_OK) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
      ctx->sm_count = sms;
  }
  if (rc == MF_OK) rc = dalloc(ctx, ctx->fixed_allocs, &ctx->D.ticket, 4);
  if (rc == MF_OK) rc = dalloc(ctx, ctx->fixed_allocs, &ctx->D.force_log, (size_t)FORCE_LOG_CAP * 2);
  if (rc == MF_OK) rc = dalloc(ctx, ctx->fixed_allocs, &ctx->D.force_last, 2);
  if (rc != MF_OK) { mf_ctx_destroy(ctx); return rc; }
  ctx->P.corr.wdeltap = 1.;  // make_corr_constants (constants_structs.cpp:31-35)
  *out = ctx;
  return MF_OK;
}

int mf_ctx_destroy(mf_ctx *ctx) {
  if (!ctx) return MF_OK;
  cudaSetDevice(ctx->device);
  mf_vtk_flush(ctx);
  if (ctx->io_stream) cudaStreamDestroy(ctx->io_stream);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graphs(ctx);
  free_list(ctx->particle_allocs);
  free_list(ctx->grid_allocs);
  free_list(ctx->fixed_allocs);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return MF_OK;
}

int mf_ctx_stream(mf_ctx *ctx, void **stream) {
  if (!ctx || !stream) return MF_ERR_INVALID;
  *stream = (void *)ctx->stream;
  return MF_OK;
}

int mf_set_flags(mf_ctx *ctx, int flags) {
  if (!ctx) return MF_ERR_INVALID;
  ctx->flags = flags;
  ctx->P.keep_derivs = (flags & MF_OPT_KEEP_DERIVATIVES) ? 1 : 0;
  drop_graphs(ctx);
  return MF_OK;
}

int mf_set_contact_conductance(mf_ctx *ctx, double h_contact, double T_tool) {
  if (!ctx || !(h_contact >= 0.) || !std::isfinite(h_contact) || !std::isfinite(T_tool)) return MF_ERR_INVALID;
  ctx->P.h_contact = h_contact;
  ctx->P.T_contact = T_tool;
  drop_graphs(ctx);  // a kernel variant and its parameters
  return MF_OK;
}

int mf_set_neighbour_skin(mf_ctx *ctx, double skin) {
  if (!ctx || !(skin == skin)) return MF_ERR_INVALID;
  ctx->skin = skin;
  drop_graphs(ctx);  // the skin is a kernel parameter
  return MF_OK;
}

int mf_list_check(mf_ctx *ctx, long long *pairs, long long *missing, int *stale) {
  if (!ctx || !pairs || !missing) return MF_ERR_INVALID;
  if (!ready(ctx) || ctx->mid_step) return MF_ERR_STATE;
  if (!ctx->P.verlet) return MF_ERR_STATE;  // the last step did not run on neighbour lists
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  dev_status st;
  CK(cudaMemcpy(&st, ctx->D.st, sizeof(st), cudaMemcpyDeviceToHost));
  const int N = ctx->N;
  const int nb = (N + BLOCK - 1) / BLOCK;
  double2 *abs = nullptr;
  unsigned long long *out = nullptr;
  unsigned long long h[2] = {0ull, 0ull};
  cudaError_t e = cudaMalloc(&abs, sizeof(double2) * (size_t)N);
  if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(h));
  if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, sizeof(h), ctx->stream);
  if (e == cudaSuccess) {
    params P = ctx->P;
    P.N = N;
    k_list_abs<<<nb, BLOCK, 0, ctx->stream>>>(N, ctx->D, abs);
    k_list_check<<<nb, BLOCK, 0, ctx->stream>>>(P, ctx->D, abs, out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (abs) cudaFree(abs);
  if (out) cudaFree(out);
  if (e != cudaSuccess) {
    ctx->last_cuda_err = (int)e;
    return e == cudaErrorMemoryAllocation ? MF_ERR_NOMEM : MF_ERR_CUDA;
  }
  *pairs = (long long)h[0];
  *missing = (long long)h[1];
  // with the fused predictor the records may already be the next step's; the lists hold for
  // them only if that step does not sort
  if (stale) *stale = (st.predicted && st.sort_now) ? 1 : 0;
  return MF_OK;
}

int mf_synchronize(mf_ctx *ctx) {
  if (!ctx) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_particles_create(mf_ctx *ctx, int N, const double *pos, const double *vel, const double *rho, const double *T,
                        const double *h, const double *fixed, const double *tool_p, const double *S) {
  if (!ctx || N <= 0 || !pos || !vel || !rho || !h) return MF_ERR_INVALID;
  for (const double *fl : {fixed, tool_p})
    if (fl)
      for (int i = 0; i < N; ++i)
        if (!(fl[i] == 0. || fl[i] == 1.)) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  TRY(alloc_particles(ctx, N));
  // the tool set so far stays the current one when the parity restarts at 0
  if (ctx->cur != 0)
    CK(cudaMemcpy(ctx->tool_buf[0], ctx->tool_buf[ctx->cur], sizeof(mf_tool_state), cudaMemcpyDeviceToDevice));
  ctx->cur = 0;
  state_set &s = ctx->set[0];
  CK(cudaMemcpy(s.pos, pos, sizeof(double) * 2 * (size_t)N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s.vel, vel, sizeof(double) * 2 * (size_t)N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s.rho, rho, sizeof(double) * (size_t)N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s.h, h, sizeof(double) * (size_t)N, cudaMemcpyHostToDevice));
  if (T) CK(cudaMemcpy(s.T, T, sizeof(double) * (size_t)N, cudaMemcpyHostToDevice));
  if (S) CK(cudaMemcpy(s.S, S, sizeof(double) * 4 * (size_t)N, cudaMemcpyHostToDevice));
  std::vector<unsigned> fl((size_t)N, 0u);
  std::vector<int> idx((size_t)N);
  for (int i = 0; i < N; ++i) {
    if (fixed && fixed[i] == 1.) fl[i] |= FLAG_FIXED;
    if (tool_p && tool_p[i] == 1.) fl[i] |= FLAG_TOOL;
    idx[i] = i;  // particle_gpu.cu:53-54
  }
  CK(cudaMemcpy(s.flags, fl.data(), sizeof(unsigned) * (size_t)N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s.idx, idx.data(), sizeof(int) * (size_t)N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s.id, idx.data(), sizeof(int) * (size_t)N, cudaMemcpyHostToDevice));
  ctx->has_particles = true;
  ctx->P.N = N;
  return MF_OK;
}

int mf_particles_count(const mf_ctx *ctx, int *N) {
  if (!ctx || !N) return MF_ERR_INVALID;
  *N = ctx->has_particles ? ctx->N : 0;
  return MF_OK;
}

int mf_get_field(mf_ctx *ctx, int field, void *host) {
  if (!ctx || !host || field < 0 || field >= MF_NUM_FIELDS) return MF_ERR_INVALID;
  if (!ctx->has_particles) return MF_ERR_STATE;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  const size_t N = (size_t)ctx->N;
  unsigned bit = flag_bit(field);
  if (bit) {
    std::vector<unsigned> fl(N);
    CK(cudaMemcpy(fl.data(), ctx->set[view_set(ctx)].flags, sizeof(unsigned) * N, cudaMemcpyDeviceToHost));
    double *o = (double *)host;
    for (size_t i = 0; i < N; ++i) o[i] = (fl[i] & bit) ? 1. : 0.;
    return MF_OK;
  }
  if (field == MF_FIELD_R) {
    double *o = (double *)host;
    if (ctx->P.precision == MF_PRECISION_MIXED && !ctx->last_staged) {
      // mixed form: R lives only in the FP32 pair records
      std::vector<float> rec(N * F_WIDTH);
      CK(cudaMemcpy(rec.data(), ctx->D.recf, sizeof(float) * N * F_WIDTH, cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < N; ++i) {
        auto at = [&](int f) { return rec[recf_word(f / 4, (int)i, (int)N) * 4 + f % 4]; };
        o[4 * i] = at(F_RXX);
        o[4 * i + 1] = at(F_RXY);
        o[4 * i + 2] = at(F_RYY);
        o[4 * i + 3] = 0.;
      }
      return MF_OK;
    }
    std::vector<double> rec(N * R_WIDTH);
    CK(cudaMemcpy(rec.data(), ctx->D.rec, sizeof(double) * N * R_WIDTH, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < N; ++i) {
      auto at = [&](int f) { return rec[(size_t)(f / 2) * N * 2 + (size_t)i * 2 + f % 2]; };
      o[4 * i] = at(R_RXX);
      o[4 * i + 1] = at(R_RXY);
      o[4 * i + 2] = at(R_RYY);
      o[4 * i + 3] = 0.;
    }
    return MF_OK;
  }
  field_desc d = describe(field);
  void *src = field_ptr(ctx, field);
  if (!src) return MF_ERR_INVALID;
  size_t bytes = N * d.width * (d.is_int ? sizeof(int) : sizeof(double));
  CK(cudaMemcpy(host, src, bytes, cudaMemcpyDeviceToHost));
  return MF_OK;
}

int mf_set_field(mf_ctx *ctx, int field, const void *host) {
  if (!ctx || !host || field < 0 || field >= MF_NUM_FIELDS) return MF_ERR_INVALID;
  if (!ctx->has_particles) return MF_ERR_STATE;
  TRY(set_device(ctx));
  TRY(invalidate_counts(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  const size_t N = (size_t)ctx->N;
  unsigned bit = flag_bit(field);
  if (bit) {
    const double *in = (const double *)host;
    for (size_t i = 0; i < N; ++i)
      if (!(in[i] == 0. || in[i] == 1.)) return MF_ERR_INVALID;
    std::vector<unsigned> fl(N);
    CK(cudaMemcpy(fl.data(), ctx->set[ctx->cur].flags, sizeof(unsigned) * N, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < N; ++i) fl[i] = in[i] == 1. ? (fl[i] | bit) : (fl[i] & ~bit);
    CK(cudaMemcpy(ctx->set[ctx->cur].flags, fl.data(), sizeof(unsigned) * N, cudaMemcpyHostToDevice));
    return MF_OK;
  }
  if (field == MF_FIELD_R) return MF_ERR_INVALID;  // recomputed every step
  field_desc d = describe(field);
  void *dst = field_ptr(ctx, field);
  if (!dst) return MF_ERR_INVALID;
  size_t bytes = N * d.width * (d.is_int ? sizeof(int) : sizeof(double));
  CK(cudaMemcpy(dst, host, bytes, cudaMemcpyHostToDevice));
  return MF_OK;
}

int mf_grid_create_locked(mf_ctx *ctx, int kind, double bbmin_x, double bbmin_y, double bbmax_x, double bbmax_y,
                          double h) {
  if (!ctx || (kind != MF_GRID_GREEN && kind != MF_GRID_ROTHLIN) || !(h > 0.)) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  // grid_base::set_geometry (grid.cu:139-158)
  geom G{};
  G.bbmin_x = bbmin_x - 1e-6;
  G.bbmin_y = bbmin_y - 1e-6;
  G.bbmax_x = bbmax_x + 1e-6;
  G.bbmax_y = bbmax_y + 1e-6;
  double kernel_width = 2.;
  G.dx = h * kernel_width / 2.;
  double lx = G.bbmax_x - G.bbmin_x, ly = G.bbmax_y - G.bbmin_y;
  double fnx = std::ceil(lx / G.dx), fny = std::ceil(ly / G.dx);
  if (!(fnx >= 1. && fny >= 1.) || fnx * fny > 2.0e9) return MF_ERR_RANGE;
  G.nx = (int)(unsigned)fnx;
  G.ny = (int)(unsigned)fny;
  G.num_cell = G.nx * G.ny;
  G.max_cell = G.num_cell;
  G.locked = 1;
  TRY(alloc_grid(ctx, G.max_cell));
  ctx->G = G;
  ctx->grid_kind = kind;
  ctx->P.grid_kind = kind;
  ctx->has_grid = true;
  TRY(upload_geom(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_grid_create_adaptive(mf_ctx *ctx, int kind, int max_cell) {
  if (!ctx || (kind != MF_GRID_GREEN && kind != MF_GRID_ROTHLIN) || max_cell < 2) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  geom G{};
  G.nx = 1; G.ny = 1; G.num_cell = 1; G.max_cell = max_cell; G.dx = 1.; G.locked = 0;
  TRY(alloc_grid(ctx, max_cell));
  ctx->G = G;
  ctx->grid_kind = kind;
  ctx->P.grid_kind = kind;
  ctx->has_grid = true;
  TRY(upload_geom(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_grid_geometry(mf_ctx *ctx, int *nx, int *ny, int *num_cell, double *out5) {
  if (!ctx) return MF_ERR_INVALID;
  if (!ctx->has_grid) return MF_ERR_STATE;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  geom G;
  CK(cudaMemcpy(&G, ctx->D.g, sizeof(geom), cudaMemcpyDeviceToHost));
  if (nx) *nx = G.nx;
  if (ny) *ny = G.ny;
  if (num_cell) *num_cell = G.num_cell;
  if (out5) { out5[0] = G.bbmin_x; out5[1] = G.bbmin_y; out5[2] = G.bbmax_x; out5[3] = G.bbmax_y; out5[4] = G.dx; }
  return MF_OK;
}

int mf_grid_build(mf_ctx *ctx) {
  nvtx_range range("mf_grid_build");
  if (!ctx) return MF_ERR_INVALID;
  if (!ctx->has_particles || !ctx->has_grid || ctx->mid_step) return MF_ERR_STATE;
  TRY(set_device(ctx));
  ctx->P.N = ctx->N;
  TRY(invalidate_counts(ctx));
  TRY(launch_cells(ctx, false));
  const int nb = (ctx->N + BLOCK - 1) / BLOCK;
  params Pg = ctx->P;
  Pg.verlet = 0;  // a sort outside a step always sorts
  k_reorder<false, false><<<nb, BLOCK, 0, ctx->stream>>>(Pg, ctx->D);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { ctx->last_cuda_err = (int)e; return MF_ERR_CUDA; }
  ctx->cur ^= 1;
  CK(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_grid_get_cells(mf_ctx *ctx, int *start, int *end) {
  if (!ctx || !start || !end) return MF_ERR_INVALID;
  if (!ctx->has_grid) return MF_ERR_STATE;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  geom G;
  CK(cudaMemcpy(&G, ctx->D.g, sizeof(geom), cudaMemcpyDeviceToHost));
  std::vector<int> off((size_t)G.num_cell + 1);
  CK(cudaMemcpy(off.data(), ctx->D.off, sizeof(int) * off.size(), cudaMemcpyDeviceToHost));
  for (int c = 0; c < G.num_cell; ++c) {
    if (ctx->grid_kind == MF_GRID_ROTHLIN) {
      start[c] = off[c];
      end[c] = off[c + 1];
    } else if (off[c + 1] > off[c]) {
      start[c] = off[c];
      end[c] = off[c + 1];
    } else {
      start[c] = -1;
      end[c] = -1;
    }
  }
  return MF_OK;
}

int mf_set_constants(mf_ctx *ctx, const mf_phys_constants *phys, const mf_corr_constants *corr,
                     const mf_joco_constants *joco, const mf_trml_constants *trml_wp,
                     const mf_trml_constants *trml_tool) {
  if (!ctx || !phys || !corr) return MF_ERR_INVALID;
  params &P = ctx->P;
  P.phys = *phys;
  P.corr = *corr;
  P.plastic = joco ? 1 : 0;
  if (joco) P.joco = *joco;
  else std::memset(&P.joco, 0, sizeof(P.joco));
  P.jc_lower_bound = joco && joco->A > 0. && joco->B >= 0. && joco->C >= 0. ? 1 : 0;
  std::memset(&P.trml_wp, 0, sizeof(P.trml_wp));
  std::memset(&P.trml_tool, 0, sizeof(P.trml_tool));
  if (trml_wp) P.trml_wp = *trml_wp;
  if (trml_tool) P.trml_tool = *trml_tool;
  P.fric_heat = P.trml_wp.eta != 0. ? 1 : 0;         // actions_gpu.cu:457-460
  P.thermal_bc = P.trml_tool.alpha != 0. ? 1 : 0;    // actions_gpu.cu:466-468
  P.thermal_wp = P.trml_wp.alpha != 0. ? 1 : 0;      // interactions_gpu.cu:443
  P.thermal_tool_on = P.trml_tool.alpha != 0. ? 1 : 0; // interactions_gpu.cu:453
  ctx->has_constants = true;
  drop_graphs(ctx);
  return MF_OK;
}

int mf_get_constants(const mf_ctx *ctx, mf_phys_constants *phys, mf_corr_constants *corr, mf_joco_constants *joco,
                     mf_trml_constants *trml_wp, mf_trml_constants *trml_tool, int *has_joco) {
  if (!ctx) return MF_ERR_INVALID;
  if (!ctx->has_constants) return MF_ERR_STATE;
  const params &P = ctx->P;
  if (phys) *phys = P.phys;
  if (corr) *corr = P.corr;
  if (joco) *joco = P.joco;
  if (trml_wp) *trml_wp = P.trml_wp;
  if (trml_tool) *trml_tool = P.trml_tool;
  if (has_joco) *has_joco = P.plastic;
  return MF_OK;
}

int mf_set_options(mf_ctx *ctx, int thermal_solver, int jc_model, int precision) {
  if (!ctx) return MF_ERR_INVALID;
  if (thermal_solver != MF_THERMAL_BROOKSHAW && thermal_solver != MF_THERMAL_PSE) return MF_ERR_INVALID;
  if (jc_model != MF_JC_JOHNSON_COOK && jc_model != MF_JC_TANH) return MF_ERR_INVALID;
  if (precision != MF_PRECISION_FP64 && precision != MF_PRECISION_MIXED) return MF_ERR_INVALID;
  ctx->P.thermal_solver = thermal_solver;
  ctx->P.jc_model = jc_model;
  ctx->P.precision = precision;
  drop_graphs(ctx);
  return MF_OK;
}

int mf_set_dt(mf_ctx *ctx, double dt) {
  if (!ctx || !(dt > 0.) || !std::isfinite(dt)) return MF_ERR_INVALID;
  if (ctx->P.dt == dt) return MF_OK;  // nothing captured goes stale (the C++ mirror sets it every step)
  ctx->P.dt = dt;
  drop_graphs(ctx);
  return MF_OK;
}

int mf_tool_set(mf_ctx *ctx, const mf_tool_state *tool) {
  if (!ctx) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  mf_tool_state t;
  std::memset(&t, 0, sizeof(t));
  if (tool) {
    if (tool->num_seg < 0 || tool->num_seg > 5 || tool->num_seg == 1 || tool->num_seg == 2 || tool->num_seg == 3)
      if (tool->num_seg != 0) return MF_ERR_INVALID;
    t = *tool;
  }
  ctx->tool = t;
  ctx->P.has_tool = t.num_seg > 0 ? 1 : 0;
  CK(cudaMemcpy(ctx->tool_buf[ctx->cur], &t, sizeof(t), cudaMemcpyHostToDevice));
  drop_graphs(ctx);
  return MF_OK;
}

int mf_tool_get(mf_ctx *ctx, mf_tool_state *tool) {
  if (!ctx || !tool) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  // during a staged step the tool advances in stage 3 (tool_gpu_update_tool after the
  // plasticity, leap_frog.cu:142-145): until then this is the tool at the start of the step
  CK(cudaMemcpy(tool, ctx->tool_buf[ctx->cur], sizeof(*tool), cudaMemcpyDeviceToHost));
  return MF_OK;
}

int mf_step(mf_ctx *ctx, int n_steps) {
  nvtx_range range("mf_step");
  if (!ctx || n_steps < 0) return MF_ERR_INVALID;
  if (!ready(ctx)) return MF_ERR_STATE;
  if (!(ctx->P.dt > 0.) || ctx->mid_step) return MF_ERR_STATE;
  TRY(set_device(ctx));
  ctx->P.N = ctx->N;
  const bool graphs = !(ctx->flags & MF_OPT_NO_GRAPHS);
  if (graphs && !ctx->graph_valid) TRY(build_graphs(ctx));
  if (n_steps > 0) ctx->last_staged = false;
  if (n_steps > 0) TRY(prime_counts(ctx));
  for (int k = 0; k < n_steps; ++k) {
    if (graphs) {
      CK(cudaGraphLaunch(ctx->graph[ctx->cur], ctx->stream));
    } else {
      TRY(launch_step(ctx));
    }
    ctx->cur ^= 1;
    ctx->steps++;
  }
  return MF_OK;
}

int mf_step_timed(mf_ctx *ctx, float *stage_ms) {
  if (!ctx || !stage_ms) return MF_ERR_INVALID;
  if (!ready(ctx)) return MF_ERR_STATE;
  if (!(ctx->P.dt > 0.) || ctx->mid_step) return MF_ERR_STATE;
  TRY(set_device(ctx));
  ctx->P.N = ctx->N;
  ctx->last_staged = false;
  TRY(prime_counts(ctx));
  cudaEvent_t ev[5] = {};
  int rc = MF_OK;
  for (int k = 0; k < 5 && rc == MF_OK; ++k)
    if (cudaEventCreate(&ev[k]) != cudaSuccess) rc = MF_ERR_CUDA;
  for (int s = 0; s < 4 && rc == MF_OK; ++s) {
    if (cudaEventRecord(ev[s], ctx->stream) != cudaSuccess) rc = MF_ERR_CUDA;
    if (rc == MF_OK) rc = launch_stage(ctx, s);
  }
  if (rc == MF_OK && cudaEventRecord(ev[4], ctx->stream) != cudaSuccess) rc = MF_ERR_CUDA;
  if (rc == MF_OK && cudaEventSynchronize(ev[4]) != cudaSuccess) rc = MF_ERR_CUDA;
  for (int s = 0; s < 4 && rc == MF_OK; ++s)
    if (cudaEventElapsedTime(&stage_ms[s], ev[s], ev[s + 1]) != cudaSuccess) rc = MF_ERR_CUDA;
  for (int k = 0; k < 5; ++k)
    if (ev[k]) cudaEventDestroy(ev[k]);
  if (rc == MF_ERR_CUDA) ctx->last_cuda_err = (int)cudaGetLastError();
  if (rc != MF_OK) return rc;
  ctx->cur ^= 1;
  ctx->steps++;
  return MF_OK;
}

namespace {

// K steps of the context captured into a graph (the cell counts must be primed); the
// context's parity is restored afterwards, so K even gives a replayable graph
int capture_steps(mf_ctx *ctx, int K, cudaGraph_t *out) {
  const int saved = ctx->cur;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int rc = MF_OK;
  for (int k = 0; k < K && rc == MF_OK; ++k) {
    rc = launch_step(ctx);
    ctx->cur ^= 1;
  }
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  ctx->cur = saved;
  if (rc != MF_OK || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) ctx->last_cuda_err = (int)e;
    return rc != MF_OK ? rc : MF_ERR_CUDA;
  }
  *out = g;
  return MF_OK;
}

int step_checks(mf_ctx *ctx) {
  if (!ready(ctx)) return MF_ERR_STATE;
  if (!(ctx->P.dt > 0.) || ctx->mid_step) return MF_ERR_STATE;
  return MF_OK;
}

}  // namespace

int mf_graph_capture(mf_ctx *ctx, int n_steps, void **graph) {
  if (!ctx || !graph || n_steps < 2 || (n_steps & 1)) return MF_ERR_INVALID;
  TRY(step_checks(ctx));
  TRY(set_device(ctx));
  ctx->P.N = ctx->N;
  ctx->last_staged = false;
  TRY(prime_counts(ctx));
  cudaGraph_t g = nullptr;
  TRY(capture_steps(ctx, n_steps, &g));
  *graph = (void *)g;
  return MF_OK;
}

int mf_graph_destroy(void *graph) {
  if (!graph) return MF_ERR_INVALID;
  return cudaGraphDestroy((cudaGraph_t)graph) == cudaSuccess ? MF_OK : MF_ERR_CUDA;
}

// ---- batched form: many contexts advanced by one graph launch ----
struct mf_batch {
  int device = 0;
  std::vector<mf_ctx *> ctx;
  std::vector<unsigned long long> gen;
  std::vector<cudaEvent_t> ev;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  int K = 0;
  // batched kernels: one launch per step phase for all systems (else one child graph per system)
  bool fused = false;
  int pair_bs = PAIR_BLOCK;          // block size of the batched pair kernel (tuned)
  batch_entry *d_entries = nullptr;  // [2][n]: every system bound to each parity of its buffers
  int *d_first = nullptr;            // 4 maps of n + 1 first blocks: scan, 256-thread phases, pair, plastic
  int grid[4] = {0, 0, 0, 0};
  // MF_BATCH_PERSISTENT: K steps in one cooperative launch of persist_bps blocks per SM
  int form = MF_BATCH_PHASES;
  int persist_bps = 0;           // 0: as many as are resident
  unsigned long long *d_bar = nullptr;  // the persistent kernel's barrier word
  double wait_s = 2.0;           // limit of one barrier wait
  int persist_used = 0;          // blocks per SM of the built persistent launch
};

namespace {

void batch_release(mf_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
}

// The batched kernels serve systems whose steps run the same kernel variants: locked grids,
// steps launched whole (not staged), no neighbour lists or contact conductance, one precision,
// heat solver, yield law and plasticity setting. Anything else keeps the child-graph batch.
bool batch_can_fuse(mf_batch *b) {
  const params &P0 = b->ctx[0]->P;
  for (mf_ctx *c : b->ctx) {
    set_list_mode(c);
    const params &P = c->P;
    if (!fused_step(c) || P.verlet || P.fuse || P.h_contact > 0. || P.precision != P0.precision ||
        P.thermal_solver != P0.thermal_solver || P.jc_model != P0.jc_model || P.plastic != P0.plastic ||
        (P.thermal_solver == MF_THERMAL_PSE && (P.thermal_wp != 0) != (P0.thermal_wp != 0)))
      return false;
  }
  return true;
}

extern "C++" {  // (this part of the file lies inside the C ABI's extern "C" block)
template <typename... KArgs, typename... Args>
int batch_kernel(mf_batch *b, void (*kernel)(KArgs...), int grid, int block, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = MF_USE_PDL ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...) == cudaSuccess ? MF_OK : MF_ERR_CUDA;
}

// the pair phase (and PSE) of one step at the tuned block size
template <int BS>
int batch_pair(mf_batch *b, const params &P0, batch_map m) {
  const bool mixed = P0.precision == MF_PRECISION_MIXED;
  if (mixed) TRY(batch_kernel(b, kb_pair_mixed<BS>, b->grid[2], BS, m));
  else TRY(batch_kernel(b, kb_pair_fp64<BS>, b->grid[2], BS, m));
  if (P0.thermal_solver == MF_THERMAL_PSE && P0.thermal_wp) {
    if (mixed) TRY(batch_kernel(b, kb_pse_mixed<BS>, b->grid[2], BS, m));
    else TRY(batch_kernel(b, kb_pse<BS>, b->grid[2], BS, m));
  }
  return MF_OK;
}
}  // extern "C++"

// Entries and block maps of every system, then K steps captured as one graph: per step one
// launch per phase for all systems (scan, scatter, reorder + predictor, pair sums, finish,
// return map), each launched as the single-system step launches it (programmatic dependent
// launch), the systems bound to the parity of their buffers at that step.
int batch_build_fused(mf_batch *b, int K) {
  batch_release(b);
  const int n = (int)b->ctx.size();
  std::vector<batch_entry> e(2 * (size_t)n);
  std::vector<int> first(4 * (size_t)(n + 1), 0);
  long long total_n = 0;
  for (mf_ctx *c : b->ctx) total_n += c->N;
  const int sms = b->ctx[0]->sm_count;
  for (int k = 0; k < n; ++k) {
    mf_ctx *c = b->ctx[k];
    c->P.N = c->N;
    c->last_staged = false;
    TRY(prime_counts(c));
    const int saved = c->cur;
    for (int par = 0; par < 2; ++par) {
      c->cur = (saved + par) & 1;
      bind_sets(c);
      batch_entry &x = e[(size_t)par * n + k];
      std::memset(&x, 0, sizeof(x));
      x.P = c->P;
      x.D = c->D;
      x.scan_tiles = c->scan_tiles;
    }
    c->cur = saved;
    bind_sets(c);
    const int pair_bs = b->form == MF_BATCH_PERSISTENT ? PERSIST_BLOCK : b->pair_bs;
    const int blocks[4] = {c->scan_tiles, (c->N + BLOCK - 1) / BLOCK, (c->N + pair_bs - 1) / pair_bs,
                           (int)std::max<long long>(1, (long long)sms * PLASTIC_BLOCKS_PER_SM * c->N / total_n)};
    for (int m = 0; m < 4; ++m) first[(size_t)m * (n + 1) + k + 1] = first[(size_t)m * (n + 1) + k] + blocks[m];
  }
  for (int m = 0; m < 4; ++m) b->grid[m] = first[(size_t)m * (n + 1) + n];
  if (!b->d_entries) {
    if (cudaMalloc(&b->d_entries, sizeof(batch_entry) * e.size()) != cudaSuccess) return MF_ERR_NOMEM;
    if (cudaMalloc(&b->d_first, sizeof(int) * first.size()) != cudaSuccess) return MF_ERR_NOMEM;
  }
  if (cudaMemcpyAsync(b->d_entries, e.data(), sizeof(batch_entry) * e.size(), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(b->d_first, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return MF_ERR_CUDA;
  const params &P0 = b->ctx[0]->P;
  const bool mixed = P0.precision == MF_PRECISION_MIXED;
  persist_args A = {};
  int pgrid = 0;
  if (b->form == MF_BATCH_PERSISTENT) {
    int resident = 0;
    if (!mixed) return MF_ERR_INVALID;
    if (persist_blocks_per_sm(&resident) != 0) return MF_ERR_CUDA;
    const int bps = b->persist_bps > 0 ? std::min(b->persist_bps, resident) : resident;
    if (bps < 1) return MF_ERR_CUDA;
    pgrid = bps * sms;
    b->persist_used = bps;
    if (!b->d_bar && cudaMalloc(&b->d_bar, sizeof(unsigned long long)) != cudaSuccess) return MF_ERR_NOMEM;
    A.e = b->d_entries;
    A.first = b->d_first;
    A.n = n;
    A.K = K;
    for (int m = 0; m < 4; ++m) A.grid[m] = b->grid[m];
    A.pse = P0.thermal_solver == MF_THERMAL_PSE && P0.thermal_wp ? 1 : 0;
    A.plastic = P0.plastic ? 1 : 0;
    A.paired = P0.jc_model == MF_JC_TANH ? 0 : 1;
    A.bar = b->d_bar;
    A.wait_ns = (unsigned long long)(b->wait_s * 1e9);
  }
  if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return MF_ERR_CUDA;
  int rc = MF_OK;
  if (b->form == MF_BATCH_PERSISTENT) {  // the barrier word starts at zero in every launch
    if (cudaMemsetAsync(b->d_bar, 0, sizeof(unsigned long long), b->stream) != cudaSuccess ||
        persist_launch(b->stream, pgrid, A) != 0)
      rc = MF_ERR_CUDA;
  }
  for (int st = 0; st < K && rc == MF_OK && b->form != MF_BATCH_PERSISTENT; ++st) {
    const batch_entry *ent = b->d_entries + (size_t)(st & 1) * n;
    const batch_map m_scan{ent, b->d_first, n}, m_256{ent, b->d_first + (n + 1), n},
        m_pair{ent, b->d_first + 2 * (n + 1), n}, m_pl{ent, b->d_first + 3 * (n + 1), n};
    rc = batch_kernel(b, kb_scan, b->grid[0], SCAN_THREADS, m_scan);
    if (rc == MF_OK) rc = batch_kernel(b, kb_scatter, b->grid[1], BLOCK, m_256);
    if (rc == MF_OK) rc = mixed ? batch_kernel(b, kb_reorder<true>, b->grid[1], BLOCK, m_256)
                                : batch_kernel(b, kb_reorder<false>, b->grid[1], BLOCK, m_256);
    if (rc == MF_OK) {
      switch (b->pair_bs) {
        case 64: rc = batch_pair<64>(b, P0, m_pair); break;
        case 256: rc = batch_pair<256>(b, P0, m_pair); break;
        default: rc = batch_pair<128>(b, P0, m_pair); break;
      }
    }
    if (rc == MF_OK) rc = batch_kernel(b, kb_finish, b->grid[1], FINISH_BLOCK, m_256);
    if (rc == MF_OK && P0.plastic)
      rc = P0.jc_model == MF_JC_TANH ? batch_kernel(b, kb_plastic<false>, b->grid[3], BLOCK, m_pl)
                                     : batch_kernel(b, kb_plastic<true>, b->grid[3], BLOCK, m_pl);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
  if (rc != MF_OK || ec != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return rc != MF_OK ? rc : MF_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(&b->exec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return MF_ERR_CUDA;
  for (int k = 0; k < n; ++k) b->gen[k] = b->ctx[k]->gen;
  b->K = K;
  return MF_OK;
}

// one parent graph: a child graph of K steps per context, no edges between them (or, where
// the systems allow it, the batched kernels)
int batch_build(mf_batch *b, int K) {
  if (b->fused) return batch_build_fused(b, K);
  batch_release(b);
  cudaGraph_t parent = nullptr;
  cudaError_t e = cudaGraphCreate(&parent, 0);
  if (e != cudaSuccess) return MF_ERR_CUDA;
  int rc = MF_OK;
  for (size_t i = 0; i < b->ctx.size() && rc == MF_OK; ++i) {
    mf_ctx *c = b->ctx[i];
    c->P.N = c->N;
    c->last_staged = false;
    rc = prime_counts(c);
    cudaGraph_t child = nullptr;
    if (rc == MF_OK) rc = capture_steps(c, K, &child);
    if (rc == MF_OK) {
      cudaGraphNode_t node;
      if (cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, child) != cudaSuccess) rc = MF_ERR_CUDA;
      cudaGraphDestroy(child);
    }
    b->gen[i] = c->gen;
  }
  if (rc == MF_OK && cudaGraphInstantiate(&b->exec, parent, 0) != cudaSuccess) rc = MF_ERR_CUDA;
  cudaGraphDestroy(parent);
  if (rc == MF_OK) b->K = K;
  return rc;
}

// the batch stream waits for every context's stream, or every context's stream for the batch
int batch_order(mf_batch *b, bool into_batch) {
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    mf_ctx *c = b->ctx[i];
    cudaStream_t from = into_batch ? c->stream : b->stream, to = into_batch ? b->stream : c->stream;
    if (cudaEventRecord(b->ev[i], from) != cudaSuccess || cudaStreamWaitEvent(to, b->ev[i], 0) != cudaSuccess)
      return MF_ERR_CUDA;
  }
  return MF_OK;
}

int batch_launch(mf_batch *b, int n) {
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    mf_ctx *c = b->ctx[i];
    if (c->gen != b->gen[i] || step_checks(c) != MF_OK) return MF_ERR_STATE;  // rebuild the batch
    c->P.N = c->N;
    TRY(prime_counts(c));  // counts discarded by a host write since the last launch
  }
  TRY(batch_order(b, true));
  for (int k = 0; k < n; ++k)
    if (cudaGraphLaunch(b->exec, b->stream) != cudaSuccess) return MF_ERR_CUDA;
  TRY(batch_order(b, false));
  for (mf_ctx *c : b->ctx) {
    c->steps += (long long)b->K * n;
    c->last_staged = false;
  }
  return MF_OK;
}

}  // namespace

int mf_batch_create(mf_ctx **ctxs, int n, int steps_per_launch, mf_batch **out) {
  if (!ctxs || n < 1 || !out || steps_per_launch < 0 || (steps_per_launch & 1)) return MF_ERR_INVALID;
  mf_batch *b = new (std::nothrow) mf_batch;
  if (!b) return MF_ERR_NOMEM;
  b->device = ctxs[0] ? ctxs[0]->device : 0;
  int rc = MF_OK;
  for (int i = 0; i < n && rc == MF_OK; ++i) {
    mf_ctx *c = ctxs[i];
    if (!c || c->device != b->device) rc = MF_ERR_INVALID;
    else if (step_checks(c) != MF_OK) rc = MF_ERR_STATE;
    for (int j = 0; j < i && rc == MF_OK; ++j)
      if (ctxs[j] == c) rc = MF_ERR_INVALID;  // one instance once
    if (rc == MF_OK) {
      b->ctx.push_back(c);
      b->gen.push_back(0);
      cudaEvent_t ev = nullptr;
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) rc = MF_ERR_CUDA;
      b->ev.push_back(ev);
    }
  }
  if (rc == MF_OK && cudaSetDevice(b->device) != cudaSuccess) rc = MF_ERR_CUDA;
  if (rc == MF_OK && cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) rc = MF_ERR_CUDA;
  if (rc == MF_OK) b->fused = batch_can_fuse(b);
  if (rc == MF_OK && steps_per_launch > 0) rc = batch_build(b, steps_per_launch);
  if (rc == MF_OK && steps_per_launch == 0) {
    // autotune over a few real launches (which advance the instances): with the batched
    // kernels first the pair kernel's block size at 4 steps per launch, then the steps per
    // launch; the highest measured throughput wins
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = MF_ERR_CUDA;
    auto measure = [&](int K, double *steps_per_ms) {
      int r = batch_build(b, K);
      if (r == MF_OK) r = batch_launch(b, 1);  // warm-up
      if (r == MF_OK && cudaEventRecord(e0, b->stream) != cudaSuccess) r = MF_ERR_CUDA;
      if (r == MF_OK) r = batch_launch(b, 2);
      if (r == MF_OK && cudaEventRecord(e1, b->stream) != cudaSuccess) r = MF_ERR_CUDA;
      float ms = 0.f;
      if (r == MF_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        r = MF_ERR_CUDA;
      *steps_per_ms = 2.0 * K / (ms > 0.f ? ms : 1e-6f);
      return r;
    };
    if (rc == MF_OK && b->fused) {
      const int bs_cand[3] = {64, 128, 256};
      double best = -1.;
      int best_bs = PAIR_BLOCK;
      for (int ci = 0; ci < 3 && rc == MF_OK; ++ci) {
        b->pair_bs = bs_cand[ci];
        double v = 0.;
        rc = measure(4, &v);
        if (rc == MF_OK && v > best) { best = v; best_bs = bs_cand[ci]; }
      }
      b->pair_bs = best_bs;
    }
    const int cand[4] = {2, 4, 8, 16};
    double best = -1.;
    int best_k = 2;
    for (int ci = 0; ci < 4 && rc == MF_OK; ++ci) {
      double v = 0.;
      rc = measure(cand[ci], &v);
      if (rc == MF_OK && v > best) { best = v; best_k = cand[ci]; }
    }
    if (rc == MF_OK && b->fused && b->ctx[0]->P.precision == MF_PRECISION_MIXED) {
      // then the persistent kernel (one launch per K steps) at 1 and 2 blocks per SM and 4 or
      // 16 steps per launch; it replaces the per-phase launches where it measures faster
      int resident = 0;
      if (persist_blocks_per_sm(&resident) != 0) resident = 0;
      int best_bps = 0, best_pk = 0;
      for (int bps = 1; bps <= std::min(resident, 2) && rc == MF_OK; ++bps) {
        for (int pk : {4, 16}) {
          b->form = MF_BATCH_PERSISTENT;
          b->persist_bps = bps;
          double v = 0.;
          const int r = measure(pk, &v);
          if (r == MF_ERR_CUDA) {  // (a launch form the device refuses: kept out)
            cudaGetLastError();
            continue;
          }
          rc = r;
          if (rc == MF_OK && v > best) { best = v; best_bps = bps; best_pk = pk; }
        }
      }
      b->form = best_bps ? MF_BATCH_PERSISTENT : MF_BATCH_PHASES;
      b->persist_bps = best_bps;
      if (best_bps) best_k = best_pk;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc == MF_OK) rc = batch_build(b, best_k);
  }
  if (rc != MF_OK) {
    mf_batch_destroy(b);
    return rc;
  }
  *out = b;
  return MF_OK;
}

int mf_batch_steps_per_launch(const mf_batch *b, int *k) {
  if (!b || !k) return MF_ERR_INVALID;
  *k = b->K;
  return MF_OK;
}

int mf_batch_config(const mf_batch *b, int *fused, int *pair_block, int *steps_per_launch) {
  if (!b) return MF_ERR_INVALID;
  if (fused) *fused = b->fused ? 1 : 0;
  if (pair_block) *pair_block = b->fused ? b->pair_bs : PAIR_BLOCK;
  if (steps_per_launch) *steps_per_launch = b->K;
  return MF_OK;
}

int mf_batch_set_form(mf_batch *b, int form, int blocks_per_sm, int steps_per_launch) {
  if (!b || (form != MF_BATCH_PHASES && form != MF_BATCH_PERSISTENT) || blocks_per_sm < 0 || steps_per_launch < 2 ||
      (steps_per_launch & 1))
    return MF_ERR_INVALID;
  // child-graph batches have no phases; the persistent kernel steps the mixed form only
  if (form == MF_BATCH_PERSISTENT && (!b->fused || b->ctx[0]->P.precision != MF_PRECISION_MIXED))
    return MF_ERR_INVALID;
  if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamSynchronize(b->stream) != cudaSuccess) return MF_ERR_CUDA;
  b->form = form;
  b->persist_bps = blocks_per_sm;
  return batch_build(b, steps_per_launch);
}

int mf_batch_form(const mf_batch *b, int *form, int *blocks_per_sm) {
  if (!b) return MF_ERR_INVALID;
  if (form) *form = b->form;
  if (blocks_per_sm) *blocks_per_sm = b->form == MF_BATCH_PERSISTENT ? b->persist_used : 0;
  return MF_OK;
}

int mf_batch_set_wait_limit(mf_batch *b, double seconds) {
  if (!b || !(seconds >= 0.) || seconds > 3600.) return MF_ERR_INVALID;
  b->wait_s = seconds;
  if (!b->exec) return MF_OK;
  if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamSynchronize(b->stream) != cudaSuccess) return MF_ERR_CUDA;
  return batch_build(b, b->K);  // the limit is an argument of the captured launch
}

int mf_batch_step(mf_batch *b, int n_launches) {
  nvtx_range range("mf_batch_step");
  if (!b || n_launches < 0) return MF_ERR_INVALID;
  if (!b->exec) return MF_ERR_STATE;
  if (cudaSetDevice(b->device) != cudaSuccess) return MF_ERR_CUDA;
  return batch_launch(b, n_launches);
}

int mf_batch_destroy(mf_batch *b) {
  if (!b) return MF_ERR_INVALID;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_release(b);
  if (b->d_entries) cudaFree(b->d_entries);
  if (b->d_first) cudaFree(b->d_first);
  if (b->d_bar) cudaFree(b->d_bar);
  for (cudaEvent_t e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return MF_OK;
}

int mf_step_stage(mf_ctx *ctx, int stage) {
  if (!ctx || stage < 0 || stage > 3) return MF_ERR_INVALID;
  if (!ready(ctx)) return MF_ERR_STATE;
  TRY(set_device(ctx));
  ctx->P.N = ctx->N;
  // stages 1..2 leave the half-built step in the other buffer; reads during the step see it
  if (stage == 0 && ctx->mid_step) return MF_ERR_STATE;
  if (stage == 0) TRY(invalidate_counts(ctx));
  ctx->P.staged = 1;
  int rc_stage = launch_stage(ctx, stage);
  ctx->P.staged = 0;
  TRY(rc_stage);
  if (stage == 1) { ctx->mid_step = true; ctx->last_staged = true; }
  if (stage == 3) {
    ctx->cur ^= 1;
    ctx->steps++;
    ctx->mid_step = false;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_report_force(mf_ctx *ctx, double out[2]) {
  if (!ctx || !out) return MF_ERR_INVALID;
  if (!ctx->has_particles) return MF_ERR_STATE;
  TRY(set_device(ctx));
  state_set &s = ctx->set[ctx->cur];
  k_force_only<<<1, BLOCK, 0, ctx->stream>>>(ctx->N, s.fc, s.ft, ctx->D);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, ctx->D.force_last, sizeof(double) * 2, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_force_last_async(mf_ctx *ctx, double *host_out2) {
  if (!ctx || !host_out2) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaMemcpyAsync(host_out2, ctx->D.force_last, sizeof(double) * 2, cudaMemcpyDeviceToHost, ctx->stream));
  return MF_OK;
}

int mf_force_log(mf_ctx *ctx, double *out, int max_entries, int *n_out) {
  if (!ctx || !n_out || max_entries < 0) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  dev_status st;
  CK(cudaMemcpy(&st, ctx->D.st, sizeof(st), cudaMemcpyDeviceToHost));
  unsigned long long head = st.force_log_head;
  unsigned long long first = ctx->force_read_head;
  if (head - first > (unsigned long long)FORCE_LOG_CAP) first = head - FORCE_LOG_CAP;
  unsigned long long n = head - first;
  if (n > (unsigned long long)max_entries) n = (unsigned long long)max_entries;
  if (n > 0 && out) {
    // at most two contiguous pieces of the ring
    unsigned long long done = 0;
    while (done < n) {
      unsigned long long slot = (first + done) % FORCE_LOG_CAP;
      unsigned long long len = std::min(n - done, (unsigned long long)FORCE_LOG_CAP - slot);
      CK(cudaMemcpy(out + 2 * done, ctx->D.force_log + 2 * slot, sizeof(double) * 2 * len, cudaMemcpyDeviceToHost));
      done += len;
    }
  }
  ctx->force_read_head = first + n;
  *n_out = (int)n;
  return MF_OK;
}

int mf_status_get(mf_ctx *ctx, mf_status *out) {
  if (!ctx || !out) return MF_ERR_INVALID;
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  dev_status st;
  CK(cudaMemcpy(&st, ctx->D.st, sizeof(st), cudaMemcpyDeviceToHost));
  out->steps = ctx->steps;
  out->blanked = 0;
  if (ctx->has_particles) {
    std::vector<unsigned> fl((size_t)ctx->N);
    CK(cudaMemcpy(fl.data(), ctx->set[ctx->cur].flags, sizeof(unsigned) * fl.size(), cudaMemcpyDeviceToHost));
    long long b = 0;
    for (unsigned f : fl) b += (f & FLAG_BLANKED) ? 1 : 0;
    out->blanked = b;
  }
  out->newly_blanked = (long long)(st.newly_blanked - ctx->status_newly_blanked_seen);
  ctx->status_newly_blanked_seen = st.newly_blanked;
  out->out_of_grid = (long long)st.out_of_grid;
  out->secant_cap_hits = (long long)st.secant_cap_hits;
  out->max_cell_occupancy = st.max_cell_occupancy;
  out->error_flags = st.error_flags;
  out->secant_iterations = (long long)st.secant_iterations;
  out->sorts = (long long)st.sorts;
  return MF_OK;
}

int mf_scene_upload(mf_ctx *ctx, const mf_scene *s, int grid_kind) {
  if (!ctx || !s) return MF_ERR_INVALID;
  TRY(mf_particles_create(ctx, s->N, s->pos, s->vel, s->rho, s->T, s->h, s->fixed, s->tool_p, nullptr));
  if (s->grid_max_cell > 0)
    TRY(mf_grid_create_adaptive(ctx, grid_kind, s->grid_max_cell));
  else
    TRY(mf_grid_create_locked(ctx, grid_kind, s->grid_bbmin[0], s->grid_bbmin[1], s->grid_bbmax[0],
                              s->grid_bbmax[1], s->grid_h));
  TRY(mf_set_constants(ctx, &s->phys, &s->corr, s->has_joco ? &s->joco : nullptr, &s->trml_wp, &s->trml_tool));
  TRY(mf_tool_set(ctx, &s->tool));
  TRY(mf_set_dt(ctx, s->dt));
  return MF_OK;
}

// vtk_writer_write(const particle_gpu*, int) (vtk_writer.cpp:20-178): the unblanked particles
}  // extern "C"

namespace {

// flag bit <-> 0/1 doubles, for the device-destination field access
__global__ void k_flag_to_double(int N, const unsigned *flags, unsigned bit, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) out[i] = (flags[i] & bit) ? 1. : 0.;
}
__global__ void k_double_to_flag(int N, const double *in, unsigned bit, unsigned *flags, unsigned *bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double v = in[i];
  if (!(v == 0. || v == 1.)) {
    atomicOr(bad, 1u);
    return;
  }
  flags[i] = v == 1. ? (flags[i] | bit) : (flags[i] & ~bit);
}

// the caller's stream waits for the context, or the context for the caller's stream
int order_streams(cudaStream_t from, cudaStream_t to) {
  if (from == to) return MF_OK;
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return MF_ERR_CUDA;
  cudaError_t r = cudaEventRecord(e, from);
  if (r == cudaSuccess) r = cudaStreamWaitEvent(to, e, 0);
  cudaEventDestroy(e);
  return r == cudaSuccess ? MF_OK : MF_ERR_CUDA;
}

int field_device_copy(mf_ctx *ctx, int field, void *dst_dev, const void *src_dev, cudaStream_t st, bool to_ctx) {
  const size_t N = (size_t)ctx->N;
  const unsigned bit = flag_bit(field);
  const int view = view_set(ctx);
  TRY(order_streams(ctx->stream, st));
  cudaError_t e = cudaSuccess;
  if (bit) {
    const int nb = (ctx->N + BLOCK - 1) / BLOCK;
    if (!to_ctx) {
      k_flag_to_double<<<nb, BLOCK, 0, st>>>(ctx->N, ctx->set[view].flags, bit, (double *)dst_dev);
    } else {
      unsigned *bad = nullptr;
      e = cudaMallocAsync(&bad, sizeof(unsigned), st);
      if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(unsigned), st);
      if (e == cudaSuccess)
        k_double_to_flag<<<nb, BLOCK, 0, st>>>(ctx->N, (const double *)src_dev, bit, ctx->set[view].flags, bad);
      unsigned hbad = 0;
      if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (bad) cudaFreeAsync(bad, st);
      if (e == cudaSuccess && hbad) return MF_ERR_INVALID;  // a value other than 0 or 1 (others kept)
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  } else {
    const field_desc d = describe(field);
    void *fp = field_ptr(ctx, field);
    if (!fp) return MF_ERR_INVALID;
    const size_t bytes = N * d.width * (d.is_int ? sizeof(int) : sizeof(double));
    e = to_ctx ? cudaMemcpyAsync(fp, src_dev, bytes, cudaMemcpyDeviceToDevice, st)
               : cudaMemcpyAsync(dst_dev, fp, bytes, cudaMemcpyDeviceToDevice, st);
  }
  if (e != cudaSuccess) {
    ctx->last_cuda_err = (int)e;
    return MF_ERR_CUDA;
  }
  return order_streams(st, ctx->stream);
}

// state file: tag, version, particle count, steps, tool, then per field (id, bytes, data),
// then an FNV-1a checksum of all the bytes before it
constexpr char STATE_TAG[8] = {'M', 'F', 'B', '2', 'S', 'T', 'A', 'T'};
constexpr int STATE_VERSION = 1;
constexpr int STATE_FIELDS[] = {MF_FIELD_POS, MF_FIELD_VEL, MF_FIELD_H, MF_FIELD_RHO, MF_FIELD_S, MF_FIELD_FC,
                                MF_FIELD_FT, MF_FIELD_N, MF_FIELD_FIXED, MF_FIELD_BLANKED, MF_FIELD_TOOL,
                                MF_FIELD_EPS_PL, MF_FIELD_EPS_PL_DOT, MF_FIELD_T, MF_FIELD_POS_T, MF_FIELD_VEL_T,
                                MF_FIELD_RHO_T, MF_FIELD_S_T, MF_FIELD_T_T, MF_FIELD_IDX, MF_FIELD_HASH, MF_FIELD_ID};

struct fnv1a {
  unsigned long long h = 1469598103934665603ull;
  void add(const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) {
      h ^= b[i];
      h *= 1099511628211ull;
    }
  }
};

}  // namespace

extern "C" {

int mf_get_field_device(mf_ctx *ctx, int field, void *device_dst, void *cuda_stream) {
  if (!ctx || !device_dst || field < 0 || field >= MF_NUM_FIELDS) return MF_ERR_INVALID;
  if (!ctx->has_particles) return MF_ERR_STATE;
  TRY(set_device(ctx));
  return field_device_copy(ctx, field, device_dst, nullptr, cuda_stream ? (cudaStream_t)cuda_stream : ctx->stream,
                           false);
}

int mf_set_field_device(mf_ctx *ctx, int field, const void *device_src, void *cuda_stream) {
  if (!ctx || !device_src || field < 0 || field >= MF_NUM_FIELDS) return MF_ERR_INVALID;
  if (!ctx->has_particles) return MF_ERR_STATE;
  if (field == MF_FIELD_R) return MF_ERR_INVALID;  // recomputed every step
  TRY(set_device(ctx));
  TRY(invalidate_counts(ctx));
  return field_device_copy(ctx, field, nullptr, device_src, cuda_stream ? (cudaStream_t)cuda_stream : ctx->stream,
                           true);
}

int mf_state_save(mf_ctx *ctx, const char *path) {
  if (!ctx || !path) return MF_ERR_INVALID;
  if (!ctx->has_particles || ctx->mid_step) return MF_ERR_STATE;
  std::vector<unsigned char> buf;
  auto put = [&](const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    buf.insert(buf.end(), b, b + n);
  };
  const int version = STATE_VERSION, N = ctx->N, nf = (int)(sizeof(STATE_FIELDS) / sizeof(int));
  const long long steps = ctx->steps;
  mf_tool_state tool{};
  TRY(mf_tool_get(ctx, &tool));
  put(STATE_TAG, 8);
  put(&version, sizeof(int));
  put(&N, sizeof(int));
  put(&nf, sizeof(int));
  put(&steps, sizeof(long long));
  put(&tool, sizeof(tool));
  std::vector<unsigned char> data;
  for (int k = 0; k < nf; ++k) {
    const int f = STATE_FIELDS[k];
    const field_desc d = describe(f);
    const long long bytes = (long long)N * d.width * (d.is_int ? sizeof(int) : sizeof(double));
    data.resize((size_t)bytes);
    TRY(mf_get_field(ctx, f, data.data()));
    put(&f, sizeof(int));
    put(&bytes, sizeof(long long));
    put(data.data(), (size_t)bytes);
  }
  fnv1a h;
  h.add(buf.data(), buf.size());
  put(&h.h, sizeof(h.h));
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return MF_ERR_IO;
  const bool ok = std::fwrite(buf.data(), 1, buf.size(), fp) == buf.size();
  if (std::fclose(fp) != 0 || !ok) return MF_ERR_IO;
  return MF_OK;
}

int mf_state_load(mf_ctx *ctx, const char *path) {
  if (!ctx || !path) return MF_ERR_INVALID;
  if (!ctx->has_particles || ctx->mid_step) return MF_ERR_STATE;
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return MF_ERR_IO;
  std::vector<unsigned char> buf;
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof(chunk), fp)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  const bool read_err = std::ferror(fp) != 0;
  std::fclose(fp);
  if (read_err) return MF_ERR_IO;
  // every check before any change to the context
  const size_t head = 8 + 3 * sizeof(int) + sizeof(long long) + sizeof(mf_tool_state);
  if (buf.size() < head + sizeof(unsigned long long)) return MF_ERR_CORRUPT;
  fnv1a h;
  h.add(buf.data(), buf.size() - sizeof(unsigned long long));
  unsigned long long stored;
  std::memcpy(&stored, buf.data() + buf.size() - sizeof(stored), sizeof(stored));
  if (stored != h.h || std::memcmp(buf.data(), STATE_TAG, 8) != 0) return MF_ERR_CORRUPT;
  size_t at = 8;
  auto get = [&](void *p, size_t n) {
    if (at + n > buf.size() - sizeof(unsigned long long)) return false;
    std::memcpy(p, buf.data() + at, n);
    at += n;
    return true;
  };
  int version = 0, N = 0, nf = 0;
  long long steps = 0;
  mf_tool_state tool{};
  if (!get(&version, sizeof(int)) || !get(&N, sizeof(int)) || !get(&nf, sizeof(int)) ||
      !get(&steps, sizeof(long long)) || !get(&tool, sizeof(tool)))
    return MF_ERR_CORRUPT;
  if (version != STATE_VERSION || N != ctx->N || nf != (int)(sizeof(STATE_FIELDS) / sizeof(int)))
    return MF_ERR_CORRUPT;
  std::vector<std::pair<int, size_t>> where;  // field, offset of its data
  for (int k = 0; k < nf; ++k) {
    int f = -1;
    long long bytes = -1;
    if (!get(&f, sizeof(int)) || !get(&bytes, sizeof(long long))) return MF_ERR_CORRUPT;
    if (f != STATE_FIELDS[k]) return MF_ERR_CORRUPT;
    const field_desc d = describe(f);
    if (bytes != (long long)N * d.width * (d.is_int ? sizeof(int) : sizeof(double))) return MF_ERR_CORRUPT;
    where.push_back({f, at});
    at += (size_t)bytes;
    if (at > buf.size() - sizeof(unsigned long long)) return MF_ERR_CORRUPT;
  }
  if (at != buf.size() - sizeof(unsigned long long)) return MF_ERR_CORRUPT;
  // apply
  for (const auto &w : where) TRY(mf_set_field(ctx, w.first, buf.data() + w.second));
  TRY(mf_tool_set(ctx, &tool));
  ctx->steps = steps;
  return MF_OK;
}

// tool_wear::eval_usui (tool_wear.cu:20-64) on the device
int mf_tool_wear_usui(mf_ctx *ctx, double K, double alpha, double out3[3]) {
  if (!ctx || !out3) return MF_ERR_INVALID;
  if (!ctx->has_particles || ctx->mid_step) return MF_ERR_STATE;
  TRY(set_device(ctx));
  double *d_out = nullptr;
  CK(cudaMalloc(&d_out, 3 * sizeof(double)));
  const state_set &S = ctx->set[ctx->cur];
  const int blocks = std::max(1, std::min((ctx->N + BLOCK - 1) / BLOCK, ctx->bbox_blocks));
  k_usui<<<blocks, BLOCK, 0, ctx->stream>>>(ctx->N, S, ctx->D, ctx->tool_buf[ctx->cur], K, alpha, d_out);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out3, d_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_out);
  if (e != cudaSuccess) { ctx->last_cuda_err = (int)e; return MF_ERR_CUDA; }
  return MF_OK;
}

}  // extern "C"

namespace {

// vtk_writer_write(const particle_gpu*, int) (vtk_writer.cpp:20-178): legacy ASCII, the
// unblanked particles, "%f" values; fields in array order
int write_vtk_particles(const char *path, int n, const double *pos, const double *vel, const double *rho,
                        const double *p, const double *T, const double *eps, const double *S,
                        const unsigned *flags) {
  FILE *fp = std::fopen(path, "w+");
  if (!fp) return MF_ERR_INVALID;
  auto live = [&](int i) { return !(flags[i] & FLAG_BLANKED); };
  int m = 0;
  for (int i = 0; i < n; ++i) m += live(i);
  std::fprintf(fp, "# vtk DataFile Version 2.0\nmfree iwf\nASCII\n\nDATASET UNSTRUCTURED_GRID\n");
  std::fprintf(fp, "POINTS %d float\n", m);
  for (int i = 0; i < n; ++i) if (live(i)) std::fprintf(fp, "%f %f %f\n", pos[2 * i], pos[2 * i + 1], 0.);
  std::fprintf(fp, "\nCELLS %d %d\n", m, 2 * m);
  for (int i = 0; i < n; ++i) if (live(i)) std::fprintf(fp, "%d %d\n", 1, i);
  std::fprintf(fp, "\nCELL_TYPES %d\n", m);
  for (int i = 0; i < n; ++i) if (live(i)) std::fprintf(fp, "%d\n", 1);
  std::fprintf(fp, "\nPOINT_DATA %d\n", m);
  auto scalars = [&](const char *name, auto value) {
    std::fprintf(fp, "SCALARS %s float 1\nLOOKUP_TABLE default\n", name);
    for (int i = 0; i < n; ++i) if (live(i)) std::fprintf(fp, "%f\n", value(i));
    std::fprintf(fp, "\n");
  };
  scalars("density", [&](int i) { return rho[i]; });
  scalars("Temperature", [&](int i) { return T[i]; });
  scalars("Fixed", [&](int i) { return (flags[i] & FLAG_FIXED) ? 1. : 0.; });
  scalars("Tool", [&](int i) { return (flags[i] & FLAG_TOOL) ? 1. : 0.; });
  scalars("EquivAccumPlasticStrain", [&](int i) { return eps[i]; });
  std::fprintf(fp, "VECTORS Velocity float\n");
  for (int i = 0; i < n; ++i) if (live(i)) std::fprintf(fp, "%f %f %f\n", vel[2 * i], vel[2 * i + 1], 0.);
  std::fprintf(fp, "\nSCALARS SvM float 1\nLOOKUP_TABLE default\n");
  for (int i = 0; i < n; ++i) {
    if (!live(i)) continue;
    double cxx = S[4 * i] - p[i], cyy = S[4 * i + 2] - p[i], czz = S[4 * i + 3] - p[i], cxy = S[4 * i + 1];
    double svm2 = (cxx * cxx + cyy * cyy + czz * czz) - cxx * cyy - cxx * czz - cyy * czz + 3.0 * cxy * cxy;
    std::fprintf(fp, "%f\n", svm2 > 0 ? std::sqrt(svm2) : 0.);
  }
  std::fprintf(fp, "\n");
  return std::fclose(fp) == 0 ? MF_OK : MF_ERR_INVALID;
}

// the fields of a dump, in snapshot order
struct vtk_src {
  const void *ptr;
  size_t doubles;  // per particle
};

}  // namespace

extern "C" {

int mf_vtk_write_particle_arrays(const char *path, int n, const double *pos, const double *vel, const double *rho,
                                 const double *p, const double *T, const double *eps_pl, const double *S,
                                 const double *fixed, const double *blanked, const double *tool_p) {
  if (!path || n < 0 || !pos || !vel || !rho || !p || !T || !eps_pl || !S || !fixed || !blanked || !tool_p)
    return MF_ERR_INVALID;
  std::vector<unsigned> flags((size_t)n);
  for (int i = 0; i < n; ++i)
    flags[i] = (fixed[i] == 1. ? FLAG_FIXED : 0u) | (blanked[i] == 1. ? FLAG_BLANKED : 0u) |
               (tool_p[i] == 1. ? FLAG_TOOL : 0u);
  return write_vtk_particles(path, n, pos, vel, rho, p, T, eps_pl, S, flags.data());
}

int mf_vtk_write_particles(mf_ctx *ctx, const char *path) {
  if (!ctx || !path) return MF_ERR_INVALID;
  if (!ctx->has_particles) return MF_ERR_STATE;
  const int n = ctx->N;
  std::vector<double> pos(2 * (size_t)n), vel(2 * (size_t)n), rho(n), p(n), T(n), eps(n), S(4 * (size_t)n);
  std::vector<unsigned> flags(n);
  TRY(mf_get_field(ctx, MF_FIELD_POS, pos.data()));
  TRY(mf_get_field(ctx, MF_FIELD_VEL, vel.data()));
  TRY(mf_get_field(ctx, MF_FIELD_RHO, rho.data()));
  TRY(mf_get_field(ctx, MF_FIELD_P, p.data()));
  TRY(mf_get_field(ctx, MF_FIELD_T, T.data()));
  TRY(mf_get_field(ctx, MF_FIELD_EPS_PL, eps.data()));
  TRY(mf_get_field(ctx, MF_FIELD_S, S.data()));
  CK(cudaMemcpy(flags.data(), ctx->set[view_set(ctx)].flags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost));
  return write_vtk_particles(path, n, pos.data(), vel.data(), rho.data(), p.data(), T.data(), eps.data(), S.data(),
                             flags.data());
}

int mf_vtk_flush(mf_ctx *ctx) {
  if (!ctx) return MF_ERR_INVALID;
  int rc = MF_OK;
  for (auto &j : ctx->vtk_jobs) {
    if (j->writer.joinable()) j->writer.join();
    if (j->rc != MF_OK && rc == MF_OK) rc = j->rc;
    if (j->snap) cudaEventDestroy(j->snap);
    if (j->landed) cudaEventDestroy(j->landed);
    if (j->dev) cudaFree(j->dev);
    if (j->dev_flags) cudaFree(j->dev_flags);
    if (j->host) cudaFreeHost(j->host);
    if (j->host_flags) cudaFreeHost(j->host_flags);
  }
  ctx->vtk_jobs.clear();
  return rc;
}

// the same file as mf_vtk_write_particles, written while the steps go on: the fields are
// copied inside the device (stream-ordered after the last step), brought to pinned host
// memory on a side stream, and written by a host thread; mf_vtk_flush waits for all dumps
int mf_vtk_write_particles_async(mf_ctx *ctx, const char *path) {
  if (!ctx || !path) return MF_ERR_INVALID;
  if (!ctx->has_particles || ctx->mid_step) return MF_ERR_STATE;
  TRY(set_device(ctx));
  if (!ctx->io_stream) CK(cudaStreamCreateWithFlags(&ctx->io_stream, cudaStreamNonBlocking));
  const int n = ctx->N;
  const state_set &s = ctx->set[ctx->cur];
  const vtk_src src[7] = {{s.pos, 2}, {s.vel, 2}, {s.rho, 1}, {s.pp, 1}, {s.T, 1}, {s.eps_pl, 1}, {s.S, 4}};
  const size_t per = 12;  // doubles per particle in the snapshot
  std::unique_ptr<vtk_job> j(new (std::nothrow) vtk_job);
  if (!j) return MF_ERR_NOMEM;
  j->n = n;
  cudaError_t e = cudaMalloc(&j->dev, sizeof(double) * per * n);
  if (e == cudaSuccess) e = cudaMalloc(&j->dev_flags, sizeof(unsigned) * n);
  if (e == cudaSuccess) e = cudaMallocHost(&j->host, sizeof(double) * per * n);
  if (e == cudaSuccess) e = cudaMallocHost(&j->host_flags, sizeof(unsigned) * n);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j->snap, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j->landed, cudaEventDisableTiming);
  size_t off = 0;
  for (int k = 0; k < 7 && e == cudaSuccess; ++k) {
    e = cudaMemcpyAsync(j->dev + off * n, src[k].ptr, sizeof(double) * src[k].doubles * n, cudaMemcpyDeviceToDevice,
                        ctx->stream);
    off += src[k].doubles;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(j->dev_flags, s.flags, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(j->snap, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->io_stream, j->snap, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(j->host, j->dev, sizeof(double) * per * n, cudaMemcpyDeviceToHost, ctx->io_stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(j->host_flags, j->dev_flags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, ctx->io_stream);
  if (e == cudaSuccess) e = cudaEventRecord(j->landed, ctx->io_stream);
  vtk_job *jp = j.get();
  ctx->vtk_jobs.push_back(std::move(j));  // released by mf_vtk_flush, also on failure
  if (e != cudaSuccess) {
    ctx->last_cuda_err = (int)e;
    return MF_ERR_CUDA;
  }
  const std::string file(path);
  const int device = ctx->device;
  jp->writer = std::thread([jp, file, device]() {
    cudaSetDevice(device);
    if (cudaEventSynchronize(jp->landed) != cudaSuccess) { jp->rc = MF_ERR_CUDA; return; }
    const int n = jp->n;
    const double *h = jp->host;
    jp->rc = write_vtk_particles(file.c_str(), n, h, h + 2 * (size_t)n, h + 4 * (size_t)n, h + 5 * (size_t)n,
                                 h + 6 * (size_t)n, h + 7 * (size_t)n, h + 8 * (size_t)n, jp->host_flags);
  });
  return MF_OK;
}

}  // extern "C"

namespace {
// the contexts the differentiable step covers: a locked Green grid, Brookshaw or no
// conduction, and the Johnson-Cook law
int tangent_check(mf_ctx *ctx) {
  if (!ready(ctx) || ctx->mid_step) return MF_ERR_STATE;
  if (!(ctx->P.dt > 0.)) return MF_ERR_STATE;
  if (!ctx->G.locked || ctx->grid_kind != MF_GRID_GREEN || ctx->P.thermal_solver == MF_THERMAL_PSE ||
      ctx->P.jc_model != MF_JC_JOHNSON_COOK || !ctx->P.plastic || ctx->P.h_contact > 0.)
    return MF_ERR_INVALID;
  return MF_OK;
}
}  // namespace

int mf_tangent_mean_force_all(mf_ctx *ctx, int skip_steps, int window_steps, double out_mean[2],
                              double out_dmean[12]) {
  nvtx_range range("mf_tangent_mean_force_all");
  if (!ctx || !out_mean || !out_dmean || skip_steps < 0 || window_steps < 1) return MF_ERR_INVALID;
  TRY(tangent_check(ctx));
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  params P = ctx->P;
  P.N = ctx->N;
  P.staged = 0;
  return mf::tg6::run_mean_force(ctx, ctx->device, P, ctx->D, skip_steps, window_steps, -1, out_mean, out_dmean);
}

int mf_tangent_mean_force(mf_ctx *ctx, int skip_steps, int window_steps, int param, double out_mean[2],
                          double out_dmean[2]) {
  nvtx_range range("mf_tangent_mean_force");
  if (!ctx || !out_mean || skip_steps < 0 || window_steps < 1 || param < -1 || param > 5) return MF_ERR_INVALID;
  TRY(tangent_check(ctx));
  TRY(set_device(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  params P = ctx->P;
  P.N = ctx->N;
  P.staged = 0;
  return mf::tg::run_mean_force(ctx, ctx->device, P, ctx->D, skip_steps, window_steps, param, out_mean, out_dmean);
}
