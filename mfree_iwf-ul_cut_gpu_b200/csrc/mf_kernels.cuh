// sm_100a kernels of one leap-frog step (leap_frog.cu:94-155).
//
// Per step, on one stream (captured once into a CUDA graph):
//   k_bbox        adaptive grid only: min/max reduction -> geometry     (grid.cu:97-136)
//   k_hash_count  cell hash per particle + atomic per-cell count       (grid.cu:34-51);
//                 with a locked grid only before the first step, after that k_finish_flat
//                 of the previous step has done it
//   k_scan        exclusive scan of the counts -> cell offsets (the cell_start/cell_end
//                 lists), each tile starting from the preceding tiles' totals
//   k_scatter     particle -> slot inside its cell (atomic cursor per cell)
//   k_reorder     stable rank fix-up inside each cell (equal to thrust's stable sort_by_key),
//                 gather of the persistent state into the other buffer, and - in a step - the
//                 predictor, EOS, artificial stress, the neighbour pair records and the rigid
//                 tool's advance (grid_gpu_green.cu:22-116, leap_frog.cu:30-66,
//                 actions_gpu.cu:41-97, tool.cpp:211-221)
//   k_pair_fp64   the pair sums over the 5x5 cell window (interactions_gpu.cu:147-345) and the
//                 rates: Jaumann, continuity, momentum, advection (actions_gpu.cu:99-224)
//   k_pse         PSE heat Laplacian (interactions_gpu.cu:88-144), PSE solver only
//   k_finish_flat corrector, friction heat, the JC elastic test, tool particles, contact,
//                 boundary conditions, invalidation and the compensated tool-force reduction;
//                 with a locked grid also the next step's hashes and counts (leap_frog.cu:68-92,
//                 actions_gpu.cu:135-162,226-349, tool_gpu.cu:151-221, output.cu:31-39)
//   k_plastic     the JC return map of the particles the elastic test did not settle
#pragma once

#include "mf_device.cuh"

namespace mf {

struct state_set {
  double2 *pos, *vel, *fc, *ft, *pos_t, *vel_t;
  double *rho, *T, *eps_pl, *eps_pl_dot, *h, *rho_t, *T_t;
  double *pp;  // predictor pressure (the reference's particles->p), of the step that wrote the set
  double4 *S, *S_t;
  unsigned *flags;
  int *idx;
  int *id;  // particle number at creation, gathered by every sort
};

// a particle that failed the elastic test of the finish kernel, with the temperature its
// return map starts from (after friction heat, before the thermal boundary condition)
struct plastic_item {
  double T;    // temperature of the yield test (after friction heat)
  double svm;  // von Mises stress of the trial state
  int q;
  int pad;
};

struct dev_buffers {
  state_set A, B;       // A: state at the start of the step (previous order), B: new order
  double2 *n;           // contact normal, indexed by array position (never permuted)
  double *rec;          // FP64 pair records: R_WIDTH / 2 planes of N double2
  float *recf;          // FP32 pair records (mixed form): F_WIDTH / 4 planes of N float4
  double4 *S_der, *v_der;
  int *hash_cur;        // cell hash per array position (sorted order)
  int *hash_new, *perm;
  int4 *perm_u;         // per sorted slot: {particle, cell, cell start, cell end} (unranked)
  int *count;           // per-cell counts (max_cell)
  int *tsum_r, *tsum_w; // per-tile totals of the counts: read by this step's scan / added to by
                        // this step's counting for the next (two arrays, swapped every step)
  int *off;             // cell offsets (max_cell + 1)
  double *partials;     // per-block partial sums (force / bbox); the force's group sums follow the
                        // block partials (at [8 * number of block partials])
  unsigned *ticket;     // last-block tickets: [0] force, [1] bbox, [2] tool wear
  unsigned *gticket;    // per-group tickets of the force sums (one per FORCE_GROUP block partials)
  double *force_log;    // FORCE_LOG_CAP x 2
  double *force_last;   // 2
  plastic_item *plastic_list;  // particles whose return map k_plastic runs (this step)
  unsigned *plastic_count;
  // neighbour lists (mixed form): entry k of particle q at nlist[q * LIST_CAP + k], ncount[q]
  // entries; pos_build[q] the predicted position the list was built from
  unsigned *nlist;
  int *ncount;
  double2 *pos_build;
  mf_tool_state *tool_prev;  // tool after the previous step (read)
  mf_tool_state *tool_next;  // tool after this step (written by k_reorder, read by k_finish_flat)
  geom *g;
  dev_status *st;
};

// Programmatic dependent launch: the step's kernels are launched so that each may be
// scheduled while its predecessor drains. Every step kernel first waits until its predecessor
// has completed and its writes are visible, then lets its own successor be scheduled (all of
// its blocks are then placed, so the successor's waiting blocks only take slots that would
// otherwise idle in this kernel's tail). Both are no-ops for a plain launch.
#define MF_PDL_WAIT() asm volatile("griddepcontrol.wait;" ::: "memory")
#define MF_PDL_TRIGGER() asm volatile("griddepcontrol.launch_dependents;" ::: "memory")

#ifndef MF_SCAN_ITEMS
#define MF_SCAN_ITEMS 8
#endif
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = MF_SCAN_ITEMS;  // cells per thread of k_scan (a multiple of 4)
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr int BLOCK = 256;
// k_finish_flat: threads per block (one particle per thread)
#ifndef FINISH_BLOCK
#define FINISH_BLOCK 256
#endif
// k_plastic: fixed grid of this many 256-thread blocks per SM over the plastic list
constexpr int PLASTIC_BLOCKS_PER_SM = 4;
#ifndef MF_PAIR_BLOCK
#define MF_PAIR_BLOCK 128
#endif
constexpr int PAIR_BLOCK = MF_PAIR_BLOCK;
// k_reorder: blocks per SM its register budget allows (REORDER_BLOCKS_PER_SM x 256 threads per
// SM, so that a ~180k-particle grid runs in one wave)
#ifndef REORDER_BLOCKS_PER_SM
#define REORDER_BLOCKS_PER_SM 3
#endif

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// A kernel body's block index and block count within its particle system: the grid's own for a
// kernel launched for one context, the system's share of the grid in a batched launch that
// steps many systems at once (mf_batch_*). Bodies use these instead of blockIdx.x / gridDim.x.
struct blk {
  int x, n;
};
__device__ __forceinline__ blk grid_blk() { return blk{(int)blockIdx.x, (int)gridDim.x}; }

// ---------------------------------------------------------------------------------------
// adaptive geometry (grid_base::update_geometry, grid.cu:97-136)
__device__ __forceinline__ void bbox_merge(double *a, const double *b) {
  a[0] = fmin(a[0], b[0]);
  a[1] = fmin(a[1], b[1]);
  a[2] = fmax(a[2], b[2]);
  a[3] = fmax(a[3], b[3]);
  a[4] = fmax(a[4], b[4]);
}

static __global__ void __launch_bounds__(BLOCK) k_bbox(int N, const double2 *__restrict__ pos,
                                                const double *__restrict__ h, dev_buffers D) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  __shared__ double sm[BLOCK / 32][5];
  __shared__ bool last;
  const double BIG = 1.7976931348623157e+308;
  double v[5] = {BIG, BIG, -BIG, -BIG, -BIG};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    double2 p = pos[i];
    double hh = h[i];
    if (isfinite(p.x)) { v[0] = fmin(v[0], p.x); v[2] = fmax(v[2], p.x); }
    if (isfinite(p.y)) { v[1] = fmin(v[1], p.y); v[3] = fmax(v[3], p.y); }
    if (isfinite(hh)) v[4] = fmax(v[4], hh);
  }
  for (int o = 16; o > 0; o >>= 1) {
    double w[5];
    for (int k = 0; k < 5; ++k) w[k] = __shfl_down_sync(0xffffffffu, v[k], o);
    bbox_merge(v, w);
  }
  if (lane_id() == 0)
    for (int k = 0; k < 5; ++k) sm[threadIdx.x >> 5][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) bbox_merge(v, sm[w]);
    for (int k = 0; k < 5; ++k) D.partials[blockIdx.x * 8 + k] = v[k];
    __threadfence();
    unsigned t = atomicAdd(&D.ticket[1], 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double r[5] = {BIG, BIG, -BIG, -BIG, -BIG};
  for (unsigned b = 0; b < gridDim.x; ++b) {
    double w[5];
    for (int k = 0; k < 5; ++k) w[k] = ((volatile double *)D.partials)[b * 8 + k];
    bbox_merge(r, w);
  }
  D.ticket[1] = 0;
  geom g = *D.g;
  double bbmin_x = r[0] - 1e-6, bbmin_y = r[1] - 1e-6, bbmax_x = r[2] + 1e-6, bbmax_y = r[3] + 1e-6;
  double dx = r[4] * 2.0 / 2;
  double lx = bbmax_x - bbmin_x, ly = bbmax_y - bbmin_y;
  unsigned nx = (unsigned)ceil(lx / dx), ny = (unsigned)ceil(ly / dx);
  unsigned long long nc = (unsigned long long)nx * ny;
  if (!(N > 0) || !(dx > 0.) || !(nc < (unsigned long long)g.max_cell)) {
    atomicOr(&D.st->error_flags, ERR_GRID_BUDGET);
    return;  // keep the previous geometry; out-of-range hashes are clamped and counted
  }
  g.bbmin_x = bbmin_x; g.bbmin_y = bbmin_y; g.bbmax_x = bbmax_x; g.bbmax_y = bbmax_y;
  g.dx = dx; g.nx = (int)nx; g.ny = (int)ny; g.num_cell = (int)nc;
  *D.g = g;
}

// ---------------------------------------------------------------------------------------
// one particle counted into its cell and into its cell's scan tile (the scan's per-tile totals);
// the lanes of a warp with the same tile add their total in one atomic
__device__ __forceinline__ void count_particle(int *count, int *tsum, int hsh) {
  atomicAdd(&count[hsh], 1);  // no return value: a fire-and-forget reduction
  const int tile = hsh / SCAN_TILE;
  const unsigned peers = __match_any_sync(__activemask(), tile);
  if ((int)lane_id() == __ffs(peers) - 1) atomicAdd(&tsum[tile], __popc(peers));
}

// ---------------------------------------------------------------------------------------
// cell hash + count (compute_hashes, grid.cu:34-51)
static __global__ void __launch_bounds__(BLOCK) k_hash_count(int N, state_set A, dev_buffers D, int num_scan_tiles) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned oog = 0;
  if (gid < N) {
    const geom g = *D.g;
    long long hh;
    if (A.flags[gid] & FLAG_BLANKED) {
      hh = D.hash_cur[gid];  // blanked particles keep their previous hash (grid.cu:39-41)
    } else {
      double2 p = A.pos[gid];
      int ix = __double2int_rz((p.x - g.bbmin_x) / g.dx);
      int iy = __double2int_rz((p.y - g.bbmin_y) / g.dx);
      hh = (long long)ix * (long long)g.ny + (long long)iy;
    }
    // outside [0, num_cell) the reference writes out of bounds; clamp and count instead
    if (hh < 0) { hh = 0; oog = 1; }
    else if (hh >= g.num_cell) { hh = g.num_cell - 1; oog = 1; }
    const int hsh = (int)hh;
    D.hash_new[gid] = hsh;
    count_particle(D.count, D.tsum_r, hsh);  // read by the scan that follows
  }
  unsigned any = __ballot_sync(0xffffffffu, oog);
  if (any && lane_id() == 0) atomicAdd(&D.st->out_of_grid, (unsigned long long)__popc(any));
}

// ---------------------------------------------------------------------------------------
// exclusive scan of the cell counts -> offsets. Whoever counted the particles into their cells
// (the previous step's finish kernel, or k_hash_count) also added each one to its tile's total
// (tsum_r, a tile = SCAN_TILE cells), so block b knows where its tile starts by summing the
// totals of the tiles before it: no block waits for another. Each block also zeroes the counts
// of its tile and the total the next counting adds to (tsum_w; one block per tile).
__device__ __forceinline__ void scan_body(const dev_buffers &D, int N, int verlet, blk bk) {
  const int num_cell = D.g->num_cell;
  if (threadIdx.x == 0) D.tsum_w[bk.x] = 0;
  if (verlet && !D.st->sort_now) {
    // neighbour lists, no sort this step: the counts the finish kernel made go unused; back
    // to zero for the next step's
    for (int c = bk.x * SCAN_TILE + threadIdx.x; c < min(num_cell, (bk.x + 1) * SCAN_TILE);
         c += SCAN_THREADS)
      D.count[c] = 0;
    return;
  }
  __shared__ int s_warp[SCAN_THREADS / 32];
  __shared__ int s_excl;
  __shared__ int s_max[SCAN_THREADS / 32];
  const int num_tiles = (num_cell + SCAN_TILE - 1) / SCAN_TILE;
  const int tile = bk.x;
  if (tile >= num_tiles) return;
  if (threadIdx.x < 32) {  // the tile's start: the totals of the tiles before it
    int v = 0;
    for (int t = (int)lane_id(); t < tile; t += 32) v += __ldcg(D.tsum_r + t);
    v = __reduce_add_sync(0xffffffffu, v);
    if (lane_id() == 0) s_excl = v;
  }
  const int base = tile * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  static_assert(SCAN_ITEMS % 4 == 0, "whole int4 per thread");
  const bool full = base + SCAN_ITEMS <= num_cell;  // base: a multiple of SCAN_ITEMS, 16-byte aligned
  int v[SCAN_ITEMS];
  if (full) {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS / 4; ++k) {
      const int4 c = reinterpret_cast<const int4 *>(D.count + base)[k];
      v[4 * k] = c.x; v[4 * k + 1] = c.y; v[4 * k + 2] = c.z; v[4 * k + 3] = c.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) v[k] = base + k < num_cell ? D.count[base + k] : 0;
  }
  int tsum = 0, tmax = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int x = v[k];
    v[k] = tsum;
    tsum += x;
    tmax = max(tmax, x);
  }
  // warp inclusive scan of thread sums
  int incl = tsum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if ((int)lane_id() >= o) incl += y;
  }
  tmax = __reduce_max_sync(0xffffffffu, tmax);
  if (lane_id() == 31) s_warp[threadIdx.x >> 5] = incl;
  if (lane_id() == 0) s_max[threadIdx.x >> 5] = tmax;
  __syncthreads();
  int warp_excl = 0, agg = 0, bmax = 0;
  for (int w = 0; w < SCAN_THREADS / 32; ++w) {
    if (w < (int)(threadIdx.x >> 5)) warp_excl += s_warp[w];
    agg += s_warp[w];
    bmax = max(bmax, s_max[w]);
  }
  if (threadIdx.x == 0 && bmax > 0) atomicMax(&D.st->max_cell_occupancy, bmax);
  const int excl = s_excl + warp_excl + incl - tsum;
  if (full) {
    int4 *o = reinterpret_cast<int4 *>(D.off + base);
    int4 *z = reinterpret_cast<int4 *>(D.count + base);  // ready for the next step
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS / 4; ++k) {
      o[k] = make_int4(excl + v[4 * k], excl + v[4 * k + 1], excl + v[4 * k + 2], excl + v[4 * k + 3]);
      z[k] = make_int4(0, 0, 0, 0);
    }
  } else {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      const int c = base + k;
      if (c < num_cell) {
        D.off[c] = excl + v[k];
        D.count[c] = 0;
      }
    }
  }
  if (tile == num_tiles - 1 && threadIdx.x == 0) D.off[num_cell] = s_excl + agg;
  (void)N;
}

static __global__ void __launch_bounds__(SCAN_THREADS) k_scan(dev_buffers D, int N, int verlet) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  scan_body(D, N, verlet, grid_blk());
}

__device__ __forceinline__ void scatter_body(int N, const dev_buffers &D, int verlet, blk bk) {
  const int q = bk.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  if (verlet && !D.st->sort_now) return;  // neighbour lists, no sort this step
  const int c = D.hash_new[q];
  const int s = D.off[c];
  // the scan left the counts at zero: they serve as per-cell cursors here (the reorder
  // zeroes them again). The cell and its bounds travel with the particle, so the reorder
  // needs one load.
  const int slot = atomicAdd(&D.count[c], 1);
  D.perm_u[s + slot] = make_int4(q, c, s, D.off[c + 1]);
}

static __global__ void __launch_bounds__(BLOCK) k_scatter(int N, dev_buffers D, int verlet) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  scatter_body(N, D, verlet, grid_blk());
}

// ---------------------------------------------------------------------------------------
// stable rank fix-up: inside a cell, the atomics gave the members in arbitrary order; the
// stable sort wants them by previous array position. The member that the scatter put at
// slot q (u = perm_u[q]: particle, cell, cell start, cell end) belongs at the cell's slot
// start + (number of members with a smaller previous position): one pass over the cell, so a
// cell of m particles costs O(m) per member (a crowded cell O(m^2) in all, not O(m^3)).
__device__ __forceinline__ int stable_rank(const int4 *__restrict__ perm_u, const int4 u) {
  if (u.w - u.z == 1) return 0;
  int r = 0;
  for (int m = u.z; m < u.w; ++m) r += perm_u[m].x < u.x ? 1 : 0;
  return r;
}

// gather into the new order (grid_gpu_green.cu:22-116) and, if PREDICT, the predictor
// (leap_frog.cu:30-66), EOS (actions_gpu.cu:41-51), artificial stress (:53-97) and the
// neighbour records read by the pair kernel.
// The predictor of a step for the particle at array position q (leap_frog.cu:30-66), EOS
// (actions_gpu.cu:41-51), artificial stress (:53-97) and the neighbour pair records, from the
// particle's state at the start of the step and its rates. Writes the predicted velocity and
// stress, the rates the pair pass will not overwrite, the flags and the pressure into set B,
// and the records. With neighbour lists, a sorting step (build) also keeps the predicted
// position its lists are built from.
template <bool MIXED>
__device__ __forceinline__ void predict_particle(const params &P, const dev_buffers &D, const state_set &B, int q,
                                                 int hsh, double2 pos, double2 vel, double4 S, double rho, double T,
                                                 const double2 &pos_t, const double2 &vel_t, const double4 &S_t,
                                                 double rho_t, double T_t, unsigned f, double h, bool build) {
  const bool blanked = f & FLAG_BLANKED;
  const bool tool = f & FLAG_TOOL;
  // the previous rates travel with the particle where this step's pair pass will not
  // overwrite them (blanked particles; tool particles' stress and density rates; the
  // kinematic rates of tool particles under PSE; the temperature rate without conduction);
  // staged, every rate is copied so that the half-built step reads whole
  bool keep_kin = true, keep_mech = true, keep_T = true;
  if (!P.staged && !blanked) {
    const bool brookshaw = P.thermal_solver == MF_THERMAL_BROOKSHAW;
    keep_kin = !brookshaw && tool;
    keep_mech = tool;
    const double alpha_T = !tool ? P.trml_wp.alpha : (P.thermal_tool_on ? P.trml_tool.alpha : 0.);
    keep_T = brookshaw ? alpha_T == 0. : !P.thermal_wp;
  }
  if (keep_kin) {
    B.pos_t[q] = pos_t;
    B.vel_t[q] = vel_t;
  }
  if (keep_mech) {
    B.S_t[q] = S_t;
    B.rho_t[q] = rho_t;
  }
  if (keep_T) B.T_t[q] = T_t;

  if (!blanked) {
    const double dt = P.dt;
    pos.x = pos.x + 0.5 * dt * pos_t.x;
    pos.y = pos.y + 0.5 * dt * pos_t.y;
    vel.x = vel.x + 0.5 * dt * vel_t.x;
    vel.y = vel.y + 0.5 * dt * vel_t.y;
    S.x = S.x + 0.5 * dt * S_t.x;
    S.y = S.y + 0.5 * dt * S_t.y;
    S.z = S.z + 0.5 * dt * S_t.z;
    S.w = S.w + 0.5 * dt * S_t.w;
    rho = rho + 0.5 * dt * rho_t;
    T = T + 0.5 * dt * T_t;
  }
  // the predicted velocity and stress are read by the pair kernels; position, density and
  // temperature live in the pair records (the full predicted state is kept when staged)
  B.vel[q] = vel;
  B.S[q] = S;
  if (P.staged) {
    B.pos[q] = pos;
    B.rho[q] = rho;
    B.T[q] = T;
  }
  B.flags[q] = f;

  const double mass = P.phys.mass, K = P.phys.K;
  double prs = 0.;
  if (!tool) prs = P.eos_c0 * P.eos_c0 * (rho - P.phys.rho0);
  B.pp[q] = prs;
  unsigned rf = f & (FLAG_BLANKED | FLAG_TOOL | FLAG_FIXED);
  float fr[F_WIDTH];
  if (!MIXED || P.staged) {
    double Rxx = 0., Rxy = 0., Ryy = 0.;
    if (!tool) artificial_stress(rho, prs, S.x, S.y, S.z, P.corr.stresseps, Rxx, Rxy, Ryy);
    const double rho21 = 1. / (rho * rho);
    const double sxx = (S.x - prs) * rho21, sxy = S.y * rho21, syy = (S.z - prs) * rho21;
    const double c = (double)sqrtf((float)(K / rho));
    const double vol = mass / rho;
    double r[R_WIDTH] = {pos.x, pos.y, vel.x, vel.y, sxx, sxy, syy, Rxx, Rxy, Ryy, h, rho, c, vol, T, 0.};
    bool finite = true;
#pragma unroll
    for (int k = 0; k < R_FLAGS; ++k) finite = finite && isfinite(r[k]);
    if (!finite) rf |= FLAG_NONFINITE;
    r[R_FLAGS] = __longlong_as_double((long long)rf);
    // the FP64 record feeds the FP64 pair kernel and its PSE pass (kept when staged, for reads);
    // eight planes of double2 (structure of arrays): plane k of particle q at [k * N + q]
    double2 *dst = reinterpret_cast<double2 *>(D.rec);
#pragma unroll
    for (int k = 0; k < R_WIDTH / 2; ++k) dst[(size_t)k * P.N + q] = make_double2(r[2 * k], r[2 * k + 1]);
    const float fv[12] = {(float)vel.x, (float)vel.y, (float)sxx, (float)sxy, (float)syy, (float)Rxx,
                          (float)Rxy, (float)Ryy, (float)h, (float)rho, (float)c, (float)vol};
#pragma unroll
    for (int k = 0; k < 12; ++k) fr[3 + k] = fv[k];
  } else {
    // the mixed form's FP32 record only: one FP64 reciprocal of rho for 1 / rho^2, c and the
    // volume, the artificial stress in float
    const double rinv = 1. / rho, rho21 = rinv * rinv;
    float Rxx = 0.f, Rxy = 0.f, Ryy = 0.f;
    if (!tool) artificial_stress_f(rho21, prs, S.x, S.y, S.z, P.corr.stresseps, Rxx, Rxy, Ryy);
    const float fv[12] = {(float)vel.x, (float)vel.y, (float)((S.x - prs) * rho21), (float)(S.y * rho21),
                          (float)((S.z - prs) * rho21), Rxx, Rxy, Ryy, (float)h, (float)rho,
                          sqrtf((float)(K * rinv)), (float)(mass * rinv)};
    bool finite = isfinite(pos.x) && isfinite(pos.y) && isfinite(T);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      fr[3 + k] = fv[k];
      finite = finite && isfinite(fv[k]);
    }
    if (!finite) rf |= FLAG_NONFINITE;
  }

  if (MIXED) {
    // FP32 record: position relative to the origin of the particle's own cell, temperature
    // relative to the initial temperature (only differences of T enter the pair sums)
    const geom g = *D.g;
    const int ci = hsh / g.ny, cj = hsh - ci * g.ny;
    const double ox = g.bbmin_x + ci * g.dx, oy = g.bbmin_y + cj * g.dx;
    fr[0] = (float)(pos.x - ox);
    fr[1] = (float)(pos.y - oy);
    fr[2] = __int_as_float((int)(rf | ((unsigned)cj << 8)));
    fr[15] = (float)(T - P.trml_wp.T_init);
    // four float4 words (recf_word: four planes, or each record's words together)
    float4 *fd = reinterpret_cast<float4 *>(D.recf);
#pragma unroll
    for (int k = 0; k < F_WIDTH / 4; ++k)
      fd[recf_word(k, q, P.N)] = make_float4(fr[4 * k], fr[4 * k + 1], fr[4 * k + 2], fr[4 * k + 3]);
    // the lists stay valid while every particle is within skin / 2 of where it was at the
    // last sort (then every pair closer than 2 h was closer than 2 h + skin there); each step's
    // finish kernel checks the next step's predicted positions against 0.45 skin
    if (P.verlet && build) D.pos_build[q] = pos;
  }
}

// the last step's contact and friction forces of the particle at slot q (start-of-step slot p):
// from the step's start set (the Rothlin grid does not gather ft: it stays in place,
// grid_gpu_rothlin.cu:138-250)
__device__ __forceinline__ void prev_contact_forces(const params &P, const dev_buffers &D, int q, int p,
                                                    double2 &fc, double2 &ft) {
  fc = D.A.fc[p];
  ft = D.A.ft[P.grid_kind == MF_GRID_GREEN ? p : q];
}

// The rigid tool of this step: tool::update_tool (tool.cpp:211-221) with IEEE-rounded
// operations (bitwise equal to the host's double arithmetic), by warp 0 of block 0 of the
// step's reorder/predictor kernel: tool_prev copied to tool_next word by word, then lane
// k < num_seg moves segment k and lane 5 the fillet. The finish kernel, which runs later in the
// step, reads tool_next; computing it there keeps this division chain out of every finish
// block's start. (A function of its own, not inlined, so that it adds no registers to the
// kernel that calls it.)
static __device__ __noinline__ void tool_advance_warp(const mf_tool_state *prev, mf_tool_state *next, double dt) {
  static_assert(sizeof(mf_tool_state) % sizeof(double) == 0, "tool state is a whole number of doubles");
  constexpr int WORDS = (int)(sizeof(mf_tool_state) / sizeof(double));
  const int l = (int)lane_id();
  const double *src = reinterpret_cast<const double *>(prev);
  double *dst = reinterpret_cast<double *>(next);
  for (int w = l; w < WORDS; w += 32) dst[w] = src[w];
  __syncwarp();  // the copy's stores before the lanes' own below
  const mf_tool_state &T0 = *prev;
  const double sx = __dmul_rn(dt, T0.vel[0]), sy = __dmul_rn(dt, T0.vel[1]);
  if (l < T0.num_seg) {
    mf_segment s = T0.seg[l];
    s.left[0] = __dadd_rn(s.left[0], sx);
    s.left[1] = __dadd_rn(s.left[1], sy);
    s.right[0] = __dadd_rn(s.right[0], sx);
    s.right[1] = __dadd_rn(s.right[1], sy);
    line_through_rn(s.left[0], s.left[1], s.right[0], s.right[1], s.a, s.b, s.vertical);
    next->seg[l] = s;
  } else if (l == 5 && T0.has_fillet) {
    next->fillet.p[0] = __dadd_rn(T0.fillet.p[0], sx);
    next->fillet.p[1] = __dadd_rn(T0.fillet.p[1], sy);
  }
}

// the step's tool (written by the pair kernel) into shared memory, copied word by word by the
// block's threads
__device__ __forceinline__ void tool_load_shared(mf_tool_state &T, const dev_buffers &D) {
  constexpr int WORDS = (int)(sizeof(mf_tool_state) / sizeof(double));
  for (int w = threadIdx.x; w < WORDS; w += blockDim.x)
    reinterpret_cast<double *>(&T)[w] = reinterpret_cast<const double *>(D.tool_next)[w];
  __syncthreads();
}

template <bool PREDICT, bool MIXED>
__device__ __forceinline__ void reorder_body(const params &P, const dev_buffers &D, blk bk) {
  if (PREDICT && P.has_tool && bk.x == 0 && threadIdx.x < 32) tool_advance_warp(D.tool_prev, D.tool_next, P.dt);
  const int t = bk.x * blockDim.x + threadIdx.x;
  if (t >= P.N) return;
  // with neighbour lists, a step without a sort keeps the order and the cells of the last
  // sort: the identity permutation
  const bool sort = !P.verlet || D.st->sort_now;
  if (t == 0) {  // re-armed for the finish kernel of this step
    *D.plastic_count = 0u;
    if (sort) D.st->sorts += 1ull;
  }
  // neighbour lists, no sort, and the previous step's finish (and plastic) kernels already ran
  // this step's predictor: nothing left to do
  if (PREDICT && !sort && D.st->predicted) return;
  // thread t takes the particle the scatter put at slot t and moves it to its stable slot q
  // (inside the same cell, so a warp's stores stay within a few neighbouring cells)
  int p = t, q = t, hsh;
  if (sort) {
    const int4 u = D.perm_u[t];
    p = u.x;
    q = u.z + stable_rank(D.perm_u, u);
    hsh = u.y;
    if (t == u.z) D.count[hsh] = 0;  // the scatter's cursor, back to zero for the next counts
    D.hash_cur[q] = hsh;
  } else {
    hsh = D.hash_cur[q];
  }
  const state_set &A = D.A;
  const state_set &B = D.B;
  // the order, numbers and smoothing lengths: unchanged on a step that keeps the order after a
  // step that kept it too (neighbour lists), when this step's set already holds them from two
  // steps ago
  const bool moved = sort || !PREDICT || P.staged || D.st->sorted_prev;
  if (moved) {
    D.perm[q] = p;
    B.idx[q] = P.grid_kind == MF_GRID_GREEN ? p : A.idx[p];
    B.id[q] = A.id[p];
  }

  double2 pos = A.pos[p], vel = A.vel[p];
  double4 S = A.S[p];
  double rho = A.rho[p], T = A.T[p];
  double2 pos_t = A.pos_t[p], vel_t = A.vel_t[p];
  double4 S_t = A.S_t[p];
  double rho_t = A.rho_t[p], T_t = A.T_t[p];
  const unsigned f = A.flags[p];
  const double h = A.h[p];
  B.eps_pl[q] = A.eps_pl[p];
  B.eps_pl_dot[q] = A.eps_pl_dot[p];
  if (!PREDICT || P.staged) {
    // the last step's contact forces: within a step the pair and finish kernels read them from
    // the start set (prev_contact_forces); a sort outside a step, or a staged step whose
    // intermediate state is read back, moves them too
    B.fc[q] = A.fc[p];
    // the Rothlin grid does not gather ft (grid_gpu_rothlin.cu:138-250): it stays in place
    B.ft[q] = P.grid_kind == MF_GRID_GREEN ? A.ft[p] : A.ft[q];
  }
  if (moved) B.h[q] = h;
  if (!PREDICT) {  // a sort outside a step: the state moves as it is
    B.pos_t[q] = pos_t;
    B.vel_t[q] = vel_t;
    B.S_t[q] = S_t;
    B.rho_t[q] = rho_t;
    B.T_t[q] = T_t;
    B.vel[q] = vel;
    B.S[q] = S;
    B.pos[q] = pos;
    B.rho[q] = rho;
    B.T[q] = T;
    B.flags[q] = f;
    return;
  }
  predict_particle<MIXED>(P, D, B, q, hsh, pos, vel, S, rho, T, pos_t, vel_t, S_t, rho_t, T_t, f, h, sort);
}

template <bool PREDICT, bool MIXED>
static __global__ void __launch_bounds__(BLOCK, REORDER_BLOCKS_PER_SM) k_reorder(params P, dev_buffers D) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  reorder_body<PREDICT, MIXED>(P, D, grid_blk());
}

// ---------------------------------------------------------------------------------------
// pair sums over the 5x5 cell window + rates, plain FP64 (interactions_gpu.cu:147-345,
// actions_gpu.cu:99-224). With hash = ix*ny + iy, the five cells of one window column are
// consecutive hashes, so their particles form one contiguous range of the sorted order;
// visiting the columns in x order and each range in array order is the reference's
// neighbour order (x-cell outer, y-cell inner, sorted order within a cell).

// plane k of the FP64 record of particle j
__device__ __forceinline__ double2 rec_plane(const double *__restrict__ rec, int N, int k, int j) {
  return __ldg(reinterpret_cast<const double2 *>(rec) + (size_t)k * N + j);
}

__device__ __forceinline__ void load_rec(const double *__restrict__ rec, int N, int j, double *r) {
#pragma unroll
  for (int k = 0; k < R_WIDTH / 2; ++k) {
    const double2 v = rec_plane(rec, N, k, j);
    r[2 * k] = v.x;
    r[2 * k + 1] = v.y;
  }
}

__device__ __forceinline__ void pair_fp64_particle(const params &P, const dev_buffers &D, int q) {
  if (q >= P.N) return;
  const double *__restrict__ rec = D.rec;
  const int N = P.N;
  double ri[R_WIDTH];
  load_rec(rec, N, q, ri);
  const unsigned fi = (unsigned)__double_as_longlong(ri[R_FLAGS]);
  if (fi & FLAG_BLANKED) return;
  const bool tool_i = fi & FLAG_TOOL;
  const bool brookshaw = P.thermal_solver == MF_THERMAL_BROOKSHAW;
  if (!brookshaw && tool_i) return;  // PSE build: tool particles return early (:160-162)

  const double mass = P.phys.mass;
  const double wdeltap = P.corr.wdeltap, alpha = P.corr.alpha, beta = P.corr.beta, eta = P.corr.eta;
  const double eps = P.corr.xspheps;
  double thermal_alpha = 0.;
  if (brookshaw) thermal_alpha = !tool_i ? P.trml_wp.alpha : (P.thermal_tool_on ? P.trml_tool.alpha : 0.);
  const bool thermal = thermal_alpha != 0.;

  const double xi = ri[R_X], yi = ri[R_Y], vxi = ri[R_VX], vyi = ri[R_VY];
  const double sxxi = ri[R_SXX], sxyi = ri[R_SXY], syyi = ri[R_SYY];
  const double Rxxi = ri[R_RXX], Rxyi = ri[R_RXY], Ryyi = ri[R_RYY];
  const double hi = ri[R_H], rhoi = ri[R_RHO], ci = ri[R_C];
  const double Ti = thermal ? ri[R_T] : 0.;
  const double h1 = 1 / hi;
  const double fourh2 = 4 * hi * hi;
  const bool nonfinite_i = fi & FLAG_NONFINITE;

  const geom g = *D.g;
  const int hashi = D.hash_cur[q];
  const int p = __ldg(D.perm + q);  // the start slot (last contact forces), loaded during the sums
  const int gi = hashi / g.ny;
  const int gj = hashi - gi * g.ny;
  const int low_i = gi - 2 < 0 ? 0 : gi - 2;
  const int low_j = gj - 2 < 0 ? 0 : gj - 2;
  const int high_i = gi + 3 > g.nx ? g.nx : gi + 3;
  const int high_j = gj + 3 > g.ny ? g.ny : gj + 3;

  double vdx = 0., vdy = 0., vdz = 0., vdw = 0.;  // v_der
  double sdx = 0., sdy = 0., sdz = 0., sdw = 0.;  // S_der
  double vtx = 0., vty = 0., xtx = 0., xty = 0.;   // vel_t (AV), pos_t (XSPH)
  double T_lapl = 0.;

  const double m_eps = -eps * mass;
  for (int ii = low_i; ii < high_i; ++ii) {
    const int j0 = __ldg(D.off + ii * g.ny + low_j);
    const int j1 = __ldg(D.off + ii * g.ny + high_j);
    // Candidates are taken in chunks of up to 32: a cheap pass marks the ones that
    // contribute, then the expensive body visits the marked ones in array order. Outside
    // the support the reference adds terms multiplied by W = 0: they change no finite sum,
    // but a NaN/Inf operand turns the sum into NaN, so those candidates are marked too.
    for (int jb = j0; jb < j1; jb += 32) {
      const int jn = min(32, j1 - jb);
      unsigned mask = 0u;
      for (int k = 0; k < jn; ++k) {
        const unsigned fj = (unsigned)__double_as_longlong(rec_plane(rec, N, 7, jb + k).y);
        const double2 xy = rec_plane(rec, N, 0, jb + k);
        const double xij = xi - xy.x;
        const double yij = yi - xy.y;
        const double rr2 = xij * xij + yij * yij;
        const bool in_support = !(rr2 >= fourh2 || rr2 < 1e-8);
        const bool take = !(fj & FLAG_BLANKED) && (in_support || nonfinite_i || (fj & FLAG_NONFINITE));
        mask |= (take ? 1u : 0u) << k;
      }
      while (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1u;
        const int j = jb + k;
        const double2 fx = rec_plane(rec, N, 7, j);    // T, flags
        const double2 xy = rec_plane(rec, N, 0, j);
        const double2 cvol = rec_plane(rec, N, 6, j);  // c, vol
        const unsigned fj = (unsigned)__double_as_longlong(fx.y);
        const double xij = xi - xy.x;
        const double yij = yi - xy.y;
        const double rr2 = xij * xij + yij * yij;
        const bool in_support = !(rr2 >= fourh2 || rr2 < 1e-8);
        double w = 0., w_x = 0., w_y = 0., dwr = 0.;
        if (in_support) cubic_spline_fp64(xij, yij, rr2, h1, w, w_x, w_y, dwr);
        const double volj = cvol.y;
        const bool tool_j = fj & FLAG_TOOL;
        if (!tool_i && !tool_j) {
          const double2 v = rec_plane(rec, N, 1, j);
          const double2 s01 = rec_plane(rec, N, 2, j);   // sxx, sxy
          const double2 s2r0 = rec_plane(rec, N, 3, j);  // syy, Rxx
          const double2 r12 = rec_plane(rec, N, 4, j);   // Rxy, Ryy
          const double2 hrho = rec_plane(rec, N, 5, j);  // h, rho
          vdx += (v.x - vxi) * w_x * volj;
          vdy += (v.x - vxi) * w_y * volj;
          vdz += (v.y - vyi) * w_x * volj;
          vdw += (v.y - vyi) * w_y * volj;
          double fab = w / wdeltap;
          fab *= fab;
          fab *= fab;
          const double Rx = fab * (Rxxi + s2r0.y);
          const double Ry = fab * (Rxyi + r12.x);
          const double Rz = fab * (Ryyi + r12.y);
          sdx += mass * (sxxi + s01.x + Rx) * w_x;
          sdy += mass * (sxyi + s01.y + Ry) * w_y;
          sdz += mass * (sxyi + s01.y + Ry) * w_x;
          sdw += mass * (syyi + s2r0.x + Rz) * w_y;
          const double vijx = vxi - v.x;
          const double vijy = vyi - v.y;
          const double vijposij = vijx * xij + vijy * yij;
          const double irhoij = 1. / (0.5 * (rhoi + hrho.y));
          if (vijposij < 0.) {
            const double cij = 0.5 * (ci + cvol.x);
            const double hij = 0.5 * (hi + hrho.x);
            const double muij = (hij * vijposij) / (rr2 + eta * eta * hij * hij);
            const double piij = (-alpha * cij * muij + beta * muij * muij) * irhoij;
            vtx += -mass * piij * w_x;
            vty += -mass * piij * w_y;
          }
          const double xs = m_eps * w * irhoij;
          xtx += xs * vijx;
          xty += xs * vijy;
        }
        // Brookshaw: 2 (m/rho_j)(Ti - Tj)(e_ij . grad W)/r, and (e_ij . grad W)/r = der*fac
        if (thermal && rr2 > 1e-16) T_lapl += 2.0 * volj * (Ti - fx.x) * dwr;
      }
    }
  }

  const state_set &B = D.B;
  if (P.keep_derivs) {
    D.S_der[q] = make_double4(sdx, sdy, sdz, sdw);
    D.v_der[q] = make_double4(vdx, vdy, vdz, vdw);
  }
  if (!tool_i) {
    const double4 S = B.S[q];  // predicted stress
    double tx, ty, tz, tw;
    jaumann(P.phys.G, vdx, vdy, vdz, vdw, S.x, S.y, S.z, S.w, tx, ty, tz, tw);
    B.S_t[q] = make_double4(tx, ty, tz, tw);
    B.rho_t[q] = -rhoi * (vdx + vdw);
    double2 fc, ft;
    prev_contact_forces(P, D, q, p, fc, ft);
    double2 vel_t;
    vel_t.x = vtx + (sdx + sdy + fc.x / mass + ft.x / mass);
    vel_t.y = vty + (sdz + sdw + fc.y / mass + ft.y / mass);
    B.vel_t[q] = vel_t;
    B.pos_t[q] = make_double2(xtx + vxi, xty + vyi);
  } else {
    B.vel_t[q] = make_double2(vtx, vty);
    B.pos_t[q] = make_double2(xtx, xty);
  }
  if (thermal) B.T_t[q] = thermal_alpha * T_lapl;
}

// the FP64 pair sums of block bk.x's particles
__device__ __forceinline__ void pair_fp64_body(const params &P, const dev_buffers &D, blk bk) {
  pair_fp64_particle(P, D, bk.x * blockDim.x + threadIdx.x);
}

// the FP64 pair kernel in blocks of 64 at 8 per SM (128 registers): 110.6 against 112.6 us in
// blocks of 128 at 4, 114.7 in blocks of 256 at 2 (the ~150k-particle cut); at 3 blocks of 128
// (153 registers, no spills) 121.8
constexpr int PAIR64_BLOCK = 64;
#ifndef MF_PAIR64_MIN_BLOCKS
#define MF_PAIR64_MIN_BLOCKS 8
#endif
static __global__ void __launch_bounds__(PAIR64_BLOCK, MF_PAIR64_MIN_BLOCKS) k_pair_fp64(params P, dev_buffers D) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  pair_fp64_body(P, D, grid_blk());
}

// PSE heat Laplacian (interactions_gpu.cu:88-144): every particle of the window, blanked
// ones included; alpha taken through the reference's half-length texture binding (:405).
__device__ __forceinline__ void pse_body(const params &P, const dev_buffers &D, blk bk) {
  const int q = bk.x * blockDim.x + threadIdx.x;
  if (q >= P.N) return;
  const double *__restrict__ rec = D.rec;
  const int N = P.N;
  const double2 fx = rec_plane(rec, N, 7, q);
  const unsigned fi = (unsigned)__double_as_longlong(fx.y);
  if (fi & FLAG_BLANKED) return;
  const double2 xy = rec_plane(rec, N, 0, q);
  const double hi = rec_plane(rec, N, 5, q).x;
  const double Ti = fx.x;
  const double mass = P.phys.mass;
  const long long tex_elems = ((long long)sizeof(int) * P.N) / 8;
  const bool tool_i = q < tex_elems ? (fi & FLAG_TOOL) != 0 : false;
  const double alpha = tool_i ? P.trml_tool.alpha : P.trml_wp.alpha;
  const geom g = *D.g;
  const int hashi = D.hash_cur[q];
  const int gi = hashi / g.ny;
  const int gj = hashi - gi * g.ny;
  const int low_i = gi - 2 < 0 ? 0 : gi - 2;
  const int low_j = gj - 2 < 0 ? 0 : gj - 2;
  const int high_i = gi + 3 > g.nx ? g.nx : gi + 3;
  const int high_j = gj + 3 > g.ny ? g.ny : gj + 3;
  double T_ti = 0.;
  for (int ii = low_i; ii < high_i; ++ii) {
    const int j0 = __ldg(D.off + ii * g.ny + low_j);
    const int j1 = __ldg(D.off + ii * g.ny + high_j);
    for (int j = j0; j < j1; ++j) {
      const double2 pj = rec_plane(rec, N, 0, j);
      const double Tj = rec_plane(rec, N, 7, j).x;
      const double rhoj = rec_plane(rec, N, 5, j).y;
      const double w2 = lapl_pse_fp64(xy.x - pj.x, xy.y - pj.y, hi);
      T_ti += (Tj - Ti) * w2 * mass / rhoj;
    }
  }
  D.B.T_t[q] = alpha * T_ti;
}

static __global__ void __launch_bounds__(PAIR_BLOCK) k_pse(params P, dev_buffers D) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  pse_body(P, D, grid_blk());
}

// ---------------------------------------------------------------------------------------

// Corrector .. invalidate for one particle (leap_frog.cu:68-92, actions_gpu.cu:135-162,
// 226-349, tool_gpu.cu:151-221), in two phases that each load, update and store their own
// fields: first velocity and position with the friction-heat input, contact, the kinematic
// boundary conditions; then stress, density and temperature with the elastic test and the
// thermal boundary condition. Fewer values are live at once than when every load is issued
// first, so the kernel runs with fewer registers and more warps per SM. (eps_pl is not touched
// here: the corrector does not change it, the return map in k_plastic does.) With FUSE_PRED and
// `fuse`, also the next step's predictor (neighbour lists, a step without a sort).
template <bool FUSE_PRED, bool CONDUCT>
__device__ __forceinline__ void finish_particle_phased(const params &P, const dev_buffers &D,
                                                       const mf_tool_state &TL, int q, double2 &pos_out,
                                                       unsigned &f_out, double2 &fc_out, double2 &ft_out,
                                                       unsigned &newly_blanked, bool &want_sort, bool identity,
                                                       bool fuse) {
  const state_set &A = D.A;
  const state_set &B = D.B;
  const double dt = P.dt;
  unsigned f = B.flags[q];
  const bool blanked = f & FLAG_BLANKED;
  const bool tool = f & FLAG_TOOL;
  const bool fixed = f & FLAG_FIXED;
  const int p = identity ? q : D.perm[q];
  // phase 1: kinematics
  double2 pos = A.pos[p], vel = A.vel[p];
  double2 pos_t = B.pos_t[q], vel_t = B.vel_t[q];
  double2 fc, ft;
  prev_contact_forces(P, D, q, p, fc, ft);
  if (!blanked) {  // correct (leap_frog.cu:68-92)
    pos.x = pos.x + dt * pos_t.x;
    pos.y = pos.y + dt * pos_t.y;
    vel.x = vel.x + dt * vel_t.x;
    vel.y = vel.y + dt * vel_t.y;
  }
  // friction heat (actions_gpu.cu:135-162), previous step's ft and n: its increment now, added
  // to the corrected temperature in phase 2
  double dT_fric = 0.;
  bool fric = false;
  if (P.has_tool && P.fric_heat && !tool) {
    const double f_fric_mag = (double)sqrtf((float)(ft.x * ft.x + ft.y * ft.y));
    if (f_fric_mag != 0.) {
      const double2 normal = D.n[q];
      const double vdx = vel.x - TL.vel[0], vdy = vel.y - TL.vel[1];
      const double vdn = vdx * normal.x + vdy * normal.y;
      const double vrx = vdx - vdn, vry = vdy - vdn;
      const double v_rel_mag = (double)sqrtf((float)(vrx * vrx + vry * vry));
      dT_fric = P.trml_wp.eta * dt * f_fric_mag * v_rel_mag / (P.trml_wp.cp * P.phys.mass);
      fric = true;
    }
  }
  // tool particles move with the tool (tool_gpu.cu:210-221); contact (:151-207)
  bool in_contact = false;
  if (P.has_tool) {
    if (tool) {
      pos.x += dt * TL.vel[0];
      pos.y += dt * TL.vel[1];
    } else {
      double cpx = 0., cpy = 0., nx = 0., ny = 0.;
      const bool inside = establish_contact(TL, pos.x, pos.y, cpx, cpy, nx, ny);
      if (!inside) {
        fc = make_double2(0., 0.);
        ft = make_double2(0., 0.);
        D.n[q] = make_double2(0., 0.);
      } else {
        const double dt2 = dt * dt;
        const double gN = (pos.x - cpx) * nx + (pos.y - cpy) * ny;
        const double sc = -TL.slave_mass * gN;
        double2 fN = make_double2(sc * nx, sc * ny);
        fN.x = fN.x / dt2 * TL.contact_alpha;
        fN.y = fN.y / dt2 * TL.contact_alpha;
        double2 fT = make_double2(0., 0.);
        if (TL.mu != 0.) {
          const double vx = vel.x - TL.vel[0], vy = vel.y - TL.vel[1];
          const double vrx = vx - vx * nx, vry = vy - vy * ny;
          const double ks = TL.contact_alpha * TL.slave_mass;
          const double kx = ks * vrx / dt, ky = ks * vry / dt;
          const double fy = TL.mu * sqrt(fN.x * fN.x + fN.y * fN.y);
          const double fsx = ft.x - kx, fsy = ft.y - ky;
          const double lfs = sqrt(fsx * fsx + fsy * fsy);
          if (lfs > fy) {
            fT.x = fy * fsx / lfs;
            fT.y = fy * fsy / lfs;
          } else {
            fT = make_double2(fsx, fsy);
          }
        }
        fc = fN;
        ft = fT;
        D.n[q] = make_double2(nx, ny);
        in_contact = true;
      }
    }
  }
  // boundary conditions (actions_gpu.cu:287-311)
  if (!tool && fixed) {
    vel = make_double2(0., 0.);
    fc = make_double2(0., 0.);
    pos_t = make_double2(0., 0.);
    vel_t = make_double2(0., 0.);
    B.pos_t[q] = pos_t;
    B.vel_t[q] = vel_t;
  }
  bool invalid = !blanked && (isnaninf(pos_t.x) || isnaninf(pos_t.y) || isnaninf(vel_t.x) || isnaninf(vel_t.y));
  // neighbour lists: the next step's predicted position against the list's build position
  bool far = false;
  if (P.verlet) {
    const double2 pb = D.pos_build[q];
    const double px = pos.x + 0.5 * dt * pos_t.x, py = pos.y + 0.5 * dt * pos_t.y;
    const double ddx = px - pb.x, ddy = py - pb.y;
    const double lim = 0.45 * (double)P.skin;
    far = !(ddx * ddx + ddy * ddy <= lim * lim);
  }
  B.pos[q] = pos;
  B.vel[q] = vel;
  B.fc[q] = fc;
  B.ft[q] = ft;
  // phase 2: stress, density, temperature
  double4 S = A.S[p];
  double rho = A.rho[p], T = A.T[p];
  const double4 S_t = B.S_t[q];
  const double rho_t = B.rho_t[q], T_t = B.T_t[q];
  if (!blanked) {
    S.x = S.x + dt * S_t.x;
    S.y = S.y + dt * S_t.y;
    S.z = S.z + dt * S_t.z;
    S.w = S.w + dt * S_t.w;
    rho = rho + dt * rho_t;
    T = T + dt * T_t;
  }
  if (fric) T += dT_fric;
  // contact conductance (no reference counterpart; off unless set): heat h (T_tool - T) per unit
  // contact length, the contact length of a particle of mass m (per unit depth) at density rho
  // being sqrt(m / rho), so dT/dt = h (T_tool - T) / (cp sqrt(m rho))
  if (CONDUCT && in_contact && !blanked && P.trml_wp.cp > 0.)
    T += dt * P.h_contact * (P.T_contact - T) / (P.trml_wp.cp * sqrt(P.phys.mass * rho));
  // JC plasticity, radial return (actions_gpu.cu:226-285): the elastic lower bound of
  // finish_particle, the rest in k_plastic
  bool elastic = false;
  if (P.plastic && !tool) {
    const double pr = B.pp[q];
    const double Sxx = S.x, Syy = S.z, Szz = S.w, Sxy = S.y;
    const double cxx = Sxx - pr, cyy = Syy - pr, czz = Szz - pr, cxy = Sxy;
    const double svm = (double)sqrtf(
        (float)((cxx * cxx + cyy * cyy + czz * czz) - cxx * cyy - cxx * czz - cyy * czz + 3.0 * cxy * cxy));
    if (P.jc_lower_bound) {
      const mf_joco_constants &JC = P.joco;
      const float theta_f = (float)(T - JC.Tref) * (1.f / (float)(JC.Tmelt - JC.Tref));
      const double pow_hi = 1.00001 * (double)powf(theta_f, (float)JC.m);
      elastic = svm < 0.999 * JC.A * (1.0 - pow_hi);
    }
    if (elastic) {
      B.eps_pl_dot[q] = 0.;
    } else {
      const unsigned am = __activemask();
      const int leader = __ffs(am) - 1;
      unsigned base = 0u;
      if ((int)lane_id() == leader) base = atomicAdd(D.plastic_count, (unsigned)__popc(am));
      base = __shfl_sync(am, base, leader);
      const unsigned rank = __popc(am & ((1u << lane_id()) - 1u));
      D.plastic_list[base + rank] = plastic_item{T, svm, q, 0};
    }
  }
  if (P.thermal_bc && fixed) T = P.trml_wp.T_init;
  invalid = invalid || (!blanked && (isnaninf(S_t.x) || isnaninf(S_t.y) || isnaninf(S_t.z) || isnaninf(S_t.w) ||
                                     isnaninf(rho_t) || isnaninf(T_t)));
  B.S[q] = S;
  B.rho[q] = rho;
  B.T[q] = T;
  if (invalid) {  // invalidate (actions_gpu.cu:317-349)
    f |= FLAG_BLANKED;
    newly_blanked += 1u;
    B.flags[q] = f;
  }
  if (far && !(f & FLAG_BLANKED)) want_sort = true;
  if (FUSE_PRED && fuse) {
    // neighbour lists, a step without a sort: the next step keeps this order, so its predictor
    // runs here, on the final state (position, velocity and the kinematic rates read back, the
    // rest still in registers), into the set the next step writes (this step's start set, read
    // above by this thread only). If the next step sorts, its reorder kernel redoes it; k_plastic
    // redoes it for the particles it changes. The next step reads the last contact forces from
    // its start set, this step's end set.
    const state_set &N1 = D.A;
    N1.idx[q] = P.grid_kind == MF_GRID_GREEN ? q : B.idx[q];
    N1.eps_pl[q] = B.eps_pl[q];
    N1.eps_pl_dot[q] = (P.plastic && !tool && elastic) ? 0. : B.eps_pl_dot[q];
    predict_particle<true>(P, D, N1, q, D.hash_cur[q], B.pos[q], B.vel[q], S, rho, T, B.pos_t[q], B.vel_t[q], S_t,
                           rho_t, T_t, f, B.h[q], false);
  }
  pos_out = pos;
  f_out = f;
  fc_out = fc;
  ft_out = ft;
}

// The step's tool force from the per-block partials (8 doubles each: the compensated sums s, c
// of fc.x, fc.y, ft.x, ft.y) in a fixed two-level tree: the partials of each group of
// FORCE_GROUP consecutive blocks summed by one warp (lane l takes the group's l-th partial,
// then a shuffle tree), then the group sums by one warp (lane l takes groups l, l + 32, ... in
// order, then the same tree). In the flat finish kernel the block that completes a group sums
// it and the block that completes the last group sums the groups: each step of the tree is one
// load per lane and a shuffle tree, so no block waits long and no warp walks a long chain.
constexpr int FORCE_GROUP = 32;

__device__ __forceinline__ void ksum4_shuffle_tree(ksum r[4]) {
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 4; ++k) {
      ksum x{__shfl_down_sync(0xffffffffu, r[k].s, o), __shfl_down_sync(0xffffffffu, r[k].c, o)};
      ksum_merge(r[k], x);
    }
}

// lane 0: the sum of group g of the nb block partials (read through L2: other blocks wrote them
// before their fence and ticket)
__device__ __forceinline__ void force_group_sum(const double *partials, int g, int nb, ksum r[4]) {
  const int b = g * FORCE_GROUP + (int)lane_id();
  for (int k = 0; k < 4; ++k) r[k] = ksum{0., 0.};
  if (b < nb) {
    const double2 *pr = reinterpret_cast<const double2 *>(partials) + (size_t)b * 4;
    for (int k = 0; k < 4; ++k) {
      const double2 v = __ldcg(pr + k);
      r[k] = ksum{v.x, v.y};
    }
  }
  ksum4_shuffle_tree(r);
}

__device__ __forceinline__ void store_ksum4(double *dst, const ksum r[4]) {
  for (int k = 0; k < 4; ++k) {
    dst[2 * k] = r[k].s;
    dst[2 * k + 1] = r[k].c;
  }
}

// lane 0: the sum of the ng group sums
__device__ __forceinline__ void force_final_sum(const double *gsums, int ng, ksum r[4]) {
  for (int k = 0; k < 4; ++k) r[k] = ksum{0., 0.};
  const double2 *pr = reinterpret_cast<const double2 *>(gsums);
  for (int g = (int)lane_id(); g < ng; g += 32)
    for (int k = 0; k < 4; ++k) {
      const double2 v = __ldcg(pr + (size_t)g * 4 + k);
      ksum x{v.x, v.y};
      ksum_merge(r[k], x);
    }
  ksum4_shuffle_tree(r);
}

// lane 0 of the warp that finished the sum: report_force (output.cu:31-39: contact plus
// friction force) into force_last and the log, the step's counters, the tickets re-armed.
// `predicted`: the next step's predictor ran in this kernel.
__device__ __forceinline__ void force_close_step(const params &P, const dev_buffers &D, const ksum r[4],
                                                 bool predicted, bool sorted) {
  const double Fx = (r[0].s + r[0].c) + (r[2].s + r[2].c);
  const double Fy = (r[1].s + r[1].c) + (r[3].s + r[3].c);
  D.force_last[0] = Fx;
  D.force_last[1] = Fy;
  const unsigned long long hd = D.st->force_log_head;
  D.force_log[2 * (hd % FORCE_LOG_CAP)] = Fx;
  D.force_log[2 * (hd % FORCE_LOG_CAP) + 1] = Fy;
  D.st->force_log_head = hd + 1;
  D.st->steps += 1;
  if (P.verlet) {  // every particle is checked: the next step sorts if one asked for it
    D.st->sort_now = D.st->want_sort;
    D.st->want_sort = 0u;
    D.st->predicted = predicted ? 1u : 0u;
  }
  D.st->sorted_prev = sorted ? 1u : 0u;
  D.ticket[0] = 0u;
}

// Corrector .. invalidate for all particles plus the tool force (output.cu:31-39): one thread
// per particle, one block per FINISH_BLOCK consecutive particles; the force sums per warp, then
// the block's warps in order, then the two-level group tree. With FUSE_HASH (locked grid) also
// the next step's hash and count; with FUSE_PRED the next step's predictor on list steps
// without a sort (MF_OPT_FUSED_PREDICTOR). (A persistent variant of the fused kernel, blocks
// taking 256-particle chunks from a counter at 128 registers, measured 44 against these 38 us
// and gave the same bits.)
#ifndef FINISH_FLAT_MIN_BLOCKS
#define FINISH_FLAT_MIN_BLOCKS 3
#endif
template <bool FUSE_HASH, bool FUSE_PRED, bool CONDUCT = false>
__device__ __forceinline__ void finish_flat_body(const params &P, const dev_buffers &D,
                                                                                    int num_scan_tiles, blk bk) {
  __shared__ mf_tool_state s_tool;
  __shared__ ksum sm[FINISH_BLOCK / 32][4];
  __shared__ unsigned smc[FINISH_BLOCK / 32][4];
  if (P.has_tool) tool_load_shared(s_tool, D);
  const int q = bk.x * FINISH_BLOCK + threadIdx.x;
  const bool identity = P.verlet && !*(volatile unsigned *)&D.st->sort_now;
  const bool fuse = FUSE_PRED && identity && P.fuse;  // the next step's predictor runs here too
  (void)num_scan_tiles;
  double2 fc = make_double2(0., 0.), ft = make_double2(0., 0.);
  unsigned newly_blanked = 0, blanked_now = 0, oog = 0;
  bool want_sort = false;
  if (q < P.N) {
    double2 pos;
    unsigned f;
    finish_particle_phased<FUSE_PRED, CONDUCT>(P, D, s_tool, q, pos, f, fc, ft, newly_blanked, want_sort, identity,
                                               fuse);
    blanked_now = (f & FLAG_BLANKED) ? 1u : 0u;
    if (FUSE_HASH) {  // compute_hashes of the next step (grid.cu:34-51)
      const geom g = *D.g;
      long long hh;
      if (f & FLAG_BLANKED) {
        hh = D.hash_cur[q];
      } else {
        const int ix = __double2int_rz(P.verlet ? (pos.x - g.bbmin_x) * (1. / g.dx) : (pos.x - g.bbmin_x) / g.dx);
        const int iy = __double2int_rz(P.verlet ? (pos.y - g.bbmin_y) * (1. / g.dx) : (pos.y - g.bbmin_y) / g.dx);
        hh = (long long)ix * (long long)g.ny + (long long)iy;
      }
      if (hh < 0) { hh = 0; oog = 1; }
      else if (hh >= g.num_cell) { hh = g.num_cell - 1; oog = 1; }
      const int hsh = (int)hh;
      D.hash_new[q] = hsh;
      count_particle(D.count, D.tsum_w, hsh);  // read by the next step's scan
    }
  }
  // the block's force sums (compensated), in a fixed tree; warps whose forces are
  // all zero skip the arithmetic ({+0, +0} is what the sums give for zeros)
  const bool nz = fc.x != 0. || fc.y != 0. || ft.x != 0. || ft.y != 0.;
  const int w = threadIdx.x >> 5;
  if (__any_sync(0xffffffffu, nz)) {
    ksum fcx{0., 0.}, fcy{0., 0.}, ftx{0., 0.}, fty{0., 0.};
    ksum_add(fcx, fc.x);
    ksum_add(fcy, fc.y);
    ksum_add(ftx, ft.x);
    ksum_add(fty, ft.y);
    for (int o = 16; o > 0; o >>= 1) {
      ksum a{__shfl_down_sync(0xffffffffu, fcx.s, o), __shfl_down_sync(0xffffffffu, fcx.c, o)};
      ksum b{__shfl_down_sync(0xffffffffu, fcy.s, o), __shfl_down_sync(0xffffffffu, fcy.c, o)};
      ksum c{__shfl_down_sync(0xffffffffu, ftx.s, o), __shfl_down_sync(0xffffffffu, ftx.c, o)};
      ksum d{__shfl_down_sync(0xffffffffu, fty.s, o), __shfl_down_sync(0xffffffffu, fty.c, o)};
      ksum_merge(fcx, a); ksum_merge(fcy, b); ksum_merge(ftx, c); ksum_merge(fty, d);
    }
    if (lane_id() == 0) {
      sm[w][0] = fcx; sm[w][1] = fcy; sm[w][2] = ftx; sm[w][3] = fty;
    }
  } else if (lane_id() == 0) {
    const ksum z{0., 0.};
    sm[w][0] = z; sm[w][1] = z; sm[w][2] = z; sm[w][3] = z;
  }
  const unsigned nb = __reduce_add_sync(0xffffffffu, newly_blanked);
  const unsigned nbl = __reduce_add_sync(0xffffffffu, blanked_now);
  const unsigned noog = __reduce_add_sync(0xffffffffu, oog);
  const unsigned nws = __ballot_sync(0xffffffffu, want_sort);
  if (lane_id() == 0) {
    smc[w][0] = nb; smc[w][1] = nbl; smc[w][2] = noog; smc[w][3] = nws;
  }
  const bool block_nz = __syncthreads_or(nz);  // sm and smc complete
  // warp 0 closes the block (the block's sums into its partial, the counters, the ticket) and,
  // in the last block, the step; the other warps are done
  if (threadIdx.x >= 32) return;
  unsigned is_last = 0u;
  if (threadIdx.x == 0) {
    ksum r[4] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
    if (block_nz) {
      for (int k = 0; k < 4; ++k) r[k] = sm[0][k];
      for (int v = 1; v < FINISH_BLOCK / 32; ++v)
        for (int k = 0; k < 4; ++k) ksum_merge(r[k], sm[v][k]);
    }
    for (int k = 0; k < 4; ++k) {
      D.partials[(size_t)bk.x * 8 + 2 * k] = r[k].s;
      D.partials[(size_t)bk.x * 8 + 2 * k + 1] = r[k].c;
    }
    unsigned long long cnt[3] = {smc[0][0], smc[0][1], smc[0][2]};
    unsigned ws = smc[0][3];
    for (int v = 1; v < FINISH_BLOCK / 32; ++v) {
      for (int k = 0; k < 3; ++k) cnt[k] += smc[v][k];
      ws |= smc[v][3];
    }
    if (ws) D.st->want_sort = 1u;  // (before the fence and the ticket below)
    if (cnt[0]) atomicAdd(&D.st->newly_blanked, cnt[0]);
    if (cnt[1]) atomicAdd(&D.st->blanked, cnt[1]);
    if (cnt[2]) atomicAdd(&D.st->out_of_grid, cnt[2]);
    __threadfence();
    const int g = bk.x / FORCE_GROUP;
    const int gsize = min(FORCE_GROUP, bk.n - g * FORCE_GROUP);
    is_last = atomicAdd(&D.gticket[g], 1u) == (unsigned)(gsize - 1) ? 1u : 0u;
  }
  if (!__shfl_sync(0xffffffffu, is_last, 0)) return;
  // this block completed its group: the group's sum, then the group ticket
  __threadfence();
  const int g = bk.x / FORCE_GROUP;
  const int ng = (bk.n + FORCE_GROUP - 1) / FORCE_GROUP;
  double *gsums = D.partials + (size_t)bk.n * 8;
  ksum r[4];
  force_group_sum(D.partials, g, bk.n, r);
  unsigned last = 0u;
  if (lane_id() == 0) {
    store_ksum4(gsums + (size_t)g * 8, r);
    D.gticket[g] = 0u;
    __threadfence();
    last = atomicAdd(&D.ticket[0], 1u) == (unsigned)(ng - 1) ? 1u : 0u;
  }
  if (!__shfl_sync(0xffffffffu, last, 0)) return;
  __threadfence();
  force_final_sum(gsums, ng, r);
  if (lane_id() == 0) force_close_step(P, D, r, fuse, !identity);
}

template <bool FUSE_HASH, bool FUSE_PRED, bool CONDUCT = false>
__global__ void __launch_bounds__(FINISH_BLOCK, FINISH_FLAT_MIN_BLOCKS) k_finish_flat(params P, dev_buffers D, int num_scan_tiles) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  finish_flat_body<FUSE_HASH, FUSE_PRED, CONDUCT>(P, D, num_scan_tiles, grid_blk());
}

// JC plasticity (actions_gpu.cu:226-285) for the particles the finish kernel listed: the
// yield test its lower bound left open, then for those that yield the secant solve
// (plasticity.cuh:85-119), the stress scaled back to the yield surface, the plastic work to
// heat, then the thermal boundary condition the finish kernel applied before the return map
// had run (actions_gpu.cu:300-311).
//
// The list is short and its time is set by the particles whose secant needs the most
// iterations, so the length of one iteration matters. With the Johnson-Cook law (PAIRED) two
// lanes share one particle: a secant iteration needs the yield stress at delta_lambda (lane 0)
// and at 1.01 delta_lambda (lane 1), each pow(eps, n) times a rate factor (log or pow); both
// lanes run the same calls on their own operands at once, and shuffles exchange the results.
// Both lanes then evaluate the reference's expressions on the same operands, so the iterates
// are those of the one-lane solve. The tanh law takes the one-lane path.
struct secant_in {
  double norm_Strial, eps_pl, eps_pl_dot, term_c;
};

// yield stress from its two transcendental factors (sigma_yield's own expression order)
__device__ __forceinline__ double jc_yield_from(const mf_joco_constants &jc, double pow_eps_n, double term_b,
                                                double term_c) {
  double Term_A = jc.A + jc.B * pow_eps_n;
  return Term_A * term_b * term_c;
}

// the rate factor of sigma_yield (plasticity.cuh:35-39)
__device__ __forceinline__ double jc_rate_factor(const mf_joco_constants &jc, double eps_pl_dot) {
  double eps_dot = eps_pl_dot / jc.eps_dot_ref;
  if (eps_dot > 1.0) return 1.0 + jc.C * log(eps_dot);
  return pow((1.0 + eps_dot), jc.C);
}

// one lane pair's secant solve; sub = lane within the pair, pmask = the pair's lanes
__device__ __forceinline__ double solve_secant_pair(const mf_joco_constants &jc, const secant_in &in, double dt,
                                                    double mu, int sub, unsigned pmask, bool &capped,
                                                    int &iterations) {
  const double tol = 1e-6;
  const double s23 = sqrt(2.0 / 3.0);
  double delta_lambda = fmax(in.eps_pl_dot * dt * sqrt(2. / 3.), 1e-8);
  double delta_lambda_old = delta_lambda;
  int iter = 0;
  const int max_iter = 100;
  capped = false;
  while (true) {
    ++iterations;
    const double delta_lambda_1 = delta_lambda * 1.01;
    // opt_fun (plasticity.cuh:74-83) at delta_lambda on lane 0, at delta_lambda_1 on lane 1
    const double dl = sub == 0 ? delta_lambda : delta_lambda_1;
    const double e = in.eps_pl + s23 * fmax(dl, 0.);
    const double ed = s23 * fmax(dl, 0.) / dt;
    const double sY = jc_yield_from(jc, pow(e, jc.n), jc_rate_factor(jc, ed), in.term_c);
    const double g_own = in.norm_Strial - 2 * mu * dl - s23 * sY;
    const double g = __shfl_sync(pmask, g_own, 0, 2);
    const double g_1 = __shfl_sync(pmask, g_own, 1, 2);
    const double slope = (g - g_1) / (delta_lambda - delta_lambda_1);
    delta_lambda_old = delta_lambda;
    delta_lambda = delta_lambda - g / slope;
    if (delta_lambda < 0.) delta_lambda = -0.1 * delta_lambda;
    if (fabs(delta_lambda - delta_lambda_old) < tol) return delta_lambda;
    if (iter > max_iter) { capped = true; return delta_lambda; }
    iter++;
  }
}

template <bool PAIRED>
__device__ __forceinline__ void plastic_body(const params &P, const dev_buffers &D, blk bk) {
  __shared__ mf_joco_constants s_jc;  // by reference into the out-of-line functions
  __shared__ unsigned long long s_cnt[BLOCK / 32][2];
  if (threadIdx.x == 0) s_jc = P.joco;
  __syncthreads();
  const mf_joco_constants &JC = s_jc;
  const unsigned n = *D.plastic_count;
  const state_set &B = D.B;
  const double dt = P.dt, mu = P.phys.G;
  // neighbour lists: the finish kernel ran the next step's predictor; redone here where the
  // return map changes the state
  const bool fuse = P.verlet && D.st->predicted;
  constexpr unsigned LANES = PAIRED ? 2u : 1u;
  const unsigned sub = PAIRED ? (lane_id() & 1u) : 0u;
  const unsigned pmask = PAIRED ? (0x3u << (lane_id() & ~1u)) : 0xffffffffu;
  unsigned capped = 0u, iters_sum = 0u;
  const unsigned stride = bk.n * blockDim.x / LANES;
  for (unsigned i = (bk.x * blockDim.x + threadIdx.x) / LANES; i < n; i += stride) {
    const plastic_item it = D.plastic_list[i];
    const int q = it.q;
    double T = it.T;
    const double eps_pl = B.eps_pl[q], eps_pl_dot = B.eps_pl_dot[q];
    // one temperature for the whole return map: its temperature-only factors once
    const jc_temp_terms tt = jc_temperature_terms(JC, P.jc_model, T);
    if (it.svm < sigma_yield(JC, eps_pl, eps_pl_dot, tt)) {  // elastic after all
      if (sub == 0) {
        B.eps_pl_dot[q] = 0.;
        if (fuse) D.A.eps_pl_dot[q] = 0.;
      }
      continue;
    }
    const double4 S = B.S[q];
    const double rho = B.rho[q];
    const unsigned f = B.flags[q];
    const double Sxx = S.x, Syy = S.z, Szz = S.w, Sxy = S.y;
    const double norm_Strial = (double)sqrtf((float)(Sxx * Sxx + Syy * Syy + Szz * Szz + Sxy * Sxy));
    bool cap = false;
    int iters = 0;
    double delta_lambda;
    if (PAIRED) {
      const secant_in in{norm_Strial, eps_pl, eps_pl_dot, tt.term_c};
      delta_lambda = solve_secant_pair(JC, in, dt, mu, (int)sub, pmask, cap, iters);
    } else {
      delta_lambda = solve_secant(JC, P.jc_model, fmax(eps_pl_dot * dt * sqrt(2. / 3.), 1e-8), 1e-6, norm_Strial,
                                  eps_pl, tt, dt, mu, cap, iters);
    }
    const float s23f = sqrtf((float)(2.0 / 3.0));
    const double eps_pl_new = eps_pl + (double)(s23f * fmaxf((float)delta_lambda, 0.f));
    const double eps_pl_dot_new = (double)(s23f * fmaxf((float)delta_lambda, 0.f)) / dt;
    if (P.trml_wp.tq != 0.) {
      double sY;
      if (PAIRED) {  // sigma_yield(eps_pl_new, eps_pl_dot_new), on both lanes
        sY = jc_yield_from(JC, pow(eps_pl_new, JC.n), jc_rate_factor(JC, eps_pl_dot_new), tt.term_c);
      } else {
        sY = sigma_yield(JC, eps_pl_new, eps_pl_dot_new, tt);
      }
      const double delta_eps_pl = eps_pl_new - eps_pl;
      T += P.trml_wp.tq / (P.trml_wp.cp * rho) * delta_eps_pl * sY;
    }
    if (P.thermal_bc && (f & FLAG_FIXED)) T = P.trml_wp.T_init;
    if (sub == 0) {
      double4 Sn;
      Sn.x = Sxx - Sxx / norm_Strial * delta_lambda * 2. * mu;
      Sn.z = Syy - Syy / norm_Strial * delta_lambda * 2. * mu;
      Sn.w = Szz - Szz / norm_Strial * delta_lambda * 2. * mu;
      Sn.y = Sxy - Sxy / norm_Strial * delta_lambda * 2. * mu;
      B.S[q] = Sn;
      B.eps_pl[q] = eps_pl_new;
      B.eps_pl_dot[q] = eps_pl_dot_new;
      B.T[q] = T;
      if (fuse) {
        const state_set &N1 = D.A;
        N1.eps_pl[q] = eps_pl_new;
        N1.eps_pl_dot[q] = eps_pl_dot_new;
        predict_particle<true>(P, D, N1, q, D.hash_cur[q], B.pos[q], B.vel[q], Sn, rho, T, B.pos_t[q], B.vel_t[q],
                               B.S_t[q], B.rho_t[q], B.T_t[q], f, B.h[q], false);
      }
      capped += cap ? 1u : 0u;
      iters_sum += (unsigned)iters;
    }
  }
  const unsigned nc = __reduce_add_sync(0xffffffffu, capped);
  const unsigned ni = __reduce_add_sync(0xffffffffu, iters_sum);
  if (lane_id() == 0) {
    s_cnt[threadIdx.x >> 5][0] = nc;
    s_cnt[threadIdx.x >> 5][1] = ni;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long c = 0, itn = 0;
    for (int w = 0; w < BLOCK / 32; ++w) {
      c += s_cnt[w][0];
      itn += s_cnt[w][1];
    }
    if (c) atomicAdd(&D.st->secant_cap_hits, c);
    if (itn) atomicAdd(&D.st->secant_iterations, itn);
  }
}

template <bool PAIRED>
static __global__ void __launch_bounds__(BLOCK, PLASTIC_BLOCKS_PER_SM) k_plastic(params P, dev_buffers D) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  plastic_body<PAIRED>(P, D, grid_blk());
}

// Usui tool wear rate (tool_wear.cu:20-64) on the current state, on the device instead of
// after six device-to-host copies: for every particle in contact (fc.x, fc.y, ft.x or fc.y
// nonzero - the reference tests fc.y twice and never ft.y), K exp(alpha/T) p |v_r| with
// p = |fc| / (2 pi h) and v_r = v - v*n component-wise, v = vel - tool velocity. out = min,
// max and mean over those particles (0 when none), the sum compensated.
static __global__ void __launch_bounds__(BLOCK) k_usui(int N, state_set S, dev_buffers D, const mf_tool_state *tool,
                                                       double K, double alpha, double *out) {
  __shared__ double smn[BLOCK / 32], smx[BLOCK / 32];
  __shared__ ksum ssum[BLOCK / 32];
  __shared__ unsigned scnt[BLOCK / 32];
  __shared__ bool last;
  const double BIG = 3.402823466e+38;  // FLT_MAX, the reference's start value
  const double tvx = tool->vel[0], tvy = tool->vel[1];
  double mn = BIG, mx = 0.;
  ksum total{0., 0.};
  unsigned count = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double2 fc = S.fc[i], ft = S.ft[i];
    if (!(fabs(fc.x) > 0. || fabs(fc.y) > 0. || fabs(ft.x) > 0. || fabs(fc.y) > 0.)) continue;
    ++count;
    const double2 v = S.vel[i], nn = D.n[i];
    const double vx = v.x - tvx, vy = v.y - tvy;
    const double vrx = vx - vx * nn.x, vry = vy - vy * nn.y;
    const double vmag = sqrt(vrx * vrx + vry * vry);
    const double fmag = sqrt(fc.x * fc.x + fc.y * fc.y);
    const double A = 2 * S.h[i] * 3.14159265358979323846;
    const double pr = fmag / A;
    const double w = K * exp(alpha / S.T[i]) * pr * vmag;
    ksum_add(total, w);
    mn = fmin(mn, w);
    mx = fmax(mx, w);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    ksum b{__shfl_down_sync(0xffffffffu, total.s, o), __shfl_down_sync(0xffffffffu, total.c, o)};
    ksum_merge(total, b);
  }
  count = __reduce_add_sync(0xffffffffu, count);
  if (lane_id() == 0) {
    smn[threadIdx.x >> 5] = mn;
    smx[threadIdx.x >> 5] = mx;
    ssum[threadIdx.x >> 5] = total;
    scnt[threadIdx.x >> 5] = count;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < BLOCK / 32; ++w) {
      mn = fmin(mn, smn[w]);
      mx = fmax(mx, smx[w]);
      ksum_merge(total, ssum[w]);
      count += scnt[w];
    }
    double *pr = D.partials + (size_t)blockIdx.x * 8;
    pr[0] = mn; pr[1] = mx; pr[2] = total.s; pr[3] = total.c; pr[4] = (double)count;
    __threadfence();
    const unsigned t = atomicAdd(&D.ticket[2], 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double rmn = BIG, rmx = 0., rc = 0.;
  ksum rs{0., 0.};
  for (unsigned b = 0; b < gridDim.x; ++b) {
    const volatile double *pr = D.partials + (size_t)b * 8;
    rmn = fmin(rmn, pr[0]);
    rmx = fmax(rmx, pr[1]);
    ksum x{pr[2], pr[3]};
    ksum_merge(rs, x);
    rc += pr[4];
  }
  out[0] = rc == 0. ? 0. : rmn;
  out[1] = rmx;
  out[2] = rc == 0. ? 0. : (rs.s + rs.c) / rc;
  D.ticket[2] = 0u;
}

// report_force on the current state without stepping (output.cu:31-39)
static __global__ void __launch_bounds__(BLOCK) k_force_only(int N, const double2 *__restrict__ fc,
                                                      const double2 *__restrict__ ft, dev_buffers D) {
  __shared__ ksum sm[BLOCK / 32][4];
  ksum r[4] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    double2 a = fc[i], b = ft[i];
    ksum_add(r[0], a.x); ksum_add(r[1], a.y); ksum_add(r[2], b.x); ksum_add(r[3], b.y);
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 4; ++k) {
      ksum x{__shfl_down_sync(0xffffffffu, r[k].s, o), __shfl_down_sync(0xffffffffu, r[k].c, o)};
      ksum_merge(r[k], x);
    }
  if (lane_id() == 0)
    for (int k = 0; k < 4; ++k) sm[threadIdx.x >> 5][k] = r[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < BLOCK / 32; ++w)
      for (int k = 0; k < 4; ++k) ksum_merge(r[k], sm[w][k]);
    D.force_last[0] = (r[0].s + r[0].c) + (r[2].s + r[2].c);
    D.force_last[1] = (r[1].s + r[1].c) + (r[3].s + r[3].c);
  }
}

}  // namespace mf
