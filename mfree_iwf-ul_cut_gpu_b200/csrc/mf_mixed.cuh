// Mixed-precision pair kernel: the pair sums, strain rates and heat fluxes in FP32, on
// particle coordinates stored relative to the origin of their own cell; the predictor,
// corrector (leap-frog accumulation), JC return map and the tool-force reduction stay FP64.
//
// Same neighbour set and order as the plain form (interactions_gpu.cu:147-345); the
// differences are the arithmetic type and these exact rewrites:
//   * x_ij = (ci - cj) * dx + (xi_rel - xj_rel) and y_ij likewise: a small integer times the
//     cell size plus a difference of in-cell offsets, instead of a difference of absolute
//     coordinates;
//   * (e_ij . grad W) / r = der * fac (Brookshaw), one rsqrt per pair for 1/r;
//   * temperatures are stored relative to the initial temperature, so Ti - Tj keeps its
//     digits near it.
// Its error against the FP64 form is measured and reported, not assumed.
#pragma once

#include "mf_kernels.cuh"

namespace mf {

// the i particle's values and the pair sums of one thread
struct mixed_i {
  float x, y, sxy, Rxy, h, rho, c, T;
  float2 nv;      // (-vx, -vy)
  float2 s_diag;  // (sxx, syy)
  float2 r_diag;  // (Rxx, Ryy)
  float h1, fourh2, fac;
  bool mech, thermal, nonfinite;
};
// Lane pairs for the packed FP32 instructions of sm_100 (two FMAs per issue). The constant
// factors of a sum are applied once at the end: the stress and viscosity sums without the
// mass, XSPH without mass * eps, the Brookshaw sum without its factor 2.
struct mixed_acc {
  float2 vd01, vd23;  // (vdx, vdy), (vdz, vdw)
  float2 sd_xw;       // (sdx, sdw) / mass
  float2 sd_zy;       // (sdz, sdy) / mass
  float2 vt;          // (vtx, vty) / mass
  float2 xt;          // (xtx, xty) / (mass * eps)
  float T_lapl;       // / 2
};
struct mixed_const {
  float inv_wdeltap, alpha, beta, eta2;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// r^2 with its one fused multiply-add written out, so that every kernel that tests or uses a
// pair's distance (window, list build, list) rounds it the same way: the list form and the
// window form then give the same sums bit for bit on a step that builds the lists
__device__ __forceinline__ float dist2(float x, float y) { return fmaf(x, x, __fmul_rn(y, y)); }

// one neighbour j (records b0..b3) of particle i at offset (xij, yij)
__device__ __forceinline__ void mixed_interact(const mixed_i &I, const mixed_const &K, mixed_acc &a, float xij,
                                               float yij, const float4 &b0, const float4 &b1, const float4 &b2,
                                               const float4 &b3) {
  const unsigned fjw = (unsigned)__float_as_int(b0.z);
  const float rr2 = dist2(xij, yij);
  const bool in_support = !(rr2 >= I.fourh2 || rr2 < 1e-8f);
  // the reference's cubic spline (kernels.cuh:30-70), its value (2 - q)^6 / 4 for q > 1 (sic:
  // _2mq2 cubed) included. (Evaluating both branches and selecting, to keep a warp's lanes
  // together, measured 8 us slower on the ~150k-particle cut.)
  float w = 0.f, dwr = 0.f;
  if (in_support) {
    const float rinv = rsqrtf(rr2);
    const float qq = rr2 * rinv * I.h1;
    float val, der;
    if (qq > 1.f) {
      const float t = 2.f - qq;
      const float t2 = t * t;
      val = 0.25f * t2 * t2 * t2;
      der = -0.75f * t2 * I.h1 * rinv;
    } else {
      val = fmaf(-1.5f * qq * qq, fmaf(-0.5f, qq, 1.f), 1.f);
      der = -3.0f * qq * fmaf(-0.75f, qq, 1.f) * I.h1 * rinv;
    }
    w = val * I.fac;
    dwr = der * I.fac;
  }
  const float2 pij = f2(xij, yij);
  const float2 w_xy = __fmul2_rn(f2(dwr, dwr), pij);
  const float volj = b3.z;
  if (I.mech && !(fjw & FLAG_TOOL)) {
    const float2 dv = __fadd2_rn(f2(b0.w, b1.x), I.nv);
    const float2 av = __fmul2_rn(dv, f2(volj, volj));
    a.vd01 = __ffma2_rn(f2(av.x, av.x), w_xy, a.vd01);
    a.vd23 = __ffma2_rn(f2(av.y, av.y), w_xy, a.vd23);
    float fab = w * K.inv_wdeltap;
    fab *= fab;
    fab *= fab;
    const float2 sd = __ffma2_rn(f2(fab, fab), __fadd2_rn(I.r_diag, f2(b2.x, b2.z)),
                                 __fadd2_rn(I.s_diag, f2(b1.y, b1.w)));
    const float sxy = fmaf(fab, I.Rxy + b2.y, I.sxy + b1.z);
    a.sd_xw = __ffma2_rn(sd, w_xy, a.sd_xw);
    a.sd_zy = __ffma2_rn(f2(sxy, sxy), w_xy, a.sd_zy);
    const float2 dvp = __fmul2_rn(dv, pij);
    const float vijposij = -(dvp.x + dvp.y);
    const float irhoij = __fdividef(2.f, I.rho + b3.x);
    if (vijposij < 0.f) {  // Monaghan viscosity for approaching pairs
      const float cij = 0.5f * (I.c + b3.y);
      const float hij = 0.5f * (I.h + b2.w);
      const float muij = hij * vijposij * __fdividef(1.f, fmaf(K.eta2 * hij, hij, rr2));
      const float npi = fmaf(K.alpha, cij, -K.beta * muij) * muij * irhoij;  // -pi_ij
      a.vt = __ffma2_rn(f2(npi, npi), w_xy, a.vt);
    }
    const float xs = w * irhoij;
    a.xt = __ffma2_rn(f2(xs, xs), dv, a.xt);
  }
  // Brookshaw: 2 (m/rho_j)(Ti - Tj)(e_ij . grad W)/r with (e_ij . grad W)/r = der*fac
  if (I.thermal && rr2 > 1e-16f) a.T_lapl = fmaf(volj * (I.T - b3.w), dwr, a.T_lapl);
}

// Records of the candidates in global memory, read through the read-only path (word k of
// record j at recf_word(k, j, N)). (A block's candidates staged in shared memory by bulk copies
// on one mbarrier measured 25-30 % slower on the ~150k-particle cut: fewer resident warps and
// the copy's wait before any arithmetic, against loads that L1 already served 84 % of.)
struct rec_global {
  const float4 *__restrict__ r;
  int N;
  __device__ __forceinline__ float4 p0(int j) const { return __ldg(r + recf_word(0, j, N)); }
  __device__ __forceinline__ void all(int j, float4 &b0, float4 &b1, float4 &b2, float4 &b3) const {
    b0 = __ldg(r + recf_word(0, j, N)); b1 = __ldg(r + recf_word(1, j, N));
    b2 = __ldg(r + recf_word(2, j, N)); b3 = __ldg(r + recf_word(3, j, N));
  }
};

// Neighbour list of particle q, built on a step that sorted: the candidates within
// 2 h_i + skin over the 7x7 cells around its own (the 5x5 window widened by one cell, which
// covers that radius for h_i up to the cell size), blanked ones left out, non-finite ones
// kept (their pair terms carry the NaN). Columns in x order and each column's range in array
// order, so the in-support candidates come in the order of the 5x5 window.
__device__ __forceinline__ int build_list(const dev_buffers &D, const rec_global &REC, int q,
                                          const mixed_i &I, const geom &g, int gi, int gj, float dxc,
                                          float skin) {
  const float R = 2.f * I.h + skin;
  const float R2 = R * R;
  const int low_i = gi - 3 < 0 ? 0 : gi - 3;
  const int low_j = gj - 3 < 0 ? 0 : gj - 3;
  const int high_i = gi + 4 > g.nx ? g.nx : gi + 4;
  const int high_j = gj + 4 > g.ny ? g.ny : gj + 4;
  unsigned *row = D.nlist + (size_t)q * LIST_CAP;
  int cnt = 0;
  for (int ii = low_i; ii < high_i; ++ii) {
    const int col = ii * g.ny;
    const int j0 = __ldg(D.off + col + low_j);
    const int j1 = __ldg(D.off + col + high_j);
    const float ox = fmaf((float)(gi - ii), dxc, I.x);
    const unsigned tag = (unsigned)(gi - ii + 3) << LIST_INDEX_BITS;
    for (int j = j0; j < j1; ++j) {
      const float4 b0 = REC.p0(j);
      const unsigned fjw = (unsigned)__float_as_int(b0.z);
      const float xij = ox - b0.x;
      const float yij = fmaf((float)(gj - (int)(fjw >> 8)), dxc, I.y - b0.y);
      const float rr2 = dist2(xij, yij);
      if (!(fjw & FLAG_BLANKED) && (!(rr2 >= R2) || (fjw & FLAG_NONFINITE))) {
        if (cnt < LIST_CAP) row[cnt] = (unsigned)j | tag;
        ++cnt;
      }
    }
  }
  if (cnt > LIST_CAP) {
    atomicOr(&D.st->error_flags, ERR_LIST_OVERFLOW);
    cnt = LIST_CAP;
  }
  D.ncount[q] = cnt;
  return cnt;
}

// The neighbour-list invariant by brute force (a diagnostic: all N^2 pairs). k_list_abs puts
// every particle's position in FP64 from its pair record (origin of the cell of the last sort
// plus the FP32 offset); k_list_check then requires of every particle i that has a list (not
// blanked, finite, not a tool particle without heat conduction) that each unblanked, finite j
// closer than 2 h_i (h_i of the record, less a 1e-5 relative margin; the pair kernel's
// zero-distance cut-off 1e-8 left out) is among the ncount[i] entries of its row.
// out[0] += such pairs, out[1] += those missing from the lists.
static __global__ void k_list_abs(int N, dev_buffers D, double2 *abs) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const float4 b0 = reinterpret_cast<const float4 *>(D.recf)[recf_word(0, j, N)];
  const geom g = *D.g;
  const int hj = D.hash_cur[j];
  const int cx = hj / g.ny, cy = hj - cx * g.ny;
  abs[j] = make_double2(g.bbmin_x + cx * g.dx + (double)b0.x, g.bbmin_y + cy * g.dx + (double)b0.y);
}

static __global__ void k_list_check(params P, dev_buffers D, const double2 *__restrict__ abs,
                                    unsigned long long *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.N) return;
  const float4 *__restrict__ r0 = reinterpret_cast<const float4 *>(D.recf);
  const unsigned fi = (unsigned)__float_as_int(r0[recf_word(0, i, P.N)].z) & 0xffu;
  if (fi & (FLAG_BLANKED | FLAG_NONFINITE)) return;
  if ((fi & FLAG_TOOL) && P.thermal_solver != MF_THERMAL_BROOKSHAW) return;  // no pair sums
  const double h = (double)r0[recf_word(2, i, P.N)].w;
  const double lim = 4. * h * h * (1. - 1e-5);
  const double2 xi = abs[i];
  const unsigned *row = D.nlist + (size_t)i * LIST_CAP;
  const int cnt = min(D.ncount[i], LIST_CAP);
  unsigned long long pairs = 0, missing = 0;
  for (int j = 0; j < P.N; ++j) {
    if (j == i) continue;
    const unsigned fj = (unsigned)__float_as_int(r0[recf_word(0, j, P.N)].z);
    if (fj & (FLAG_BLANKED | FLAG_NONFINITE)) continue;
    const double2 xj = abs[j];
    const double dx = xi.x - xj.x, dy = xi.y - xj.y;
    const double rr2 = dx * dx + dy * dy;
    if (!(rr2 < lim) || rr2 < 1e-8) continue;
    ++pairs;
    bool found = false;
    for (int k = 0; k < cnt && !found; ++k) found = (row[k] & LIST_INDEX_MASK) == (unsigned)j;
    if (!found) ++missing;
  }
  if (pairs) atomicAdd(out, pairs);
  if (missing) atomicAdd(out + 1, missing);
}

// The i particle of slot q: its records and the constants of its sums. False when q has no
// pair sums (past the end, blanked, a tool particle without Brookshaw heat).
__device__ __forceinline__ bool mixed_begin(const params &P, const dev_buffers &D, int q, mixed_i &I,
                                            mixed_const &K, double &thermal_alpha) {
  if (q >= P.N) return false;
  const float4 *__restrict__ r0 = reinterpret_cast<const float4 *>(D.recf);
  const float4 a0 = __ldg(r0 + recf_word(0, q, P.N));  // x, y, flags|cy, vx
  const unsigned fi = (unsigned)__float_as_int(a0.z) & 0xffu;
  if (fi & FLAG_BLANKED) return false;
  const bool tool_i = fi & FLAG_TOOL;
  const bool brookshaw = P.thermal_solver == MF_THERMAL_BROOKSHAW;
  if (!brookshaw && tool_i) return false;
  const float4 a1 = __ldg(r0 + recf_word(1, q, P.N));  // vy, sxx, sxy, syy
  const float4 a2 = __ldg(r0 + recf_word(2, q, P.N));  // Rxx, Rxy, Ryy, h
  const float4 a3 = __ldg(r0 + recf_word(3, q, P.N));  // rho, c, vol, T - T_init

  K.inv_wdeltap = (float)(1. / P.corr.wdeltap);
  K.alpha = (float)P.corr.alpha;
  K.beta = (float)P.corr.beta;
  const float eta = (float)P.corr.eta;
  K.eta2 = eta * eta;
  thermal_alpha = 0.;
  if (brookshaw) thermal_alpha = !tool_i ? P.trml_wp.alpha : (P.thermal_tool_on ? P.trml_tool.alpha : 0.);

  I.thermal = thermal_alpha != 0.;
  I.nonfinite = fi & FLAG_NONFINITE;
  I.mech = !tool_i;
  I.x = a0.x; I.y = a0.y; I.nv = f2(-a0.w, -a1.x);
  I.s_diag = f2(a1.y, a1.w); I.sxy = a1.z;
  I.r_diag = f2(a2.x, a2.z); I.Rxy = a2.y; I.h = a2.w;
  I.rho = a3.x; I.c = a3.y; I.T = I.thermal ? a3.w : 0.f;
  I.h1 = 1.f / I.h;
  I.fourh2 = 4.f * I.h * I.h;
  I.fac = 0.454728408833987f * I.h1 * I.h1;
  return true;
}

// The candidates j0 .. j1 - 1 of one window column (indices into R), in chunks of up to 32: mark
// the contributing ones, then visit them in order.
template <class REC>
__device__ __forceinline__ void mixed_column(const REC &R, int j0, int j1, float ox, int gj, float dxc,
                                             const mixed_i &I, const mixed_const &K, mixed_acc &acc) {
  for (int jb = j0; jb < j1; jb += 32) {
    const int jn = min(32, j1 - jb);
    unsigned mask = 0u;
#pragma unroll 4
    for (int k = 0; k < jn; ++k) {
      const float4 b0 = R.p0(jb + k);
      const unsigned fjw = (unsigned)__float_as_int(b0.z);
      const float xij = ox - b0.x;
      const float yij = fmaf((float)(gj - (int)(fjw >> 8)), dxc, I.y - b0.y);
      const float rr2 = dist2(xij, yij);
      const bool in_support = !(rr2 >= I.fourh2 || rr2 < 1e-8f);
      const bool take = !(fjw & FLAG_BLANKED) && (in_support || I.nonfinite || (fjw & FLAG_NONFINITE));
      mask |= (take ? 1u : 0u) << k;
    }
    while (mask) {
      const int k = __ffs(mask) - 1;
      mask &= mask - 1u;
      // all four planes at once: one load latency per neighbour
      float4 b0, b1, b2, b3;
      R.all(jb + k, b0, b1, b2, b3);
      const float yij = fmaf((float)(gj - (int)((unsigned)__float_as_int(b0.z) >> 8)), dxc, I.y - b0.y);
      mixed_interact(I, K, acc, ox - b0.x, yij, b0, b1, b2, b3);
    }
  }
}

// the rates of slot q from its pair sums: Jaumann stress rate, continuity, momentum, advection
// and heat (actions_gpu.cu:100-132, interactions_gpu.cu:331-345)
__device__ __forceinline__ void mixed_end(const params &P, const dev_buffers &D, int q, int p, const mixed_i &I,
                                          const mixed_acc &acc, double thermal_alpha) {
  const float mass = (float)P.phys.mass;
  const float m_eps = (float)P.corr.xspheps * mass;
  const float vdx = acc.vd01.x, vdy = acc.vd01.y, vdz = acc.vd23.x, vdw = acc.vd23.y;
  const float sdx = mass * acc.sd_xw.x, sdy = mass * acc.sd_zy.y, sdz = mass * acc.sd_zy.x,
              sdw = mass * acc.sd_xw.y;
  const float vtx = mass * acc.vt.x, vty = mass * acc.vt.y;
  const float xtx = m_eps * acc.xt.x, xty = m_eps * acc.xt.y, T_lapl = 2.f * acc.T_lapl;
  const bool mech_i = I.mech, thermal = I.thermal;
  const float rhoi = I.rho;

  const state_set &B = D.B;
  if (P.keep_derivs) {
    D.S_der[q] = make_double4(sdx, sdy, sdz, sdw);
    D.v_der[q] = make_double4(vdx, vdy, vdz, vdw);
  }
  if (mech_i) {
    const double4 S = B.S[q];
    const float G = (float)P.phys.G;
    const float e01 = 0.5f * (vdy + vdz);
    const float w01 = 0.5f * (vdz - vdy);
    const float t3 = (1.f / 3.f) * (vdx + vdw);
    const float Sxx = (float)S.x, Sxy = (float)S.y, Syy = (float)S.z;
    const float g2 = 2.f * G;
    // Jaumann rate with omega_10 = -omega_01 (actions_gpu.cu:120-132)
    const float tx = g2 * (vdx - t3) - 2.f * w01 * Sxy;
    const float ty = g2 * e01 + w01 * (Sxx - Syy);
    const float tz = g2 * (vdw - t3) + 2.f * w01 * Sxy;
    const float tw = -g2 * t3;
    B.S_t[q] = make_double4(tx, ty, tz, tw);
    B.rho_t[q] = -(double)rhoi * (double)(vdx + vdw);
    double2 fc, ft;
    prev_contact_forces(P, D, q, p, fc, ft);
    const double m = P.phys.mass;
    const double2 vp = B.vel[q];
    B.vel_t[q] = make_double2((double)(vtx + (sdx + sdy)) + fc.x / m + ft.x / m,
                              (double)(vty + (sdz + sdw)) + fc.y / m + ft.y / m);
    B.pos_t[q] = make_double2((double)xtx + vp.x, (double)xty + vp.y);
  } else {
    B.vel_t[q] = make_double2(vtx, vty);
    B.pos_t[q] = make_double2(xtx, xty);
  }
  if (thermal) B.T_t[q] = thermal_alpha * (double)T_lapl;
}

// LIST: the neighbour-list form (steps with P.verlet)
template <bool LIST>
__device__ __forceinline__ void pair_mixed_particle(const params &P, const dev_buffers &D, int q) {
  mixed_i I;
  mixed_const K;
  double thermal_alpha;
  if (!mixed_begin(P, D, q, I, K, thermal_alpha)) return;
  const rec_global R{reinterpret_cast<const float4 *>(D.recf), P.N};
  // the particle's slot at the start of the step (its last contact forces are read there at the
  // end): loaded now, so that the load's latency passes during the sums; a list step without a
  // sort keeps the order
  const bool sorting = !LIST || D.st->sort_now;
  const int p = sorting ? __ldg(D.perm + q) : q;

  const geom g = *D.g;
  const float dxc = (float)g.dx;
  const int hashi = D.hash_cur[q];
  const int gi = hashi / g.ny;
  const int gj = hashi - gi * g.ny;

  mixed_acc acc;
  acc.vd01 = acc.vd23 = acc.sd_xw = acc.sd_zy = acc.vt = acc.xt = f2(0.f, 0.f);
  acc.T_lapl = 0.f;

  if (LIST && !I.nonfinite) {
    // neighbour list: built on a sorting step, then read; each entry passes the same
    // support test as a window candidate. A particle's row is contiguous: four entries per
    // 16-byte load; an entry past the count reads the particle's own record (always valid,
    // so the loads need no guard) and is skipped.
    const int cnt = sorting ? build_list(D, R, q, I, g, gi, gj, dxc, P.skin) : D.ncount[q];
    const uint4 *row = reinterpret_cast<const uint4 *>(D.nlist + (size_t)q * LIST_CAP);
    uint4 e4 = row[0];  // (a row is LIST_CAP entries: the first four are always there)
    const unsigned self = (unsigned)q | (3u << LIST_INDEX_BITS);
    // software pipeline: the next entry's four record planes are in flight while one entry is
    // summed (c0..c3 hold entry k's at the top of its iteration; past the count, the particle's
    // own record, always a valid address). Measured on the ~150k-particle cut: pair kernel 48.1
    // against 50.1 us at 5 blocks per SM (96 registers, 4 B of spills); at 4 blocks per SM (108
    // registers) 54.2 us.
    float4 c0, c1, c2, c3;
    R.all((int)((cnt > 0 ? e4.x : self) & LIST_INDEX_MASK), c0, c1, c2, c3);
    for (int k0 = 0; k0 < cnt; k0 += 4) {
      const unsigned ev[4] = {e4.x, e4.y, e4.z, e4.w};
      if (k0 + 4 < cnt) e4 = row[(k0 >> 2) + 1];  // the next four, in flight during these
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool live = k0 + u < cnt;
        const unsigned e = live ? ev[u] : self;
        const unsigned en = (k0 + u + 1 < cnt) ? (u < 3 ? ev[u + 1] : e4.x) : self;
        const float ox = fmaf((float)((int)(e >> LIST_INDEX_BITS) - 3), dxc, I.x);
        const float4 b0 = c0, b1 = c1, b2 = c2, b3 = c3;
        R.all((int)(en & LIST_INDEX_MASK), c0, c1, c2, c3);
        const unsigned fjw = (unsigned)__float_as_int(b0.z);
        const float xij = ox - b0.x;
        const float yij = fmaf((float)(gj - (int)(fjw >> 8)), dxc, I.y - b0.y);
        const float rr2 = dist2(xij, yij);
        const bool in_support = !(rr2 >= I.fourh2 || rr2 < 1e-8f);
        if (live && !(fjw & FLAG_BLANKED) && (in_support || (fjw & FLAG_NONFINITE)))
          mixed_interact(I, K, acc, xij, yij, b0, b1, b2, b3);
      }
    }
  } else {  // the 5x5 window (interactions_gpu.cu:147-345)
    const int low_i = gi - 2 < 0 ? 0 : gi - 2;
    const int low_j = gj - 2 < 0 ? 0 : gj - 2;
    const int high_i = gi + 3 > g.nx ? g.nx : gi + 3;
    const int high_j = gj + 3 > g.ny ? g.ny : gj + 3;
    for (int ii = low_i; ii < high_i; ++ii) {
      const int col = ii * g.ny;
      const int j0 = __ldg(D.off + col + low_j);
      const int j1 = __ldg(D.off + col + high_j);
      mixed_column(R, j0, j1, fmaf((float)(gi - ii), dxc, I.x), gj, dxc, I, K, acc);
    }
  }
  mixed_end(P, D, q, p, I, acc, thermal_alpha);
}

// the mixed pair sums of block bk.x's particles
template <bool LIST>
__device__ __forceinline__ void pair_mixed_body(const params &P, const dev_buffers &D, blk bk) {
  pair_mixed_particle<LIST>(P, D, bk.x * blockDim.x + threadIdx.x);
}

// blocks per SM: the window kernel at 6 (80 registers, no spills); the list kernel at 5 (96
// registers with its software pipeline, 4 B of spills; before the pipeline, at 6 it spilled a
// little and ran ~1.5 us slower than at 5, at 9 with 56 registers 13 us slower)
template <bool LIST>
static __global__ void __launch_bounds__(PAIR_BLOCK, LIST ? 5 : 6) k_pair_mixed(params P, dev_buffers D) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  pair_mixed_body<LIST>(P, D, grid_blk());
}

// PSE heat Laplacian (interactions_gpu.cu:88-144, kernels.cuh:72-89) in FP32 for the mixed
// form, on the FP32 records: the same window (every particle of the 5x5 cells, blanked ones
// included, no support cut-off) and the same alpha through the half-length texture binding;
// exp from the hardware approximation, temperatures relative to the initial temperature.
__device__ __forceinline__ void pse_mixed_body(const params &P, const dev_buffers &D, blk bk) {
  const int q = bk.x * blockDim.x + threadIdx.x;
  if (q >= P.N) return;
  const float4 *__restrict__ r = reinterpret_cast<const float4 *>(D.recf);
  const float4 a0 = __ldg(r + recf_word(0, q, P.N));  // x, y, flags|cy, vx
  const unsigned fi = (unsigned)__float_as_int(a0.z) & 0xffu;
  if (fi & FLAG_BLANKED) return;
  const float hi = __ldg(r + recf_word(2, q, P.N)).w;
  const float Ti = __ldg(r + recf_word(3, q, P.N)).w;
  const long long tex_elems = ((long long)sizeof(int) * P.N) / 8;
  const bool tool_i = q < tex_elems ? (fi & FLAG_TOOL) != 0 : false;
  const double alpha = tool_i ? P.trml_tool.alpha : P.trml_wp.alpha;
  const float h2 = hi * hi;
  const float inv_h2 = 1.f / h2;
  const float coef = (float)(4. / 3.14159265358979323846) / (h2 * h2);
  const geom g = *D.g;
  const float dxc = (float)g.dx;
  const int hashi = D.hash_cur[q];
  const int gi = hashi / g.ny;
  const int gj = hashi - gi * g.ny;
  const int low_i = gi - 2 < 0 ? 0 : gi - 2;
  const int low_j = gj - 2 < 0 ? 0 : gj - 2;
  const int high_i = gi + 3 > g.nx ? g.nx : gi + 3;
  const int high_j = gj + 3 > g.ny ? g.ny : gj + 3;
  float T_ti = 0.f;
  for (int ii = low_i; ii < high_i; ++ii) {
    const int j0 = __ldg(D.off + ii * g.ny + low_j);
    const int j1 = __ldg(D.off + ii * g.ny + high_j);
    const float ox = (float)(gi - ii) * dxc + a0.x;
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
      const float4 b0 = __ldg(r + recf_word(0, j, P.N));
      const float4 b3 = __ldg(r + recf_word(3, j, P.N));  // rho, c, vol, T - T_init
      const float xij = ox - b0.x;
      const float yij = fmaf((float)(gj - (int)((unsigned)__float_as_int(b0.z) >> 8)), dxc, a0.y - b0.y);
      const float w2 = coef * __expf(-(xij * xij + yij * yij) * inv_h2);
      T_ti += (b3.w - Ti) * w2 * b3.z;
    }
  }
  D.B.T_t[q] = alpha * (double)T_ti;
}

static __global__ void __launch_bounds__(PAIR_BLOCK) k_pse_mixed(params P, dev_buffers D) {
  MF_PDL_WAIT();
  MF_PDL_TRIGGER();
  pse_mixed_body(P, D, grid_blk());
}

}  // namespace mf
