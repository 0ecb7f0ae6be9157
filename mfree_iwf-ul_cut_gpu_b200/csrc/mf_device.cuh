// Device-side types and per-particle physics shared by the sm_100a kernels.
//
// Each function cites the reference file:line whose arithmetic it keeps. The plain FP64
// form evaluates every expression in the reference's order and calls the same
// float-precision functions the reference calls on double arguments (sqrtf, atan2f, cosf,
// sinf, fmaxf), so that it matches the reference's FP64 build to rounding.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "mfree_b200.h"

namespace mf {

// particle flag bits (the reference stores fixed / blanked / tool_particle as 0/1 doubles)
constexpr unsigned FLAG_FIXED = 1u;
constexpr unsigned FLAG_BLANKED = 2u;
constexpr unsigned FLAG_TOOL = 4u;
constexpr unsigned FLAG_NONFINITE = 8u;  // pair record holds a NaN/Inf (set per step)

// one FP64 pair record per particle: what a neighbour j contributes to the pair sums,
// written once per step by the predictor kernel (16 doubles = one 128-byte line)
enum : int {
  R_X = 0, R_Y, R_VX, R_VY, R_SXX, R_SXY, R_SYY, R_RXX, R_RXY, R_RYY, R_H, R_RHO, R_C, R_VOL, R_T, R_FLAGS,
  R_WIDTH
};

// FP32 pair record of the mixed form (16 floats = 64 bytes): coordinates relative to the
// origin of the particle's own cell; the first 16 bytes (x, y, flags | cell_y << 8, vx) are
// all the distance test needs
enum : int {
  F_X = 0, F_Y, F_FLAGS, F_VX, F_VY, F_SXX, F_SXY, F_SYY, F_RXX, F_RXY, F_RYY, F_H, F_RHO, F_C, F_VOL, F_T,
  F_WIDTH
};

// index of float4 word k (0..3) of particle j's FP32 pair record among N records: four planes,
// word k of every particle together at k N + j. (Each particle's 64 bytes together, at 4 j + k,
// measured 68 % slower in the list pair kernel: a warp's 16-byte loads then touch four times as
// many cache lines, and L1 throughput becomes the limit.)
__host__ __device__ __forceinline__ size_t recf_word(int k, int j, int N) {
  return (size_t)k * (size_t)N + (size_t)j;
}

struct params {
  int N;
  int grid_kind;
  int thermal_solver;
  int jc_model;
  int precision;
  int plastic, fric_heat, thermal_bc, thermal_wp, thermal_tool_on, has_tool, keep_derivs;
  int staged;  // step run stage by stage (mf_step_stage): keep every intermediate array
  int jc_lower_bound;  // A > 0, B >= 0, C >= 0: the yield stress is bounded below by A (1 - theta^m)
  // mixed form with neighbour lists: the cell list is sorted only on steps where some
  // particle's predicted position is more than 0.45 skin from where its list was built; in
  // between, each particle's candidates within 2 h + skin are kept in a list
  int verlet;
  int fuse;  // neighbour lists: the finish kernel also runs the next step's predictor
  float skin;
  double eos_c0;  // (double)sqrtf((float)(K / rho0)), the EOS sound speed (actions_gpu.cu:41-51)
  double dt;
  // tool-workpiece contact conductance (an extension without a reference counterpart, off at
  // 0): a workpiece particle in contact with the tool exchanges h_contact (T_contact - T) per
  // unit contact length with a tool surface at T_contact
  double h_contact, T_contact;
  mf_phys_constants phys;
  mf_corr_constants corr;
  mf_joco_constants joco;
  mf_trml_constants trml_wp, trml_tool;
};

struct geom {
  int nx, ny, num_cell, max_cell;
  double bbmin_x, bbmin_y, bbmax_x, bbmax_y, dx;
  int locked;
  int pad;
};

// device status counters (reset by the host)
struct dev_status {
  unsigned long long out_of_grid;
  unsigned long long newly_blanked;
  unsigned long long secant_cap_hits;
  unsigned long long blanked;
  unsigned long long steps;
  int max_cell_occupancy;
  int error_flags;
  unsigned int force_ticket;
  unsigned int scan_tile_counter;  // (unused: the cell scan takes no tile tickets)
  unsigned long long force_log_head;
  unsigned long long secant_iterations;
  unsigned long long sorts;  // cell-list sorts (every step, except with neighbour lists)
  unsigned int sort_now;     // neighbour lists: this step sorts (set by the previous step)
  unsigned int want_sort;    // neighbour lists: a particle's next predicted position is more
                             // than 0.45 skin from where its list was built
  unsigned int sorted_prev;  // the last step sorted the cell list: the set this step writes
                             // holds the order of two steps ago, so this step's reorder writes
                             // the order, particle numbers and smoothing lengths again
  unsigned int predicted;    // neighbour lists: the last finish kernel also ran the next step's
                             // predictor (it did not follow a sort); the next step, if it does
                             // not sort, skips the reorder kernel
};

constexpr int FORCE_LOG_CAP = 1 << 16;
constexpr int ERR_SCAN_WAIT = 1;  // (no longer raised: the cell scan has no bounded waits)
constexpr int ERR_GRID_BUDGET = 2;
constexpr int ERR_LIST_OVERFLOW = 4;  // a neighbour list was full: neighbours were dropped
constexpr int ERR_BATCH_WAIT = 8;     // a persistent batch launch's grid barrier wait expired

// neighbour list entry: particle index in the low LIST_INDEX_BITS bits, above them the
// column offset of the pair's cells (i's column - j's column) + 3, in [0, 6]
constexpr int LIST_CAP = 64;
constexpr int LIST_INDEX_BITS = 26;
constexpr unsigned LIST_INDEX_MASK = (1u << LIST_INDEX_BITS) - 1u;

// ---------------------------------------------------------------------------------------
// SPH kernel function: cubic spline (kernels.cuh:30-70). hi enters through h1 = 1/hi and
// fourh2 = 4*hi*hi, computed once per particle i exactly as the reference computes them
// per pair. Returns false (w = 0) outside the support or for r^2 < 1e-8.
// Also returns dwr = der*fac, the radial factor of the gradient (grad W = dwr * x_ij), which
// is (e_ij . grad W) / r of the Brookshaw Laplacian.
__device__ __forceinline__ void cubic_spline_fp64(double xij, double yij, double rr2, double h1,
                                                  double &w, double &w_x, double &w_y, double &dwr) {
  constexpr double PI_FAC = 0.454728408833987;
  double der, val;
  double rad = (double)sqrtf((float)rr2);
  double q = rad * h1;
  double fac = PI_FAC * h1 * h1;
  if (q > 1) {
    double _2mq = 2 - q;
    double _2mq2 = _2mq * _2mq;
    val = 0.25 * _2mq2 * _2mq2 * _2mq2;
    der = -0.75 * _2mq2 * h1 / rad;
  } else {
    val = 1 - 1.5 * q * q * (1 - 0.5 * q);
    der = -3.0 * q * (1 - 0.75 * q) * h1 / rad;
  }
  w = val * fac;
  w_x = der * xij * fac;
  w_y = der * yij * fac;
  dwr = der * fac;
}

// PSE Laplacian kernel (kernels.cuh:72-89)
__device__ __forceinline__ double lapl_pse_fp64(double xij, double yij, double hi) {
  double xx = sqrt(xij * xij + yij * yij);
  double h2 = hi * hi;
  double h4 = h2 * h2;
  return +4. / (h4 * 3.14159265358979323846) * exp(-xx * xx / (h2));
}

// ---------------------------------------------------------------------------------------
// artificial stress (actions_gpu.cu:35-39, 53-97)
__device__ __forceinline__ void artificial_stress(double rhoi, double pi, double Sx, double Sy, double Sz,
                                                  double eps, double &Rxx, double &Rxy, double &Ryy) {
  double sxx = Sx - pi;
  double sxy = Sy;
  double syy = Sz - pi;
  double rhoi21 = 1. / (rhoi * rhoi);
  double numer = 2. * sxy;
  double denom = sxx - syy + 0.;
  double theta = 0.5 * (double)atan2f((float)numer, (float)denom);
  double cos_theta = (double)cosf((float)theta);
  double sin_theta = (double)sinf((float)theta);
  double cos_theta2 = cos_theta * cos_theta;
  double sin_theta2 = sin_theta * sin_theta;
  double rot_sxx = cos_theta2 * sxx + 2.0 * cos_theta * sin_theta * sxy + sin_theta2 * syy;
  double rot_syy = sin_theta2 * sxx - 2.0 * cos_theta * sin_theta * sxy + cos_theta2 * syy;
  double rot_rxx = 0., rot_ryy = 0.;
  if (rot_sxx > 0) rot_rxx = -eps * rot_sxx * rhoi21;
  if (rot_syy > 0) rot_ryy = -eps * rot_syy * rhoi21;
  Rxx = cos_theta2 * rot_rxx + sin_theta2 * rot_ryy;
  Rxy = cos_theta * sin_theta * (rot_rxx - rot_ryy);
  Ryy = sin_theta2 * rot_rxx + cos_theta2 * rot_ryy;
}

// The same in float for the mixed form's FP32 records, from rho21 = 1 / rho^2: the angle and
// its cosine and sine are the reference's float ones; the deviatoric parts are rounded once.
__device__ __forceinline__ void artificial_stress_f(double rhoi21, double pi, double Sx, double Sy, double Sz,
                                                    double eps, float &Rxx, float &Rxy, float &Ryy) {
  const float sxx = (float)(Sx - pi), sxy = (float)Sy, syy = (float)(Sz - pi);
  const float theta = 0.5f * atan2f(2.f * sxy, (float)((Sx - pi) - (Sz - pi)));
  const float c = cosf(theta), s = sinf(theta);
  const float c2 = c * c, s2 = s * s, cs = c * s;
  const float rot_sxx = c2 * sxx + 2.f * cs * sxy + s2 * syy;
  const float rot_syy = s2 * sxx - 2.f * cs * sxy + c2 * syy;
  const float er = -(float)eps * (float)rhoi21;
  const float rot_rxx = rot_sxx > 0.f ? er * rot_sxx : 0.f;
  const float rot_ryy = rot_syy > 0.f ? er * rot_syy : 0.f;
  Rxx = c2 * rot_rxx + s2 * rot_ryy;
  Rxy = cs * (rot_rxx - rot_ryy);
  Ryy = s2 * rot_rxx + c2 * rot_ryy;
}

// Jaumann stress rate (actions_gpu.cu:99-133). The reference builds 3x3 GLM matrices; the
// entries that are structurally zero drop out exactly, leaving these sums in GLM's order.
__device__ __forceinline__ void jaumann(double G, double vx_x, double vx_y, double vy_x, double vy_y, double Sxx,
                                        double Sxy, double Syy, double Szz, double &tx, double &ty, double &tz,
                                        double &tw) {
  double e01 = 0.5 * (vx_y + vy_x);
  double w01 = 0.5 * (vy_x - vx_y);  // omega[0][1]
  double w10 = 0.5 * (vx_y - vy_x);  // omega[1][0]
  double tr = vx_x + vy_y + 0.;
  double t3 = (double)(1. / 3.) * tr;
  double g2 = (double)(2.) * G;
  // (omega*S)[c][r] = omega[0][r] S[c][0] + omega[1][r] S[c][1] + omega[2][r] S[c][2]
  double oS00 = 0. * Sxx + w10 * Sxy;  // + 0*0
  double oS01 = w01 * Sxx + 0. * Sxy;
  double oS11 = w01 * Sxy + 0. * Syy;
  // (S*omega^T)[c][r] = S[0][r] omega[0][c] + S[1][r] omega[1][c] + S[2][r] omega[2][c]
  double So00 = Sxx * 0. + Sxy * w10;
  double So01 = Sxy * 0. + Syy * w10;
  double So11 = Sxy * w01 + Syy * 0.;
  tx = (g2 * (vx_x - t3) + (oS00 + 0.)) + (So00 + 0.);
  ty = (g2 * (e01 - t3 * 0.) + (oS01 + 0.)) + (So01 + 0.);
  tz = (g2 * (vy_y - t3) + (oS11 + 0.)) + (So11 + 0.);
  tw = (g2 * (0. - t3) + 0.) + 0.;
}

// ---------------------------------------------------------------------------------------
// Johnson-Cook flow stress (plasticity.cuh:30-46) and the tanh variant (:48-70). Kept out of
// line: each call holds several pow/log expansions, and one copy keeps the instruction cache
// and the caller's register budget small.
// The yield stress (plasticity.cuh:30-46, 48-70). The factors that depend on the temperature
// alone are computed once per particle (jc_temperature_terms) and passed in: the return map
// evaluates the yield stress many times at one temperature. Every factor is the value the
// reference computes, combined in the reference's order, so the result is the same double.
struct jc_temp_terms {
  double term_c;  // 1 - theta^m
  double tanh_d;  // tanh model: 1 - (T/Tm)^d
  double tanh_s;  // tanh model: (T/Tm)^b
};

__device__ __forceinline__ jc_temp_terms jc_temperature_terms(const mf_joco_constants &jc, int model, double t) {
  jc_temp_terms r;
  const double theta = (t - jc.Tref) / (jc.Tmelt - jc.Tref);
  r.term_c = 1.0 - pow(theta, jc.m);
  r.tanh_d = 0.;
  r.tanh_s = 0.;
  if (model == MF_JC_TANH) {
    r.tanh_d = 1.0 - pow((t / jc.Tmelt), jc.tanh_d);
    r.tanh_s = pow(t / jc.Tmelt, jc.tanh_b);
  }
  return r;
}

static __device__ __noinline__ double sigma_yield(const mf_joco_constants &jc, double eps_pl, double eps_pl_dot,
                                              const jc_temp_terms &tt) {
  double Term_A = jc.A + jc.B * pow(eps_pl, jc.n);
  double Term_B = 1.0;
  double eps_dot = eps_pl_dot / jc.eps_dot_ref;
  if (eps_dot > 1.0) Term_B = 1.0 + jc.C * log(eps_dot);
  else Term_B = pow((1.0 + eps_dot), jc.C);
  return Term_A * Term_B * tt.term_c;
}

static __device__ __noinline__ double sigma_yield_tanh(const mf_joco_constants &jc, double eps_pl, double eps_dot_pl,
                                                   const jc_temp_terms &tt) {
  double Term_A = jc.A + jc.B * pow(eps_pl, jc.n) * 1.0 / exp(pow(eps_pl, jc.tanh_a));
  double Term_B = 1.0;
  double eps_dot = eps_dot_pl / jc.eps_dot_ref;
  if (eps_dot > 1.0) Term_B = 1.0 + jc.C * log(eps_dot);
  else Term_B = pow((1.0 + eps_dot), jc.C);
  double Term_D = tt.tanh_d + (1.0 - tt.tanh_d) * tanh(1.0 / (pow(eps_pl + tt.tanh_s, jc.tanh_c)));
  return Term_A * Term_B * tt.term_c * Term_D;
}

// consistency function of the radial return (plasticity.cuh:74-83)
__device__ __forceinline__ double opt_fun(const mf_joco_constants &jc, int model, double delta_lambda,
                                          double norm_Strial, double eps_pl_init, const jc_temp_terms &tt,
                                          double delta_t, double mu) {
  const double s23 = sqrt(2.0 / 3.0);
  double eps_pl_equiv = eps_pl_init + s23 * fmax(delta_lambda, 0.);
  double eps_pl_equiv_dot = s23 * fmax(delta_lambda, 0.) / delta_t;
  double sigmaY = model == MF_JC_TANH ? sigma_yield_tanh(jc, eps_pl_equiv, eps_pl_equiv_dot, tt)
                                      : sigma_yield(jc, eps_pl_equiv, eps_pl_equiv_dot, tt);
  return norm_Strial - 2 * mu * delta_lambda - s23 * sigmaY;
}

// secant iteration (plasticity.cuh:85-119): at most 102 evaluation pairs; capped -> flag
static __device__ __noinline__ double solve_secant(const mf_joco_constants &jc, int model, double init, double tol,
                                               double norm_Strial, double eps_pl_init, const jc_temp_terms &tt,
                                               double delta_t, double mu, bool &capped, int &iterations) {
  double delta_lambda = init;
  double delta_lambda_old = delta_lambda;
  int iter = 0;
  const int max_iter = 100;
  capped = false;
  while (true) {
    ++iterations;
    double g = opt_fun(jc, model, delta_lambda, norm_Strial, eps_pl_init, tt, delta_t, mu);
    double delta_lambda_1 = delta_lambda * 1.01;
    double g_1 = opt_fun(jc, model, delta_lambda_1, norm_Strial, eps_pl_init, tt, delta_t, mu);
    double slope = (g - g_1) / (delta_lambda - delta_lambda_1);
    delta_lambda_old = delta_lambda;
    delta_lambda = delta_lambda - g / slope;
    if (delta_lambda < 0.) delta_lambda = -0.1 * delta_lambda;
    if (fabs(delta_lambda - delta_lambda_old) < tol) return delta_lambda;
    if (iter > max_iter) { capped = true; return delta_lambda; }
    iter++;
  }
}

// ---------------------------------------------------------------------------------------
// rigid-tool contact (tool_gpu.cu:29-207)
__device__ __forceinline__ double angle_0_2pi(double y, double x) {
  double t = atan2(y, x);
  return t > 0. ? t : t + 2 * 3.14159265358979323846;
}

__device__ __forceinline__ double circle_segment_distance(const mf_fillet &f, double qx, double qy) {
  double Ax = f.p[0], Ay = f.p[1], Bx = qx, By = qy, r = f.r;
  double Cx = Ax + r * (Bx - Ax) / sqrt((Bx - Ax) * (Bx - Ax) + (By - Ay) * (By - Ay));
  double Cy = Ay + r * (By - Ay) / sqrt((Bx - Ax) * (Bx - Ax) + (By - Ay) * (By - Ay));
  double t = angle_0_2pi(f.p[1] - Cy, f.p[0] - Cx);
  bool valid = t > fmin(f.t1, f.t2) && t < fmax(f.t1, f.t2);
  if (valid) {
    double dx = Cx - qx, dy = Cy - qy;
    return sqrt(dx * dx + dy * dy);
  }
  return 3.402823466e+38;  // FLT_MAX
}

// penetration test and closest feature (tool_gpu.cu:87-139)
__device__ __forceinline__ bool establish_contact(const mf_tool_state &T, double qx, double qy, double &cpx,
                                                  double &cpy, double &nx, double &ny) {
  const bool has_fillet = T.num_seg == 5;
  bool in = true;
  for (int i = 0; i < T.num_seg; i++) {
    double dx = T.seg[i].left[0] - qx, dy = T.seg[i].left[1] - qy;
    in = in && (dx * T.seg[i].n[0] + dy * T.seg[i].n[1]) < 0.;
  }
  if (has_fillet) {
    double dx = T.fillet.p[0] - qx, dy = T.fillet.p[1] - qy;
    in = in || sqrt(dx * dx + dy * dy) < T.fillet.r;
  }
  if (!in) return false;
  double depth = 3.402823466e+38;
  for (int i = 0; i < T.num_seg; i++) {
    double d;
    if (T.seg[i].vertical) {
      d = fabs(T.seg[i].left[0] - qx);
      if (d < depth) {
        depth = d;
        double vx = T.seg[i].left[0] - qx, vy = 0.;
        double inv = 1. / sqrt(vx * vx + vy * vy);
        nx = vx * inv;
        ny = vy * inv;
        cpx = T.seg[i].left[0];
        cpy = qy;
      }
    } else if (has_fillet && i == 2) {
      d = circle_segment_distance(T.fillet, qx, qy);
      if (d < depth) {
        depth = d;
        double vx = qx - T.fillet.p[0], vy = qy - T.fillet.p[1];
        double inv = 1. / sqrt(vx * vx + vy * vy);
        nx = vx * inv;
        ny = vy * inv;
        cpx = T.fillet.p[0] + nx * T.fillet.r;
        cpy = T.fillet.p[1] + ny * T.fillet.r;
      }
    } else {
      double px, py;
      {
        const double bb = -1, cc = T.seg[i].b, aa = T.seg[i].a;
        px = (bb * (bb * qx - aa * qy) - aa * cc) / (aa * aa + bb * bb);
        py = (aa * (-bb * qx + aa * qy) - bb * cc) / (aa * aa + bb * bb);
      }
      double dx = px - qx, dy = py - qy;
      d = sqrt(dx * dx + dy * dy);
      if (d < depth) {
        depth = d;
        nx = -T.seg[i].n[0];
        ny = -T.seg[i].n[1];
        cpx = px;
        cpy = py;
      }
    }
  }
  return true;
}

// tool::update_tool (tool.cpp:211-221) on the device, with explicitly rounded operations so
// that the result equals the host's IEEE double arithmetic bit for bit.
__device__ __forceinline__ void line_through_rn(double x1, double y1, double x2, double y2, double &a, double &b,
                                                int &vertical) {
  double detM = __dsub_rn(__dmul_rn(x1, 1.), __dmul_rn(1., x2));
  if (fabs(detM) < 1e-12) {
    vertical = 1;
    a = 1.7976931348623157e+308;
    b = x1;
    return;
  }
  vertical = 0;
  a = __ddiv_rn(__dsub_rn(__dmul_rn(y1, 1.), __dmul_rn(1., y2)), detM);
  b = __ddiv_rn(__dsub_rn(__dmul_rn(y2, x1), __dmul_rn(x2, y1)), detM);
}

__device__ __forceinline__ void tool_translate_rn(mf_tool_state &T, double dt) {
  double sx = __dmul_rn(dt, T.vel[0]), sy = __dmul_rn(dt, T.vel[1]);
  for (int i = 0; i < T.num_seg; ++i) {
    mf_segment &s = T.seg[i];
    s.left[0] = __dadd_rn(s.left[0], sx);
    s.left[1] = __dadd_rn(s.left[1], sy);
    s.right[0] = __dadd_rn(s.right[0], sx);
    s.right[1] = __dadd_rn(s.right[1], sy);
    line_through_rn(s.left[0], s.left[1], s.right[0], s.right[1], s.a, s.b, s.vertical);
  }
  if (T.has_fillet) {
    T.fillet.p[0] = __dadd_rn(T.fillet.p[0], sx);
    T.fillet.p[1] = __dadd_rn(T.fillet.p[1], sy);
  }
}

__device__ __forceinline__ bool isnaninf(double v) { return isnan(v) || isinf(v); }

// Neumaier two-sum accumulation (compensated summation of the tool force)
struct ksum {
  double s, c;
};
__device__ __forceinline__ void ksum_add(ksum &a, double x) {
  double t = a.s + x;
  if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x;
  else a.c += (x - t) + a.s;
  a.s = t;
}
__device__ __forceinline__ void ksum_merge(ksum &a, const ksum &b) {
  ksum_add(a, b.s);
  a.c += b.c;
}

}  // namespace mf
