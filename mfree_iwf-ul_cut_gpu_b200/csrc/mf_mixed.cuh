// Mixed-precision pair kernel: the pair sums, strain rates and heat fluxes in FP32, on
// particle coordinates stored relative to the origin of their own cell; the predictor,
// corrector (leap-frog accumulation), JC return map and the tool-force reduction stay FP64.
//
// Same neighbour set and order as the plain form (interactions_gpu.cu:147-345); the
// differences are the arithmetic type and these exact rewrites:
//   * x_ij = (ci - cj) * dx + (xi_rel - xj_rel): small integers times the cell size plus
//     a difference of in-cell offsets, instead of a difference of absolute coordinates;
//   * e_ij . grad W / r = (x_ij w_x + y_ij w_y) / r^2 (Brookshaw);
//   * divisions by r use one rsqrt per pair;
//   * temperatures are stored relative to the initial temperature, so Ti - Tj keeps its
//     digits near it.
// Its error against the FP64 oracle is measured and reported, not assumed.
#pragma once

#include "mf_kernels.cuh"

namespace mf {

static __global__ void __launch_bounds__(PAIR_BLOCK) k_pair_mixed(params P, dev_buffers D) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= P.N) return;
  const float *__restrict__ rec = D.recf;
  const float4 *si = reinterpret_cast<const float4 *>(rec + (size_t)q * F_WIDTH);
  const float4 a0 = __ldg(si + 0), a1 = __ldg(si + 1), a2 = __ldg(si + 2), a3 = __ldg(si + 3);
  const unsigned fi = (unsigned)__float_as_int(a3.w);
  if (fi & FLAG_BLANKED) return;
  const bool tool_i = fi & FLAG_TOOL;
  const bool brookshaw = P.thermal_solver == MF_THERMAL_BROOKSHAW;
  if (!brookshaw && tool_i) return;

  const float mass = (float)P.phys.mass;
  const float inv_wdeltap = (float)(1. / P.corr.wdeltap);
  const float alpha = (float)P.corr.alpha, beta = (float)P.corr.beta, eta = (float)P.corr.eta;
  const float eps = (float)P.corr.xspheps;
  double thermal_alpha = 0.;
  if (brookshaw) thermal_alpha = !tool_i ? P.trml_wp.alpha : (P.thermal_tool_on ? P.trml_tool.alpha : 0.);
  const bool thermal = thermal_alpha != 0.;
  const bool nonfinite_i = fi & FLAG_NONFINITE;

  const float xi = a0.x, yi = a0.y, vxi = a0.z, vyi = a0.w;
  const float sxxi = a1.x, sxyi = a1.y, syyi = a1.z, Rxxi = a1.w;
  const float Rxyi = a2.x, Ryyi = a2.y, hi = a2.z, rhoi = a2.w;
  const float ci = a3.x, Ti = thermal ? a3.z : 0.f;
  const float h1 = 1.f / hi;
  const float fourh2 = 4.f * hi * hi;
  const float fac = 0.454728408833987f * h1 * h1;
  const float eta2 = eta * eta;

  const geom g = *D.g;
  const float dxc = (float)g.dx;
  const int hashi = D.hash_cur[q];
  const int gi = hashi / g.ny;
  const int gj = hashi - gi * g.ny;
  const int low_i = gi - 2 < 0 ? 0 : gi - 2;
  const int low_j = gj - 2 < 0 ? 0 : gj - 2;
  const int high_i = gi + 3 > g.nx ? g.nx : gi + 3;
  const int high_j = gj + 3 > g.ny ? g.ny : gj + 3;

  float vdx = 0.f, vdy = 0.f, vdz = 0.f, vdw = 0.f;
  float sdx = 0.f, sdy = 0.f, sdz = 0.f, sdw = 0.f;
  float vtx = 0.f, vty = 0.f, xtx = 0.f, xty = 0.f;
  float T_lapl = 0.f;

  for (int ii = low_i; ii < high_i; ++ii) {
    const int col = ii * g.ny;
    const int j0 = __ldg(D.off + col + low_j);
    const int j1 = __ldg(D.off + col + high_j);
    const float ox = (float)(gi - ii) * dxc;
    for (int j = j0; j < j1; ++j) {
      const float4 *sj = reinterpret_cast<const float4 *>(rec + (size_t)j * F_WIDTH);
      const float4 b3 = __ldg(sj + 3);  // c, vol, T, flags|cell_y
      const unsigned fjw = (unsigned)__float_as_int(b3.w);
      const unsigned fj = fjw & 0xffu;
      if (fj & FLAG_BLANKED) continue;
      const int cyj = (int)(fjw >> 8);
      const float4 b0 = __ldg(sj + 0);  // x_rel, y_rel, vx, vy
      const float xij = ox + (xi - b0.x);
      const float yij = (float)(gj - cyj) * dxc + (yi - b0.y);
      const float rr2 = xij * xij + yij * yij;
      const bool in_support = !(rr2 >= fourh2 || rr2 < 1e-8f);
      if (!in_support && !(nonfinite_i || (fj & FLAG_NONFINITE))) continue;
      float w = 0.f, w_x = 0.f, w_y = 0.f, rinv = 0.f;
      if (in_support) {
        rinv = rsqrtf(rr2);
        const float rad = rr2 * rinv;
        const float qq = rad * h1;
        float val, der;
        if (qq > 1.f) {
          const float t = 2.f - qq;
          const float t2 = t * t;
          val = 0.25f * t2 * t2 * t2;
          der = -0.75f * t2 * h1 * rinv;
        } else {
          val = 1.f - 1.5f * qq * qq * (1.f - 0.5f * qq);
          der = -3.0f * qq * (1.f - 0.75f * qq) * h1 * rinv;
        }
        w = val * fac;
        w_x = der * xij * fac;
        w_y = der * yij * fac;
      }
      const float volj = b3.y;
      const bool tool_j = fj & FLAG_TOOL;
      if (!tool_i && !tool_j) {
        const float4 b1 = __ldg(sj + 1);  // sxx, sxy, syy, Rxx
        const float4 b2 = __ldg(sj + 2);  // Rxy, Ryy, h, rho
        const float dvx = b0.z - vxi, dvy = b0.w - vyi;
        vdx += dvx * w_x * volj;
        vdy += dvx * w_y * volj;
        vdz += dvy * w_x * volj;
        vdw += dvy * w_y * volj;
        float fab = w * inv_wdeltap;
        fab *= fab;
        fab *= fab;
        const float Rx = fab * (Rxxi + b1.w);
        const float Ry = fab * (Rxyi + b2.x);
        const float Rz = fab * (Ryyi + b2.y);
        const float sxy = sxyi + b1.y + Ry;
        sdx += mass * (sxxi + b1.x + Rx) * w_x;
        sdy += mass * sxy * w_y;
        sdz += mass * sxy * w_x;
        sdw += mass * (syyi + b1.z + Rz) * w_y;
        const float vijposij = -(dvx * xij + dvy * yij);
        const float rhoij = 0.5f * (rhoi + b2.w);
        const float irhoij = __frcp_rn(rhoij);
        if (vijposij < 0.f) {
          const float cij = 0.5f * (ci + b3.x);
          const float hij = 0.5f * (hi + b2.z);
          const float muij = hij * vijposij * __frcp_rn(rr2 + eta2 * hij * hij);
          const float piij = (-alpha * cij * muij + beta * muij * muij) * irhoij;
          vtx -= mass * piij * w_x;
          vty -= mass * piij * w_y;
        }
        const float xs = eps * w * mass * irhoij;
        xtx += xs * dvx;
        xty += xs * dvy;
      }
      if (thermal && rr2 > 1e-16f) {
        // 2 (m/rho_j) (Ti - Tj) (e_ij . grad W) / r
        T_lapl += 2.0f * volj * (Ti - b3.z) * (xij * w_x + yij * w_y) * (rinv * rinv);
      }
    }
  }

  const state_set &B = D.B;
  if (P.keep_derivs) {
    D.S_der[q] = make_double4(sdx, sdy, sdz, sdw);
    D.v_der[q] = make_double4(vdx, vdy, vdz, vdw);
  }
  if (!tool_i) {
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
    const double2 fc = B.fc[q], ft = B.ft[q];
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

}  // namespace mf
