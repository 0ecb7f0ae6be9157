// Mixed-precision pair kernel: the pair sums, strain rates and heat fluxes in FP32, on
// particle coordinates stored relative to the origin of their own cell; the predictor,
// corrector (leap-frog accumulation), JC return map and the tool-force reduction stay FP64.
//
// Same neighbour set and order as the plain form (interactions_gpu.cu:147-345); the
// differences are the arithmetic type and these exact rewrites:
//   * x_ij = (ci - cj) * dx + (xi_rel - xj_rel): small integers times the cell size plus
//     a difference of in-cell offsets, instead of a difference of absolute coordinates;
//   * (e_ij . grad W) / r = der * fac (Brookshaw), one rsqrt per pair for 1/r;
//   * temperatures are stored relative to the initial temperature, so Ti - Tj keeps its
//     digits near it.
// Its error against the FP64 form is measured and reported, not assumed.
#pragma once

#include "mf_kernels.cuh"

namespace mf {

static __global__ void __launch_bounds__(PAIR_BLOCK, 8) k_pair_mixed(params P, dev_buffers D) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= P.N) return;
  const float4 *__restrict__ rec = reinterpret_cast<const float4 *>(D.recf);
  const float4 a0 = __ldg(rec + 4 * q + 0);  // x, y, flags|cy, vx
  const unsigned fi = (unsigned)__float_as_int(a0.z) & 0xffu;
  if (fi & FLAG_BLANKED) return;
  const bool tool_i = fi & FLAG_TOOL;
  const bool brookshaw = P.thermal_solver == MF_THERMAL_BROOKSHAW;
  if (!brookshaw && tool_i) return;
  const float4 a1 = __ldg(rec + 4 * q + 1);  // vy, sxx, sxy, syy
  const float4 a2 = __ldg(rec + 4 * q + 2);  // Rxx, Rxy, Ryy, h
  const float4 a3 = __ldg(rec + 4 * q + 3);  // rho, c, vol, T - T_init

  const float mass = (float)P.phys.mass;
  const float inv_wdeltap = (float)(1. / P.corr.wdeltap);
  const float alpha = (float)P.corr.alpha, beta = (float)P.corr.beta, eta = (float)P.corr.eta;
  double thermal_alpha = 0.;
  if (brookshaw) thermal_alpha = !tool_i ? P.trml_wp.alpha : (P.thermal_tool_on ? P.trml_tool.alpha : 0.);
  const bool thermal = thermal_alpha != 0.;
  const bool nonfinite_i = fi & FLAG_NONFINITE;
  const bool mech_i = !tool_i;

  const float xi = a0.x, yi = a0.y, vxi = a0.w, vyi = a1.x;
  const float sxxi = a1.y, sxyi = a1.z, syyi = a1.w;
  const float Rxxi = a2.x, Rxyi = a2.y, Ryyi = a2.z, hi = a2.w;
  const float rhoi = a3.x, ci = a3.y, Ti = thermal ? a3.w : 0.f;
  const float h1 = 1.f / hi;
  const float fourh2 = 4.f * hi * hi;
  const float fac = 0.454728408833987f * h1 * h1;
  const float eta2 = eta * eta;
  const float m_eps = (float)P.corr.xspheps * mass;

  const geom g = *D.g;
  const float dxc = (float)g.dx;
  const int hashi = D.hash_cur[q];
  const int gi = hashi / g.ny;
  const int gj = hashi - gi * g.ny;
  const int low_i = gi - 2 < 0 ? 0 : gi - 2;
  const int low_j = gj - 2 < 0 ? 0 : gj - 2;
  const int high_i = gi + 3 > g.nx ? g.nx : gi + 3;
  const int high_j = gj + 3 > g.ny ? g.ny : gj + 3;
  // y offset between cell rows: (gj - r) * dx = oy0 - r * dx
  const float oy0 = (float)gj * dxc;

  float vdx = 0.f, vdy = 0.f, vdz = 0.f, vdw = 0.f;
  float sdx = 0.f, sdy = 0.f, sdz = 0.f, sdw = 0.f;
  float vtx = 0.f, vty = 0.f, xtx = 0.f, xty = 0.f;
  float T_lapl = 0.f;

  for (int ii = low_i; ii < high_i; ++ii) {
    const int col = ii * g.ny;
    const int j0 = __ldg(D.off + col + low_j);
    const int j1 = __ldg(D.off + col + high_j);
    const float ox = (float)(gi - ii) * dxc + xi;
    // chunks of up to 32 candidates: mark the contributing ones, then visit them in order
    for (int jb = j0; jb < j1; jb += 32) {
      const int jn = min(32, j1 - jb);
      unsigned mask = 0u;
#pragma unroll 4
      for (int k = 0; k < jn; ++k) {
        const float4 b0 = __ldg(rec + 4 * (jb + k));
        const unsigned fjw = (unsigned)__float_as_int(b0.z);
        const float xij = ox - b0.x;
        const float yij = (oy0 - (float)(int)(fjw >> 8) * dxc) + (yi - b0.y);
        const float rr2 = xij * xij + yij * yij;
        const bool in_support = !(rr2 >= fourh2 || rr2 < 1e-8f);
        const bool take = !(fjw & FLAG_BLANKED) && (in_support || nonfinite_i || (fjw & FLAG_NONFINITE));
        mask |= (take ? 1u : 0u) << k;
      }
      while (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1u;
        const float4 *sj = rec + 4 * (jb + k);
        const float4 b0 = __ldg(sj + 0);  // x, y, flags|cy, vx
        const float4 b3 = __ldg(sj + 3);  // rho, c, vol, T - T_init
        const unsigned fjw = (unsigned)__float_as_int(b0.z);
        const float xij = ox - b0.x;
        const float yij = (oy0 - (float)(int)(fjw >> 8) * dxc) + (yi - b0.y);
        const float rr2 = xij * xij + yij * yij;
        const bool in_support = !(rr2 >= fourh2 || rr2 < 1e-8f);
        float w = 0.f, w_x = 0.f, w_y = 0.f, dwr = 0.f;
        if (in_support) {
          const float rinv = rsqrtf(rr2);
          const float qq = rr2 * rinv * h1;
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
          dwr = der * fac;
          w_x = dwr * xij;
          w_y = dwr * yij;
        }
        const float volj = b3.z;
        if (mech_i && !(fjw & FLAG_TOOL)) {
          const float4 b1 = __ldg(sj + 1);  // vy, sxx, sxy, syy
          const float4 b2 = __ldg(sj + 2);  // Rxx, Rxy, Ryy, h
          const float dvx = b0.w - vxi, dvy = b1.x - vyi;
          const float ax = dvx * volj, ay = dvy * volj;
          vdx += ax * w_x;
          vdy += ax * w_y;
          vdz += ay * w_x;
          vdw += ay * w_y;
          float fab = w * inv_wdeltap;
          fab *= fab;
          fab *= fab;
          const float sxy = mass * (sxyi + b1.z + fab * (Rxyi + b2.y));
          sdx += mass * (sxxi + b1.y + fab * (Rxxi + b2.x)) * w_x;
          sdy += sxy * w_y;
          sdz += sxy * w_x;
          sdw += mass * (syyi + b1.w + fab * (Ryyi + b2.z)) * w_y;
          const float vijposij = -(dvx * xij + dvy * yij);
          const float irhoij = __frcp_rn(0.5f * (rhoi + b3.x));
          if (vijposij < 0.f) {
            const float cij = 0.5f * (ci + b3.y);
            const float hij = 0.5f * (hi + b2.w);
            const float muij = hij * vijposij * __frcp_rn(rr2 + eta2 * hij * hij);
            const float piij = (-alpha * cij * muij + beta * muij * muij) * irhoij;
            vtx -= mass * piij * w_x;
            vty -= mass * piij * w_y;
          }
          const float xs = m_eps * w * irhoij;
          xtx += xs * dvx;
          xty += xs * dvy;
        }
        // Brookshaw: 2 (m/rho_j)(Ti - Tj)(e_ij . grad W)/r with (e_ij . grad W)/r = der*fac
        if (thermal && rr2 > 1e-16f) T_lapl += 2.0f * volj * (Ti - b3.w) * dwr;
      }
    }
  }

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
