// Body of the differentiable step (included by mf_tangent.cu once per number of derivative
// directions): MF_TG_ND directions in namespace mf::MF_TG_NS. No include guard: each
// inclusion instantiates it for one MF_TG_ND.
namespace mf {
namespace MF_TG_NS {

constexpr int ND = MF_TG_ND;
using DN = dn<ND>;

// one particle's persistent state on duals (array-of-structures: the kernels here favour
// simplicity over bandwidth)
struct tpart {
  DN pos[2], vel[2], S[4], rho, T, eps, epsd, fc[2], ft[2], pos_t[2], vel_t[2], rho_t, S_t[4], T_t;
  double h;
  unsigned flags;
  int id;
};

// the per-step neighbour record (predicted state)
struct trec {
  DN x, y, vx, vy, sxx, sxy, syy, Rxx, Rxy, Ryy, rho, c, vol, T;
  double h;
  unsigned flags;
};

// the differentiated parameters, duals seeded in the chosen direction
struct tparams {
  DN A, B, n, C, m, mu;
};

struct tbuf {
  tpart *a, *b;   // state at the start of the step / in the new order
  DN *n2;         // contact normal, position-indexed (2 per particle)
  DN *pp;         // predictor pressure
  trec *rec;
  double2 *posv;  // value positions for the hash
  unsigned *flagsv;
  DN *blk;        // per-block force partials (4 per block: fc.x, fc.y, ft.x, ft.y)
  DN *wsum;       // window sums of (Fc, Ff)
};

__global__ void k_t_posv(int N, tbuf T) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  T.posv[q] = make_double2(T.a[q].pos[0].v, T.a[q].pos[1].v);
  T.flagsv[q] = T.a[q].flags;
}

// artificial stress (actions_gpu.cu:35-39, 53-97) on duals
__device__ void t_artificial_stress(const DN &rhoi, const DN &pi, const DN &Sx, const DN &Sy, const DN &Sz,
                                    double eps, DN &Rxx, DN &Rxy, DN &Ryy) {
  const DN sxx = Sx - pi, sxy = Sy, syy = Sz - pi;
  const DN rhoi21 = 1. / (rhoi * rhoi);
  const DN theta = 0.5 * datan2f_narrow(2. * sxy, sxx - syy);
  const DN ct = dcosf_narrow(theta), st = dsinf_narrow(theta);
  const DN ct2 = ct * ct, st2 = st * st;
  const DN rot_sxx = ct2 * sxx + 2.0 * ct * st * sxy + st2 * syy;
  const DN rot_syy = st2 * sxx - 2.0 * ct * st * sxy + ct2 * syy;
  DN rot_rxx = dconst<ND>(0.), rot_ryy = dconst<ND>(0.);
  if (rot_sxx.v > 0) rot_rxx = -eps * rot_sxx * rhoi21;
  if (rot_syy.v > 0) rot_ryy = -eps * rot_syy * rhoi21;
  Rxx = ct2 * rot_rxx + st2 * rot_ryy;
  Rxy = ct * st * (rot_rxx - rot_ryy);
  Ryy = st2 * rot_rxx + ct2 * rot_ryy;
}

// gather into the new order + predictor + EOS + artificial stress + records
__global__ void k_t_reorder(params P, dev_buffers D, tbuf T) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.N) return;
  const int4 u = D.perm_u[t];
  const int p = u.x;
  const int q = u.z + stable_rank(D.perm_u, u);  // the particle's stable slot in its cell
  if (t == u.z) D.count[u.y] = 0;
  D.perm[q] = p;
  D.hash_cur[q] = u.y;
  tpart s = T.a[p];
  const bool blanked = s.flags & FLAG_BLANKED, tool = s.flags & FLAG_TOOL;
  if (!blanked) {  // predict (leap_frog.cu:42-66)
    const double hdt = 0.5 * P.dt;
    for (int k = 0; k < 2; ++k) {
      s.pos[k] = s.pos[k] + hdt * s.pos_t[k];
      s.vel[k] = s.vel[k] + hdt * s.vel_t[k];
    }
    for (int k = 0; k < 4; ++k) s.S[k] = s.S[k] + hdt * s.S_t[k];
    s.rho = s.rho + hdt * s.rho_t;
    s.T = s.T + hdt * s.T_t;
  }
  T.b[q] = s;
  DN prs = dconst<ND>(0.), Rxx = dconst<ND>(0.), Rxy = dconst<ND>(0.), Ryy = dconst<ND>(0.);
  if (!tool) {
    const double rho0 = P.phys.rho0;
    const double c0 = (double)sqrtf((float)(P.phys.K / rho0));
    prs = c0 * c0 * (s.rho - rho0);
    t_artificial_stress(s.rho, prs, s.S[0], s.S[1], s.S[2], P.corr.stresseps, Rxx, Rxy, Ryy);
  }
  T.pp[q] = prs;
  const DN rho21 = 1. / (s.rho * s.rho);
  trec r;
  r.x = s.pos[0]; r.y = s.pos[1]; r.vx = s.vel[0]; r.vy = s.vel[1];
  r.sxx = (s.S[0] - prs) * rho21; r.sxy = s.S[1] * rho21; r.syy = (s.S[2] - prs) * rho21;
  r.Rxx = Rxx; r.Rxy = Rxy; r.Ryy = Ryy;
  r.rho = s.rho;
  r.c = dsqrtf_narrow(P.phys.K / s.rho);
  r.vol = P.phys.mass / s.rho;
  r.T = s.T;
  r.h = s.h;
  r.flags = s.flags;
  T.rec[q] = r;
}

// pair sums over the 5x5 window (interactions_gpu.cu:147-345) and the rates
// (actions_gpu.cu:99-224), on duals
__global__ void k_t_pair(params P, dev_buffers D, tbuf T) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= P.N) return;
  const trec ri = T.rec[q];
  if (ri.flags & FLAG_BLANKED) return;
  const bool tool_i = ri.flags & FLAG_TOOL;
  const bool brookshaw = P.thermal_solver == MF_THERMAL_BROOKSHAW;
  const double mass = P.phys.mass;
  const double wdeltap = P.corr.wdeltap, alpha = P.corr.alpha, beta = P.corr.beta, eta = P.corr.eta;
  double thermal_alpha = 0.;
  if (brookshaw) thermal_alpha = !tool_i ? P.trml_wp.alpha : (P.thermal_tool_on ? P.trml_tool.alpha : 0.);
  const bool thermal = thermal_alpha != 0.;
  const double h1 = 1 / ri.h;
  const double fourh2 = 4 * ri.h * ri.h;
  const double fac = 0.454728408833987 * h1 * h1;
  const geom g = *D.g;
  const int hashi = D.hash_cur[q];
  const int gi = hashi / g.ny, gj = hashi - gi * g.ny;
  const int low_i = gi - 2 < 0 ? 0 : gi - 2, low_j = gj - 2 < 0 ? 0 : gj - 2;
  const int high_i = gi + 3 > g.nx ? g.nx : gi + 3, high_j = gj + 3 > g.ny ? g.ny : gj + 3;
  DN vdx = dconst<ND>(0.), vdy = vdx, vdz = vdx, vdw = vdx, sdx = vdx, sdy = vdx, sdz = vdx, sdw = vdx;
  DN vtx = vdx, vty = vdx, xtx = vdx, xty = vdx, T_lapl = vdx;
  const double m_eps = -P.corr.xspheps * mass;
  for (int ii = low_i; ii < high_i; ++ii) {
    const int j0 = D.off[ii * g.ny + low_j], j1 = D.off[ii * g.ny + high_j];
    for (int j = j0; j < j1; ++j) {
      const trec &rj = T.rec[j];
      if (rj.flags & FLAG_BLANKED) continue;
      const DN xij = ri.x - rj.x, yij = ri.y - rj.y;
      const DN rr2 = xij * xij + yij * yij;
      if (rr2.v >= fourh2 || rr2.v < 1e-8) continue;  // outside the support: W = 0
      // cubic spline (kernels.cuh:30-70), rad = (double)sqrtf((float)rr2)
      const DN rad = dsqrtf_narrow(rr2);
      const DN qq = rad * h1;
      DN val, der;
      if (qq.v > 1) {
        const DN t = 2. - qq;
        const DN t2 = t * t;
        val = 0.25 * t2 * t2 * t2;
        der = -0.75 * t2 * h1 / rad;
      } else {
        val = 1. - 1.5 * qq * qq * (1. - 0.5 * qq);
        der = -3.0 * qq * (1. - 0.75 * qq) * h1 / rad;
      }
      const DN w = val * fac;
      const DN w_x = der * xij * fac, w_y = der * yij * fac;
      const DN dwr = der * fac;
      const bool tool_j = rj.flags & FLAG_TOOL;
      if (!tool_i && !tool_j) {
        vdx += (rj.vx - ri.vx) * w_x * rj.vol;
        vdy += (rj.vx - ri.vx) * w_y * rj.vol;
        vdz += (rj.vy - ri.vy) * w_x * rj.vol;
        vdw += (rj.vy - ri.vy) * w_y * rj.vol;
        DN fab = w / wdeltap;
        fab = fab * fab;
        fab = fab * fab;
        const DN Rx = fab * (ri.Rxx + rj.Rxx), Ry = fab * (ri.Rxy + rj.Rxy), Rz = fab * (ri.Ryy + rj.Ryy);
        sdx += mass * (ri.sxx + rj.sxx + Rx) * w_x;
        sdy += mass * (ri.sxy + rj.sxy + Ry) * w_y;
        sdz += mass * (ri.sxy + rj.sxy + Ry) * w_x;
        sdw += mass * (ri.syy + rj.syy + Rz) * w_y;
        const DN vijx = ri.vx - rj.vx, vijy = ri.vy - rj.vy;
        const DN vijposij = vijx * xij + vijy * yij;
        const DN irhoij = 1. / (0.5 * (ri.rho + rj.rho));
        if (vijposij.v < 0.) {
          const DN cij = 0.5 * (ri.c + rj.c);
          const double hij = 0.5 * (ri.h + rj.h);
          const DN muij = (hij * vijposij) / (rr2 + eta * eta * hij * hij);
          const DN piij = (-alpha * cij * muij + beta * muij * muij) * irhoij;
          vtx += -mass * piij * w_x;
          vty += -mass * piij * w_y;
        }
        const DN xs = m_eps * w * irhoij;
        xtx += xs * vijx;
        xty += xs * vijy;
      }
      if (thermal && rr2.v > 1e-16) T_lapl += 2.0 * rj.vol * (ri.T - rj.T) * dwr;
    }
  }
  tpart &B = T.b[q];
  if (!tool_i) {
    // Jaumann rate (actions_gpu.cu:99-133); the structurally zero GLM entries dropped
    const DN e01 = 0.5 * (vdy + vdz), w01 = 0.5 * (vdz - vdy), w10 = 0.5 * (vdy - vdz);
    const DN t3 = (1. / 3.) * (vdx + vdw);
    const double g2 = 2. * P.phys.G;
    const DN Sxx = B.S[0], Sxy = B.S[1], Syy = B.S[2];
    B.S_t[0] = g2 * (vdx - t3) + w10 * Sxy + Sxy * w10;
    B.S_t[1] = g2 * e01 + w01 * Sxx + Syy * w10;
    B.S_t[2] = g2 * (vdw - t3) + w01 * Sxy + Sxy * w01;
    B.S_t[3] = g2 * (0. - t3);
    B.rho_t = -ri.rho * (vdx + vdw);
    B.vel_t[0] = vtx + (sdx + sdy + B.fc[0] / mass + B.ft[0] / mass);
    B.vel_t[1] = vty + (sdz + sdw + B.fc[1] / mass + B.ft[1] / mass);
    B.pos_t[0] = xtx + ri.vx;
    B.pos_t[1] = xty + ri.vy;
  } else {
    B.vel_t[0] = vtx;
    B.vel_t[1] = vty;
    B.pos_t[0] = xtx;
    B.pos_t[1] = xty;
  }
  if (thermal) B.T_t = thermal_alpha * T_lapl;
}

// the Johnson-Cook yield stress (plasticity.cuh:30-46) on duals
__device__ DN t_sigma_yield(const params &P, const tparams &TP, const DN &eps_pl, const DN &eps_pl_dot, const DN &t) {
  const mf_joco_constants &jc = P.joco;
  const DN theta = (t - jc.Tref) / (jc.Tmelt - jc.Tref);
  const DN Term_A = TP.A + TP.B * dpow(eps_pl, TP.n);
  const DN eps_dot = eps_pl_dot / jc.eps_dot_ref;
  const DN Term_B = eps_dot.v > 1.0 ? 1.0 + TP.C * dlog(eps_dot) : dpow(1.0 + eps_dot, TP.C);
  const DN Term_C = 1.0 - dpow(theta, TP.m);
  return Term_A * Term_B * Term_C;
}

// secant radial return (plasticity.cuh:74-119) iterated on duals: the derivative of the
// iterate the reference returns
__device__ DN t_solve_secant(const params &P, const tparams &TP, const DN &init, const DN &norm_Strial,
                             const DN &eps_pl_init, const DN &t, double delta_t, double mu) {
  const double s23 = sqrt(2.0 / 3.0), tol = 1e-6;
  DN dl = init, dl_old = init;
  int iter = 0;
  while (true) {
    const DN dl_1 = dl * 1.01;
    const DN e0 = eps_pl_init + s23 * dfmax0(dl), ed0 = s23 * dfmax0(dl) / delta_t;
    const DN e1 = eps_pl_init + s23 * dfmax0(dl_1), ed1 = s23 * dfmax0(dl_1) / delta_t;
    const DN g = norm_Strial - 2 * mu * dl - s23 * t_sigma_yield(P, TP, e0, ed0, t);
    const DN g_1 = norm_Strial - 2 * mu * dl_1 - s23 * t_sigma_yield(P, TP, e1, ed1, t);
    const DN slope = (g - g_1) / (dl - dl_1);
    dl_old = dl;
    dl = dl - g / slope;
    if (dl.v < 0.) dl = -0.1 * dl;
    if (fabs(dl.v - dl_old.v) < tol) return dl;
    if (iter > 100) return dl;
    iter++;
  }
}

// contact (tool_gpu.cu:87-207) on duals; the closest feature is chosen on values
__device__ bool t_contact(const mf_tool_state &TL, const DN &qx, const DN &qy, DN &cpx, DN &cpy, DN &nx, DN &ny) {
  double cpxv, cpyv, nxv, nyv;
  if (!establish_contact(TL, qx.v, qy.v, cpxv, cpyv, nxv, nyv)) return false;
  // repeat the selection of establish_contact to know which feature won
  const bool has_fillet = TL.num_seg == 5;
  double depth = 3.402823466e+38;
  int best = -1;
  for (int i = 0; i < TL.num_seg; i++) {
    double d;
    if (TL.seg[i].vertical) d = fabs(TL.seg[i].left[0] - qx.v);
    else if (has_fillet && i == 2) d = circle_segment_distance(TL.fillet, qx.v, qy.v);
    else {
      const double bb = -1, cc = TL.seg[i].b, aa = TL.seg[i].a;
      const double px = (bb * (bb * qx.v - aa * qy.v) - aa * cc) / (aa * aa + bb * bb);
      const double py = (aa * (-bb * qx.v + aa * qy.v) - bb * cc) / (aa * aa + bb * bb);
      d = sqrt((px - qx.v) * (px - qx.v) + (py - qy.v) * (py - qy.v));
    }
    if (d < depth) { depth = d; best = i; }
  }
  if (best < 0) return false;
  const mf_segment &s = TL.seg[best];
  if (s.vertical) {
    nx = dconst<ND>(nxv);
    ny = dconst<ND>(nyv);
    cpx = dconst<ND>(s.left[0]);
    cpy = qy;
  } else if (has_fillet && best == 2) {
    const DN vx = qx - TL.fillet.p[0], vy = qy - TL.fillet.p[1];
    const DN inv = 1. / dsqrt(vx * vx + vy * vy);
    nx = vx * inv;
    ny = vy * inv;
    cpx = TL.fillet.p[0] + nx * TL.fillet.r;
    cpy = TL.fillet.p[1] + ny * TL.fillet.r;
  } else {
    const double bb = -1, cc = s.b, aa = s.a;
    cpx = (bb * (bb * qx - aa * qy) - aa * cc) / (aa * aa + bb * bb);
    cpy = (aa * (-bb * qx + aa * qy) - bb * cc) / (aa * aa + bb * bb);
    nx = dconst<ND>(-s.n[0]);
    ny = dconst<ND>(-s.n[1]);
  }
  return true;
}

// corrector .. invalidate (leap_frog.cu:68-92, actions_gpu.cu:135-349, tool_gpu.cu:151-221)
// on duals, plus the block's share of report_force
__global__ void __launch_bounds__(128) k_t_finish(params P, dev_buffers D, tbuf T, tparams TP, mf_tool_state TL) {
  __shared__ DN sh[4][128];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  DN fsum[4] = {dconst<ND>(0.), dconst<ND>(0.), dconst<ND>(0.), dconst<ND>(0.)};
  if (q < P.N) {
    const double dt = P.dt;
    tpart &B = T.b[q];
    const tpart A = T.a[D.perm[q]];
    unsigned f = B.flags;
    const bool blanked = f & FLAG_BLANKED, tool = f & FLAG_TOOL, fixed = f & FLAG_FIXED;
    DN pos[2] = {A.pos[0], A.pos[1]}, vel[2] = {A.vel[0], A.vel[1]};
    DN S[4] = {A.S[0], A.S[1], A.S[2], A.S[3]};
    DN rho = A.rho, Tm = A.T;
    if (!blanked) {
      for (int k = 0; k < 2; ++k) {
        pos[k] = pos[k] + dt * B.pos_t[k];
        vel[k] = vel[k] + dt * B.vel_t[k];
      }
      for (int k = 0; k < 4; ++k) S[k] = S[k] + dt * B.S_t[k];
      rho = rho + dt * B.rho_t;
      Tm = Tm + dt * B.T_t;
    }
    DN eps_pl = B.eps, eps_pl_dot = B.epsd;
    DN fc[2] = {B.fc[0], B.fc[1]}, ft[2] = {B.ft[0], B.ft[1]};
    if (P.has_tool && P.fric_heat && !tool) {  // friction heat (actions_gpu.cu:135-162)
      const DN f_fric_mag = dsqrtf_narrow(ft[0] * ft[0] + ft[1] * ft[1]);
      if (f_fric_mag.v != 0.) {
        const DN vdx = vel[0] - TL.vel[0], vdy = vel[1] - TL.vel[1];
        const DN vdn = vdx * T.n2[2 * q] + vdy * T.n2[2 * q + 1];
        const DN vrx = vdx - vdn, vry = vdy - vdn;
        const DN v_rel_mag = dsqrtf_narrow(vrx * vrx + vry * vry);
        Tm += P.trml_wp.eta * dt * f_fric_mag * v_rel_mag / (P.trml_wp.cp * P.phys.mass);
      }
    }
    if (P.plastic && !tool) {  // JC radial return (actions_gpu.cu:226-285)
      const double mu = P.phys.G;
      const DN Sxx = S[0], Syy = S[2], Szz = S[3], Sxy = S[1];
      const DN norm_Strial = dsqrtf_narrow(Sxx * Sxx + Syy * Syy + Szz * Szz + Sxy * Sxy);
      const DN pr = T.pp[q];
      const DN cxx = Sxx - pr, cyy = Syy - pr, czz = Szz - pr, cxy = Sxy;
      const DN svm = dsqrtf_narrow((cxx * cxx + cyy * cyy + czz * czz) - cxx * cyy - cxx * czz - cyy * czz +
                                   3.0 * cxy * cxy);
      const DN sigma_Y = t_sigma_yield(P, TP, eps_pl, eps_pl_dot, Tm);
      if (svm.v < sigma_Y.v) {
        eps_pl_dot = dconst<ND>(0.);
      } else {
        DN init = eps_pl_dot * dt * sqrt(2. / 3.);
        if (!(init.v > 1e-8)) init = dconst<ND>(fmax(init.v, 1e-8));
        const DN dl = t_solve_secant(P, TP, init, norm_Strial, eps_pl, Tm, dt, mu);
        // (double)(sqrtf(2/3) * fmaxf((float)dl, 0)): float-rounded value, exact derivative
        const float s23f = sqrtf((float)(2.0 / 3.0));
        const double inc_v = (double)(s23f * fmaxf((float)dl.v, 0.f));
        const DN inc = dl.v > 0. ? dchain(inc_v, sqrt(2.0 / 3.0), dl) : dconst<ND>(inc_v);
        const DN eps_pl_new = eps_pl + inc;
        const DN eps_pl_dot_new = inc / dt;
        S[0] = Sxx - Sxx / norm_Strial * dl * 2. * mu;
        S[2] = Syy - Syy / norm_Strial * dl * 2. * mu;
        S[3] = Szz - Szz / norm_Strial * dl * 2. * mu;
        S[1] = Sxy - Sxy / norm_Strial * dl * 2. * mu;
        if (P.trml_wp.tq != 0.) {
          const DN sY = t_sigma_yield(P, TP, eps_pl_new, eps_pl_dot_new, Tm);
          Tm += P.trml_wp.tq / (P.trml_wp.cp * rho) * (eps_pl_new - eps_pl) * sY;
        }
        eps_pl = eps_pl_new;
        eps_pl_dot = eps_pl_dot_new;
      }
    }
    if (P.has_tool) {
      if (tool) {
        pos[0] += dt * TL.vel[0];
        pos[1] += dt * TL.vel[1];
      } else {
        DN cpx, cpy, nx, ny;
        if (!t_contact(TL, pos[0], pos[1], cpx, cpy, nx, ny)) {
          fc[0] = fc[1] = ft[0] = ft[1] = dconst<ND>(0.);
          T.n2[2 * q] = T.n2[2 * q + 1] = dconst<ND>(0.);
        } else {
          const double dt2 = dt * dt;
          const DN gN = (pos[0] - cpx) * nx + (pos[1] - cpy) * ny;
          const DN sc = -TL.slave_mass * gN;
          const DN fNx = sc * nx / dt2 * TL.contact_alpha, fNy = sc * ny / dt2 * TL.contact_alpha;
          DN fTx = dconst<ND>(0.), fTy = dconst<ND>(0.);
          if (TP.mu.v != 0.) {
            const DN vx = vel[0] - TL.vel[0], vy = vel[1] - TL.vel[1];
            const DN vrx = vx - vx * nx, vry = vy - vy * ny;
            const double ks = TL.contact_alpha * TL.slave_mass;
            const DN kx = ks * vrx / dt, ky = ks * vry / dt;
            const DN fy = TP.mu * dsqrt(fNx * fNx + fNy * fNy);
            const DN fsx = ft[0] - kx, fsy = ft[1] - ky;
            const DN lfs = dsqrt(fsx * fsx + fsy * fsy);
            if (lfs.v > fy.v) {
              fTx = fy * fsx / lfs;
              fTy = fy * fsy / lfs;
            } else {
              fTx = fsx;
              fTy = fsy;
            }
          }
          fc[0] = fNx; fc[1] = fNy; ft[0] = fTx; ft[1] = fTy;
          T.n2[2 * q] = nx;
          T.n2[2 * q + 1] = ny;
        }
      }
    }
    if (!tool && fixed) {  // boundary conditions (actions_gpu.cu:287-311)
      vel[0] = vel[1] = fc[0] = fc[1] = dconst<ND>(0.);
      B.pos_t[0] = B.pos_t[1] = B.vel_t[0] = B.vel_t[1] = dconst<ND>(0.);
    }
    if (P.thermal_bc && fixed) Tm = dconst<ND>(P.trml_wp.T_init);
    if (!blanked) {  // invalidate (actions_gpu.cu:317-349)
      bool bad = isnaninf(B.pos_t[0].v) || isnaninf(B.pos_t[1].v) || isnaninf(B.vel_t[0].v) ||
                 isnaninf(B.vel_t[1].v) || isnaninf(B.rho_t.v) || isnaninf(B.T_t.v);
      for (int k = 0; k < 4; ++k) bad = bad || isnaninf(B.S_t[k].v);
      if (bad) f |= FLAG_BLANKED;
    }
    B.flags = f;
    B.pos[0] = pos[0]; B.pos[1] = pos[1];
    B.vel[0] = vel[0]; B.vel[1] = vel[1];
    for (int k = 0; k < 4; ++k) B.S[k] = S[k];
    B.rho = rho;
    B.T = Tm;
    B.eps = eps_pl;
    B.epsd = eps_pl_dot;
    B.fc[0] = fc[0]; B.fc[1] = fc[1];
    B.ft[0] = ft[0]; B.ft[1] = ft[1];
    fsum[0] = fc[0]; fsum[1] = fc[1]; fsum[2] = ft[0]; fsum[3] = ft[1];
  }
  // the block's partial sums in a fixed order (report_force, output.cu:31-39)
  for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = fsum[k];
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = sh[k][threadIdx.x] + sh[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) T.blk[4 * blockIdx.x + k] = sh[k][0];
}

// the step's total force Fc = sum(fc.x + ft.x), Ff = sum(fc.y + ft.y), added to the window sums
__global__ void k_t_force(int nblocks, tbuf T, int accumulate) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  DN s[4] = {dconst<ND>(0.), dconst<ND>(0.), dconst<ND>(0.), dconst<ND>(0.)};
  for (int b = 0; b < nblocks; ++b)
    for (int k = 0; k < 4; ++k) s[k] += T.blk[4 * b + k];
  if (accumulate) {
    T.wsum[0] += s[0] + s[2];
    T.wsum[1] += s[1] + s[3];
  }
}

struct tg_alloc {
  std::vector<void *> ptrs;
  cudaError_t err = cudaSuccess;
  template <class T>
  T *get(size_t n) {
    void *p = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&p, (n ? n : 1) * sizeof(T));
    if (err == cudaSuccess) err = cudaMemset(p, 0, (n ? n : 1) * sizeof(T));
    if (p) ptrs.push_back(p);
    return (T *)p;
  }
  ~tg_alloc() {
    for (void *p : ptrs) cudaFree(p);
  }
};

template <class T>
int download(std::vector<T> &v, int field, mf_ctx *ctx, int width, int N) {
  v.resize((size_t)N * width);
  return mf_get_field(ctx, field, v.data());
}

// runs from the context's current state; P and Dctx are the context's parameters and buffers
int run_mean_force(mf_ctx *ctx, int device, params P, const dev_buffers &Dctx, int skip_steps, int window_steps,
                   int param, double out_mean[2], double out_dmean[2]) {
  int N = 0;
  if (mf_particles_count(ctx, &N) != MF_OK || N <= 0) return MF_ERR_STATE;
  mf_tool_state TL;
  if (mf_tool_get(ctx, &TL) != MF_OK) return MF_ERR_STATE;

  // initial state from the context, in its current array order
  std::vector<double> pos, vel, S, rho, T, eps, epsd, fc, ft, n, pos_t, vel_t, rho_t, S_t, T_t, h, fixed, blanked,
      toolp;
  std::vector<int> id;
  if (download(pos, MF_FIELD_POS, ctx, 2, N) || download(vel, MF_FIELD_VEL, ctx, 2, N) ||
      download(S, MF_FIELD_S, ctx, 4, N) || download(rho, MF_FIELD_RHO, ctx, 1, N) ||
      download(T, MF_FIELD_T, ctx, 1, N) || download(eps, MF_FIELD_EPS_PL, ctx, 1, N) ||
      download(epsd, MF_FIELD_EPS_PL_DOT, ctx, 1, N) || download(fc, MF_FIELD_FC, ctx, 2, N) ||
      download(ft, MF_FIELD_FT, ctx, 2, N) || download(n, MF_FIELD_N, ctx, 2, N) ||
      download(pos_t, MF_FIELD_POS_T, ctx, 2, N) || download(vel_t, MF_FIELD_VEL_T, ctx, 2, N) ||
      download(rho_t, MF_FIELD_RHO_T, ctx, 1, N) || download(S_t, MF_FIELD_S_T, ctx, 4, N) ||
      download(T_t, MF_FIELD_T_T, ctx, 1, N) || download(h, MF_FIELD_H, ctx, 1, N) ||
      download(fixed, MF_FIELD_FIXED, ctx, 1, N) || download(blanked, MF_FIELD_BLANKED, ctx, 1, N) ||
      download(toolp, MF_FIELD_TOOL, ctx, 1, N) || download(id, MF_FIELD_ID, ctx, 1, N))
    return MF_ERR_STATE;
  std::vector<tpart> host((size_t)N);
  for (int i = 0; i < N; ++i) {
    tpart &p = host[i];
    auto c = [](double v) { return dconst<ND>(v); };
    for (int k = 0; k < 2; ++k) {
      p.pos[k] = c(pos[2 * i + k]); p.vel[k] = c(vel[2 * i + k]); p.fc[k] = c(fc[2 * i + k]);
      p.ft[k] = c(ft[2 * i + k]); p.pos_t[k] = c(pos_t[2 * i + k]); p.vel_t[k] = c(vel_t[2 * i + k]);
    }
    for (int k = 0; k < 4; ++k) { p.S[k] = c(S[4 * i + k]); p.S_t[k] = c(S_t[4 * i + k]); }
    p.rho = c(rho[i]); p.T = c(T[i]); p.eps = c(eps[i]); p.epsd = c(epsd[i]);
    p.rho_t = c(rho_t[i]); p.T_t = c(T_t[i]);
    p.h = h[i];
    p.flags = (fixed[i] == 1. ? FLAG_FIXED : 0u) | (blanked[i] == 1. ? FLAG_BLANKED : 0u) |
              (toolp[i] == 1. ? FLAG_TOOL : 0u);
    p.id = id[i];
  }
  std::vector<DN> n2((size_t)2 * N);
  for (int i = 0; i < 2 * N; ++i) n2[i] = dconst<ND>(n[i]);

  if (cudaSetDevice(device) != cudaSuccess) return MF_ERR_CUDA;
  tg_alloc al;
  tbuf TB;
  TB.a = al.get<tpart>(N);
  TB.b = al.get<tpart>(N);
  TB.n2 = al.get<DN>((size_t)2 * N);
  TB.pp = al.get<DN>(N);
  TB.rec = al.get<trec>(N);
  TB.posv = al.get<double2>(N);
  TB.flagsv = al.get<unsigned>(N);
  const int nb = (N + 127) / 128;
  TB.blk = al.get<DN>((size_t)4 * nb);
  TB.wsum = al.get<DN>(2);
  // cell lists on the product's kernels, with buffers of their own
  dev_buffers D = {};
  geom G;
  if (al.err == cudaSuccess) al.err = cudaMemcpy(&G, Dctx.g, sizeof(G), cudaMemcpyDeviceToHost);
  D.g = Dctx.g;
  D.count = al.get<int>((size_t)G.max_cell);
  D.off = al.get<int>((size_t)G.max_cell + 1);
  const int scan_tiles = (G.max_cell + SCAN_TILE - 1) / SCAN_TILE + 1;
  D.tsum_r = al.get<int>((size_t)scan_tiles);
  D.tsum_w = al.get<int>((size_t)scan_tiles);
  D.st = al.get<dev_status>(1);
  D.hash_cur = al.get<int>(N);
  D.hash_new = al.get<int>(N);
  D.perm = al.get<int>(N);
  D.perm_u = al.get<int4>(N);
  if (al.err != cudaSuccess) return al.err == cudaErrorMemoryAllocation ? MF_ERR_NOMEM : MF_ERR_CUDA;
  if (cudaMemcpy(TB.a, host.data(), sizeof(tpart) * N, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(TB.n2, n2.data(), sizeof(DN) * 2 * N, cudaMemcpyHostToDevice) != cudaSuccess)
    return MF_ERR_CUDA;
  {  // the context's hashes (blanked particles keep theirs)
    std::vector<int> hc((size_t)N);
    if (mf_get_field(ctx, MF_FIELD_HASH, hc.data()) != MF_OK) return MF_ERR_STATE;
    if (cudaMemcpy(D.hash_cur, hc.data(), sizeof(int) * N, cudaMemcpyHostToDevice) != cudaSuccess) return MF_ERR_CUDA;
  }
  tparams TP;
  const mf_joco_constants &jc = P.joco;
  // one direction: the parameter `param` (none for -1); six directions: A, B, n, C, m, mu
  auto dir = [param](int k) { return ND == 1 ? (param == k ? 0 : -1) : k; };
  TP.A = dseed<ND>(jc.A, dir(0));
  TP.B = dseed<ND>(jc.B, dir(1));
  TP.n = dseed<ND>(jc.n, dir(2));
  TP.C = dseed<ND>(jc.C, dir(3));
  TP.m = dseed<ND>(jc.m, dir(4));
  TP.mu = dseed<ND>(TL.mu, dir(5));
  P.N = N;

  const int hb = std::max(nb, (scan_tiles + 127) / 128);
  for (int step = 0; step < skip_steps + window_steps; ++step) {
    state_set As = {};
    As.pos = TB.posv;
    As.flags = TB.flagsv;
    k_t_posv<<<nb, 128>>>(N, TB);
    k_hash_count<<<hb, 128>>>(N, As, D, scan_tiles);
    k_scan<<<scan_tiles, SCAN_THREADS>>>(D, N, 0);
    std::swap(D.tsum_r, D.tsum_w);  // the scan zeroed the other one for the next count
    k_scatter<<<(N + BLOCK - 1) / BLOCK, BLOCK>>>(N, D, 0);
    k_t_reorder<<<nb, 128>>>(P, D, TB);
    k_t_pair<<<nb, 128>>>(P, D, TB);
    if (P.has_tool) mf_tool_translate(&TL, P.dt);  // tool::update_tool, before contact
    k_t_finish<<<nb, 128>>>(P, D, TB, TP, TL);
    k_t_force<<<1, 32>>>(nb, TB, step >= skip_steps ? 1 : 0);
    std::swap(TB.a, TB.b);
    if (cudaGetLastError() != cudaSuccess) return MF_ERR_CUDA;
  }
  DN w[2];
  if (cudaMemcpy(w, TB.wsum, sizeof(w), cudaMemcpyDeviceToHost) != cudaSuccess) return MF_ERR_CUDA;
  dev_status st;
  if (cudaMemcpy(&st, D.st, sizeof(st), cudaMemcpyDeviceToHost) != cudaSuccess) return MF_ERR_CUDA;
  if (st.error_flags) return MF_ERR_CUDA;
  out_mean[0] = w[0].v / window_steps;
  out_mean[1] = w[1].v / window_steps;
  if (out_dmean) {  // per direction k: d(mean Fc), d(mean Ff) at [2k], [2k + 1]
    if (ND == 1) {
      out_dmean[0] = param >= 0 ? w[0].d[0] / window_steps : 0.;
      out_dmean[1] = param >= 0 ? w[1].d[0] / window_steps : 0.;
    } else {
      for (int k = 0; k < ND; ++k) {
        out_dmean[2 * k] = w[0].d[k] / window_steps;
        out_dmean[2 * k + 1] = w[1].d[k] / window_steps;
      }
    }
  }
  return MF_OK;
}

}  // namespace MF_TG_NS
}  // namespace mf
