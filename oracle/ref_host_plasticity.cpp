// Oracle recipe: the reference's plasticity.cuh compiled for the host (test infrastructure only).
//
// plasticity.cuh holds __device__ functions (sigma_yield, sigma_yield_tanh, opt_fun,
// solve_secant and the m_s_yield function pointer). Compiled by the host compiler, CUDA's
// host_defines.h turns __device__ into an attribute the compiler ignores, so the same
// source lines become plain host functions using the host libm. Built into
// oracle/_ref/libref_host.so by oracle/build_oracle.py.
#include <cmath>
#include <cfloat>
#include <cstdio>

#include "types.h"
#include "constants_structs.h"
#include "plasticity.cuh"

extern "C" {

static joco_constants make_jc(const double *p) {
  joco_constants jc;
  jc.A = p[0]; jc.B = p[1]; jc.C = p[2]; jc.n = p[3]; jc.m = p[4]; jc.Tmelt = p[5];
  jc.Tref = p[6]; jc.eps_dot_ref = p[7]; jc.tanh_a = p[8]; jc.tanh_b = p[9];
  jc.tanh_c = p[10]; jc.tanh_d = p[11];
  return jc;
}

double refh_sigma_yield(const double *jc12, double eps_pl, double eps_pl_dot, double T) {
  return sigma_yield(make_jc(jc12), eps_pl, eps_pl_dot, T);
}

double refh_sigma_yield_tanh(const double *jc12, double eps_pl, double eps_pl_dot, double T) {
  return sigma_yield_tanh(make_jc(jc12), eps_pl, eps_pl_dot, T);
}

// model: 0 -> m_s_yield = sigma_yield (the reference default), 1 -> sigma_yield_tanh
double refh_solve_secant(const double *jc12, int model, double init, double tol, double norm_Strial,
                         double eps_pl_init, double T, double dt, double mu) {
  m_s_yield = model == 1 ? sigma_yield_tanh : sigma_yield;
  double r = solve_secant(make_jc(jc12), init, tol, norm_Strial, eps_pl_init, T, dt, mu);
  m_s_yield = sigma_yield;
  return r;
}

// solve_secant with the reference's default yield law (m_s_yield = sigma_yield, untouched):
// safe to call from several threads at once
double refh_solve_secant_jc(const double *jc12, double init, double tol, double norm_Strial, double eps_pl_init,
                            double T, double dt, double mu) {
  return solve_secant(make_jc(jc12), init, tol, norm_Strial, eps_pl_init, T, dt, mu);
}

}  // extern "C"
