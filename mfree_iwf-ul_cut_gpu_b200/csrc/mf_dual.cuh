// Forward-mode dual numbers for the tangent (differentiable) step: a value and ND directional
// derivatives, with the chain rule of every operation the step uses. The functions the
// reference evaluates in float on double arguments (sqrtf, atan2f, cosf, sinf, fmaxf) keep
// that value here; their derivative is the one of the exact function (the float rounding is
// piecewise constant and has none).
#pragma once

#include <cmath>

namespace mf {

template <int ND>
struct dn {
  double v;
  double d[ND];
};

template <int ND>
__host__ __device__ __forceinline__ dn<ND> dconst(double v) {
  dn<ND> r;
  r.v = v;
#pragma unroll
  for (int k = 0; k < ND; ++k) r.d[k] = 0.;
  return r;
}

// value v with derivative 1 in direction `dir` (a parameter being differentiated)
template <int ND>
__host__ __device__ __forceinline__ dn<ND> dseed(double v, int dir) {
  dn<ND> r = dconst<ND>(v);
  if (dir >= 0 && dir < ND) r.d[dir] = 1.;
  return r;
}

// r = a * x (value f, derivative scale fp applied to x's derivatives)
template <int ND>
__device__ __forceinline__ dn<ND> dchain(double f, double fp, const dn<ND> &x) {
  dn<ND> r;
  r.v = f;
#pragma unroll
  for (int k = 0; k < ND; ++k) r.d[k] = fp * x.d[k];
  return r;
}

#define MF_DN_BINOP(OP, VAL, DER)                                                        \
  template <int ND>                                                                       \
  __device__ __forceinline__ dn<ND> operator OP(const dn<ND> &a, const dn<ND> &b) {      \
    dn<ND> r;                                                                             \
    r.v = VAL;                                                                            \
    _Pragma("unroll") for (int k = 0; k < ND; ++k) r.d[k] = DER;                          \
    return r;                                                                             \
  }                                                                                       \
  template <int ND>                                                                       \
  __device__ __forceinline__ dn<ND> operator OP(const dn<ND> &a, double bv) {            \
    return a OP dconst<ND>(bv);                                                           \
  }                                                                                       \
  template <int ND>                                                                       \
  __device__ __forceinline__ dn<ND> operator OP(double av, const dn<ND> &b) {            \
    return dconst<ND>(av) OP b;                                                           \
  }

MF_DN_BINOP(+, a.v + b.v, a.d[k] + b.d[k])
MF_DN_BINOP(-, a.v - b.v, a.d[k] - b.d[k])
MF_DN_BINOP(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
MF_DN_BINOP(/, a.v / b.v, (a.d[k] * b.v - a.v * b.d[k]) / (b.v * b.v))
#undef MF_DN_BINOP

template <int ND>
__device__ __forceinline__ dn<ND> operator-(const dn<ND> &a) {
  return dchain(-a.v, -1., a);
}

template <int ND> __device__ __forceinline__ dn<ND> &operator+=(dn<ND> &a, const dn<ND> &b) { return a = a + b; }
template <int ND> __device__ __forceinline__ dn<ND> &operator-=(dn<ND> &a, const dn<ND> &b) { return a = a - b; }
template <int ND> __device__ __forceinline__ dn<ND> &operator*=(dn<ND> &a, const dn<ND> &b) { return a = a * b; }
template <int ND> __device__ __forceinline__ dn<ND> &operator+=(dn<ND> &a, double b) { a.v += b; return a; }

template <int ND>
__device__ __forceinline__ dn<ND> dsqrt(const dn<ND> &x) {
  const double s = sqrt(x.v);
  return dchain(s, s > 0. ? 0.5 / s : 0., x);
}

// (double)sqrtf((float)x): the reference's float-rounded root
template <int ND>
__device__ __forceinline__ dn<ND> dsqrtf_narrow(const dn<ND> &x) {
  const double s = (double)sqrtf((float)x.v);
  const double se = sqrt(x.v);
  return dchain(s, se > 0. ? 0.5 / se : 0., x);
}

template <int ND>
__device__ __forceinline__ dn<ND> dlog(const dn<ND> &x) {
  return dchain(log(x.v), 1. / x.v, x);
}

template <int ND>
__device__ __forceinline__ dn<ND> dexp(const dn<ND> &x) {
  const double e = exp(x.v);
  return dchain(e, e, x);
}

// x^y with both operands carrying derivatives: d = x^y (y' ln x + y x'/x); at x = 0 the
// value is pow's and the derivative is taken as 0 (the limit of the y' term for y > 0)
template <int ND>
__device__ __forceinline__ dn<ND> dpow(const dn<ND> &x, const dn<ND> &y) {
  dn<ND> r;
  r.v = pow(x.v, y.v);
  if (x.v > 0.) {
    const double lx = log(x.v);
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = r.v * (y.d[k] * lx + y.v * x.d[k] / x.v);
  } else {
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = 0.;
  }
  return r;
}

template <int ND>
__device__ __forceinline__ dn<ND> dfmax0(const dn<ND> &x) {  // fmax(x, 0)
  return x.v > 0. ? x : dconst<ND>(fmax(x.v, 0.));
}

template <int ND>
__device__ __forceinline__ dn<ND> dfabs(const dn<ND> &x) {
  return x.v < 0. ? -x : x;
}

// (double)atan2f((float)y, (float)x)
template <int ND>
__device__ __forceinline__ dn<ND> datan2f_narrow(const dn<ND> &y, const dn<ND> &x) {
  dn<ND> r;
  r.v = (double)atan2f((float)y.v, (float)x.v);
  const double den = x.v * x.v + y.v * y.v;
#pragma unroll
  for (int k = 0; k < ND; ++k) r.d[k] = den > 0. ? (x.v * y.d[k] - y.v * x.d[k]) / den : 0.;
  return r;
}

template <int ND>
__device__ __forceinline__ dn<ND> dcosf_narrow(const dn<ND> &x) {
  return dchain((double)cosf((float)x.v), -sin(x.v), x);
}

template <int ND>
__device__ __forceinline__ dn<ND> dsinf_narrow(const dn<ND> &x) {
  return dchain((double)sinf((float)x.v), cos(x.v), x);
}

}  // namespace mf
