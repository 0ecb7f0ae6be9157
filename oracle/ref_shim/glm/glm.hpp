// Minimal GLM-compatible header, written for this project (test infrastructure only).
//
// The reference sources include <glm/glm.hpp>, and GLM is not installed in this image.
// This header lets the oracle recipe compile the reference's own host-compilable files
// (tool.cpp, geometric_primitives.cpp, benchmarks.cpp, kernels.cuh, plasticity.cuh) where
// they lie. It implements only the subset the reference uses, following GLM's documented
// semantics:
//   * vectors: component-wise arithmetic, including vec*vec; vec/scalar is a true division;
//   * dot(a,b) = a.x*b.x + a.y*b.y (+ a.z*b.z), summed left to right;
//   * length(v) = sqrt(dot(v,v)); normalize(v) = v * (1/sqrt(dot(v,v)));
//   * matrices are column-major: m[c][r]; the scalar constructors take columns in order;
//     mat(s) is s on the diagonal; (A*B)[c][r] = sum_k A[k][r]*B[c][k];
//   * row-vector times matrix: (v*m)[c] = dot(v, m[c]);
//   * determinant of a 3x3 matrix by cofactor expansion along the first column.
// Nothing here is product code; only the oracle recipe under oracle/ includes it.
#ifndef MF_ORACLE_GLM_SHIM_HPP
#define MF_ORACLE_GLM_SHIM_HPP

#include <cmath>
#include <cfloat>
#include <cstddef>

#if defined(__CUDACC__)
#define GSHIM_FN __host__ __device__ inline
#else
#define GSHIM_FN inline
#endif

namespace glm {

template <typename T> struct tvec2 {
  T x, y;
  GSHIM_FN tvec2() : x(T(0)), y(T(0)) {}
  GSHIM_FN explicit tvec2(T s) : x(s), y(s) {}
  GSHIM_FN tvec2(T a, T b) : x(a), y(b) {}
  GSHIM_FN T &operator[](int i) { return i == 0 ? x : y; }
  GSHIM_FN const T &operator[](int i) const { return i == 0 ? x : y; }
  GSHIM_FN tvec2 &operator+=(const tvec2 &o) { x = x + o.x; y = y + o.y; return *this; }
  GSHIM_FN tvec2 &operator-=(const tvec2 &o) { x = x - o.x; y = y - o.y; return *this; }
  GSHIM_FN tvec2 &operator*=(T s) { x = x * s; y = y * s; return *this; }
  GSHIM_FN tvec2 &operator/=(T s) { x = x / s; y = y / s; return *this; }
};

template <typename T> struct tvec3 {
  T x, y, z;
  GSHIM_FN tvec3() : x(T(0)), y(T(0)), z(T(0)) {}
  GSHIM_FN explicit tvec3(T s) : x(s), y(s), z(s) {}
  GSHIM_FN tvec3(T a, T b, T c) : x(a), y(b), z(c) {}
  GSHIM_FN T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  GSHIM_FN const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

// vec2 operators
template <typename T> GSHIM_FN tvec2<T> operator+(const tvec2<T> &a, const tvec2<T> &b) { return tvec2<T>(a.x + b.x, a.y + b.y); }
template <typename T> GSHIM_FN tvec2<T> operator-(const tvec2<T> &a, const tvec2<T> &b) { return tvec2<T>(a.x - b.x, a.y - b.y); }
template <typename T> GSHIM_FN tvec2<T> operator*(const tvec2<T> &a, const tvec2<T> &b) { return tvec2<T>(a.x * b.x, a.y * b.y); }
template <typename T> GSHIM_FN tvec2<T> operator/(const tvec2<T> &a, const tvec2<T> &b) { return tvec2<T>(a.x / b.x, a.y / b.y); }
template <typename T> GSHIM_FN tvec2<T> operator*(const tvec2<T> &a, T s) { return tvec2<T>(a.x * s, a.y * s); }
template <typename T> GSHIM_FN tvec2<T> operator*(T s, const tvec2<T> &a) { return tvec2<T>(s * a.x, s * a.y); }
template <typename T> GSHIM_FN tvec2<T> operator/(const tvec2<T> &a, T s) { return tvec2<T>(a.x / s, a.y / s); }
template <typename T> GSHIM_FN tvec2<T> operator-(const tvec2<T> &a) { return tvec2<T>(-a.x, -a.y); }

// vec3 operators
template <typename T> GSHIM_FN tvec3<T> operator+(const tvec3<T> &a, const tvec3<T> &b) { return tvec3<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T> GSHIM_FN tvec3<T> operator-(const tvec3<T> &a, const tvec3<T> &b) { return tvec3<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> GSHIM_FN tvec3<T> operator*(const tvec3<T> &a, const tvec3<T> &b) { return tvec3<T>(a.x * b.x, a.y * b.y, a.z * b.z); }
template <typename T> GSHIM_FN tvec3<T> operator*(const tvec3<T> &a, T s) { return tvec3<T>(a.x * s, a.y * s, a.z * s); }
template <typename T> GSHIM_FN tvec3<T> operator*(T s, const tvec3<T> &a) { return tvec3<T>(s * a.x, s * a.y, s * a.z); }
template <typename T> GSHIM_FN tvec3<T> operator/(const tvec3<T> &a, T s) { return tvec3<T>(a.x / s, a.y / s, a.z / s); }

template <typename T> GSHIM_FN T dot(const tvec2<T> &a, const tvec2<T> &b) { tvec2<T> t = a * b; return t.x + t.y; }
template <typename T> GSHIM_FN T dot(const tvec3<T> &a, const tvec3<T> &b) { tvec3<T> t = a * b; return (t.x + t.y) + t.z; }
template <typename T> GSHIM_FN T length(const tvec2<T> &v) { return sqrt(dot(v, v)); }
template <typename T> GSHIM_FN T length(const tvec3<T> &v) { return sqrt(dot(v, v)); }
template <typename T> GSHIM_FN tvec2<T> normalize(const tvec2<T> &v) { return v * (T(1) / sqrt(dot(v, v))); }
template <typename T> GSHIM_FN tvec3<T> normalize(const tvec3<T> &v) { return v * (T(1) / sqrt(dot(v, v))); }

// column-major 2x2
template <typename T> struct tmat2x2 {
  tvec2<T> c[2];
  GSHIM_FN tmat2x2() { c[0] = tvec2<T>(T(1), T(0)); c[1] = tvec2<T>(T(0), T(1)); }
  GSHIM_FN explicit tmat2x2(T s) { c[0] = tvec2<T>(s, T(0)); c[1] = tvec2<T>(T(0), s); }
  GSHIM_FN tmat2x2(T x0, T y0, T x1, T y1) { c[0] = tvec2<T>(x0, y0); c[1] = tvec2<T>(x1, y1); }
  GSHIM_FN tvec2<T> &operator[](int i) { return c[i]; }
  GSHIM_FN const tvec2<T> &operator[](int i) const { return c[i]; }
};

// column-major 3x3
template <typename T> struct tmat3x3 {
  tvec3<T> c[3];
  GSHIM_FN tmat3x3() { c[0] = tvec3<T>(T(1), T(0), T(0)); c[1] = tvec3<T>(T(0), T(1), T(0)); c[2] = tvec3<T>(T(0), T(0), T(1)); }
  GSHIM_FN explicit tmat3x3(T s) { c[0] = tvec3<T>(s, T(0), T(0)); c[1] = tvec3<T>(T(0), s, T(0)); c[2] = tvec3<T>(T(0), T(0), s); }
  GSHIM_FN tmat3x3(T x0, T y0, T z0, T x1, T y1, T z1, T x2, T y2, T z2) {
    c[0] = tvec3<T>(x0, y0, z0); c[1] = tvec3<T>(x1, y1, z1); c[2] = tvec3<T>(x2, y2, z2);
  }
  GSHIM_FN tvec3<T> &operator[](int i) { return c[i]; }
  GSHIM_FN const tvec3<T> &operator[](int i) const { return c[i]; }
};

// row vector times matrix: (v*m)[col] = dot(v, m[col])
template <typename T> GSHIM_FN tvec2<T> operator*(const tvec2<T> &v, const tmat2x2<T> &m) {
  return tvec2<T>(v.x * m[0][0] + v.y * m[0][1], v.x * m[1][0] + v.y * m[1][1]);
}
// matrix times column vector
template <typename T> GSHIM_FN tvec2<T> operator*(const tmat2x2<T> &m, const tvec2<T> &v) {
  return tvec2<T>(m[0][0] * v.x + m[1][0] * v.y, m[0][1] * v.x + m[1][1] * v.y);
}

template <typename T> GSHIM_FN tmat3x3<T> operator+(const tmat3x3<T> &a, const tmat3x3<T> &b) {
  tmat3x3<T> r;
  for (int i = 0; i < 3; ++i) r[i] = a[i] + b[i];
  return r;
}
template <typename T> GSHIM_FN tmat3x3<T> operator-(const tmat3x3<T> &a, const tmat3x3<T> &b) {
  tmat3x3<T> r;
  for (int i = 0; i < 3; ++i) r[i] = a[i] - b[i];
  return r;
}
template <typename T> GSHIM_FN tmat3x3<T> operator*(T s, const tmat3x3<T> &a) {
  tmat3x3<T> r;
  for (int i = 0; i < 3; ++i) r[i] = s * a[i];
  return r;
}
template <typename T> GSHIM_FN tmat3x3<T> operator*(const tmat3x3<T> &a, T s) {
  tmat3x3<T> r;
  for (int i = 0; i < 3; ++i) r[i] = a[i] * s;
  return r;
}
template <typename T> GSHIM_FN tmat3x3<T> operator*(const tmat3x3<T> &a, const tmat3x3<T> &b) {
  tmat3x3<T> r;
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row)
      r[col][row] = (a[0][row] * b[col][0] + a[1][row] * b[col][1]) + a[2][row] * b[col][2];
  return r;
}
template <typename T> GSHIM_FN tmat3x3<T> transpose(const tmat3x3<T> &m) {
  tmat3x3<T> r;
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row) r[col][row] = m[row][col];
  return r;
}
template <typename T> GSHIM_FN T determinant(const tmat3x3<T> &m) {
  return m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2])
       - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2])
       + m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}

typedef tvec2<double> dvec2;
typedef tvec3<double> dvec3;
typedef tmat2x2<double> dmat2x2;
typedef tmat3x3<double> dmat3x3;
typedef tvec2<float> vec2;
typedef tvec3<float> vec3;
typedef tmat2x2<float> mat2x2;
typedef tmat3x3<float> mat3x3;

}  // namespace glm

#endif
