// Minimal stand-in for the subset of the blaze linear-algebra API (blaze >= 3.7) that the
// blazeRT headers use, so that those headers compile unchanged for the CPU oracle and the CPU
// baseline.  blaze itself is a third-party dependency that is not vendored with blazeRT
// (blazert/datatypes.h:9-10 includes <blaze/Math.h>; CMakeLists.txt:47-52 and the CI workflow
// download blaze-3.7) and is absent from this machine.
//
// This file is TEST INFRASTRUCTURE for the oracle.  It is written from the mathematics of the
// operations, not from blaze's sources.  Because the reference's own tests pin these operations
// only to doctest's Approx (~1e-5 relative), the exact floating-point ORDER of every operation is
// defined HERE, and the CUDA kernels and the C restatement follow the same order:
//
//   a +- b, a * b (Schur), a / b      element-wise, one rounding per element
//   a * s, s * a                       element-wise a[i] * s
//   a / s                              element-wise a[i] / s   (true division, not * (1/s))
//   s / a                              element-wise s / a[i]
//   a +- s                             element-wise
//   dot(a, b)                          (a0*b0 + a1*b1) + a2*b2, left to right, no FMA
//   cross(a, b)                        (a1*b2 - a2*b1, a2*b0 - a0*b2, a0*b1 - a1*b0)
//   norm(a)                            sqrt(dot(a, a))
//   normalize(a)                       a * (1 / norm(a)); the zero vector stays zero
//   M * v                              row i: (M(i,0)*v0 + M(i,1)*v1) + M(i,2)*v2
//   trans(M)                           transpose (exact)
//   abs/min/max(a[, b])                element-wise std:: functions
//
// Like blaze's own Math.h, it makes <cstdint>, <complex>, <memory> and <limits> available to its
// includers.
//
// Builds that must be bit-comparable with the CUDA path compile with -ffp-contract=off.
#pragma once
#ifndef BZR_ORACLE_BLAZE_SHIM_MATH_H_
#define BZR_ORACLE_BLAZE_SHIM_MATH_H_

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <iostream>
#include <limits>
#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

// plane.h:210 calls an unqualified abs() on a double.  Make the floating-point overloads visible
// at global scope so that it binds to abs(double) (the evident intent), not to C's int abs(int).
using std::abs;

namespace blaze {

enum AlignmentFlag : bool { unaligned = false, aligned = true };
enum PaddingFlag : bool { unpadded = false, padded = true };
constexpr bool columnVector = false;
constexpr bool rowVector = true;
constexpr bool rowMajor = false;
constexpr bool columnMajor = true;

template <typename Type, std::size_t N, bool TF = columnVector, AlignmentFlag AF = unaligned,
          PaddingFlag PF = unpadded>
class StaticVector {
 public:
  using ElementType = Type;
  Type v_[N];

  StaticVector() : v_{} {}
  explicit StaticVector(const Type &init) {
    for (std::size_t i = 0; i < N; ++i) v_[i] = init;
  }
  // Element-wise construction from N values of any arithmetic type (braced or parenthesised).
  template <typename U0, typename U1, typename... Us,
            typename = std::enable_if_t<(2 + sizeof...(Us) == N)>>
  StaticVector(U0 a, U1 b, Us... rest)
      : v_{static_cast<Type>(a), static_cast<Type>(b), static_cast<Type>(rest)...} {}
  template <typename O, bool TF2, AlignmentFlag AF2, PaddingFlag PF2>
  StaticVector(const StaticVector<O, N, TF2, AF2, PF2> &o) {
    for (std::size_t i = 0; i < N; ++i) v_[i] = static_cast<Type>(o[i]);
  }
  StaticVector(const StaticVector &) = default;
  StaticVector &operator=(const StaticVector &) = default;
  StaticVector &operator=(const Type &s) {
    for (std::size_t i = 0; i < N; ++i) v_[i] = s;
    return *this;
  }

  static constexpr std::size_t size() { return N; }
  Type &operator[](std::size_t i) { return v_[i]; }
  const Type &operator[](std::size_t i) const { return v_[i]; }
  Type *begin() { return v_; }
  Type *end() { return v_ + N; }
  const Type *begin() const { return v_; }
  const Type *end() const { return v_ + N; }
  Type *data() { return v_; }
  const Type *data() const { return v_; }

  StaticVector &operator+=(const StaticVector &o) {
    for (std::size_t i = 0; i < N; ++i) v_[i] = v_[i] + o[i];
    return *this;
  }
  StaticVector &operator-=(const StaticVector &o) {
    for (std::size_t i = 0; i < N; ++i) v_[i] = v_[i] - o[i];
    return *this;
  }
  template <typename S, typename = std::enable_if_t<std::is_arithmetic<S>::value>>
  StaticVector &operator*=(S s) {
    for (std::size_t i = 0; i < N; ++i) v_[i] = v_[i] * s;
    return *this;
  }
  template <typename S, typename = std::enable_if_t<std::is_arithmetic<S>::value>>
  StaticVector &operator/=(S s) {
    for (std::size_t i = 0; i < N; ++i) v_[i] = v_[i] / s;
    return *this;
  }
};

template <typename T>
struct is_static_vector : std::false_type {};
template <typename Type, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
struct is_static_vector<StaticVector<Type, N, TF, AF, PF>> : std::true_type {};

#define BZR_SHIM_VV(op)                                                                           \
  template <typename A, typename B, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF,    \
            AlignmentFlag AF2, PaddingFlag PF2>                                                   \
  inline auto operator op(const StaticVector<A, N, TF, AF, PF> &a,                                \
                          const StaticVector<B, N, TF, AF2, PF2> &b) {                            \
    using R = decltype(a[0] op b[0]);                                                             \
    StaticVector<R, N, TF, AF, PF> r;                                                             \
    for (std::size_t i = 0; i < N; ++i) r[i] = a[i] op b[i];                                      \
    return r;                                                                                     \
  }
BZR_SHIM_VV(+)
BZR_SHIM_VV(-)
BZR_SHIM_VV(*)
BZR_SHIM_VV(/)
#undef BZR_SHIM_VV

#define BZR_SHIM_VS(op)                                                                           \
  template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF, typename S,     \
            typename = std::enable_if_t<std::is_arithmetic<S>::value>>                            \
  inline auto operator op(const StaticVector<A, N, TF, AF, PF> &a, S s) {                         \
    using R = decltype(a[0] op s);                                                                \
    StaticVector<R, N, TF, AF, PF> r;                                                             \
    for (std::size_t i = 0; i < N; ++i) r[i] = a[i] op s;                                         \
    return r;                                                                                     \
  }                                                                                               \
  template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF, typename S,     \
            typename = std::enable_if_t<std::is_arithmetic<S>::value>>                            \
  inline auto operator op(S s, const StaticVector<A, N, TF, AF, PF> &a) {                         \
    using R = decltype(s op a[0]);                                                                \
    StaticVector<R, N, TF, AF, PF> r;                                                             \
    for (std::size_t i = 0; i < N; ++i) r[i] = s op a[i];                                         \
    return r;                                                                                     \
  }
BZR_SHIM_VS(+)
BZR_SHIM_VS(-)
BZR_SHIM_VS(*)
BZR_SHIM_VS(/)
#undef BZR_SHIM_VS

template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline StaticVector<A, N, TF, AF, PF> operator-(const StaticVector<A, N, TF, AF, PF> &a) {
  StaticVector<A, N, TF, AF, PF> r;
  for (std::size_t i = 0; i < N; ++i) r[i] = -a[i];
  return r;
}

template <typename A, typename B, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF,
          AlignmentFlag AF2, PaddingFlag PF2>
inline bool operator==(const StaticVector<A, N, TF, AF, PF> &a,
                       const StaticVector<B, N, TF, AF2, PF2> &b) {
  for (std::size_t i = 0; i < N; ++i)
    if (!(a[i] == b[i])) return false;
  return true;
}
template <typename A, typename B, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF,
          AlignmentFlag AF2, PaddingFlag PF2>
inline bool operator!=(const StaticVector<A, N, TF, AF, PF> &a,
                       const StaticVector<B, N, TF, AF2, PF2> &b) {
  return !(a == b);
}

template <typename A, typename B, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF,
          AlignmentFlag AF2, PaddingFlag PF2>
inline auto dot(const StaticVector<A, N, TF, AF, PF> &a, const StaticVector<B, N, TF, AF2, PF2> &b) {
  auto s = a[0] * b[0];
  for (std::size_t i = 1; i < N; ++i) s = s + a[i] * b[i];
  return s;
}

template <typename A, typename B, bool TF, AlignmentFlag AF, PaddingFlag PF, AlignmentFlag AF2,
          PaddingFlag PF2>
inline auto cross(const StaticVector<A, 3, TF, AF, PF> &a, const StaticVector<B, 3, TF, AF2, PF2> &b) {
  using R = decltype(a[0] * b[0]);
  StaticVector<R, 3, TF, AF, PF> r;
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
  return r;
}

template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline A sqrNorm(const StaticVector<A, N, TF, AF, PF> &a) {
  return dot(a, a);
}
template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline A norm(const StaticVector<A, N, TF, AF, PF> &a) {
  return std::sqrt(dot(a, a));
}
template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline A length(const StaticVector<A, N, TF, AF, PF> &a) {
  return norm(a);
}
template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline A l2Norm(const StaticVector<A, N, TF, AF, PF> &a) {
  return norm(a);
}
template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline StaticVector<A, N, TF, AF, PF> normalize(const StaticVector<A, N, TF, AF, PF> &a) {
  const A len = norm(a);
  const A ilen = (len != A(0)) ? A(1) / len : A(0);
  StaticVector<A, N, TF, AF, PF> r;
  for (std::size_t i = 0; i < N; ++i) r[i] = a[i] * ilen;
  return r;
}

template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline StaticVector<A, N, TF, AF, PF> abs(const StaticVector<A, N, TF, AF, PF> &a) {
  StaticVector<A, N, TF, AF, PF> r;
  for (std::size_t i = 0; i < N; ++i) r[i] = std::abs(a[i]);
  return r;
}
template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline StaticVector<A, N, TF, AF, PF> min(const StaticVector<A, N, TF, AF, PF> &a,
                                          const StaticVector<A, N, TF, AF, PF> &b) {
  StaticVector<A, N, TF, AF, PF> r;
  for (std::size_t i = 0; i < N; ++i) r[i] = std::min(a[i], b[i]);
  return r;
}
template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline StaticVector<A, N, TF, AF, PF> max(const StaticVector<A, N, TF, AF, PF> &a,
                                          const StaticVector<A, N, TF, AF, PF> &b) {
  StaticVector<A, N, TF, AF, PF> r;
  for (std::size_t i = 0; i < N; ++i) r[i] = std::max(a[i], b[i]);
  return r;
}
template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
inline bool isZero(const StaticVector<A, N, TF, AF, PF> &a) {
  for (std::size_t i = 0; i < N; ++i)
    if (a[i] != A(0)) return false;
  return true;
}

template <typename A, std::size_t N, bool TF, AlignmentFlag AF, PaddingFlag PF>
std::ostream &operator<<(std::ostream &os, const StaticVector<A, N, TF, AF, PF> &a) {
  os << "(";
  for (std::size_t i = 0; i < N; ++i) os << (i ? " " : "") << a[i];
  return os << ")";
}

// Identity matrix of run-time size; only 3x3 is used by blazeRT and its tests.
template <typename Type>
class IdentityMatrix {
 public:
  explicit IdentityMatrix(std::size_t n) : n_(n) {}
  std::size_t rows() const { return n_; }
  Type operator()(std::size_t i, std::size_t j) const { return i == j ? Type(1) : Type(0); }

 private:
  std::size_t n_;
};

template <typename Type, std::size_t M, std::size_t N, bool SO = rowMajor,
          AlignmentFlag AF = unaligned, PaddingFlag PF = unpadded>
class StaticMatrix {
 public:
  using ElementType = Type;
  Type m_[M][N];

  StaticMatrix() : m_{} {}
  explicit StaticMatrix(const Type &init) {
    for (std::size_t i = 0; i < M; ++i)
      for (std::size_t j = 0; j < N; ++j) m_[i][j] = init;
  }
  StaticMatrix(std::initializer_list<std::initializer_list<Type>> rows) : m_{} {
    std::size_t i = 0;
    for (const auto &row : rows) {
      std::size_t j = 0;
      for (const auto &x : row) m_[i][j++] = x;
      ++i;
    }
  }
  StaticMatrix(const IdentityMatrix<Type> &id) : m_{} {
    for (std::size_t i = 0; i < M; ++i)
      for (std::size_t j = 0; j < N; ++j) m_[i][j] = id(i, j);
  }
  StaticMatrix(const StaticMatrix &) = default;
  StaticMatrix &operator=(const StaticMatrix &) = default;

  static constexpr std::size_t rows() { return M; }
  static constexpr std::size_t columns() { return N; }
  Type &operator()(std::size_t i, std::size_t j) { return m_[i][j]; }
  const Type &operator()(std::size_t i, std::size_t j) const { return m_[i][j]; }
};

template <typename Type, std::size_t M, std::size_t N, bool SO, AlignmentFlag AF, PaddingFlag PF>
inline StaticMatrix<Type, N, M, SO, AF, PF> trans(const StaticMatrix<Type, M, N, SO, AF, PF> &a) {
  StaticMatrix<Type, N, M, SO, AF, PF> r;
  for (std::size_t i = 0; i < M; ++i)
    for (std::size_t j = 0; j < N; ++j) r(j, i) = a(i, j);
  return r;
}

template <typename Type, std::size_t M, std::size_t N, bool SO, AlignmentFlag AF, PaddingFlag PF,
          typename B, bool TF, AlignmentFlag AF2, PaddingFlag PF2>
inline auto operator*(const StaticMatrix<Type, M, N, SO, AF, PF> &a,
                      const StaticVector<B, N, TF, AF2, PF2> &v) {
  using R = decltype(a(0, 0) * v[0]);
  StaticVector<R, M, TF, AF2, PF2> r;
  for (std::size_t i = 0; i < M; ++i) {
    R s = a(i, 0) * v[0];
    for (std::size_t j = 1; j < N; ++j) s = s + a(i, j) * v[j];
    r[i] = s;
  }
  return r;
}

template <typename Type, std::size_t M, std::size_t K, std::size_t N, bool SO, AlignmentFlag AF,
          PaddingFlag PF, AlignmentFlag AF2, PaddingFlag PF2>
inline StaticMatrix<Type, M, N, SO, AF, PF> operator*(const StaticMatrix<Type, M, K, SO, AF, PF> &a,
                                                      const StaticMatrix<Type, K, N, SO, AF2, PF2> &b) {
  StaticMatrix<Type, M, N, SO, AF, PF> r;
  for (std::size_t i = 0; i < M; ++i)
    for (std::size_t j = 0; j < N; ++j) {
      Type s = a(i, 0) * b(0, j);
      for (std::size_t k = 1; k < K; ++k) s = s + a(i, k) * b(k, j);
      r(i, j) = s;
    }
  return r;
}

template <typename Type, std::size_t M, std::size_t N, bool SO, AlignmentFlag AF, PaddingFlag PF>
std::ostream &operator<<(std::ostream &os, const StaticMatrix<Type, M, N, SO, AF, PF> &a) {
  for (std::size_t i = 0; i < M; ++i) {
    os << "(";
    for (std::size_t j = 0; j < N; ++j) os << (j ? " " : "") << a(i, j);
    os << ")\n";
  }
  return os;
}

}  // namespace blaze

#endif  // BZR_ORACLE_BLAZE_SHIM_MATH_H_
