// oracle/shim/blitz/array.h — minimal blitz++ API for building the reference.
//
// TEST INFRASTRUCTURE ONLY.  blitz++ is not installed in this image; this
// header implements, from blitz's documented interface, the subset that the
// BlockSp v1.0 headers use (TinyVector, TinyMatrix, Array<T,1|2>, Range,
// dot/min/max/abs/conj/product, stream output) so that the reference headers
// compile *unmodified* for the CPU oracle and the timed CPU baseline.
//
// Semantics that matter for the reference's arithmetic:
//   * TinyVector / TinyMatrix are fixed-size, contiguous, row-major values;
//     arithmetic is elementwise, and recurses into nested TinyVectors
//     (solArray elements are TinyVector<TinyVector<T,B>,D>).
//   * Array<T,N> is contiguous row-major; assignment from an Array copies the
//     elements, assignment from a scalar fills; Array<T,2>(n) is n x n.
//   * dot(a, b) sums a(i)*b(i) left to right.
// Deviation (documented, off the solve path): copy-construction and slicing
// make deep copies, where blitz would share the memory block.
#ifndef BSP_ORACLE_BLITZ_SHIM_H
#define BSP_ORACLE_BLITZ_SHIM_H

#include <algorithm>
#include <cassert>
#include <cmath>
#include <complex>
#include <cstddef>
#include <initializer_list>
#include <iostream>
#include <type_traits>
#include <vector>

namespace blitz {

template <typename T, int N> class TinyVector;
template <typename T, int M, int N> class TinyMatrix;
template <typename T, int N> class Array;

template <typename T> struct is_tiny : std::false_type {};
template <typename T, int N> struct is_tiny<TinyVector<T, N>> : std::true_type {};
template <typename T, int M, int N> struct is_tiny<TinyMatrix<T, M, N>> : std::true_type {};
template <typename T> inline constexpr bool is_tiny_v = is_tiny<std::decay_t<T>>::value;

template <typename T> struct is_array : std::false_type {};
template <typename T, int N> struct is_array<Array<T, N>> : std::true_type {};
template <typename T> inline constexpr bool is_array_v = is_array<std::decay_t<T>>::value;

template <typename S> inline constexpr bool is_scalar_like_v = !is_tiny_v<S> && !is_array_v<S>;

// placeholder for blitz's expression-template node type (named by the reference)
template <typename T> class _bz_ArrayExpr {};

// ------------------------------------------------------------------ TinyVector
template <typename T, int N>
class TinyVector {
 public:
  using T_numtype = T;
  T d_[N > 0 ? N : 1];

  TinyVector() = default;
  TinyVector(const TinyVector&) = default;
  TinyVector& operator=(const TinyVector&) = default;
  template <typename S, std::enable_if_t<is_scalar_like_v<S> && std::is_constructible_v<T, const S&>, bool> = true>
  explicit(false) TinyVector(const S& s) {
    for (int i = 0; i < N; ++i) d_[i] = T(s);
  }
  template <typename A0, typename A1, typename... Rest>
  TinyVector(const A0& a0, const A1& a1, const Rest&... rest) {
    static_assert(2 + sizeof...(Rest) == N, "TinyVector: wrong number of elements");
    const T tmp[N] = {T(a0), T(a1), T(rest)...};
    for (int i = 0; i < N; ++i) d_[i] = tmp[i];
  }
  template <typename S, std::enable_if_t<!std::is_same_v<S, T>, bool> = true>
  TinyVector(const TinyVector<S, N>& o) {
    for (int i = 0; i < N; ++i) d_[i] = T(o(i));
  }

  T& operator()(int i) { return d_[i]; }
  const T& operator()(int i) const { return d_[i]; }
  T& operator[](int i) { return d_[i]; }
  const T& operator[](int i) const { return d_[i]; }
  T* data() { return d_; }
  const T* data() const { return d_; }
  T* begin() { return d_; }
  T* end() { return d_ + N; }
  const T* begin() const { return d_; }
  const T* end() const { return d_ + N; }
  static constexpr int length() { return N; }

  template <typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true>
  TinyVector& operator=(const S& s) {
    for (int i = 0; i < N; ++i) d_[i] = s;
    return *this;
  }
  // smaller TinyVector assigned into a larger one (utility tvM1 assigns N -> N-1)
  template <int M, std::enable_if_t<M != N, bool> = true>
  TinyVector& operator=(const TinyVector<T, M>& o) {
    for (int i = 0; i < std::min(N, M); ++i) d_[i] = o(i);
    return *this;
  }

#define BSP_TV_COMPOUND(op)                                                     \
  template <typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true>   \
  TinyVector& operator op(const S& s) {                                        \
    for (int i = 0; i < N; ++i) d_[i] op s;                                    \
    return *this;                                                              \
  }                                                                            \
  template <typename S>                                                        \
  TinyVector& operator op(const TinyVector<S, N>& o) {                         \
    for (int i = 0; i < N; ++i) d_[i] op o(i);                                 \
    return *this;                                                              \
  }
  BSP_TV_COMPOUND(+=)
  BSP_TV_COMPOUND(-=)
  BSP_TV_COMPOUND(*=)
  BSP_TV_COMPOUND(/=)
#undef BSP_TV_COMPOUND
};

// elementwise binary operators (recursive through nested TinyVectors)
#define BSP_TV_BINOP(op)                                                                        \
  template <typename A, typename B, int N>                                                      \
  auto operator op(const TinyVector<A, N>& a, const TinyVector<B, N>& b) {                      \
    using R = std::decay_t<decltype(a(0) op b(0))>;                                             \
    TinyVector<R, N> r;                                                                         \
    for (int i = 0; i < N; ++i) r(i) = a(i) op b(i);                                            \
    return r;                                                                                   \
  }                                                                                             \
  template <typename A, int N, typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true>  \
  auto operator op(const TinyVector<A, N>& a, const S& s) {                                     \
    using R = std::decay_t<decltype(a(0) op s)>;                                                \
    TinyVector<R, N> r;                                                                         \
    for (int i = 0; i < N; ++i) r(i) = a(i) op s;                                               \
    return r;                                                                                   \
  }                                                                                             \
  template <typename A, int N, typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true>  \
  auto operator op(const S& s, const TinyVector<A, N>& a) {                                     \
    using R = std::decay_t<decltype(s op a(0))>;                                                \
    TinyVector<R, N> r;                                                                         \
    for (int i = 0; i < N; ++i) r(i) = s op a(i);                                               \
    return r;                                                                                   \
  }
BSP_TV_BINOP(+)
BSP_TV_BINOP(-)
BSP_TV_BINOP(*)
BSP_TV_BINOP(/)
#undef BSP_TV_BINOP

template <typename A, int N>
TinyVector<A, N> operator-(const TinyVector<A, N>& a) {
  TinyVector<A, N> r;
  for (int i = 0; i < N; ++i) r(i) = -a(i);
  return r;
}

// ------------------------------------------------------------------ TinyMatrix
template <typename T, int M, int N>
class TinyMatrix {
 public:
  using T_numtype = T;
  T d_[M * N];

  TinyMatrix() = default;
  TinyMatrix(const TinyMatrix&) = default;
  TinyMatrix& operator=(const TinyMatrix&) = default;
  template <typename S, std::enable_if_t<is_scalar_like_v<S> && std::is_constructible_v<T, const S&>, bool> = true>
  explicit(false) TinyMatrix(const S& s) {
    for (int i = 0; i < M * N; ++i) d_[i] = T(s);
  }

  T& operator()(int i, int j) { return d_[i * N + j]; }
  const T& operator()(int i, int j) const { return d_[i * N + j]; }
  T* data() { return d_; }
  const T* data() const { return d_; }
  T* begin() { return d_; }
  T* end() { return d_ + M * N; }
  const T* begin() const { return d_; }
  const T* end() const { return d_ + M * N; }
  static constexpr int rows() { return M; }
  static constexpr int columns() { return N; }

  template <typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true>
  TinyMatrix& operator=(const S& s) {
    for (int i = 0; i < M * N; ++i) d_[i] = s;
    return *this;
  }
#define BSP_TM_COMPOUND(op)                                                   \
  template <typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true> \
  TinyMatrix& operator op(const S& s) {                                      \
    for (int i = 0; i < M * N; ++i) d_[i] op s;                              \
    return *this;                                                            \
  }                                                                          \
  TinyMatrix& operator op(const TinyMatrix& o) {                             \
    for (int i = 0; i < M * N; ++i) d_[i] op o.d_[i];                        \
    return *this;                                                            \
  }
  BSP_TM_COMPOUND(+=)
  BSP_TM_COMPOUND(-=)
  BSP_TM_COMPOUND(*=)
  BSP_TM_COMPOUND(/=)
#undef BSP_TM_COMPOUND
};

#define BSP_TM_BINOP(op)                                                                      \
  template <typename T, int M, int N>                                                         \
  TinyMatrix<T, M, N> operator op(const TinyMatrix<T, M, N>& a, const TinyMatrix<T, M, N>& b) { \
    TinyMatrix<T, M, N> r;                                                                    \
    for (int i = 0; i < M * N; ++i) r.d_[i] = a.d_[i] op b.d_[i];                             \
    return r;                                                                                 \
  }                                                                                           \
  template <typename T, int M, int N, typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true> \
  TinyMatrix<T, M, N> operator op(const TinyMatrix<T, M, N>& a, const S& s) {                 \
    TinyMatrix<T, M, N> r;                                                                    \
    for (int i = 0; i < M * N; ++i) r.d_[i] = a.d_[i] op s;                                   \
    return r;                                                                                 \
  }                                                                                           \
  template <typename T, int M, int N, typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true> \
  TinyMatrix<T, M, N> operator op(const S& s, const TinyMatrix<T, M, N>& a) {                 \
    TinyMatrix<T, M, N> r;                                                                    \
    for (int i = 0; i < M * N; ++i) r.d_[i] = s op a.d_[i];                                   \
    return r;                                                                                 \
  }
BSP_TM_BINOP(+)
BSP_TM_BINOP(-)
BSP_TM_BINOP(*)
BSP_TM_BINOP(/)
#undef BSP_TM_BINOP

// ------------------------------------------------------------------ Range
class Range {
 public:
  int first_, last_;
  Range() : first_(0), last_(-1) {}
  Range(int f, int l) : first_(f), last_(l) {}
  static Range all() { return Range(0, -2); }
  bool is_all() const { return last_ == -2; }
};

// ------------------------------------------------------------------ Array
template <typename T, int N>
class Array {
  static_assert(N == 1 || N == 2, "shim supports rank 1 and 2");

 public:
  using T_numtype = T;
  std::vector<T> v_;
  int ext_[2] = {0, 0};

  Array() = default;
  explicit Array(int n0) { resize(n0); }
  Array(int n0, int n1) { resize(n0, n1); }
  explicit Array(const TinyVector<int, N>& e) { resize(e); }
  Array(const Array& o) = default;  // deep copy (see header note)
  Array(Array&&) noexcept = default;
  Array& operator=(Array&& o) noexcept = default;

  Array& operator=(const Array& o) {
    if (this == &o) return *this;
    if (size() == 0 && o.size() != 0) {
      v_ = o.v_;
      ext_[0] = o.ext_[0];
      ext_[1] = o.ext_[1];
      return *this;
    }
    assert(o.size() == size());
    for (size_t i = 0; i < v_.size(); ++i) v_[i] = o.v_[i];
    return *this;
  }
  template <typename S, std::enable_if_t<is_scalar_like_v<S> || is_tiny_v<S>, bool> = true>
  Array& operator=(const S& s) {
    for (auto& e : v_) e = s;
    return *this;
  }
  template <typename R>
  Array& operator=(const _bz_ArrayExpr<R>&) {
    static_assert(sizeof(R) == 0, "blitz expression objects are not provided by the shim");
    return *this;
  }

  void resize(int n0) {
    if constexpr (N == 1) {
      ext_[0] = n0;
      v_.assign((size_t)std::max(n0, 0), T());
    } else {
      resize(n0, n0);
    }
  }
  void resize(int n0, int n1) {
    static_assert(N == 2 || N == 1, "");
    ext_[0] = n0;
    ext_[1] = n1;
    v_.assign((size_t)std::max(n0, 0) * (size_t)std::max(n1, 0), T());
  }
  void resize(const TinyVector<int, N>& e) {
    if constexpr (N == 1) resize(e(0));
    else resize(e(0), e(1));
  }
  void resizeAndPreserve(int n0) {
    if constexpr (N == 1) {
      v_.resize((size_t)std::max(n0, 0));
      ext_[0] = n0;
    } else {
      resizeAndPreserve(n0, n0);
    }
  }
  void resizeAndPreserve(int n0, int n1) {
    std::vector<T> nv((size_t)std::max(n0, 0) * (size_t)std::max(n1, 0), T());
    for (int i = 0; i < std::min(n0, ext_[0]); ++i)
      for (int j = 0; j < std::min(n1, ext_[1]); ++j) nv[(size_t)i * n1 + j] = v_[(size_t)i * ext_[1] + j];
    v_.swap(nv);
    ext_[0] = n0;
    ext_[1] = n1;
  }
  void reset() {
    v_.clear();
    ext_[0] = ext_[1] = 0;
  }
  Array copy() const { return Array(*this); }

  int extent(int d) const { return ext_[d]; }
  TinyVector<int, N> extent() const {
    TinyVector<int, N> e;
    for (int d = 0; d < N; ++d) e(d) = ext_[d];
    return e;
  }
  TinyVector<int, N> shape() const { return extent(); }
  int rows() const { return ext_[0]; }
  int cols() const { return N == 2 ? ext_[1] : 1; }
  size_t size() const { return v_.size(); }
  size_t numElements() const { return v_.size(); }
  T* data() { return v_.data(); }
  const T* data() const { return v_.data(); }
  T* dataFirst() { return v_.data(); }
  auto begin() { return v_.begin(); }
  auto end() { return v_.end(); }
  auto begin() const { return v_.begin(); }
  auto end() const { return v_.end(); }

  T& operator()(int i) { return v_[(size_t)i]; }
  const T& operator()(int i) const { return v_[(size_t)i]; }
  T& operator()(int i, int j) { return v_[(size_t)i * ext_[1] + j]; }
  const T& operator()(int i, int j) const { return v_[(size_t)i * ext_[1] + j]; }
  T& operator()(const TinyVector<int, N>& ix) {
    if constexpr (N == 1) return (*this)(ix(0));
    else return (*this)(ix(0), ix(1));
  }
  // slices (copies; see header note)
  Array<T, 1> operator()(const Range& r) const {
    const int f = r.is_all() ? 0 : r.first_, l = r.is_all() ? ext_[0] - 1 : r.last_;
    Array<T, 1> out(l - f + 1);
    for (int i = f; i <= l; ++i) out(i - f) = v_[(size_t)i];
    return out;
  }
  Array<T, 2> operator()(const Range& r, const Range& c) const {
    const int rf = r.is_all() ? 0 : r.first_, rl = r.is_all() ? ext_[0] - 1 : r.last_;
    const int cf = c.is_all() ? 0 : c.first_, cl = c.is_all() ? ext_[1] - 1 : c.last_;
    Array<T, 2> out(rl - rf + 1, cl - cf + 1);
    for (int i = rf; i <= rl; ++i)
      for (int j = cf; j <= cl; ++j) out(i - rf, j - cf) = (*this)(i, j);
    return out;
  }
  Array<T, 1> operator()(const Range& r, int c) const {
    const int rf = r.is_all() ? 0 : r.first_, rl = r.is_all() ? ext_[0] - 1 : r.last_;
    Array<T, 1> out(rl - rf + 1);
    for (int i = rf; i <= rl; ++i) out(i - rf) = (*this)(i, c);
    return out;
  }

#define BSP_AR_COMPOUND(op)                                                             \
  template <typename S, std::enable_if_t<is_scalar_like_v<S> || is_tiny_v<S>, bool> = true> \
  Array& operator op(const S& s) {                                                     \
    for (auto& e : v_) e op s;                                                         \
    return *this;                                                                      \
  }                                                                                    \
  Array& operator op(const Array& o) {                                                 \
    assert(o.size() == size());                                                        \
    for (size_t i = 0; i < v_.size(); ++i) v_[i] op o.v_[i];                           \
    return *this;                                                                      \
  }
  BSP_AR_COMPOUND(+=)
  BSP_AR_COMPOUND(-=)
  BSP_AR_COMPOUND(*=)
  BSP_AR_COMPOUND(/=)
#undef BSP_AR_COMPOUND
};

#define BSP_AR_BINOP(op)                                                                  \
  template <typename T, int N>                                                            \
  Array<T, N> operator op(const Array<T, N>& a, const Array<T, N>& b) {                   \
    Array<T, N> r(a);                                                                     \
    r op## = b;                                                                           \
    return r;                                                                             \
  }                                                                                       \
  template <typename T, int N, typename S, std::enable_if_t<is_scalar_like_v<S>, bool> = true> \
  Array<T, N> operator op(const Array<T, N>& a, const S& s) {                             \
    Array<T, N> r(a);                                                                     \
    r op## = s;                                                                           \
    return r;                                                                             \
  }
BSP_AR_BINOP(+)
BSP_AR_BINOP(-)
BSP_AR_BINOP(*)
BSP_AR_BINOP(/)
#undef BSP_AR_BINOP

// ------------------------------------------------------------------ reductions
template <typename A, typename B, int N>
auto dot(const TinyVector<A, N>& a, const TinyVector<B, N>& b) {
  auto s = a(0) * b(0);
  for (int i = 1; i < N; ++i) s += a(i) * b(i);
  return s;
}
template <typename T>
T dot(const Array<T, 1>& a, const Array<T, 1>& b) {
  T s = T(0);
  for (size_t i = 0; i < a.size(); ++i) s += a(i) * b(i);
  return s;
}

template <typename T, int N>
auto abs(const TinyVector<T, N>& a) {
  using R = std::decay_t<decltype(std::abs(a(0)))>;
  TinyVector<R, N> r;
  for (int i = 0; i < N; ++i) r(i) = std::abs(a(i));
  return r;
}
template <typename T, int N>
auto abs(const Array<T, N>& a) {
  using R = std::decay_t<decltype(std::abs(a.v_[0]))>;
  Array<R, N> r;
  r.ext_[0] = a.ext_[0];
  r.ext_[1] = a.ext_[1];
  r.v_.resize(a.v_.size());
  for (size_t i = 0; i < a.v_.size(); ++i) r.v_[i] = std::abs(a.v_[i]);
  return r;
}
template <typename T, int N>
TinyVector<T, N> conj(const TinyVector<T, N>& a) {
  TinyVector<T, N> r;
  for (int i = 0; i < N; ++i) {
    if constexpr (std::is_arithmetic_v<T>) r(i) = a(i);
    else r(i) = std::conj(a(i));
  }
  return r;
}
template <typename T>
Array<T, 1> conj(const Array<T, 1>& a) {
  Array<T, 1> r(a);
  if constexpr (!std::is_arithmetic_v<T>)
    for (auto& e : r.v_) e = std::conj(e);
  return r;
}
template <typename T, int N> T max(const TinyVector<T, N>& a) {
  T m = a(0);
  for (int i = 1; i < N; ++i) m = std::max(m, a(i));
  return m;
}
template <typename T, int N> T min(const TinyVector<T, N>& a) {
  T m = a(0);
  for (int i = 1; i < N; ++i) m = std::min(m, a(i));
  return m;
}
template <typename T, int N> T max(const Array<T, N>& a) {
  return *std::max_element(a.v_.begin(), a.v_.end());
}
template <typename T, int N> T min(const Array<T, N>& a) {
  return *std::min_element(a.v_.begin(), a.v_.end());
}
template <typename T, int N> T sum(const TinyVector<T, N>& a) {
  T s = a(0);
  for (int i = 1; i < N; ++i) s += a(i);
  return s;
}
template <typename T, int N> T product(const TinyVector<T, N>& a) {
  T s = a(0);
  for (int i = 1; i < N; ++i) s *= a(i);
  return s;
}

// ------------------------------------------------------------------ output
template <typename T, int N>
std::ostream& operator<<(std::ostream& os, const TinyVector<T, N>& a) {
  os << "(";
  for (int i = 0; i < N; ++i) os << a(i) << (i + 1 < N ? "," : "");
  return os << ")";
}
template <typename T, int M, int N>
std::ostream& operator<<(std::ostream& os, const TinyMatrix<T, M, N>& a) {
  os << "(" << M << " x " << N << ")\n[";
  for (int i = 0; i < M; ++i) {
    for (int j = 0; j < N; ++j) os << " " << a(i, j);
    os << (i + 1 < M ? "\n " : " ]");
  }
  return os;
}
template <typename T, int N>
std::ostream& operator<<(std::ostream& os, const Array<T, N>& a) {
  os << "(" << a.extent(0);
  if (N == 2) os << " x " << a.extent(1);
  os << ")\n[ ";
  for (size_t i = 0; i < a.size(); ++i) os << a.v_[i] << " ";
  return os << "]";
}

}  // namespace blitz

#endif
