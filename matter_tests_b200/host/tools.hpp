// tools.hpp — the setup-facing basics of the reference's src/tools.hpp
// (types T/TV/TM/TA, the enums, debug printing, linspace/arange), for setup
// files that build a Simulation for the B200 step.
//
// The reference selects the dimension and spline degree at compile time
// (tools.hpp:19-21); so does this header: THREEDIM unless MATTER_TWODIM is
// defined, SPLINEDEG 2 unless defined otherwise.  TV/TM are this project's
// own small fixed-size, column-major vector and matrix types covering the
// operations setup code and object classes use; Eigen is not needed.
#ifndef TOOLS_HPP
#define TOOLS_HPP

#include <assert.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

typedef double T;
#ifndef MATTER_TWODIM
#define THREEDIM
#endif
#ifndef SPLINEDEG
#define SPLINEDEG 2
#endif
#ifdef THREEDIM
#define DIMENSION 3
#else
#define DIMENSION 2
#endif

namespace matter {

template <int R, int C>
struct Mat {
  T d[R * C];  // column-major: (r, c) at c*R + r

  Mat() {
    for (int i = 0; i < R * C; ++i) d[i] = T(0);
  }
  template <typename A, typename B>
  Mat(A a, B b) {
    static_assert(R * C == 2, "two-component constructor");
    d[0] = T(a);
    d[1] = T(b);
  }
  template <typename A, typename B, typename D>
  Mat(A a, B b, D c) {
    static_assert(R * C == 3, "three-component constructor");
    d[0] = T(a);
    d[1] = T(b);
    d[2] = T(c);
  }
  static Mat Zero() { return Mat(); }
  static Mat Zero(int) { return Mat(); }
  static Mat Constant(T v) {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = v;
    return m;
  }
  static Mat Ones() { return Constant(T(1)); }
  static Mat Ones(int) { return Constant(T(1)); }
  static Mat Identity() {
    Mat m;
    for (int i = 0; i < R && i < C; ++i) m(i, i) = T(1);
    return m;
  }
  static constexpr int rows() { return R; }
  static constexpr int cols() { return C; }
  static constexpr int size() { return R * C; }
  T* data() { return d; }
  const T* data() const { return d; }
  T& operator()(int r, int c) { return d[c * R + r]; }
  const T& operator()(int r, int c) const { return d[c * R + r]; }
  T& operator()(int i) { return d[i]; }
  const T& operator()(int i) const { return d[i]; }
  T& operator[](int i) { return d[i]; }
  const T& operator[](int i) const { return d[i]; }
  void setZero() { *this = Mat(); }
  void setOnes() { *this = Ones(); }
  void setIdentity() { *this = Identity(); }

  struct Comma {  // out << a, b, c;  (row by row, like Eigen)
    Mat* m;
    int i;
    Comma& operator,(T v) {
      m->d[(i % C) * R + i / C] = v;
      ++i;
      return *this;
    }
  };
  Comma operator<<(T v) {
    d[0] = v;
    return Comma{this, 1};
  }

  Mat operator-() const {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = -d[i];
    return m;
  }
  Mat operator+(const Mat& o) const {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = d[i] + o.d[i];
    return m;
  }
  Mat operator-(const Mat& o) const {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = d[i] - o.d[i];
    return m;
  }
  Mat& operator+=(const Mat& o) { return *this = *this + o; }
  Mat& operator-=(const Mat& o) { return *this = *this - o; }
  Mat operator*(T s) const {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = d[i] * s;
    return m;
  }
  Mat operator/(T s) const {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = d[i] / s;
    return m;
  }
  Mat& operator*=(T s) { return *this = *this * s; }
  Mat& operator/=(T s) { return *this = *this / s; }
  template <int K>
  Mat<R, K> operator*(const Mat<C, K>& o) const {
    Mat<R, K> m;
    for (int i = 0; i < R; ++i)
      for (int j = 0; j < K; ++j) {
        T acc = (*this)(i, 0) * o(0, j);
        for (int k = 1; k < C; ++k) acc += (*this)(i, k) * o(k, j);
        m(i, j) = acc;
      }
    return m;
  }
  Mat<C, R> transpose() const {
    Mat<C, R> m;
    for (int i = 0; i < R; ++i)
      for (int j = 0; j < C; ++j) m(j, i) = (*this)(i, j);
    return m;
  }
  T determinant() const {
    static_assert(R == C, "square");
    const Mat& a = *this;
    if (R == 2) return a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0);
    return a(0, 0) * (a(1, 1) * a(2, 2) - a(2, 1) * a(1, 2)) - a(1, 0) * (a(0, 1) * a(2, 2) - a(2, 1) * a(0, 2)) +
           a(2, 0) * (a(0, 1) * a(1, 2) - a(1, 1) * a(0, 2));
  }
  Mat inverse() const {  // adjugate / determinant
    static_assert(R == C, "square");
    const Mat& a = *this;
    const T det = determinant();
    Mat t;
    if (R == 2) {
      t(0, 0) = a(1, 1) / det;
      t(0, 1) = -a(0, 1) / det;
      t(1, 0) = -a(1, 0) / det;
      t(1, 1) = a(0, 0) / det;
    } else {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          const int i1 = (j + 1) % 3, i2 = (j + 2) % 3, j1 = (i + 1) % 3, j2 = (i + 2) % 3;
          t(i, j) = (a(i1, j1) * a(i2, j2) - a(i1, j2) * a(i2, j1)) / det;
        }
    }
    return t;
  }
  T trace() const {
    T acc = 0;
    for (int i = 0; i < R && i < C; ++i) acc += (*this)(i, i);
    return acc;
  }
  T sum() const {
    T acc = 0;
    for (int i = 0; i < R * C; ++i) acc += d[i];
    return acc;
  }
  T squaredNorm() const {
    T acc = 0;
    for (int i = 0; i < R * C; ++i) acc += d[i] * d[i];
    return acc;
  }
  T norm() const { return std::sqrt(squaredNorm()); }
  Mat normalized() const {
    const T z = squaredNorm();
    return z > T(0) ? *this / std::sqrt(z) : *this;
  }
  void normalize() { *this = normalized(); }
  T dot(const Mat& o) const {
    T acc = 0;
    for (int i = 0; i < R * C; ++i) acc += d[i] * o.d[i];
    return acc;
  }
  Mat cwiseProduct(const Mat& o) const {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = d[i] * o.d[i];
    return m;
  }
  Mat cwiseAbs() const {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = std::abs(d[i]);
    return m;
  }
  T maxCoeff() const { return *std::max_element(d, d + R * C); }
  T minCoeff() const { return *std::min_element(d, d + R * C); }
  template <typename F>
  Mat unaryExpr(F f) const {
    Mat m;
    for (int i = 0; i < R * C; ++i) m.d[i] = f(d[i]);
    return m;
  }
};

template <int R, int C>
Mat<R, C> operator*(T s, const Mat<R, C>& m) {
  return m * s;
}

template <int R, int C>
std::ostream& operator<<(std::ostream& os, const Mat<R, C>& m) {
  for (int i = 0; i < R; ++i) {
    for (int j = 0; j < C; ++j) os << (j ? " " : "") << m(i, j);
    if (i + 1 < R) os << "\n";
  }
  return os;
}

}  // namespace matter

typedef matter::Mat<DIMENSION, DIMENSION> TM;
typedef matter::Mat<DIMENSION, 1> TV;
typedef matter::Mat<DIMENSION, 1> TA;

// tools.hpp:53-57 (same order, so the numeric values match)
enum class PlateType { top, bottom, left, right, front, back };
enum class ElasticModel { Hencky, NeoHookean };
enum class PlasticModel { NoPlasticity, VM, DP, DPSoft, MCC, VMVisc, DPVisc, MCCVisc, DPMui, MCCMui, Snow };
enum class HardeningLaw { NoHard, ExpoExpl, ExpoImpl, SinhExpl, SinhImpl };
enum class BC { NoSlip, SlipStick, SlipFree };

// debug(...) prints its arguments on one line (tools.hpp:61-88)
inline void debug_print_all(std::ostream&) {}
template <typename A, typename... Rest>
void debug_print_all(std::ostream& os, const A& a, const Rest&... rest) {
  os << a;
  debug_print_all(os, rest...);
}
template <typename... Args>
void debug(const Args&... args) {
  std::cout << std::setprecision(12);
  debug_print_all(std::cout, args...);
  std::cout << std::endl;
}

inline int sgn(T val) { return (T(0) < val) - (val < T(0)); }

inline T selfDoubleDot(const TM& A) { return A.squaredNorm(); }

// N points spanning [a, b] (tools.hpp:279-287)
inline std::vector<T> linspace(T a, T b, size_t N) {
  const T h = (b - a) / static_cast<T>(N - 1);
  std::vector<T> xs(N);
  T val = a;
  for (size_t i = 0; i < N; ++i, val += h) xs[i] = val;
  return xs;
}

// start, start+step, ... while < stop, accumulated (tools.hpp:291-296)
inline std::vector<T> arange(T start, T stop, T step) {
  std::vector<T> values;
  for (T value = start; value < stop; value += step) values.push_back(value);
  return values;
}

#endif  // TOOLS_HPP
