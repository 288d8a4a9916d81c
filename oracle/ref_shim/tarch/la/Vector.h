// Minimal stand-in for Peano's tarch::la::Vector, written for this project so that the
// reference's header-only generic ADER-DG kernels (ExaHyPE/kernels/aderdg/generic/c/*)
// compile without the absent Peano submodule. Test infrastructure only: it builds the
// oracle/_ref checker library and is never linked into the product.
#pragma once
#include <cmath>
#include <initializer_list>

namespace tarch {
namespace la {

template <int N, typename T>
class Vector {
 public:
  T v[N];
  Vector() { for (int i = 0; i < N; i++) v[i] = T(); }
  Vector(const T& s) { for (int i = 0; i < N; i++) v[i] = s; }
  Vector(const T& a, const T& b) { v[0] = a; if (N > 1) v[1] = b; for (int i = 2; i < N; i++) v[i] = T(); }
  Vector(const T& a, const T& b, const T& c) {
    v[0] = a; if (N > 1) v[1] = b; if (N > 2) v[2] = c; for (int i = 3; i < N; i++) v[i] = T();
  }
  Vector(std::initializer_list<T> l) {
    int i = 0;
    for (auto x : l) { if (i < N) v[i] = x; i++; }
    for (; i < N; i++) v[i] = T();
  }
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
  T& operator()(int i) { return v[i]; }
  const T& operator()(int i) const { return v[i]; }
  int size() const { return N; }
  T* data() { return v; }
  const T* data() const { return v; }
};

template <int N, typename T>
Vector<N, T> operator+(const Vector<N, T>& a, const Vector<N, T>& b) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = a[i] + b[i]; return r;
}
template <int N, typename T>
Vector<N, T> operator-(const Vector<N, T>& a, const Vector<N, T>& b) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = a[i] - b[i]; return r;
}
template <int N, typename T>
Vector<N, T> operator*(const T& s, const Vector<N, T>& a) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = s * a[i]; return r;
}
template <int N, typename T>
Vector<N, T> operator*(const Vector<N, T>& a, const T& s) { return s * a; }
template <int N, typename T>
Vector<N, T> operator/(const Vector<N, T>& a, const T& s) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = a[i] / s; return r;
}
template <int N, typename T>
Vector<N, T> invertEntries(const Vector<N, T>& a) {
  Vector<N, T> r; for (int i = 0; i < N; i++) r[i] = T(1) / a[i]; return r;
}
template <int N, typename T>
T volume(const Vector<N, T>& a) {
  T r = T(1); for (int i = 0; i < N; i++) r *= a[i]; return r;
}
template <int N, typename T>
T norm2(const Vector<N, T>& a) {
  T r = T(0); for (int i = 0; i < N; i++) r += a[i] * a[i]; return std::sqrt(r);
}
inline int aPowI(int i, int a) { int r = 1; for (int k = 0; k < i; k++) r *= a; return r; }
inline bool equals(double a, double b, double tol = 1e-12) { return std::abs(a - b) <= tol; }

}  // namespace la
}  // namespace tarch
