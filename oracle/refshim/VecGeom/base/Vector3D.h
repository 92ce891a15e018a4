// Shim (oracle test infrastructure): a scalar 3-vector with the members the
// reference's ConstFieldHelixStepper uses.  VecGeom itself is an empty
// submodule in the reference; Unit() here divides by the magnitude.
#pragma once
#include "VecGeom/base/Global.h"
#include "VecCore/VecCore"
namespace vecgeom {
template <typename T> struct Vector3D {
  T v[3];
  Vector3D() : v{T(0), T(0), T(0)} {}
  Vector3D(T a, T b, T c) : v{a, b, c} {}
  T &x() { return v[0]; }
  T &y() { return v[1]; }
  T &z() { return v[2]; }
  T x() const { return v[0]; }
  T y() const { return v[1]; }
  T z() const { return v[2]; }
  T &operator[](int i) { return v[i]; }
  T operator[](int i) const { return v[i]; }
  void Set(T a, T b, T c) { v[0] = a; v[1] = b; v[2] = c; }
  T Dot(const Vector3D &o) const { return v[0] * o.v[0] + v[1] * o.v[1] + v[2] * o.v[2]; }
  T Mag2() const { return Dot(*this); }
  T Mag() const { return std::sqrt(Mag2()); }
  Vector3D Unit() const { T m = Mag(); return m > 0 ? Vector3D(v[0] / m, v[1] / m, v[2] / m) : *this; }
  Vector3D Cross(const Vector3D &o) const {
    return Vector3D(v[1] * o.v[2] - v[2] * o.v[1], v[2] * o.v[0] - v[0] * o.v[2], v[0] * o.v[1] - v[1] * o.v[0]);
  }
  void Normalize() { *this = Unit(); }
  Vector3D operator+(const Vector3D &o) const { return Vector3D(v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]); }
  Vector3D operator-(const Vector3D &o) const { return Vector3D(v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]); }
};
template <typename T> Vector3D<T> operator*(T s, const Vector3D<T> &a) { return Vector3D<T>(s * a.v[0], s * a.v[1], s * a.v[2]); }
} // namespace vecgeom
