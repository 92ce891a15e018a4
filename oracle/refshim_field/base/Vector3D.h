// Shim (oracle test infrastructure): the scalar 3-vector the reference's
// ScalarCMSmagField uses (VecGeom is an empty submodule in the reference).
#pragma once
#include <cmath>
namespace vecgeom {
template <typename T> struct Vector3D {
  T v[3];
  Vector3D() : v{T(0), T(0), T(0)} {}
  Vector3D(T a, T b, T c) : v{a, b, c} {}
  template <typename U> Vector3D &operator=(const Vector3D<U> &o)
  {
    for (int i = 0; i < 3; ++i) v[i] = (T)o.v[i];
    return *this;
  }
  T &x() { return v[0]; }
  T &y() { return v[1]; }
  T &z() { return v[2]; }
  T x() const { return v[0]; }
  T y() const { return v[1]; }
  T z() const { return v[2]; }
  Vector3D &operator*=(double s)
  {
    for (int i = 0; i < 3; ++i) v[i] *= s;
    return *this;
  }
};
} // namespace vecgeom
