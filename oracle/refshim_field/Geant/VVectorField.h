// Shim (oracle test infrastructure): GeantV's field base classes, absent from
// the reference.  ScalarCMSmagField refers to two members it does not declare
// (rInv, fVcMagVector3); the shim base declares them, with Vc's vector as
// std::vector.
#pragma once
#include "base/Vector3D.h"
#include <vector>
namespace Vc {
template <class T> using vector = std::vector<T>;
}
class VVectorField {
public:
  virtual ~VVectorField() {}
  virtual VVectorField *Clone() const = 0;
};
class GUVMagneticField : public VVectorField {
public:
  virtual void GetFieldValue(const vecgeom::Vector3D<double> &pos, vecgeom::Vector3D<float> &field) = 0;

protected:
  float rInv = 0.0f;
  void *fVcMagVector3 = nullptr;
};
