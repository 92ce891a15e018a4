// Shim (oracle test infrastructure): the part of the reference's Material
// (source/Geant/material/Material.hpp) the cut converter reads: elements,
// atoms per volume and density (internal units).
#pragma once
#include "Geant/material/Element.hpp"
#include "Geant/material/MaterialProperties.hpp"
#include "Geant/core/PhysicalConstants.hpp" // the real Material.hpp brings it in
namespace geantx {
inline namespace GEANT_IMPL_NAMESPACE {
class Material {
public:
  Vector_t<Element *> fElements;
  MaterialProperties fProps;
  double fDensity = 0.0;
  const Vector_t<Element *> &GetElementVector() const { return fElements; }
  const MaterialProperties *GetMaterialProperties() const { return &fProps; }
  double GetDensity() const { return fDensity; }
};
} // namespace GEANT_IMPL_NAMESPACE
} // namespace geantx
