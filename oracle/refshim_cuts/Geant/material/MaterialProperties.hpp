// Shim (oracle test infrastructure): atoms per volume of each element of a
// material (source/Geant/material/MaterialProperties.hpp).
#pragma once
#include "Geant/material/Types.hpp"
namespace geantx {
inline namespace GEANT_IMPL_NAMESPACE {
class MaterialProperties {
public:
  Vector_t<double> fNumOfAtomsPerVolume;
  const double *GetNumOfAtomsPerVolumeVect() const { return fNumOfAtomsPerVolume.data(); }
};
} // namespace GEANT_IMPL_NAMESPACE
} // namespace geantx
