// Shim (oracle test infrastructure): the container aliases the reference's
// cut converter and spline (source/Geant/cuts) take from material/Types.hpp,
// without its VecGeom device declarations.
#pragma once
#include "Geant/core/Config.hpp"
#include <map>
#include <vector>
namespace geantx {
inline namespace GEANT_IMPL_NAMESPACE {
template <class T> using Vector_t = std::vector<T>;
template <class K, class V> using Map_t = std::map<K, V>;
} // namespace GEANT_IMPL_NAMESPACE
} // namespace geantx
