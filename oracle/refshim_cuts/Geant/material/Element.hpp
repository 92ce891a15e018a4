// Shim (oracle test infrastructure): the part of the reference's Element
// (source/Geant/material/Element.hpp) the cut converter reads: Z and the
// global element table.
#pragma once
#include "Geant/material/Types.hpp"
namespace geantx {
inline namespace GEANT_IMPL_NAMESPACE {
class Element {
public:
  explicit Element(double z) : fZ(z) { GetTheElementTable().push_back(this); }
  double GetZ() const { return fZ; }
  static Vector_t<Element *> &GetTheElementTable()
  {
    static Vector_t<Element *> table;
    return table;
  }

private:
  double fZ;
};
} // namespace GEANT_IMPL_NAMESPACE
} // namespace geantx
