// Shim (oracle test infrastructure): the Process base of
// source/Geant/processes/Process.hpp reduced to its constructors.
#pragma once
#include "Geant/track/TrackState.hpp"
#include <cfloat>
namespace geantx {
class Process {
public:
  Process() {}
  explicit Process(int) {}
};
} // namespace geantx
