// Shim (oracle test infrastructure): the reference's ProxyRandom
// (source/Geant/proxy/ProxyRandom.hpp:21-51) gives every process and model its
// own MRG32k3a stream.  This stand-in draws, through the reference's own
// MRG32k3a::Kernel, from a state the harness selects before each call, so a
// model can be fed exactly the stream the CUDA kernels are fed.
#pragma once
#include "Geant/random/MRG32k3a.hpp"
namespace geantx {
MRG32k3a::State_t *gxref_current_state();
MRG32k3a &gxref_engine();
class ProxyRandom {
public:
  ProxyRandom() {}
  double uniform() { return gxref_engine().Uniform(gxref_current_state()); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  void uniform_array(size_t n, double *array, const double min = 0., const double max = 1.) {
    for (size_t i = 0; i < n; ++i) array[i] = uniform(min, max);
  }
};
} // namespace geantx
