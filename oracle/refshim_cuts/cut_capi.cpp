// cut_capi.cpp -- ORACLE (test infrastructure only).
//
// Drives the reference's production-cut converter (source/Geant/cuts:
// CutConverter, CutConverterForGamma/Electron/Positron, Spline) compiled in
// place through the material shims in this directory, to pin the oracle's and
// the library's restatement of it.  Built into its own library
// (oracle/_ref/libgxref_cuts.so) because these shims define Material and
// Element differently from the model harness's shims.
#include "Geant/cuts/CutConverterForElectron.hpp"
#include "Geant/cuts/CutConverterForGamma.hpp"
#include "Geant/cuts/CutConverterForPositron.hpp"

#include <map>

using namespace geantx;

namespace {
Element *element(double Z)
{
  static std::map<int, Element *> table;
  Element *&e = table[(int)(Z + 0.5)];
  if (!e) e = new Element(Z);
  return e;
}
} // namespace

extern "C" {

// Registers the elements first: a converter sizes its per-Z tables from the
// element table when it is built.
void gxref_cut_elements(int n, const double *Z)
{
  for (int i = 0; i < n; ++i) element(Z[i]);
}

// CutConverter::Convert (cuts/src/CutConverter.cpp:107-128) for particle
// 0 gamma / 1 e- / 2 e+ with the reference's settings (301 bins, 990 eV to
// 10 GeV, MaterialCuts.cpp:88-93): the energy (MeV) of a production cut given
// as a length (mm), or the length of a cut given as an energy when
// from_length is 0.  Material: nelem elements Z with atoms per mm^3, density
// in g/cm^3.
double gxref_cut_convert(int particle, int nelem, const double *Z, const double *n_atoms, double density,
                         double cut, int from_length)
{
  Material m;
  for (int i = 0; i < nelem; ++i) {
    m.fElements.push_back(element(Z[i]));
    m.fProps.fNumOfAtomsPerVolume.push_back(n_atoms[i] / (geantx::units::mm * geantx::units::mm * geantx::units::mm));
  }
  m.fDensity = density * geantx::units::g / geantx::units::cm3;
  const double emin = 990.0 * geantx::units::eV, emax = 10.0 * geantx::units::GeV;
  CutConverter *c = nullptr;
  if (particle == 0)
    c = new CutConverterForGamma(301, emin, emax);
  else if (particle == 1)
    c = new CutConverterForElectron(301, emin, emax);
  else
    c = new CutConverterForPositron(301, emin, emax);
  double v = c->Convert(&m, from_length ? cut * geantx::units::mm : cut * geantx::units::MeV, from_length != 0);
  delete c;
  return from_length ? v / geantx::units::MeV : v / geantx::units::mm;
}

} // extern "C"
