// gx_cuts.cu -- production-cut conversion (range cut -> energy threshold) on
// the host, and the context's cut table built from it instead of read from
// the Geant4-dumped cut.dat.
//
// The reference's converter (source/Geant/cuts/src/CutConverter.cpp:54-280,
// CutConverterForGamma.cpp:45-121, CutConverterForElectron.cpp:43-100,
// CutConverterForPositron.cpp:43-104, Spline.cpp:185-294), with its settings
// (301 log-spaced energies from 990 eV to 10 GeV, MaterialCuts.cpp:88-93):
// per element an empirical photo-absorption cross section (photons) or an
// approximate dE/dx (e-, e+); per material the absorption length 5 / Sum n
// sigma or the range Integral E / (dE/dx) d(log E); the length cut converted
// to energy by bisection (to 1%) on a not-a-knot spline of length(E); for
// e-/e+ below 30 keV the reference's low-energy correction.  This is a few
// thousand scalar operations per (particle, material), run once per context:
// host code, not a kernel.
#include "gx_internal.cuh"

#include <cmath>
#include <cstring>
#include <vector>

namespace gx {

namespace {

constexpr int kBins = 301;
constexpr double kCutEmin = 990.0e-6, kCutEmax = 10.0e3; // MeV

// the reference's unit chain (core/SystemOfUnits.hpp, core/PhysicalConstants.hpp)
struct CutUnits {
  double g, cm2, cm3, barn, rcl;
  CutUnits()
  {
    const double e_SI = 1.602176487e-19, eplus = 1., eVu = 1.e-6, s = 1.e+9, m = 1000.;
    const double joule = eVu / e_SI, kg = joule * s * s / (m * m);
    g = 1.e-3 * kg;
    cm2 = 100.;
    cm3 = 1000.;
    barn = 1.e-28 * (m * m);
    const double coulomb = eplus / e_SI, ampere = coulomb / s, volt = 1.e-6 * (1. / eplus);
    const double weber = volt * s, henry = weber / ampere;
    const double c_light = 2.99792458e+8 * m / s, mu0 = 4 * kPi * 1.e-7 * henry / m;
    const double eps0 = 1. / (c_light * c_light * mu0);
    rcl = eplus * eplus / (4 * kPi * eps0) / kEMass;
  }
};
const CutUnits &units()
{
  static const CutUnits u;
  return u;
}

// empirical photo-absorption cross section per atom, mm^2
double gamma_absorption_xs(double Z, double e)
{
  const double t1keV = 1.0e-3, t200keV = 200.0e-3, t100MeV = 100.0;
  const double Zsq = Z * Z, Zlog = std::log(Z), Zlogsq = Zlog * Zlog;
  const double s200 = (0.2651 - 0.1501 * Zlog + 0.02283 * Zlogsq) * Zsq;
  const double tmin = (0.552 + 218.5 / Z + 557.17 / Zsq);
  const double smin = (0.01239 + 0.005585 * Zlog - 0.000923 * Zlogsq) * std::exp(1.5 * Zlog);
  const double cmin = std::log(s200 / smin) / (std::log(tmin / t200keV) * std::log(tmin / t200keV));
  const double tlow = 0.2 * std::exp(-7.355 / std::sqrt(Z));
  const double slow = s200 * std::exp(0.042 * Z * std::log(t200keV / tlow) * std::log(t200keV / tlow));
  const double s1keV = 300.0 * Zsq;
  const double clow = std::log(s1keV / slow) / std::log(tlow / t1keV);
  const double chigh = (7.55e-5 - 0.0542e-5 * Z) * Zsq * Z / std::log(t100MeV / tmin);
  double xs;
  if (e < tlow)
    xs = e < t1keV ? slow * std::exp(clow * std::log(tlow / t1keV)) : slow * std::exp(clow * std::log(tlow / e));
  else if (e < t200keV)
    xs = s200 * std::exp(0.042 * Z * std::log(t200keV / e) * std::log(t200keV / e));
  else if (e < tmin) {
    const double dum = std::log(tmin / e);
    xs = smin * std::exp(cmin * dum * dum);
  } else
    xs = smin + chigh * std::log(e / tmin);
  return xs * units().barn;
}

// approximate dE/dx per atom of an e- or an e+ (ionisation, plus brems above 10 keV), MeV mm^2
double charged_loss(bool positron, double Z, double e)
{
  const double cbr1 = 0.02, cbr2 = -5.7e-5, cbr3 = 1., cbr4 = 0.072;
  const double tlow = 10.e-3, thigh = 1.e3, mass = kEMass, taul = tlow / mass, cpot = 1.6e-5;
  const double rcl = units().rcl, fact = 2 * kPi * kEMass * rcl * rcl;
  const double ionpot = cpot * std::exp(0.9 * std::log(Z)) / mass, ionpotlog = std::log(ionpot);
  const double tau = e / mass, x = tau < taul ? taul : tau;
  const double t1 = x + 1., t2 = x + 2., tsq = x * x, beta2 = x * t2 / (t1 * t1);
  const double f =
      positron ? 2. * std::log(x) -
                     (6. * x + 1.5 * tsq - x * (1. - tsq / 3.) / t2 - tsq * (0.5 - tsq / 12.) / (t2 * t2)) / (t1 * t1)
               : 1. - beta2 + std::log(tsq / 2.) + (0.5 + 0.25 * tsq + (1. + 2. * x) * std::log(0.5)) / (t1 * t1);
  double dedx = (std::log(2. * x + 4.) - 2. * ionpotlog + f) / beta2;
  dedx = fact * Z * dedx;
  if (tau < taul) return dedx * std::sqrt(taul) / std::sqrt(tau);
  double cbrem = (cbr1 + cbr2 * Z) * (cbr3 + cbr4 * std::log(e / thigh));
  cbrem = 0.1 * Z * (Z + 1.) * cbrem * tau / beta2;
  return dedx + fact * cbrem;
}

// Cubic spline through (x, y), not-a-knot second derivatives, evaluated per
// interval as a + dx (b + dx (c + dx d)); needs at least 5 points.
struct Spline {
  const double *x, *y;
  int n;
  std::vector<double> a, b, c, d;
  Spline(const double *xs, const double *ys, int N) : x(xs), y(ys), n(N), a(N), b(N), c(N), d(N)
  {
    const int m = N - 1;
    std::vector<double> u(N, 0.0), d2(N, 0.0);
    u[1] = ((y[2] - y[1]) / (x[2] - x[1]) - (y[1] - y[0]) / (x[1] - x[0]));
    u[1] = 6.0 * u[1] * (x[2] - x[1]) / ((x[2] - x[0]) * (x[2] - x[0]));
    d2[1] = (2.0 * x[1] - x[0] - x[2]) / (2.0 * x[2] - x[0] - x[1]);
    for (int i = 2; i < m - 1; ++i) {
      const double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
      const double p = sig * d2[i - 1] + 2.0;
      d2[i] = (sig - 1.0) / p;
      u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
      u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1])) - sig * u[i - 1] / p;
    }
    double sig = (x[m - 1] - x[m - 2]) / (x[m] - x[m - 2]);
    double p = sig * d2[m - 3] + 2.0;
    u[m - 1] = (y[m] - y[m - 1]) / (x[m] - x[m - 1]) - (y[m - 1] - y[m - 2]) / (x[m - 1] - x[m - 2]);
    u[m - 1] = 6.0 * sig * u[m - 1] / (x[m] - x[m - 2]) - (2.0 * sig - 1.0) * u[m - 2] / p;
    p = (1.0 + sig) + (2.0 * sig - 1.0) * d2[m - 2];
    d2[m - 1] = u[m - 1] / p;
    for (int k = m - 2; k > 1; --k) d2[k] *= (d2[k + 1] - u[k] * (x[k + 1] - x[k - 1]) / (x[k + 1] - x[k]));
    d2[m] = (d2[m - 1] - (1.0 - sig) * d2[m - 2]) / sig;
    sig = 1.0 - ((x[2] - x[1]) / (x[2] - x[0]));
    d2[1] *= (d2[2] - u[1] / (1.0 - sig));
    d2[0] = (d2[1] - sig * d2[2]) / (1.0 - sig);
    for (int i = 0; i < m; ++i) {
      const double dx = x[i + 1] - x[i];
      a[i] = y[i];
      b[i] = (y[i + 1] - y[i]) / dx - (2.0 * d2[i] + d2[i + 1]) * dx / 6.0;
      c[i] = 0.5 * d2[i];
      d[i] = (d2[i + 1] - d2[i]) / (6.0 * dx);
    }
  }
  double operator()(double v) const
  {
    int lo = 0, hi = n - 1; // first node >= v among x[0 .. n-2], then one back
    while (lo < hi) {
      const int mid = (lo + hi) / 2;
      if (x[mid] < v)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int m = lo > 0 ? lo - 1 : 0;
    if (y[m] + y[m + 1] == 0.0) return 0.0;
    v -= x[m];
    return a[m] + v * (b[m] + v * (c[m] + v * d[m]));
  }
};

} // namespace

// Energy (MeV) of a cut given as a length (mm), or length of a cut given as
// an energy (from_length false); particle 0 gamma, 1 e-, 2 e+.
double cut_convert(int particle, int nelem, const double *Z, const double *n_atoms, double density, double cut,
                   bool from_length)
{
  double E[kBins], L[kBins];
  const double delta = std::log(kCutEmax / kCutEmin) / (kBins - 1), base = std::log(kCutEmin) / delta;
  for (int i = 0; i < kBins - 1; ++i) E[i] = std::exp((base + i) * delta);
  E[kBins - 1] = kCutEmax;
  int maxidx = -1;
  if (particle == 0) {
    double maxlen = -1.0;
    for (int i = 0; i < kBins; ++i) {
      double mac = 0.0;
      for (int k = 0; k < nelem; ++k) mac += n_atoms[k] * gamma_absorption_xs(Z[k], E[i]);
      L[i] = 5.0 / mac;
      if (maxlen < L[i]) {
        maxlen = L[i];
        maxidx = i;
      }
    }
  } else {
    double loss[kBins];
    for (int i = 0; i < kBins; ++i) {
      double l = 0.0;
      for (int k = 0; k < nelem; ++k) l += n_atoms[k] * charged_loss(particle == 2, Z[k], E[i]);
      loss[i] = l;
    }
    double de = std::log(kCutEmax / kCutEmin);
    de /= (kBins - 1);
    L[0] = E[0] / loss[0] * de;
    double sum = 0.5 * E[0] / loss[0];
    for (int i = 1; i < kBins; ++i) {
      const double q = E[i] / loss[i];
      sum += q;
      L[i] = (sum - 0.5 * q) * de;
    }
  }
  if (!from_length) {
    if (cut <= kCutEmin) return L[0];
    if (cut >= kCutEmax) return L[kBins - 1];
    int istart = 0, num = kBins;
    if (maxidx > -1) {
      if (cut < E[maxidx])
        num = maxidx + 1;
      else {
        istart = maxidx;
        num = kBins - maxidx;
      }
    }
    if (num < 5) { // below the spline's minimum: linear in the first interval
      const int m = istart;
      return L[m] + (L[m + 1] - L[m]) * (cut - E[m]) / (E[m + 1] - E[m]);
    }
    return Spline(E + istart, L + istart, num)(cut);
  }
  const double eps = 0.01;
  double rmax = -1.0, T1 = kCutEmin, r1 = L[0], T2 = kCutEmax, e;
  if (cut <= r1) {
    e = T1;
  } else {
    for (int i = 0; i < kBins; ++i) {
      const double T = E[i], r = L[i];
      if (r > rmax) rmax = r;
      if (r < cut) {
        T1 = T;
        r1 = r;
      } else if (r > cut) {
        T2 = T;
        break;
      }
    }
    if (cut >= rmax) {
      e = kCutEmax;
    } else {
      const Spline sp(E, L, kBins);
      double T3 = std::sqrt(T1 * T2), r3 = sp(T3);
      for (int itr = 0; itr < 1000; ++itr) {
        if (std::fabs(1.0 - r3 / cut) < eps) break;
        if (cut <= r3)
          T2 = T3;
        else
          T1 = T3;
        T3 = std::sqrt(T1 * T2);
        r3 = sp(T3);
      }
      e = T3;
    }
  }
  const CutUnits &u = units();
  const double lowen = 30.0e-3, tune = 0.0025 * u.g / u.cm2;
  if ((particle == 1 || particle == 2) && e < lowen)
    e /= (1.0 + (1.0 - e / lowen) * tune / (cut * (density * u.g / u.cm3)));
  return e < kCutEmin ? kCutEmin : (e > kCutEmax ? kCutEmax : e);
}

} // namespace gx

using namespace gx;

extern "C" {

int gx_cut_convert(int particle, int nelem, const double *Z, const double *n_atoms, double density, double cut,
                   int from_length, double *out)
{
  if (!out || particle < 0 || particle > 2 || nelem <= 0 || nelem > 64 || !Z || !n_atoms || !(cut > 0.0) ||
      !(density > 0.0))
    return set_error(GX_ERR_ARG, "gx_cut_convert: bad arguments");
  for (int k = 0; k < nelem; ++k)
    if (!(Z[k] >= 1.0 && Z[k] <= 120.0) || !(n_atoms[k] > 0.0))
      return set_error(GX_ERR_ARG, "gx_cut_convert: element %d: Z %g, atoms per mm^3 %g", k, Z[k], n_atoms[k]);
  *out = cut_convert(particle, nelem, Z, n_atoms, density, cut, from_length != 0);
  return GX_OK;
}

int gx_ctx_compute_cuts(gx_ctx *ctx, double cut_mm)
{
  if (!ctx || !(cut_mm > 0.0)) return set_error(GX_ERR_ARG, "gx_ctx_compute_cuts: bad arguments");
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  Data &d = c->host;
  for (int m = 0; m < kNMat; ++m) {
    const double Z = d.mat_Z[m], n_atoms = d.mat_nel[m] / d.mat_Z[m];
    for (int p = 0; p < 3; ++p) {
      const double e = cut_convert(p, 1, &Z, &n_atoms, d.mat_density[m], cut_mm, true);
      d.cut_energy[p][m] = e;
      d.cut_length[p][m] = cut_mm;
      d.cut_raw[p * kNMat + m] = e * 1.0e3; // keV, in the file's order
    }
    // protons: 100 keV per mm of range cut (Geant4's converter for protons;
    // the reference has none, its cut.dat holds 70 keV for 0.7 mm)
    d.cut_energy[3][m] = 0.1 * cut_mm;
    d.cut_length[3][m] = cut_mm;
    d.cut_raw[3 * kNMat + m] = 100.0 * cut_mm;
  }
  cudaError_t e = cudaSetDevice(c->device);
  if (e == cudaSuccess) e = cudaMemcpy(c->dev, &d, sizeof(Data), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? GX_OK : cuda_error(e, "gx_ctx_compute_cuts: upload");
}

} // extern "C"
