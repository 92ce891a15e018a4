/*
 * gxo_cuts.c -- ORACLE (test infrastructure only): the production-cut
 * converter, restated in C.
 *
 *   CutConverter::Initialise / Convert / BuildLengthVector /
 *     ConvertLengthToKineticEnergy / ConvertKineticEnergyToLength
 *     (source/Geant/cuts/src/CutConverter.cpp:54-280)
 *   CutConverterForGamma::BuildLengthVector, ComputeELossOrAbsXsecPerAtom
 *     (cuts/src/CutConverterForGamma.cpp:45-121)
 *   CutConverterForElectron / ForPositron::ComputeELossOrAbsXsecPerAtom
 *     (cuts/src/CutConverterForElectron.cpp:43-100, ForPositron.cpp:43-104)
 *   Spline with the accurate second derivatives (cuts/src/Spline.cpp:21-294)
 * with the reference's settings: 301 log-spaced energies from 990 eV to
 * 10 GeV (cuts/src/MaterialCuts.cpp:88-93, particles/src/PhysicsParameters.cpp:17-22).
 */
#include "gxo.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NBIN 301
#define EMIN 990.0e-6
#define EMAX 10.0e3

/* the reference's unit system (core/SystemOfUnits.hpp, core/PhysicalConstants.hpp) */
static const double kPi = 3.14159265358979323846;
static double u_g, u_cm2, u_cm3, u_barn, k_emass = 0.510998910, k_rcl;
static void cut_units(void)
{
  if (k_rcl != 0.0) return;
  const double e_SI = 1.602176487e-19, eplus = 1., eV = 1.e-6, s = 1.e+9, m = 1000.;
  const double joule = eV / e_SI, kg = joule * s * s / (m * m);
  u_g = 1.e-3 * kg;
  u_cm2 = 100.;
  u_cm3 = 1000.;
  u_barn = 1.e-28 * (m * m);
  const double coulomb = eplus / e_SI, ampere = coulomb / s, volt = 1.e-6 * (1. / eplus);
  const double weber = volt * s, henry = weber / ampere;
  const double c_light = 2.99792458e+8 * m / s, mu0 = 4 * kPi * 1.e-7 * henry / m;
  const double eps0 = 1. / (c_light * c_light * mu0);
  k_rcl = eplus * eplus / (4 * kPi * eps0) / k_emass;
}

/* photo-absorption cross section per atom (empirical), mm^2 */
static double gamma_xs(double Z, double e)
{
  const double t1keV = 1.0e-3, t200keV = 200.0e-3, t100MeV = 100.0;
  double Zsq = Z * Z, Zlog = log(Z), Zlogsq = Zlog * Zlog;
  double s200 = (0.2651 - 0.1501 * Zlog + 0.02283 * Zlogsq) * Zsq;
  double tmin = (0.552 + 218.5 / Z + 557.17 / Zsq);
  double smin = (0.01239 + 0.005585 * Zlog - 0.000923 * Zlogsq) * exp(1.5 * Zlog);
  double cmin = log(s200 / smin) / (log(tmin / t200keV) * log(tmin / t200keV));
  double tlow = 0.2 * exp(-7.355 / sqrt(Z));
  double slow = s200 * exp(0.042 * Z * log(t200keV / tlow) * log(t200keV / tlow));
  double s1keV = 300.0 * Zsq;
  double clow = log(s1keV / slow) / log(tlow / t1keV);
  double chigh = (7.55e-5 - 0.0542e-5 * Z) * Zsq * Z / log(t100MeV / tmin);
  double xs;
  if (e < tlow)
    xs = e < t1keV ? slow * exp(clow * log(tlow / t1keV)) : slow * exp(clow * log(tlow / e));
  else if (e < t200keV)
    xs = s200 * exp(0.042 * Z * log(t200keV / e) * log(t200keV / e));
  else if (e < tmin) {
    double dum = log(tmin / e);
    xs = smin * exp(cmin * dum * dum);
  } else
    xs = smin + chigh * log(e / tmin);
  return xs * u_barn;
}

/* approximate dE/dx per atom of e- (positron 0) or e+ (positron 1), MeV mm^2 */
static double charged_loss(int positron, double Z, double e)
{
  const double cbr1 = 0.02, cbr2 = -5.7e-5, cbr3 = 1., cbr4 = 0.072;
  const double tlow = 10.e-3, thigh = 1.e3, mass = k_emass, taul = tlow / mass;
  const double cpot = 1.6e-5, fact = 2 * kPi * k_emass * k_rcl * k_rcl;
  double ionpot = cpot * exp(0.9 * log(Z)) / mass, ionpotlog = log(ionpot);
  double tau = e / mass, x = tau < taul ? taul : tau;
  double t1 = x + 1., t2 = x + 2., tsq = x * x, beta2 = x * t2 / (t1 * t1), f;
  if (!positron)
    f = 1. - beta2 + log(tsq / 2.) + (0.5 + 0.25 * tsq + (1. + 2. * x) * log(0.5)) / (t1 * t1);
  else
    f = 2. * log(x) - (6. * x + 1.5 * tsq - x * (1. - tsq / 3.) / t2 - tsq * (0.5 - tsq / 12.) / (t2 * t2)) / (t1 * t1);
  double dedx = (log(2. * x + 4.) - 2. * ionpotlog + f) / beta2;
  dedx = fact * Z * dedx;
  if (tau < taul) return dedx * sqrt(taul) / sqrt(tau);
  double cbrem = (cbr1 + cbr2 * Z) * (cbr3 + cbr4 * log(e / thigh));
  cbrem = 0.1 * Z * (Z + 1.) * cbrem * tau / beta2;
  return dedx + fact * cbrem;
}

/* cubic spline through (x, y) with not-a-knot second derivatives, evaluated
 * as a + dx (b + dx (c + dx d)) per interval (Spline.cpp:185-294) */
typedef struct { const double *x, *y; int n; double a[NBIN], b[NBIN], c[NBIN], d[NBIN]; } spline_t;

static void spline_init(spline_t *s, const double *x, const double *y, int N)
{
  s->x = x;
  s->y = y;
  s->n = N;
  int n = N - 1;
  double u[NBIN], d2[NBIN];
  memset(d2, 0, sizeof(d2));
  u[1] = ((y[2] - y[1]) / (x[2] - x[1]) - (y[1] - y[0]) / (x[1] - x[0]));
  u[1] = 6.0 * u[1] * (x[2] - x[1]) / ((x[2] - x[0]) * (x[2] - x[0]));
  d2[1] = (2.0 * x[1] - x[0] - x[2]) / (2.0 * x[2] - x[0] - x[1]);
  for (int i = 2; i < n - 1; ++i) {
    double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
    double p = sig * d2[i - 1] + 2.0;
    d2[i] = (sig - 1.0) / p;
    u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
    u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1])) - sig * u[i - 1] / p;
  }
  double sig = (x[n - 1] - x[n - 2]) / (x[n] - x[n - 2]);
  double p = sig * d2[n - 3] + 2.0;
  u[n - 1] = (y[n] - y[n - 1]) / (x[n] - x[n - 1]) - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
  u[n - 1] = 6.0 * sig * u[n - 1] / (x[n] - x[n - 2]) - (2.0 * sig - 1.0) * u[n - 2] / p;
  p = (1.0 + sig) + (2.0 * sig - 1.0) * d2[n - 2];
  d2[n - 1] = u[n - 1] / p;
  for (int k = n - 2; k > 1; --k) d2[k] *= (d2[k + 1] - u[k] * (x[k + 1] - x[k - 1]) / (x[k + 1] - x[k]));
  d2[n] = (d2[n - 1] - (1.0 - sig) * d2[n - 2]) / sig;
  sig = 1.0 - ((x[2] - x[1]) / (x[2] - x[0]));
  d2[1] *= (d2[2] - u[1] / (1.0 - sig));
  d2[0] = (d2[1] - sig * d2[2]) / (1.0 - sig);
  for (int i = 0; i < n; ++i) {
    double dx = x[i + 1] - x[i];
    s->a[i] = y[i];
    s->b[i] = (y[i + 1] - y[i]) / dx - (2.0 * d2[i] + d2[i + 1]) * dx / 6.0;
    s->c[i] = 0.5 * d2[i];
    s->d[i] = (d2[i + 1] - d2[i]) / (6.0 * dx);
  }
}

static double spline_value(const spline_t *s, double v)
{
  /* first node >= v among x[0 .. n-2], then one back */
  int lo = 0, hi = s->n - 1;
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (s->x[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  int m = lo > 0 ? lo - 1 : 0;
  if (s->y[m] + s->y[m + 1] == 0.0) return 0.0;
  v -= s->x[m];
  return s->a[m] + v * (s->b[m] + v * (s->c[m] + v * s->d[m]));
}

/* The energy (MeV) of a cut given as a length (mm), or the length of a cut
 * given as an energy (from_length 0), for particle 0 gamma / 1 e- / 2 e+ in a
 * material of nelem elements Z with n_atoms per mm^3 and density in g/cm^3. */
double gxo_cut_convert(int particle, int nelem, const double *Z, const double *n_atoms, double density, double cut,
                       int from_length)
{
  cut_units();
  double E[NBIN], L[NBIN];
  double delta = log(EMAX / EMIN) / (NBIN - 1), base = log(EMIN) / delta;
  for (int i = 0; i < NBIN - 1; ++i) E[i] = exp((base + i) * delta);
  E[NBIN - 1] = EMAX;
  int maxidx = -1;
  if (particle == 0) {
    /* absorption length: 5 / macroscopic absorption cross section */
    double maxlen = -1.0;
    for (int i = 0; i < NBIN; ++i) {
      double mac = 0.0;
      for (int k = 0; k < nelem; ++k) mac += n_atoms[k] * gamma_xs(Z[k], E[i]);
      L[i] = 5.0 / mac;
      if (maxlen < L[i]) {
        maxlen = L[i];
        maxidx = i;
      }
    }
  } else {
    /* range: integral of E / (dE/dx) d(log E), trapezoidal on the log grid */
    double loss[NBIN];
    for (int i = 0; i < NBIN; ++i) {
      double l = 0.0;
      for (int k = 0; k < nelem; ++k) l += n_atoms[k] * charged_loss(particle == 2, Z[k], E[i]);
      loss[i] = l;
    }
    double de = log(EMAX / EMIN);
    de /= (NBIN - 1);
    L[0] = E[0] / loss[0] * de;
    double sum = 0.5 * E[0] / loss[0];
    for (int i = 1; i < NBIN; ++i) {
      double q = E[i] / loss[i];
      sum += q;
      L[i] = (sum - 0.5 * q) * de;
    }
  }
  static spline_t sp; /* large: keep it off the stack */
  if (!from_length) {
    if (cut <= EMIN) return L[0];
    if (cut >= EMAX) return L[NBIN - 1];
    int istart = 0, num = NBIN;
    if (maxidx > -1) {
      if (cut < E[maxidx])
        num = maxidx + 1;
      else {
        istart = maxidx;
        num = NBIN - maxidx;
      }
    }
    spline_init(&sp, E + istart, L + istart, num);
    return spline_value(&sp, cut);
  }
  /* length -> energy by bisection on the spline of L(E), to 1% (Geant4's way) */
  const double eps = 0.01;
  double rmax = -1.0, T1 = EMIN, r1 = L[0], T2 = EMAX, e;
  if (cut <= r1) {
    e = T1;
  } else {
    for (int i = 0; i < NBIN; ++i) {
      double T = E[i], r = L[i];
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
      e = EMAX;
    } else {
      spline_init(&sp, E, L, NBIN);
      double T3 = sqrt(T1 * T2), r3 = spline_value(&sp, T3);
      for (int itr = 0; itr < 1000; ++itr) {
        if (fabs(1.0 - r3 / cut) < eps) break;
        if (cut <= r3)
          T2 = T3;
        else
          T1 = T3;
        T3 = sqrt(T1 * T2);
        r3 = spline_value(&sp, T3);
      }
      e = T3;
    }
  }
  /* low-energy correction for e-/e+ */
  const double lowen = 30.0e-3, tune = 0.0025 * u_g / u_cm2;
  if ((particle == 1 || particle == 2) && e < lowen) e /= (1.0 + (1.0 - e / lowen) * tune / (cut * (density * u_g / u_cm3)));
  if (e < EMIN)
    e = EMIN;
  else if (e > EMAX)
    e = EMAX;
  return e;
}
