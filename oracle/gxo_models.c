/*
 * gxo_models.c -- ORACLE (test infrastructure only): the reference's EM
 * interaction models, process step limits, ionisation along-step loss and the
 * constant-field helix step, restated in plain C.
 *
 * Every model has two modes sharing one code path:
 *   GXO_MODE_QUIRK   reproduces the reference exactly (hard-coded Z = 10,
 *                    inverted photo-electron shell choice, Tsai angle used as
 *                    a cosine, 1 keV cuts, ...), so it can be compared with
 *                    the reference's own code at 1e-12;
 *   GXO_MODE_PHYSICS uses the element of the material, the production cuts
 *                    and the corrected formulas, for whole showers.
 */
#include "gxo.h"

#include <float.h>
#include <math.h>
#include <string.h>

/* --- constants: the derivation chain of source/Geant/proxy/ProxySystemOfUnits.hpp
 *     and ProxyPhysicalConstants.hpp (CLHEP definitions), in the same order. */
#define PI 3.14159265358979323846
#define TWOPI (2 * PI)
#define MEV 1.0
#define KEV 1.e-3
#define EV 1.e-6
#define TEV 1.e+6
#define EMASS 0.510998910
static double g_rcl = 0, g_twopi_mc2_rcl2 = 0, g_pi_rcl2 = 0, g_compton_len = 0, g_alpha = 0;
static void init_constants(void)
{
  if (g_rcl != 0) return;
  const double eplus = 1., e_SI = 1.602176487e-19;
  const double coulomb = eplus / e_SI, second = 1.e+9, meter = 1000.;
  const double ampere = coulomb / second;
  const double megavolt = 1. / eplus, volt = 1.e-6 * megavolt;
  const double weber = volt * second, henry = weber / ampere;
  const double mu0 = 4 * PI * 1.e-7 * henry / meter;
  const double c_light = 2.99792458e+8 * meter / second;
  const double c_squared = c_light * c_light;
  const double epsilon0 = 1. / (c_squared * mu0);
  const double elm_coupling = eplus * eplus / (4 * PI * epsilon0);
  const double joule = EV / e_SI;
  const double h_Planck = 6.62606896e-34 * joule * second;
  const double hbarc = h_Planck / TWOPI * c_light;
  g_rcl = elm_coupling / EMASS;
  g_twopi_mc2_rcl2 = TWOPI * EMASS * g_rcl * g_rcl;
  g_pi_rcl2 = PI * g_rcl * g_rcl;
  g_compton_len = hbarc / EMASS;
  g_alpha = elm_coupling / hbarc;
}

/* Tsai's radiation-length factor of an element (ProxyElementUtils.cu:40-61,
 * with its Coulomb correction ComputeCoulombFactor, :24-37). */
static double lrad_tsai_factor(double Z)
{
  static const double lrad_light[] = {5.31, 4.79, 4.74, 4.71};
  static const double lprad_light[] = {6.144, 5.621, 5.805, 5.924};
  double logZ3 = log(Z) / 3.;
  double lrad, lprad;
  int iz = (int)(Z + 0.5) - 1;
  if (iz <= 3) {
    lrad = lrad_light[iz];
    lprad = lprad_light[iz];
  } else {
    lrad = log(184.15) - logZ3;
    lprad = log(1194.) - 2 * logZ3;
  }
  double az1 = g_alpha * Z, az2 = az1 * az1, az4 = az2 * az2;
  double fc = (0.0083 * az4 + 0.20206 + 1. / (1. + az2)) * az2 - (0.0020 * az4 + 0.0369) * az4;
  return 4 * g_alpha * g_rcl * g_rcl * Z * (Z * (lrad - fc) + lprad);
}

/* Math::RotateToLabFrame, source/Geant/core/math_wrappers.hpp:194-212 */
void gxo_rotate_to_lab(double *u, double *v, double *w, double u1, double u2, double u3)
{
  double up = u1 * u1 + u2 * u2;
  int m1 = up > 0.0;
  up = sqrt(up);
  double px = *u, py = *v, pz = *w;
  if (m1) {
    *u = (u3 * px * u1 - u2 * py) * (1.0 / up) + u1 * pz;
    *v = (u3 * px * u2 + u1 * py) * (1.0 / up) + u2 * pz;
    *w = -up * px + u3 * pz;
  } else if (u3 < 0.) {
    *u = -*u;
    *w = -*w;
  }
}

/* ThreeVector::Unit as the shim-compiled reference evaluates it: v / |v| */
static void unit3(double *x, double *y, double *z)
{
  double m = sqrt(*x * *x + *y * *y + *z * *z);
  if (m > 0) {
    *x /= m;
    *y /= m;
    *z /= m;
  }
}

static void add_sec(gxo_inter_t *io, int type, double e, double dx, double dy, double dz)
{
  int k = io->nsec++;
  io->sec_type[k] = type;
  io->sec_E[k] = e;
  io->sec_dir[k][0] = dx;
  io->sec_dir[k][1] = dy;
  io->sec_dir[k][2] = dz;
}

/* ProxyEmModel::ComputeCoulombFactor, source/Geant/proxy/ProxyEmModel.hpp:114-128 */
double gxo_coulomb_factor(double Zeff)
{
  double k1 = 0.0083, k2 = 0.20206, k3 = 0.0020, k4 = 0.0369;
  double fine_structure_const = (1.0 / 137);
  double az1 = fine_structure_const * Zeff;
  double az2 = az1 * az1;
  double az4 = az2 * az2;
  return (k1 * az4 + k2 + 1. / (1. + az2)) * az2 - (k3 * az4 + k4) * az4;
}

/* ---------------------------------------------------------- Klein-Nishina */
/* ProxyKleinNishina::CrossSectionPerAtom, ProxyKleinNishina.hpp:62-93.  The
 * low-energy threshold T0 is 15 * geantx::units::keV in the reference, a
 * GeV-based unit, i.e. 1.5e-5 in the MeV-based arithmetic around it. */
double gxo_kn_xs_per_atom(double Z, double e)
{
  double Z2 = Z * Z;
  double p1 = 2.7965e-1 + 1.9756e-5 * Z + -3.9178e-7 * Z2;
  double p2 = -1.8300e-1 + -1.0205e-2 * Z + 6.8241e-5 * Z2;
  double p3 = 6.7527 + -7.3913e-2 * Z + 6.0480e-5 * Z2;
  double p4 = -1.9798e+1 + 2.7079e-2 * Z + 3.0274e-4 * Z2;
  double T0 = (Z < 1.5) ? 40.0 * KEV : 15.0 * 1.e-6;
  double X = fmax(e, T0) / EMASS;
  double X2 = X * X;
  double xs = p1 * log(1. + 2. * X) / X + (p2 + p3 * X + p4 * X2) / (1. + 20. * X + 230. * X2 + 440. * X2 * X);
  if (e < T0) {
    const double dT0 = KEV;
    X = (T0 + dT0) / EMASS;
    X2 = X * X;
    double sigma = p1 * log(1. + 2. * X) / X + (p2 + p3 * X + p4 * X2) / (1. + 20. * X + 230. * X2 + 440. * X2 * X);
    double c1 = -T0 * (sigma - xs) / (xs * dT0);
    double c2 = (Z > 1.5) ? 0.375 - 0.0556 * log(Z) : 0.150;
    double y = log(e / T0);
    xs *= exp(-y * (c1 + c2 * y));
  }
  return Z * xs * (1.e-28 * (1000. * 1000.)); /* barn = 1e-28 * meter2 */
}

/* ProxyKleinNishina::SampleSecondaries, ProxyKleinNishina.hpp:96-166 */
int gxo_kn_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io)
{
  const double low = 100.0 * EV;
  double E0 = io->E;
  io->nsec = 0;
  if (E0 < low) return 0;
  double d0x = io->dir[0], d0y = io->dir[1], d0z = io->dir[2];
  double epsilon, epsilonsq, onecost, sint2, greject;
  double E0_m = E0 / EMASS;
  double eps0 = 1. / (1. + 2. * E0_m);
  double epsilon0sq = eps0 * eps0;
  double alpha1 = -gxo_log(eps0);
  double alpha2 = 0.5 * (1. - epsilon0sq);
  do {
    if (alpha1 / (alpha1 + alpha2) > gxo_mrg_u01(r)) {
      epsilon = gxo_exp(-alpha1 * gxo_mrg_u01(r));
      epsilonsq = epsilon * epsilon;
    } else {
      epsilonsq = epsilon0sq + (1. - epsilon0sq) * gxo_mrg_u01(r);
      epsilon = sqrt(epsilonsq);
    }
    onecost = (1. - epsilon) / (epsilon * E0_m);
    sint2 = onecost * (2. - onecost);
    greject = 1. - epsilon * sint2 / (1. + epsilonsq);
  } while (greject < gxo_mrg_u01(r));
  double sinTheta = (sint2 < 0.0) ? 0.0 : sqrt(sint2);
  double phi = TWOPI * gxo_mrg_u01(r);
  double gE = epsilon * E0;
  double gx = sinTheta * gxo_cos(phi), gy = sinTheta * gxo_sin(phi), gz = 1. - onecost;
  gxo_rotate_to_lab(&gx, &gy, &gz, d0x, d0y, d0z);
  if (gE > low) {
    io->dir[0] = gx;
    io->dir[1] = gy;
    io->dir[2] = gz;
    io->E = gE;
  } else {
    io->status = 1;
    io->edep += gE;
  }
  double eKin = E0 - gE;
  /* the reference tests the scattered photon energy here (:151); physics mode
   * tests the electron's own energy as Geant4's Klein-Nishina model does */
  int make_e = (p->mode == GXO_MODE_QUIRK) ? (gE > low) : (eKin > low);
  if (make_e) {
    double ex = E0 * d0x - gE * gx, ey = E0 * d0y - gE * gy, ez = E0 * d0z - gE * gz;
    unit3(&ex, &ey, &ez);
    add_sec(io, 1, eKin, ex, ey, ez);
  } else {
    io->edep += eKin;
  }
  return io->nsec;
}

/* --------------------------------------------------------- Sauter-Gavrila */
/* ProxySauterGavrila::GetPhotoElectronEnergy, ProxySauterGavrila.hpp:132-145.
 * Quirk: the loop stops at the first shell whose binding energy exceeds the
 * photon energy and returns E minus that shell (or the next element's K shell).
 * Physics: shells are stored K first, so the first shell with B <= E is the
 * innermost one the photon can ionise; 0 if there is none. */
double gxo_sg_photo_electron_energy(const gxo_data_t *d, int Z, double e, int mode)
{
  int n = d->nshell[Z];
  const double *b = &d->binding[d->ishell[Z]];
  int i = 0;
  if (mode == GXO_MODE_QUIRK) {
    while (i < n && e >= b[i] * EV) i++;
    return i <= n ? e - b[i] * EV : 0.0;
  }
  while (i < n && e < b[i] * EV) i++;
  return (i < n) ? e - b[i] * EV : 0.0;
}

/* ProxySauterGavrila::SampleSecondaries, ProxySauterGavrila.hpp:67-130 */
int gxo_sg_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io)
{
  double gE = io->E;
  io->nsec = 0;
  int Z = (p->mode == GXO_MODE_QUIRK) ? 10 : p->Z;
  double eE = gxo_sg_photo_electron_energy(p->data, Z, gE, p->mode);
  if (p->mode == GXO_MODE_PHYSICS && eE <= 0.0) {
    io->edep += gE;
    io->E = 0.0;
    io->status = 1;
    return 0;
  }
  double tau = gE / EMASS;
  double cost = -1.0;
  if (tau > 50.0) {
    cost = 1.0;
  } else {
    double gam = tau + 1.;
    double beta = sqrt(tau * (tau + 2.)) / gam;
    double A = (1 - beta) / beta;
    double Ap2 = A + 2.;
    double B = 0.5 * beta * gam * (gam - 1.) * (gam - 2.);
    double grej = 2. * (1. + A * B) / A;
    double z, g;
    do {
      double q = gxo_mrg_u01(r);
      z = 2 * A * (2 * q + Ap2 * sqrt(q)) / (Ap2 * Ap2 - 4 * q);
      g = (2 - z) * (1.0 / (A + z) + B);
    } while (g < gxo_mrg_u01(r) * grej);
    cost = 1 - z;
  }
  double sint = sqrt((1 + cost) * (1 - cost));
  double phi = TWOPI * gxo_mrg_u01(r);
  double xh = sint * gxo_cos(phi), yh = sint * gxo_sin(phi), zh = cost;
  gxo_rotate_to_lab(&xh, &yh, &zh, io->dir[0], io->dir[1], io->dir[2]);
  add_sec(io, 1, eE, xh, yh, zh);
  if (p->mode == GXO_MODE_PHYSICS) io->edep += gE - eE; /* binding energy, local */
  io->E = 0.0;
  io->status = 1;
  return io->nsec;
}

/* ---------------------------------------------------------- Bethe-Heitler */
/* ScreenFunction1/2, ProxyBetheHeitler.hpp:184-210 */
static double screen1(double s)
{
  return (s > 1.) ? 42.24 - 8.368 * gxo_log(s + 0.952) : 42.392 - s * (7.796 - 1.961 * s);
}
static double screen2(double s)
{
  return (s > 1.) ? 42.24 - 8.368 * gxo_log(s + 0.952) : 41.405 - s * (5.828 - 0.8945 * s);
}

/* ProxyBetheHeitler::SampleSecondaries, ProxyBetheHeitler.hpp:64-182.  Quirk:
 * the Tsai angle u m/E is used as the cosine (:146,:162); physics uses cos(u m/E). */
int gxo_bh_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io)
{
  double gE = io->E;
  io->nsec = 0;
  double epsil0 = EMASS / gE;
  if (epsil0 > 0.5) return 0;
  int Z = (p->mode == GXO_MODE_QUIRK) ? 10 : p->Z;
  const double Egsmall = 2. * MEV;
  double epsil;
  if (gE < Egsmall) {
    epsil = epsil0 + (0.5 - epsil0) * gxo_mrg_u01(r);
  } else {
    double logZ3 = gxo_log(1.0 * (int)(Z + 0.5)) / 3.0;
    double FZ = 8. * logZ3;
    if (gE > 50. * MEV) FZ += 8. * gxo_coulomb_factor(Z);
    double Z3 = gxo_pow(1.0 * (int)(Z + 0.5), 1 / 3.0);
    double screenfac = 136. * epsil0 / Z3;
    double screenmax = gxo_exp((42.24 - FZ) / 8.368) - 0.952;
    double screenmin = fmin(4. * screenfac, screenmax);
    double epsil1 = 0.5 - 0.5 * sqrt(1. - screenmin / screenmax);
    double epsilmin = fmax(epsil0, epsil1);
    double epsilrange = 0.5 - epsilmin;
    double screenvar, greject;
    double F10 = screen1(screenmin) - FZ;
    double F20 = screen2(screenmin) - FZ;
    double NormF1 = fmax(F10 * epsilrange * epsilrange, 0.);
    double NormF2 = fmax(1.5 * F20, 0.);
    do {
      if (NormF1 / (NormF1 + NormF2) > gxo_mrg_u01(r)) {
        epsil = 0.5 - epsilrange * gxo_pow(gxo_mrg_u01(r), 0.333333);
        screenvar = screenfac / (epsil * (1 - epsil));
        greject = (screen1(screenvar) - FZ) / F10;
      } else {
        epsil = epsilmin + epsilrange * gxo_mrg_u01(r);
        screenvar = screenfac / (epsil * (1 - epsil));
        greject = (screen2(screenvar) - FZ) / F20;
      }
    } while (greject < gxo_mrg_u01(r));
  }
  double eTot = (gxo_mrg_u01(r) > 0.5) ? (1. - epsil) * gE : epsil * gE;
  double pTot = gE - eTot;
  double u1 = gxo_mrg_u01(r);
  double u2 = gxo_mrg_u01(r);
  double aa0 = -gxo_log(u1 * u2);
  double u = (0.25 > gxo_mrg_u01(r)) ? aa0 / 0.625 : aa0 / 1.875;
  double phi = TWOPI * gxo_mrg_u01(r);
  double cosp = gxo_cos(phi), sinp = gxo_sin(phi);
  double cost = u * EMASS / eTot;
  if (p->mode == GXO_MODE_PHYSICS) cost = gxo_cos(cost);
  double sint = sqrt((1. - cost) * (1. + cost));
  double xh = sint * cosp, yh = sint * sinp, zh = cost;
  gxo_rotate_to_lab(&xh, &yh, &zh, io->dir[0], io->dir[1], io->dir[2]);
  add_sec(io, 1, eTot - EMASS, xh, yh, zh);
  cost = u * EMASS / pTot;
  if (p->mode == GXO_MODE_PHYSICS) cost = gxo_cos(cost);
  sint = sqrt((1. - cost) * (1. + cost));
  xh = -sint * cosp;
  yh = -sint * sinp;
  zh = cost;
  gxo_rotate_to_lab(&xh, &yh, &zh, io->dir[0], io->dir[1], io->dir[2]);
  add_sec(io, 2, pTot - EMASS, xh, yh, zh);
  io->E = 0.0;
  io->status = 1;
  return io->nsec;
}

/* --------------------------------------------------------- Seltzer-Berger */
/* ProxySeltzerBerger::SamplePhotonDirection, ProxySeltzerBerger.hpp:288-315
 * (dipole-boosted angle).  The reference feeds it the photon energy (:272);
 * physics mode feeds the electron kinetic energy, the quantity the angular
 * generator is defined for. */
static void sb_photon_direction(gxo_mrg_t *r, double energyIn, double *dx, double *dy, double *dz)
{
  double c = 4.0 - 8.0 * gxo_mrg_u01(r);
  double signc = (c < 0) ? -1 : 1;
  double a = fabs(c);
  double delta = 0.5 * (sqrt(4.0 + a * a) + a);
  double cofA = -signc * gxo_pow(delta, 1.0 / 3.0);
  double cosTheta = cofA - 1.0 / cofA;
  double tau = energyIn / EMASS;
  double beta = sqrt(tau * (tau + 2.0)) / (tau + 1.0);
  cosTheta = (cosTheta + beta) / (1.0 + cosTheta * beta);
  double sinTheta = sqrt((1.0 - cosTheta) * (1.0 + cosTheta));
  double phi = TWOPI * gxo_mrg_u01(r);
  *dx = sinTheta * gxo_cos(phi);
  *dy = sinTheta * gxo_sin(phi);
  *dz = cosTheta;
}

/* ProxySeltzerBerger::SampleSecondaries, ProxySeltzerBerger.hpp:204-286 */
int gxo_sb_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io)
{
  double kin = io->E;
  io->nsec = 0;
  int quirk = p->mode == GXO_MODE_QUIRK;
  double cut = fmin(quirk ? 1.0 * KEV : p->cut, kin);
  double emax = fmin(1.0 * TEV, kin);
  if (cut >= emax) return 0;
  const gxo_sb_t *T = p->sb;
  double totalEnergy = kin + EMASS;
  double densityCorr = p->density_factor * totalEnergy * totalEnergy;
  double xmin = gxo_log(cut * cut + densityCorr);
  double xmax = gxo_log(emax * emax + densityCorr);
  double y = gxo_log(kin / MEV);
  double x0 = cut / kin;
  double vmax = gxo_sb_value(T, x0, y) * 1.02;
  double epeaklimit = 300 * MEV, elowlimit = 10 * KEV;
  if (x0 < 0.97 && ((kin > epeaklimit) || (kin < elowlimit))) {
    double ylim = fmin(gxo_sb_value(T, 0.97, 4 * log(10.)), 1.1 * gxo_sb_value(T, 0.97, y));
    if (ylim > vmax) vmax = ylim;
  }
  if (x0 < 0.05) vmax *= 1.2;
  double gE = 0, v;
  do {
    double auxrand = gxo_mrg_u01(r);
    double x = gxo_exp(xmin + auxrand * (xmax - xmin)) - densityCorr;
    if (x < 0.0) x = 0.0;
    gE = sqrt(x);
    double x1 = gE / kin;
    v = gxo_sb_value(T, x1, y);
  } while (v < vmax * gxo_mrg_u01(r));
  double gx, gy, gz;
  sb_photon_direction(r, quirk ? gE : kin, &gx, &gy, &gz);
  gxo_rotate_to_lab(&gx, &gy, &gz, io->dir[0], io->dir[1], io->dir[2]);
  add_sec(io, 0, gE, gx, gy, gz);
  double totalMomentum = sqrt(kin * (totalEnergy + EMASS));
  io->E -= gE;
  double nx = totalMomentum * io->dir[0] - gE * gx;
  double ny = totalMomentum * io->dir[1] - gE * gy;
  double nz = totalMomentum * io->dir[2] - gE * gz;
  unit3(&nx, &ny, &nz);
  io->dir[0] = nx;
  io->dir[1] = ny;
  io->dir[2] = nz;
  return io->nsec;
}

/* ------------------------------------------------------- Moller / Bhabha */
/* ProxyMollerScattering::CrossSectionPerAtom, ProxyMollerScattering.hpp:61-89 */
double gxo_mb_xs_per_atom(double Z, double kin)
{
  init_constants();
  const double cutEnergy = 10.0 * EV;
  double tmax = fmin(100.0 * TEV, 0.5 * kin);
  if (cutEnergy > tmax) return 0.0;
  double xmin = cutEnergy / kin, xmax = tmax / kin;
  double tau = kin / EMASS, gam = tau + 1.0, gamma2 = gam * gam;
  double beta2 = tau * (tau + 2) / gamma2;
  double gg = (2.0 * gam - 1.0) / gamma2;
  double xs = ((xmax - xmin) * (1.0 - gg + 1.0 / (xmin * xmax) + 1.0 / ((1.0 - xmin) * (1.0 - xmax))) -
               gg * log(xmax * (1.0 - xmin) / (xmin * (1.0 - xmax)))) /
              beta2;
  xs *= g_twopi_mc2_rcl2 / kin;
  return Z * xs;
}

/* delta-ray kinematics shared by Moller and Bhabha, ProxyMollerScattering.hpp:128-156 */
static void delta_ray(gxo_mrg_t *r, gxo_inter_t *io, double kin, double x)
{
  double energy = kin + EMASS;
  double deltaKin = x * kin;
  double totalMomentum = sqrt(kin * (kin + 2.0 * EMASS));
  double deltaMomentum = sqrt(deltaKin * (deltaKin + 2.0 * EMASS));
  double cost = deltaKin * (energy + EMASS) / (deltaMomentum * totalMomentum);
  if (cost > 1.0) cost = 1.0;
  double sint = sqrt((1.0 - cost) * (1. + cost));
  double phi = TWOPI * gxo_mrg_u01(r);
  double xh = sint * gxo_cos(phi), yh = sint * gxo_sin(phi), zh = cost;
  gxo_rotate_to_lab(&xh, &yh, &zh, io->dir[0], io->dir[1], io->dir[2]);
  add_sec(io, 1, deltaKin, xh, yh, zh);
  io->E -= deltaKin;
  double nx = totalMomentum * io->dir[0] - deltaMomentum * xh;
  double ny = totalMomentum * io->dir[1] - deltaMomentum * yh;
  double nz = totalMomentum * io->dir[2] - deltaMomentum * zh;
  unit3(&nx, &ny, &nz);
  io->dir[0] = nx;
  io->dir[1] = ny;
  io->dir[2] = nz;
}

/* ProxyMollerScattering::SampleSecondaries, ProxyMollerScattering.hpp:92-159 */
int gxo_mb_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io)
{
  double kin = io->E;
  io->nsec = 0;
  double maxEnergy = 1.0 * TEV;
  double cutEnergy = (p->mode == GXO_MODE_QUIRK) ? 1.0 * KEV : p->cut;
  double tmin = cutEnergy, tmax = 0.5 * kin;
  if (maxEnergy < tmax) tmax = maxEnergy;
  if (tmin >= tmax) return 0;
  double energy = kin + EMASS;
  double xmin = tmin / kin, xmax = tmax / kin;
  double gam = energy / EMASS, gamma2 = gam * gam;
  double x, z, grej;
  double gg = (2.0 * gam - 1.0) / gamma2;
  double y = 1.0 - xmax;
  grej = 1.0 - gg * xmax + xmax * xmax * (1.0 - gg + (1.0 - gg * y) / (y * y));
  do {
    double rndm = gxo_mrg_u01(r);
    x = xmin * xmax / (xmin * (1.0 - rndm) + xmax * rndm);
    y = 1.0 - x;
    z = 1.0 - gg * x + x * x * (1.0 - gg + (1.0 - gg * y) / (y * y));
  } while (grej * gxo_mrg_u01(r) > z);
  delta_ray(r, io, kin, x);
  return io->nsec;
}

/* Bhabha (e+ e-) scattering.  The reference has no positron model; this is the
 * published Geant4 Moller-Bhabha sampling (G4MollerBhabhaModel, Geant4 Physics
 * Reference Manual), restated.  Physics mode only; parity unpinned. */
int gxo_bhabha_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io)
{
  double kin = io->E;
  io->nsec = 0;
  double tmin = p->cut, tmax = kin;
  if (tmin >= tmax) return 0;
  double energy = kin + EMASS;
  double xmin = tmin / kin, xmax = tmax / kin;
  double gam = energy / EMASS, gamma2 = gam * gam;
  double beta2 = 1.0 - 1.0 / gamma2;
  double y = 1.0 / (1.0 + gam);
  double y2 = y * y;
  double y12 = 1.0 - 2.0 * y;
  double b1 = 2.0 - y2;
  double b2 = y12 * (3.0 + y2);
  double y122 = y12 * y12;
  double b4 = y122 * y12;
  double b3 = b4 + y122;
  y = xmax * xmax;
  double grej = 1.0 + (y * y * b4 - xmin * xmin * xmin * b3 + y * b2 - xmin * b1) * beta2;
  double x, z;
  do {
    double rndm = gxo_mrg_u01(r);
    x = xmin * xmax / (xmin * (1.0 - rndm) + xmax * rndm);
    y = x * x;
    z = 1.0 + (y * y * b4 - x * y * b3 + y * b2 - x * b1) * beta2;
  } while (grej * gxo_mrg_u01(r) > z);
  delta_ray(r, io, kin, x);
  return io->nsec;
}

/* ---------------------------------------------------- e+ annihilation */
/* Heitler cross section per target electron for e+ e- -> 2 gamma (Geant4
 * eeToTwoGamma model, published formula). */
double gxo_annih_xs_per_electron(double kin)
{
  init_constants();
  double ekin = fmax(EV, kin);
  double tau = ekin / EMASS;
  double gam = tau + 1.0;
  double gamma2 = gam * gam;
  double bg2 = tau * (tau + 2.0);
  double bg = sqrt(bg2);
  return g_pi_rcl2 * ((gamma2 + 4 * gam + 1.) * gxo_log(gam + bg) - (gam + 3.) * bg) / (bg2 * (gam + 1.));
}

/* Two-photon annihilation (Geant4 eeToTwoGamma sampling, published algorithm).
 * At rest (E == 0) the photons are back to back, isotropic, m_e c^2 each. */
int gxo_annih_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io)
{
  (void)p;
  double kin = io->E;
  io->nsec = 0;
  if (kin <= 0.0) {
    double cost = 2. * gxo_mrg_u01(r) - 1.;
    double sint = sqrt((1. - cost) * (1. + cost));
    double phi = TWOPI * gxo_mrg_u01(r);
    double dx = sint * gxo_cos(phi), dy = sint * gxo_sin(phi), dz = cost;
    add_sec(io, 0, EMASS, dx, dy, dz);
    add_sec(io, 0, EMASS, -dx, -dy, -dz);
  } else {
    double tau = kin / EMASS;
    double gam = tau + 1.0;
    double tau2 = tau + 2.0;
    double sqgrate = sqrt(tau / tau2) * 0.5;
    double sqg2m1 = sqrt(tau * tau2);
    double epsilmin = 0.5 - sqgrate;
    double epsilmax = 0.5 + sqgrate;
    double epsilqot = epsilmax / epsilmin;
    double epsil, greject;
    do {
      epsil = epsilmin * gxo_exp(gxo_log(epsilqot) * gxo_mrg_u01(r));
      greject = 1. - epsil + (2. * gam * epsil - 1.) / (epsil * tau2 * tau2);
    } while (greject < gxo_mrg_u01(r));
    double cost = (epsil * tau2 - 1.) / (epsil * sqg2m1);
    if (cost > 1.0) cost = 1.0;
    if (cost < -1.0) cost = -1.0;
    double sint = sqrt((1. + cost) * (1. - cost));
    double phi = TWOPI * gxo_mrg_u01(r);
    double tot = kin + 2.0 * EMASS;
    double e1 = epsil * tot, e2 = (1. - epsil) * tot;
    double dx = sint * gxo_cos(phi), dy = sint * gxo_sin(phi), dz = cost;
    gxo_rotate_to_lab(&dx, &dy, &dz, io->dir[0], io->dir[1], io->dir[2]);
    double pp = sqrt(kin * (kin + 2. * EMASS));
    double ex = pp * io->dir[0] - e1 * dx, ey = pp * io->dir[1] - e1 * dy, ez = pp * io->dir[2] - e1 * dz;
    unit3(&ex, &ey, &ez);
    add_sec(io, 0, e1, dx, dy, dz);
    add_sec(io, 0, e2, ex, ey, ez);
  }
  io->E = 0.0;
  io->status = 1;
  return io->nsec;
}

/* ------------------------------------------------ photo-electric cross section */
/* Below 200 keV the reference's tables have no photo-electric entry (its
 * LambdaPrim.phot table starts at 0.2 MeV); Geant4 computes the cross section
 * there from the Sandia parametrisation sigma/rho = sum_k a_k / E^k of the
 * element, in the interval that contains E.  Returns 1/mm. */
double gxo_pe_xs_sandia(const gxo_data_t *d, int Z, double density, double e)
{
  double ekev = e / KEV;
  int first = d->cumint[Z - 1], n = d->nint[Z];
  int row = first + n - 1;
  while (row > first && ekev < d->sandia[row][0]) --row;
  if (ekev < d->sandia[row][0]) return 0.0;
  const double *a = d->sandia[row];
  /* a1/E + a2/E^2 + a3/E^3 + a4/E^4 as a polynomial in 1/E (Horner), the
   * CUDA library's form, so that both round alike */
  double i1 = 1.0 / ekev;
  double s = i1 * (a[1] + i1 * (a[2] + i1 * (a[3] + i1 * a[4])));
  return fmax(s, 0.0) * density * 0.1; /* cm2/g * g/cm3 = 1/cm -> 1/mm */
}

/* --------------------------------------------------------------- materials */
void gxo_material_make(double Z, double A, double density, gxo_material_t *m)
{
  init_constants();
  const double avogadro = 6.02214179e+23;
  m->Z = Z;
  m->A = A;
  m->density = density;
  m->n_atoms = avogadro * density / A * 1.e-3;
  m->n_el = Z * m->n_atoms;
  double migdal = 4.0 * PI * g_rcl * g_compton_len * g_compton_len;
  m->density_factor = m->n_el * migdal;
  double radinv = m->n_atoms * lrad_tsai_factor(Z);
  m->radlen = radinv <= 0.0 ? DBL_MAX : 1. / radinv;
}

/* ------------------------------------------------------- batch front end */
void gxo_interact_batch(int model, const gxo_model_params_t *p, int n, double *states,
                        const double *E, const double *dir, double *E_out, double *dir_out,
                        double *edep, int *status, int *nsec, int *sec_type, double *sec_E,
                        double *sec_dir)
{
  for (int i = 0; i < n; ++i) {
    gxo_mrg_t r;
    memcpy(r.s, &states[6 * i], sizeof(r.s));
    gxo_inter_t io;
    memset(&io, 0, sizeof(io));
    io.E = E[i];
    io.dir[0] = dir[3 * i];
    io.dir[1] = dir[3 * i + 1];
    io.dir[2] = dir[3 * i + 2];
    switch (model) {
    case 0: gxo_kn_sample(&r, p, &io); break;
    case 1: gxo_sg_sample(&r, p, &io); break;
    case 2: gxo_bh_sample(&r, p, &io); break;
    case 3: gxo_sb_sample(&r, p, &io); break;
    case 4: gxo_mb_sample(&r, p, &io); break;
    case 5: gxo_bhabha_sample(&r, p, &io); break;
    case 6: gxo_annih_sample(&r, p, &io); break;
    default: break;
    }
    memcpy(&states[6 * i], r.s, sizeof(r.s));
    E_out[i] = io.E;
    for (int k = 0; k < 3; ++k) dir_out[3 * i + k] = io.dir[k];
    edep[i] = io.edep;
    status[i] = io.status;
    nsec[i] = io.nsec;
    for (int s = 0; s < 2; ++s) {
      sec_type[2 * i + s] = s < io.nsec ? io.sec_type[s] : -1;
      sec_E[2 * i + s] = s < io.nsec ? io.sec_E[s] : 0.0;
      for (int k = 0; k < 3; ++k) sec_dir[6 * i + 3 * s + k] = s < io.nsec ? io.sec_dir[s][k] : 0.0;
    }
  }
}

/* ------------------------------------------------------------ processes */
/* ProxyEmProcess<T>::PostStepGPIL, ProxyEmProcess.hpp:122-151 (the material
 * index is chosen by the caller; the reference forces index 2 at :133). */
double gxo_post_step_gpil(gxo_mrg_t *r, double lambda, double pstep_prev, double *nil,
                          double *inv_lambda_saved)
{
  if (*nil <= 0.0)
    *nil = -gxo_log(gxo_mrg_u01(r));
  else
    *nil -= pstep_prev / *inv_lambda_saved;
  double step = *nil / lambda;
  *inv_lambda_saved = 1.0 / lambda;
  return step;
}

/* ProxyIonization::AlongStepGPIL, ProxyIonization.hpp:108-128.  Quirk: the cut
 * is GetCutValue(index, 1), an energy in keV read with stride 4, used as a
 * length, and the step function uses 2 finR/range.  Physics: the length cut,
 * and Geant4's step function range dR + finR (1 - dR)(2 - finR/range). */
double gxo_ioni_along_gpil(const gxo_data_t *d, int mode, int charge, int mat, double e)
{
  const double dRoverRange = 0.2, finalRange = 10.0, minE = 100.0 * EV;
  int rt = (mode == GXO_MODE_PHYSICS && charge > 0) ? GXO_Range_ep : GXO_Range_em;
  double range = gxo_table_value(d, rt, mat, e);
  if (e < minE) range *= e / minE;
  double cut;
  if (mode == GXO_MODE_QUIRK)
    cut = gxo_get_cut_value(d, mat, 1);
  else
    cut = d->cut_length[1][mat];
  double finR = (finalRange < cut) ? finalRange : cut;
  if (range <= finR) return range;
  if (mode == GXO_MODE_QUIRK) return range * dRoverRange + finR * (1.0 - dRoverRange) * (2.0 * finR / range);
  return range * dRoverRange + finR * (1.0 - dRoverRange) * (2.0 - finR / range);
}

/* ProxyIonization::AlongStepDoIt, ProxyIonization.hpp:130-168.  Quirk: the
 * inverse range is read through Value() (:100-104,154), i.e. the log-grid bin
 * search applied to the range-indexed vector; the bin is clamped to the vector
 * here so the lookup stays in memory.  Physics: InvRangeValue. */
void gxo_ioni_along_doit(const gxo_data_t *d, int mode, int charge, int mat, double step,
                         double *e, double *edep)
{
  const double minE = 100.0 * EV, linLossLimit = 0.01;
  int ep = (mode == GXO_MODE_PHYSICS && charge > 0);
  double energy = *e;
  double range = gxo_table_value(d, ep ? GXO_Range_ep : GXO_Range_em, mat, energy);
  if (step >= range || energy <= minE) {
    *e = 0.0;
    *edep += energy;
    return;
  }
  double dedx = gxo_table_value(d, ep ? GXO_DEDX_eIoni_ep : GXO_DEDX_eIoni_em, mat, energy);
  if (energy < minE) dedx *= sqrt(energy / minE);
  double eloss = step * dedx;
  if (eloss > energy * linLossLimit) {
    range -= step;
    const gxo_pvec_t *iv = &d->vec[ep ? GXO_InverseRange_ep : GXO_InverseRange_em][mat];
    double einv;
    if (mode == GXO_MODE_QUIRK) {
      if (range <= iv->emin)
        einv = iv->y[0];
      else if (range >= iv->emax)
        einv = iv->y[iv->n - 1];
      else {
        int bin = (int)(gxo_log(range) / iv->dbin - iv->base);
        if (bin > 0 && range < iv->x[bin]) --bin;
        if (bin < 0) bin = 0;
        if (bin > iv->n - 2) bin = iv->n - 2;
        double x1 = iv->x[bin], x2 = iv->x[bin + 1], delta = x2 - x1;
        double a = (x2 - range) / delta, b = (range - x1) / delta;
        einv = a * iv->y[bin] + b * iv->y[bin + 1] +
               ((a * a * a - a) * iv->d2[bin] + (b * b * b - b) * iv->d2[bin + 1]) * delta * delta / 6.0;
      }
    } else {
      einv = gxo_pvec_invrange_value(iv, range);
    }
    eloss = energy - einv;
  }
  double finalE = energy - eloss;
  if (finalE < minE) {
    eloss += finalE;
    finalE = 0.0;
  }
  eloss = fmax(eloss, 0.0);
  *e = finalE;
  *edep += eloss;
}

/* --------------------------------------------------------------- helix */
/* ConstFieldHelixStepper::DoStep, ConstFieldHelixStepper.hpp:164-239, with the
 * reference's constant kB2C = -0.299792458e-3 (GeV, kilogauss, cm).  A caller
 * in mm / MeV / tesla passes the same numbers scaled: kB2C B / p is unit-free
 * up to the length unit, see the transport. */
static void helix_core(double kB2C, const double B[3], const double pos[3], const double dir[3],
                       double charge, double momentum, double step, double np[3], double nd[3])
{
  const double kSmall = 1.E-30;
  double Bmag = sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
  double ux = B[0], uy = B[1], uz = B[2];
  if (Bmag > 0) {
    ux /= Bmag;
    uy /= Bmag;
    uz /= Bmag;
  }
  double UVdotUB = dir[0] * ux + dir[1] * uy + dir[2] * uz;
  double dt2 = fmax(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2] - UVdotUB * UVdotUB, 0.0);
  double sinVB = sqrt(dt2) + kSmall;
  double R = momentum * sinVB / (kB2C * charge * Bmag);
  double vx = dir[0] - UVdotUB * ux, vy = dir[1] - UVdotUB * uy, vz = dir[2] - UVdotUB * uz;
  unit3(&vx, &vy, &vz);
  double cx = vy * uz - vz * uy, cy = vz * ux - vx * uz, cz = vx * uy - vy * ux;
  double phi = -step * charge * Bmag * kB2C / momentum;
  double sinphi = gxo_sin(phi), cosphi = gxo_cos(phi);
  np[0] = pos[0] + R * (cosphi - 1) * cx - R * sinphi * vx + step * UVdotUB * ux;
  np[1] = pos[1] + R * (cosphi - 1) * cy - R * sinphi * vy + step * UVdotUB * uy;
  np[2] = pos[2] + R * (cosphi - 1) * cz - R * sinphi * vz + step * UVdotUB * uz;
  nd[0] = UVdotUB * ux + cosphi * sinVB * vx + sinphi * sinVB * cx;
  nd[1] = UVdotUB * uy + cosphi * sinVB * vy + sinphi * sinVB * cy;
  nd[2] = UVdotUB * uz + cosphi * sinVB * vz + sinphi * sinVB * cz;
}

void gxo_helix_dostep(const double B[3], const double pos[3], const double dir[3], double charge,
                      double momentum, double step, double newpos[3], double newdir[3])
{
  helix_core(-0.299792458e-3, B, pos, dir, charge, momentum, step, newpos, newdir);
}

void gxo_helix_dostep_mm(double Bz_tesla, const double pos[3], const double dir[3], double charge,
                         double momentum, double step, double newpos[3], double newdir[3])
{
  double B[3] = {0.0, 0.0, Bz_tesla};
  helix_core(-0.299792458, B, pos, dir, charge, momentum, step, newpos, newdir);
}

void gxo_helix_batch(const double B[3], int n, const double *pos, const double *dir,
                     const double *charge, const double *mom, const double *step, double *newpos,
                     double *newdir)
{
  for (int i = 0; i < n; ++i)
    gxo_helix_dostep(B, &pos[3 * i], &dir[3 * i], charge[i], mom[i], step[i], &newpos[3 * i], &newdir[3 * i]);
}
