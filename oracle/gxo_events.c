/*
 * gxo_events.c -- ORACLE (test infrastructure only): primary generation, the
 * reference's event generators restated in C.
 *
 *   gxo_egamma_gun   ProxyEgammaGun::GenerateOneEvent (proxy/src/ProxyEgammaGun.cpp:43-85)
 *   gxo_egamma_dir   ProxyEgammaGun::SetDirectionXYZ (proxy/src/ProxyEgammaGun.cpp:35-41)
 *   gxo_hepevt_read  ProxyHepEvtGenerator::GenerateOneEvent (proxy/src/ProxyHepEvtGenerator.cpp:48-132)
 */
#include "gxo.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define EMASS 0.510998910 /* clhep::electron_mass_c2, ProxyPhysicalConstants.hpp:51 */

/* Four draws per particle from one stream, in this order: the type (gamma
 * below gamma_fraction, else e-), the momentum (uniform in [minp, maxp]),
 * eta and phi (uniform in their ranges); events one after another.  The
 * kinetic energy is p^2 / (sqrt(p^2 + m^2) + m) with m = m_e q^2; the
 * direction is (sin t cos phi, sin t sin phi, cos t), t = 2 atan(exp(-eta)). */
int gxo_egamma_gun(gxo_mrg_t *r, int nevents, int nparticles, double gamma_fraction, double minp, double maxp,
                   double mineta, double maxeta, double minphi, double maxphi, int *pdg, double *p, double *ekin,
                   double *dir)
{
  int k = 0;
  for (int e = 0; e < nevents; ++e)
    for (int i = 0; i < nparticles; ++i, ++k) {
      double charge;
      if (gxo_mrg_u01(r) < gamma_fraction) {
        pdg[k] = 22;
        charge = 0.0;
      } else {
        pdg[k] = 11;
        charge = -1.0;
      }
      double pp = minp + (maxp - minp) * gxo_mrg_u01(r);
      double mass = EMASS * charge * charge;
      p[k] = pp;
      ekin[k] = pp * pp / (sqrt(pp * pp + mass * mass) + mass);
      double eta = mineta + (maxeta - mineta) * gxo_mrg_u01(r);
      double phi = minphi + (maxphi - minphi) * gxo_mrg_u01(r);
      double theta = 2. * atan(exp(-eta));
      dir[3 * k + 0] = sin(theta) * cos(phi);
      dir[3 * k + 1] = sin(theta) * sin(phi);
      dir[3 * k + 2] = cos(theta);
    }
  return k;
}

/* The eta and phi SetDirectionXYZ sets (both ranges collapse to them).  The
 * reference takes theta = atan(rho / z) and phi = atan(y / z) (quirk mode:
 * right only for z > 0 and, for phi, y / z in place of y / x); physics mode
 * uses atan2(rho, z) and atan2(y, x). */
void gxo_egamma_dir(int physics, double x, double y, double z, double *eta, double *phi)
{
  double rho = sqrt(x * x + y * y);
  double theta = physics ? atan2(rho, z) : atan(rho / z);
  *eta = -log(tan(0.5 * theta));
  *phi = physics ? atan2(y, x) : atan(y / z);
}

/* HEPEVT ASCII events: per event NHEP, then NHEP lines
 * ISTHEP IDHEP JDAHEP1 JDAHEP2 PHEP1 PHEP2 PHEP3 PHEP4 (momentum, mass in GeV).
 * Every daughter (entries jda1..jda2, 1-based, of an entry with JDAHEP1 > 0)
 * whose ISTHEP is positive is marked -1; the primaries are the marked entries
 * without daughters, in file order.  Their kinetic energy is
 * p^2 / (sqrt(p^2 + m^2) + m) and their direction p / |p|.  Quirk mode keeps
 * the reference's m = PHEP4^2 and its GeV numbers read as MeV; physics mode
 * uses m = PHEP4 and converts GeV to MeV.  Daughter indices outside the event
 * are skipped (the reference reads out of bounds there) and counted in
 * *bad.  Returns the number of primaries written (at most cap); *nev_read
 * receives the number of complete events read (at most max_events). */
int gxo_hepevt_read(const char *path, int physics, int max_events, int cap, int *event, int *pdg, double *p,
                    double *ekin, double *dir, int *nev_read, int *bad)
{
  FILE *f = fopen(path, "r");
  int k = 0, nev = 0;
  *bad = 0;
  if (!f) {
    *nev_read = 0;
    return -1;
  }
  const double unit = physics ? 1000.0 : 1.0;
  for (int e = 0; e < max_events; ++e) {
    int nhep;
    if (fscanf(f, "%d", &nhep) != 1 || nhep < 0) break;
    int *ist = malloc(sizeof(int) * (nhep + 1)), *id = malloc(sizeof(int) * (nhep + 1));
    int *j1 = malloc(sizeof(int) * (nhep + 1)), *j2 = malloc(sizeof(int) * (nhep + 1));
    double *ph = malloc(sizeof(double) * 4 * (nhep + 1));
    int ok = 1;
    for (int i = 0; i < nhep; ++i)
      if (fscanf(f, "%d %d %d %d %lf %lf %lf %lf", &ist[i], &id[i], &j1[i], &j2[i], &ph[4 * i], &ph[4 * i + 1],
                 &ph[4 * i + 2], &ph[4 * i + 3]) != 8) {
        ok = 0;
        break;
      }
    if (ok) {
      for (int i = 0; i < nhep; ++i) {
        if (j1[i] <= 0) continue;
        for (int j = j1[i] - 1; j <= j2[i] - 1; ++j) {
          if (j < 0 || j >= nhep) {
            ++*bad;
            continue;
          }
          if (ist[j] > 0) ist[j] = -1;
        }
      }
      for (int i = 0; i < nhep && k < cap; ++i) {
        if (!(ist[i] == -1 && j1[i] == 0)) continue;
        double px = ph[4 * i], py = ph[4 * i + 1], pz = ph[4 * i + 2];
        double pp = sqrt(px * px + py * py + pz * pz);
        double mass = physics ? ph[4 * i + 3] * unit : ph[4 * i + 3] * ph[4 * i + 3];
        event[k] = e;
        pdg[k] = id[i];
        p[k] = pp * unit;
        ekin[k] = p[k] * p[k] / (sqrt(p[k] * p[k] + mass * mass) + mass);
        dir[3 * k] = pp > 0 ? px / pp : px;
        dir[3 * k + 1] = pp > 0 ? py / pp : py;
        dir[3 * k + 2] = pp > 0 ? pz / pp : pz;
        ++k;
      }
      ++nev;
    }
    free(ist);
    free(id);
    free(j1);
    free(j2);
    free(ph);
    if (!ok) break;
  }
  fclose(f);
  *nev_read = nev;
  return k;
}

/* The beam-spot gun of the throughput workloads (the library's gx_spot_gun;
 * the reference has no such gun: its benchmarks start from ProxyEgammaGun or
 * HEPEVT files).  Stream `stream` of the seed (SetNextStream applied
 * stream + 1 times, MRG32k3a.cpp:51-58); primary i takes draws 5i .. 5i+4,
 * drawn here in sequence from draw 0: kinetic energy emin (emax / emin)^u0,
 * cos theta = 1 - u1 (1 - cos cone), phi = 2 pi u2 about +axis (transverse
 * axes in cyclic order), start centre +- half (2u - 1) in the two transverse
 * coordinates, type = types[i % ntypes]. */
int gxo_spot_gun(const double seed[6], long stream, long first, int n, int ntypes, const int *types, double emin,
                 double emax, double cone_deg, int axis, const double centre[3], const double half[2], int *type,
                 double *E, double *pos, double *dir)
{
  double sd[6];
  gxo_mrg_t r;
  for (int k = 0; k < 6; ++k) sd[k] = seed[k];
  for (long s = 0; s <= stream; ++s) gxo_mrg_next_stream(sd, &r);
  for (long j = 0; j < 5 * first; ++j) gxo_mrg_u01(&r);
  const double pi = 3.14159265358979323846;
  const double cc = cos(cone_deg * pi / 180.0);
  const int b = (axis + 1) % 3, c = (axis + 2) % 3;
  for (int i = 0; i < n; ++i) {
    double u[5];
    for (int j = 0; j < 5; ++j) u[j] = gxo_mrg_u01(&r);
    type[i] = types[(first + i) % ntypes];
    E[i] = emin * exp(u[0] * log(emax / emin));
    double ct = 1.0 - u[1] * (1.0 - cc), st = sqrt((1.0 - ct) * (1.0 + ct)), phi = 2.0 * pi * u[2];
    double *d = dir + 3 * i, *p = pos + 3 * i;
    d[axis] = ct;
    d[b] = st * cos(phi);
    d[c] = st * sin(phi);
    p[axis] = centre[axis];
    p[b] = centre[b] + half[0] * (2.0 * u[3] - 1.0);
    p[c] = centre[c] + half[1] * (2.0 * u[4] - 1.0);
  }
  return n;
}
