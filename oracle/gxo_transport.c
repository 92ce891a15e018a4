/*
 * gxo_transport.c -- ORACLE (test infrastructure only): the per-track step
 * loop, restated on the CPU.
 *
 * The reference's only transport driver (source/Geant/proxy/test/
 * test_BasicCpuTransport.cpp:358-550, OneStep/InnerStep/DoStep) needs VecGeom
 * navigation, which is absent, and runs with every EM process commented out
 * (BasicCpuTransport/Types.hpp:110-128).  This file restates its step
 * structure in physics mode with an analytic layered-box navigator:
 *
 *   OneStep (:408-497): post-step GPIL of every discrete process (NIL against
 *     the macroscopic cross section, ProxyEmProcess.hpp:122-151), the
 *     continuous range limit (ProxyIonization.hpp:108-128), then
 *     FindNextBoundary (geometry/NavigationInterface.hpp:63-98);
 *   InnerStep (:358-403): propagation -- straight line
 *     (core/src/LinearPropagationHandler.cpp:12-56) or helix sub-steps in the
 *     uniform field (magneticfield/src/FieldPropagationHandler.cpp:87-139,
 *     142-360) -- then the along-step loss (ProxyIonization.hpp:130-168) and
 *     the selected post-step interaction (ProxyEmProcess.hpp:153-163).
 *
 * The same algorithm, in the same order of random draws, is what the CUDA
 * engine runs; tests compare the two on identical MRG32k3a streams.
 */
#include "gxo.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define EMASS 0.510998910
#define MINE 1.0e-4 /* 100 eV: the models' low-energy limit used as minE */
#define PI 3.14159265358979323846
#define TWOPI (2 * PI)

typedef struct {
  int type;
  double E, pos[3], dir[3];
  int vol;
  double nil[3];
  gxo_mrg_t rng;
  int event;
  int primary;   /* index of the primary if this is the primary track, else -1 */
  double msc_r0; /* multiple scattering: range scale of the step limit in this volume (<= 0: unset) */
} track_t;

typedef struct {
  track_t *a;
  int n, cap;
} stack_t;

static void push(stack_t *s, const track_t *t)
{
  if (s->n == s->cap) {
    s->cap = s->cap ? 2 * s->cap : 256;
    s->a = (track_t *)realloc(s->a, sizeof(track_t) * s->cap);
  }
  s->a[s->n++] = *t;
}

typedef struct {
  const gxo_data_t *d;
  const gxo_config_t *c;
  gxo_material_t mat[3];
  double pitch;
  struct msc_mat { double X0, th1, th2, ca, cb, cc, cd; } msc[3];
} world_t;

/* ---------------------------------------------------------------- geometry */
/* Volumes: calorimeter: vol = 2 * layer + slab (slab 0 absorber = material 1
 * (Pb), slab 1 gap = material 2 (LAr)); box: vol 0 = box material; -1 outside. */
static int vol_material(const world_t *w, int vol)
{
  if (w->c->geometry == 2) return w->c->csg->node[vol].mat;
  if (w->c->geometry == 0) return w->c->box_mat;
  return (vol & 1) ? 2 : 1;
}

static void slab_bounds(const world_t *w, int vol, double *lo, double *hi)
{
  const gxo_config_t *c = w->c;
  if (c->geometry == 0) {
    *lo = c->box_centre[c->axis] - c->box_half[c->axis];
    *hi = c->box_centre[c->axis] + c->box_half[c->axis];
    return;
  }
  double x0 = -0.5 * c->nlayers * w->pitch;
  int layer = vol >> 1;
  double base = x0 + layer * w->pitch;
  if (vol & 1) {
    *lo = base + c->t_abs;
    *hi = base + w->pitch;
  } else {
    *lo = base;
    *hi = base + c->t_abs;
  }
}

static double trans_half(const world_t *w, int b)
{
  return w->c->geometry == 0 ? w->c->box_half[b] : w->c->half_trans;
}
static double trans_centre(const world_t *w, int b)
{
  return w->c->geometry == 0 ? w->c->box_centre[b] : 0.0;
}

/* Locate a point; on a plane (within 1e-12 mm) the direction picks the side. */
static int locate(const world_t *w, const double *p, const double *d)
{
  const gxo_config_t *c = w->c;
  if (c->geometry == 2) return gxo_csg_locate(c->csg, 0, p, d, GXO_CSG_TOL);
  const double tol = 1e-12;
  int a = c->axis;
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    double h = trans_half(w, b), q = p[b] - trans_centre(w, b);
    if (q > h || q < -h) return -1;
    if ((q > h - tol && d[b] > 0) || (q < -h + tol && d[b] < 0)) return -1;
  }
  if (c->geometry == 0) {
    double q = p[a] - c->box_centre[a], h = c->box_half[a];
    if (q > h || q < -h) return -1;
    if ((q > h - tol && d[a] > 0) || (q < -h + tol && d[a] < 0)) return -1;
    return 0;
  }
  double x0 = -0.5 * c->nlayers * w->pitch;
  double u = p[a] - x0;
  double total = c->nlayers * w->pitch;
  if (u < -tol || u > total + tol) return -1;
  if ((u < tol && d[a] < 0) || (u > total - tol && d[a] > 0)) return -1;
  int layer = (int)floor(u / w->pitch);
  if (layer < 0) layer = 0;
  if (layer >= c->nlayers) layer = c->nlayers - 1;
  double q = u - layer * w->pitch;
  if (q < tol && d[a] < 0 && layer > 0) return 2 * (layer - 1) + 1;
  if (q > w->pitch - tol && d[a] > 0 && layer + 1 < c->nlayers) return 2 * (layer + 1);
  if (fabs(q - c->t_abs) < tol) return 2 * layer + (d[a] > 0 ? 1 : 0);
  return 2 * layer + (q < c->t_abs ? 0 : 1);
}

/* Straight-line distance to the boundary of vol along d; *plane = -1 for the
 * low axis plane, +1 high axis plane, 2 transverse wall (csg: the child
 * entered, -1 leaving vol). */
static double dist_to_out(const world_t *w, int vol, const double *p, const double *d, int *plane)
{
  const gxo_config_t *c = w->c;
  if (c->geometry == 2) return gxo_csg_step(c->csg, vol, p, d, DBL_MAX, plane);
  int a = c->axis;
  double lo, hi, dist = DBL_MAX;
  slab_bounds(w, vol, &lo, &hi);
  *plane = 0;
  if (d[a] > 0) {
    dist = (hi - p[a]) / d[a];
    *plane = 1;
  } else if (d[a] < 0) {
    dist = (lo - p[a]) / d[a];
    *plane = -1;
  }
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    double h = trans_half(w, b), q = p[b] - trans_centre(w, b), t = DBL_MAX;
    if (d[b] > 0)
      t = (h - q) / d[b];
    else if (d[b] < 0)
      t = (-h - q) / d[b];
    if (t < dist) {
      dist = t;
      *plane = 2;
    }
  }
  return dist < 0 ? 0 : dist;
}

static double safety(const world_t *w, int vol, const double *p)
{
  const gxo_config_t *c = w->c;
  if (c->geometry == 2) return gxo_csg_safety(c->csg, vol, p);
  int a = c->axis;
  double lo, hi;
  slab_bounds(w, vol, &lo, &hi);
  double s = fmin(p[a] - lo, hi - p[a]);
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    double h = trans_half(w, b), q = p[b] - trans_centre(w, b);
    s = fmin(s, h - fabs(q));
  }
  return s < 0 ? 0 : s;
}

/* Volume entered through a plane of vol (straight-line crossing). */
static int next_volume(const world_t *w, int vol, int plane)
{
  if (plane == 2 || w->c->geometry == 0) return -1;
  int nv = vol + (plane > 0 ? 1 : -1);
  return (nv < 0 || nv >= 2 * w->c->nlayers) ? -1 : nv;
}

/* Volume after a helix sub-step started in vol: an end point within 1e-6 mm
 * of a face it moves out through (or past it) is put on the face and enters
 * the neighbour; otherwise the point is located (the engine's rule, so that
 * crossings do not hinge on rounding near the reference's 2e-9 mm push). */
static int relocate(const world_t *w, int vol, double *p, const double *d)
{
  const double snap = 1e-6;
  if (w->c->geometry == 2) return gxo_csg_locate(w->c->csg, vol, p, d, snap);
  int a = w->c->axis;
  double lo, hi;
  slab_bounds(w, vol, &lo, &hi);
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    double h = trans_half(w, b), q = p[b] - trans_centre(w, b);
    if ((d[b] > 0 && h - q < snap) || (d[b] < 0 && q + h < snap)) return -1;
  }
  if (d[a] > 0 && hi - p[a] < snap) {
    p[a] = hi;
    return next_volume(w, vol, 1);
  }
  if (d[a] < 0 && p[a] - lo < snap) {
    p[a] = lo;
    return next_volume(w, vol, -1);
  }
  return locate(w, p, d);
}

/* -------------------------------------------------------- cross sections */
static double lambda_table(const world_t *w, int table, int mat, double e)
{
  const gxo_pvec_t *v = &w->d->vec[table][mat];
  if (e <= v->emin) return 0.0;
  return gxo_pvec_value(v, e);
}

/* Macroscopic cross sections (1/mm) of the discrete processes of a particle:
 * gamma {Compton, conversion, photo-electric}, e- {ionisation, brems},
 * e+ {ionisation, brems, annihilation}. */
static void cross_sections(const world_t *w, int type, int mat, double e, double xs[3])
{
  const gxo_data_t *d = w->d;
  xs[0] = xs[1] = xs[2] = 0.0;
  if (type == 0) {
    xs[0] = (e < 1.0) ? gxo_table_value(d, GXO_Lambda_compt, mat, e)
                      : gxo_table_value(d, GXO_LambdaPrim_compt, mat, e) / e;
    xs[1] = lambda_table(w, GXO_Lambda_conv, mat, e);
    if (e >= 0.2)
      xs[2] = gxo_table_value(d, GXO_LambdaPrim_phot, mat, e) / e;
    else
      xs[2] = gxo_pe_xs_sandia(d, (int)w->mat[mat].Z, w->mat[mat].density, e);
  } else if (type == 1) {
    xs[0] = lambda_table(w, GXO_Lambda_eIoni_em, mat, e);
    xs[1] = lambda_table(w, GXO_Lambda_eBrem_em, mat, e);
  } else {
    xs[0] = lambda_table(w, GXO_Lambda_eIoni_ep, mat, e);
    xs[1] = lambda_table(w, GXO_Lambda_eBrem_ep, mat, e);
    xs[2] = w->mat[mat].n_el * gxo_annih_xs_per_electron(e);
  }
  for (int i = 0; i < 3; ++i)
    if (!(xs[i] > 0.0)) xs[i] = 0.0;
}

static int nproc(int type) { return type == 1 ? 2 : 3; }

/* ------------------------------------------------------ multiple scattering
 * Multiple scattering of e-/e+ (physics mode, config msc = 1; 2 adds the
 * lateral displacement): the Urban
 * model as published (L. Urban, CERN-OPEN-2006-077): the reference has only a
 * placeholder (proxy/ProxyScattering.hpp:53-71); it ships the transport mean
 * free path tables (LambdaMod1.msc.e-/e+: E^2 / lambda1, MeV^2 / mm).
 *   step limit: t <= max(MSC_FR r0, MSC_FS safety, MSC_TMIN), r0 = max(range,
 *     lambda1) taken at the first step in each volume (safety-based stepping);
 *   path lengths: geometric z = lambda1 (1 - exp(-t / lambda1)) from the true
 *     length t, and back when a boundary stops the step;
 *   deflection after the along-step loss: cos(theta) from the model's mixture
 *     (a central exponential part with the Highland-type width theta0, a power
 *     tail, a uniform part), normalised so that <cos theta> = exp(-tau),
 *     tau = t / lambda1 (averaged over the loss); phi uniform.  Where the
 *     published weights would need a uniform part above 1, the uniform part is
 *     dropped and the central/tail split set to keep that mean (a choice of
 *     this restatement);
 *   lateral displacement (msc = 2) after a step that ends inside its volume:
 *     0.73 sqrt(t^2 - z^2) perpendicular to the starting direction at the
 *     deflection's azimuth, cut to 0.99 of the end point's safety, none when
 *     that safety is below MSC_TMIN.
 * Not modelled: the e+ correction of theta0. */
#define MSC_FR 0.04
#define MSC_FS 0.6
#define MSC_TMIN 1.0e-5
#define MSC_TAUBIG 8.0
#define MSC_TAUSMALL 1.0e-16
#define MSC_TAULIM 1.0e-6

/* Z-dependent constants of the model: the theta0 correction and the tail
 * parameter's coefficients. */
static void msc_material(double Z, double X0, struct msc_mat *m)
{
  double z16 = exp(log(Z) / 6.0), z13 = z16 * z16;
  double facz = 0.990395 + z16 * (-0.168386 + z16 * 0.093286);
  m->X0 = X0;
  m->th1 = facz * (1.0 - 8.7780e-2 / Z);
  m->th2 = facz * (4.0780e-2 + 1.7315e-4 * Z);
  m->ca = 2.3785 - z13 * (4.1981e-1 - z13 * 6.3100e-2);
  m->cb = 4.7526e-1 + z13 * (1.7694 - z13 * 3.3885e-1);
  m->cc = 2.3683e-1 - z13 * (1.8111 - z13 * 3.2774e-1);
  m->cd = 1.7888e-2 + z13 * (1.9659e-2 - z13 * 2.6664e-3);
}

/* transport mean free path lambda1 (mm); 0 when the table has nothing */
static double msc_lambda1(const world_t *w, int type, int mat, double e)
{
  const gxo_pvec_t *v = &w->d->vec[type == 2 ? GXO_LambdaMod1_msc_ep : GXO_LambdaMod1_msc_em][mat];
  double t = gxo_pvec_value(v, e);
  return t > 0.0 ? e * e / t : 0.0;
}

static double msc_range(const world_t *w, int type, int mat, double e)
{
  double r = gxo_table_value(w->d, type == 2 ? GXO_Range_ep : GXO_Range_em, mat, e);
  if (e < MINE) r *= e / MINE;
  return r;
}

static double msc_true_to_geom(double t, double lam)
{
  double tau = t / lam;
  return tau < MSC_TAULIM ? t : -lam * gxo_expm1(-tau);
}

static double msc_geom_to_true(double z, double lam, double tmax)
{
  double x = z / lam;
  if (x < MSC_TAULIM) return z;
  double t = x < 1.0 ? -lam * gxo_log1p(-x) : tmax;
  return t < tmax ? t : tmax;
}

/* the model's two-function form for large angles: exact first and second moments */
static double msc_simple(gxo_mrg_t *r, double xm, double x2m)
{
  double a = (2 * xm + 9 * x2m - 3) / (2 * xm - 3 * x2m + 1);
  double prob = (a + 2) * xm / a;
  double r0 = gxo_mrg_u01(r), r1 = gxo_mrg_u01(r);
  if (r0 < prob) return -1 + 2 * gxo_exp(gxo_log(r1) / (a + 1));
  return -1 + 2 * r1;
}

/* cos(theta) after a true path t; lam0 / lam1 and e0 / e1 at the start and
 * the end of the step */
static double msc_cos_theta(gxo_mrg_t *r, const struct msc_mat *m, double t, double lam0, double lam1, double e0,
                            double e1)
{
  double tau = t / lam0;
  if (lam1 > 0.0 && fabs(lam1 - lam0) > 0.01 * lam0) tau = t * gxo_log(lam0 / lam1) / (lam0 - lam1);
  if (tau >= MSC_TAUBIG) return -1 + 2 * gxo_mrg_u01(r);
  if (tau < MSC_TAUSMALL) return 1.0;
  double xm, x2m;
  if (tau < 0.01) {
    xm = 1 - tau * (1 - 0.5 * tau);
    x2m = 1 - tau * (5 - 6.25 * tau) / 3;
  } else {
    xm = gxo_exp(-tau);
    x2m = (1 + 2 * gxo_exp(-2.5 * tau)) / 3;
  }
  if (1.0 - e1 / e0 > 0.5) return msc_simple(r, xm, x2m);
  /* Highland-type width with the model's Z-dependent correction; 1 / (beta c p)
   * taken at the geometric mean of the start and end energies */
  double inv0 = (e0 + EMASS) / (e0 * (e0 + 2 * EMASS)), inv1 = (e1 + EMASS) / (e1 * (e1 + 2 * EMASS));
  double y = t / m->X0;
  double th0 = 13.6 * sqrt(y) * sqrt(inv0 * inv1) * (m->th1 + m->th2 * gxo_log(y));
  double th2 = th0 * th0;
  if (th2 < MSC_TAUSMALL) return 1.0;
  if (th0 > PI / 6) return msc_simple(r, xm, x2m);
  double x = th2 * (1 - th2 / 12);
  if (th2 > 0.01) {
    double s = 2 * gxo_sin(0.5 * th0);
    x = s * s;
  }
  double u = gxo_exp(gxo_log(tau) / 6);
  double xsi = m->ca + u * (m->cb + m->cc * u) + m->cd * gxo_log((t / tau) / m->X0);
  if (xsi < 1.9) xsi = 1.9;
  double c = xsi;
  if (fabs(c - 3) < 0.001)
    c = 3.001;
  else if (fabs(c - 2) < 0.001)
    c = 2.001;
  double c1 = c - 1;
  double ea = gxo_exp(-xsi), eaa = 1 - ea;
  double xmean1 = 1 - (1 - (1 + xsi) * ea) * x / eaa;
  if (xmean1 <= 0.999 * xm) return msc_simple(r, xm, x2m);
  double x0 = 1 - xsi * x;
  double b = 1 + (c - xsi) * x, b1 = b + 1, bx = c * x;
  double d = gxo_exp(c1 * gxo_log(bx)) / gxo_exp(c1 * gxo_log(b1));
  double xmean2 = (x0 + d - (bx - b1 * d) / (c - 2)) / (1 - d);
  double f1x0 = ea / eaa, f2x0 = c1 / (c * (1 - d));
  double prob = f2x0 / (f1x0 + f2x0);
  double qprob = xm / (prob * xmean1 + (1 - prob) * xmean2);
  if (qprob > 1.0) {
    /* the published normalisation would need a negative uniform part: keep
     * q = 1 and move weight from the tail to the central part so that
     * <cos theta> = exp(-tau) still holds (xmean2 < xm < xmean1 here) */
    qprob = 1.0;
    prob = (xm - xmean2) / (xmean1 - xmean2);
  }
  double r0 = gxo_mrg_u01(r), r1 = gxo_mrg_u01(r);
  if (r0 < qprob) {
    if (r1 < prob) return 1 + gxo_log(ea + gxo_mrg_u01(r) * eaa) * x;
    double var = (1 - d) * gxo_mrg_u01(r);
    if (var < 0.01 * d) {
      var /= d * c1;
      return -1 + var * (1 - 0.5 * var * c) * (2 + (c - xsi) * x);
    }
    return 1 + x * (c - xsi - c * gxo_exp(-gxo_log(var + d) / c1));
  }
  return -1 + 2 * r1;
}

/* deflect the direction by the sampled angle (no draw for phi when it is 0) */
/* returns 0 when the direction is kept (no azimuth drawn); *phi: the azimuth */
static int msc_deflect(const world_t *w, track_t *tr, int mat, double t, double lam0, double e0, double *phi_out)
{
  double lam1 = msc_lambda1(w, tr->type, mat, tr->E);
  double ct = msc_cos_theta(&tr->rng, &w->msc[mat], t, lam0, lam1, e0, tr->E);
  if (ct >= 1.0) return 0;
  if (ct < -1.0) ct = -1.0;
  double st = sqrt((1 - ct) * (1 + ct));
  double phi = TWOPI * gxo_mrg_u01(&tr->rng);
  double u = st * gxo_cos(phi), v = st * gxo_sin(phi), z = ct;
  gxo_rotate_to_lab(&u, &v, &z, tr->dir[0], tr->dir[1], tr->dir[2]);
  tr->dir[0] = u;
  tr->dir[1] = v;
  tr->dir[2] = z;
  *phi_out = phi;
  return 1;
}

/* ---------------------------------------------------------- one track step */
typedef struct {
  double *edep; /* [events][nvol] */
  int nvol;
  double escaped;
  long long steps, substeps, tracks, sec[3], npair, nannih, errors;
  int *pstep;
  const gxo_csg_t *csg; /* geometry 2: tally bins are the touchables' score indices */
} tally_t;

static void deposit(tally_t *t, int event, int vol, double e)
{
  if (vol >= 0 && t->csg) vol = t->csg->node[vol].score; /* unscored touchables: -1 */
  if (vol >= 0 && e != 0.0) t->edep[(long)event * t->nvol + vol] += e;
}

static void make_secondary(const world_t *w, track_t *parent, stack_t *st, tally_t *t, int type,
                           double e, const double *dir)
{
  if (w->c->charged_local && type != 0) {
    deposit(t, parent->event, parent->vol, e);
    return;
  }
  track_t s;
  memset(&s, 0, sizeof(s));
  s.type = type;
  s.E = e;
  for (int k = 0; k < 3; ++k) {
    s.pos[k] = parent->pos[k];
    s.dir[k] = dir[k];
  }
  s.vol = parent->vol;
  s.nil[0] = s.nil[1] = s.nil[2] = -1.0;
  s.msc_r0 = -1.0;
  gxo_mrg_seed_child(&parent->rng, &s.rng);
  s.event = parent->event;
  s.primary = -1;
  t->sec[type]++;
  push(st, &s);
}

/* One classical fourth-order Runge-Kutta step of length s through the field
 * map: du/ds = k u x B(x), k = 0.299792458 q / p; direction renormalised.
 * (The reference has no stepper for non-uniform fields; this is the textbook
 * method, the same operations as the CUDA engine's.) */
static void rk4_map_step(const float *map, double k, double s, double x[3], double u[3], const double B0[3])
{
  double xs[3], us[3], B[3], kx[4][3], ku[4][3];
  const double h[3] = {0.5 * s, 0.5 * s, s};
  for (int j = 0; j < 3; ++j) kx[0][j] = u[j];
  ku[0][0] = k * (u[1] * B0[2] - u[2] * B0[1]);
  ku[0][1] = k * (u[2] * B0[0] - u[0] * B0[2]);
  ku[0][2] = k * (u[0] * B0[1] - u[1] * B0[0]);
  for (int st = 1; st < 4; ++st) {
    for (int j = 0; j < 3; ++j) {
      xs[j] = x[j] + h[st - 1] * kx[st - 1][j];
      us[j] = u[j] + h[st - 1] * ku[st - 1][j];
    }
    gxo_field_map_value(map, xs, B);
    for (int j = 0; j < 3; ++j) kx[st][j] = us[j];
    ku[st][0] = k * (us[1] * B[2] - us[2] * B[1]);
    ku[st][1] = k * (us[2] * B[0] - us[0] * B[2]);
    ku[st][2] = k * (us[0] * B[1] - us[1] * B[0]);
  }
  double m = 0.0;
  for (int j = 0; j < 3; ++j) {
    x[j] += s / 6.0 * (kx[0][j] + 2.0 * kx[1][j] + 2.0 * kx[2][j] + kx[3][j]);
    u[j] += s / 6.0 * (ku[0][j] + 2.0 * ku[1][j] + 2.0 * ku[2][j] + ku[3][j]);
    m += u[j] * u[j];
  }
  m = 1.0 / sqrt(m);
  for (int j = 0; j < 3; ++j) u[j] *= m;
}

/* Helix sub-steps in Bz (FieldPropagationHandler::Propagate/PropagateInVolume).
 * Returns the path length; *crossed and *newvol report a boundary crossing. */
static double field_propagate(const world_t *w, track_t *tr, double pstep, int *crossed, int *newvol,
                              tally_t *t)
{
  const double eps = 0.1;         /* gEpsDeflection = 1e-2 cm */
  double charge = (tr->type == 1) ? -1.0 : 1.0;
  double p = sqrt(tr->E * (tr->E + 2.0 * EMASS));
  double Bz = w->c->Bz;
  double remaining = pstep, total = 0.0;
  *crossed = 0;
  *newvol = tr->vol;
  for (int it = 0; it < 10000; ++it) {
    int plane;
    double saf = safety(w, tr->vol, tr->pos);
    double snext;
    if (saf > remaining)
      snext = remaining;
    else
      snext = fmax(2e-9, fmin(dist_to_out(w, tr->vol, tr->pos, tr->dir, &plane), remaining) + 2e-9);
    double step_gp = fmax(fmin(remaining, 1e-4), snext);
    double np[3], nd[3], s;
    if (w->c->field_map) {
      /* the field map: the sub-step length from the field at the start
       * point, then a Runge-Kutta step */
      double B0[3];
      gxo_field_map_value(w->c->field_map, tr->pos, B0);
      const double *u = tr->dir;
      double cx = u[1] * B0[2] - u[2] * B0[1], cy = u[2] * B0[0] - u[0] * B0[2], cz = u[0] * B0[1] - u[1] * B0[0];
      double bperp = sqrt(cx * cx + cy * cy + cz * cz);
      double step_field = DBL_MAX;
      if (bperp > 0.0) step_field = fmax(2.0 * sqrt(eps * p / (0.299792458 * bperp)), saf);
      s = fmin(fmin(step_gp, step_field), remaining);
      for (int k = 0; k < 3; ++k) {
        np[k] = tr->pos[k];
        nd[k] = tr->dir[k];
      }
      if (bperp > 0.0)
        rk4_map_step(w->c->field_map, 0.299792458 * charge / p, s, np, nd, B0);
      else
        for (int k = 0; k < 3; ++k) np[k] += s * nd[k];
    } else {
    double pt = p * sqrt(fmax(1.0 - tr->dir[2] * tr->dir[2], 0.0));
    double step_field = DBL_MAX;
    if (pt > 0.0) {
      double curv = 0.299792458 * fabs(Bz) / pt;
      step_field = fmax(2.0 * sqrt(eps / curv), saf);
    }
    s = fmin(fmin(step_gp, step_field), remaining);
    if (pt > 0.0) {
      gxo_helix_dostep_mm(Bz, tr->pos, tr->dir, charge, p, s, np, nd);
      double m = sqrt(nd[0] * nd[0] + nd[1] * nd[1] + nd[2] * nd[2]);
      nd[0] /= m;
      nd[1] /= m;
      nd[2] /= m;
    } else {
      for (int k = 0; k < 3; ++k) {
        np[k] = tr->pos[k] + s * tr->dir[k];
        nd[k] = tr->dir[k];
      }
    }
    }
    for (int k = 0; k < 3; ++k) {
      tr->pos[k] = np[k];
      tr->dir[k] = nd[k];
    }
    total += s;
    remaining -= s;
    t->substeps++;
    int v = relocate(w, tr->vol, tr->pos, tr->dir);
    if (v != tr->vol) {
      *crossed = 1;
      *newvol = v;
      return total;
    }
    if (remaining <= 1e-10) return total;
  }
  t->errors++;
  *crossed = 1;
  *newvol = -2; /* stuck: killed by the caller */
  return total;
}

static void run_model(const world_t *w, track_t *tr, int proc, stack_t *st, tally_t *t)
{
  int mat = vol_material(w, tr->vol);
  gxo_model_params_t mp;
  memset(&mp, 0, sizeof(mp));
  mp.mode = GXO_MODE_PHYSICS;
  mp.Z = (int)w->mat[mat].Z;
  mp.data = w->d;
  mp.density_factor = w->mat[mat].density_factor;
  mp.sb = (mat == 1) ? &w->d->sb_pb : &w->d->sb_ar;
  gxo_inter_t io;
  memset(&io, 0, sizeof(io));
  io.E = tr->E;
  memcpy(io.dir, tr->dir, sizeof(io.dir));
  if (tr->type == 0) {
    if (proc == 0)
      gxo_kn_sample(&tr->rng, &mp, &io);
    else if (proc == 1) {
      gxo_bh_sample(&tr->rng, &mp, &io);
      if (io.nsec == 2) t->npair++;
    } else
      gxo_sg_sample(&tr->rng, &mp, &io);
  } else if (proc == 0) {
    mp.cut = w->d->cut_energy[1][mat];
    if (tr->type == 1)
      gxo_mb_sample(&tr->rng, &mp, &io);
    else
      gxo_bhabha_sample(&tr->rng, &mp, &io);
  } else if (proc == 1) {
    mp.cut = w->d->cut_energy[0][mat];
    gxo_sb_sample(&tr->rng, &mp, &io);
  } else {
    gxo_annih_sample(&tr->rng, &mp, &io);
    t->nannih++;
  }
  deposit(t, tr->event, tr->vol, io.edep);
  tr->E = io.E;
  memcpy(tr->dir, io.dir, sizeof(io.dir));
  for (int s = 0; s < io.nsec; ++s) make_secondary(w, tr, st, t, io.sec_type[s], io.sec_E[s], io.sec_dir[s]);
  if (io.status == 1) tr->E = 0.0;
}

/* One OneStep of one track; returns 0 when the track is finished. */
static int one_step(const world_t *w, track_t *tr, stack_t *st, tally_t *t)
{
  int mat = vol_material(w, tr->vol);
  int np = nproc(tr->type);
  int charged = tr->type != 0;
  double xs[3];
  cross_sections(w, tr->type, mat, tr->E, xs);
  for (int i = 0; i < np; ++i)
    if (tr->nil[i] <= 0.0) tr->nil[i] = -gxo_log(gxo_mrg_u01(&tr->rng));
  double pstep = DBL_MAX;
  int sel = -1;
  for (int i = 0; i < np; ++i)
    if (xs[i] > 0.0) {
      double s = tr->nil[i] / xs[i];
      if (s < pstep) {
        pstep = s;
        sel = i;
      }
    }
  if (charged) {
    double slim = gxo_ioni_along_gpil(w->d, GXO_MODE_PHYSICS, tr->type == 2 ? 1 : -1, mat, tr->E);
    if (slim < pstep) {
      pstep = slim;
      sel = -1;
    }
  }
  /* multiple scattering: its step limit, then the true step pstep becomes the
   * geometric length to move */
  const int msc = charged && w->c->msc;
  double lam0 = 0.0, ttrue = 0.0, e0 = tr->E;
  if (msc) {
    lam0 = msc_lambda1(w, tr->type, mat, tr->E);
    if (tr->msc_r0 <= 0.0) tr->msc_r0 = fmax(msc_range(w, tr->type, mat, tr->E), lam0);
    double tlim = fmax(fmax(MSC_FR * tr->msc_r0, MSC_FS * safety(w, tr->vol, tr->pos)), MSC_TMIN);
    if (tlim < pstep) {
      pstep = tlim;
      sel = -1;
    }
    ttrue = pstep;
    if (lam0 > 0.0) pstep = msc_true_to_geom(pstep, lam0);
  }
  int vol0 = tr->vol, crossed = 0, newvol = tr->vol;
  double step;
  if (!charged || (w->c->Bz == 0.0 && !w->c->field_map)) {
    int plane;
    double d = dist_to_out(w, tr->vol, tr->pos, tr->dir, &plane);
    if (d < pstep) {
      step = d;
      crossed = 1;
      for (int k = 0; k < 3; ++k) tr->pos[k] += step * tr->dir[k];
      if (w->c->geometry == 2)
        newvol = gxo_csg_cross(w->c->csg, tr->vol, plane, tr->pos, tr->dir);
      else
        newvol = next_volume(w, tr->vol, plane);
      if (plane != 2 && w->c->geometry != 2) {
        double lo, hi;
        slab_bounds(w, tr->vol, &lo, &hi);
        tr->pos[w->c->axis] = plane > 0 ? hi : lo;
      }
    } else {
      step = pstep;
      for (int k = 0; k < 3; ++k) tr->pos[k] += step * tr->dir[k];
    }
  } else {
    step = field_propagate(w, tr, pstep, &crossed, &newvol, t);
  }
  /* the true length of the step: all of it, or back from where a boundary
   * stopped it */
  const double zgeom = step; /* the geometric length moved */
  if (msc && lam0 > 0.0) step = crossed ? msc_geom_to_true(step, lam0, ttrue) : ttrue;
  for (int i = 0; i < np; ++i) tr->nil[i] -= step * xs[i];
  t->steps++;
  if (newvol == -2) { /* stuck in field: deposit and stop */
    deposit(t, tr->event, vol0, tr->E);
    return 0;
  }
  if (charged) {
    double edep = 0.0;
    gxo_ioni_along_doit(w->d, GXO_MODE_PHYSICS, tr->type == 2 ? 1 : -1, mat, step, &tr->E, &edep);
    deposit(t, tr->event, vol0, edep);
    if (tr->E <= 0.0) {
      /* a stopped e+ annihilates at rest where it stopped (ProxyIonization has
       * no e+ branch; Geant4 semantics) */
      if (tr->type == 2) {
        int v = crossed ? newvol : vol0;
        if (v >= 0) {
          tr->vol = v;
          run_model(w, tr, 2, st, t);
        } else {
          t->escaped += 2.0 * EMASS;
        }
      }
      return 0;
    }
    if (msc && lam0 > 0.0) {
      const double d0 = tr->dir[0], d1 = tr->dir[1], d2 = tr->dir[2];
      double phi = 0.0;
      int turned = msc_deflect(w, tr, mat, step, lam0, e0, &phi);
      if (w->c->msc == 2 && turned && !crossed) { /* lateral displacement */
        const double rmax2 = (step - zgeom) * (step + zgeom);
        const double saf = rmax2 > 0.0 ? safety(w, tr->vol, tr->pos) : 0.0;
        if (saf > MSC_TMIN) {
          double r = fmin(0.73 * sqrt(rmax2), 0.99 * saf);
          double u = gxo_cos(phi), v = gxo_sin(phi), z = 0.0;
          gxo_rotate_to_lab(&u, &v, &z, d0, d1, d2);
          tr->pos[0] += r * u;
          tr->pos[1] += r * v;
          tr->pos[2] += r * z;
        }
      }
    }
  }
  if (crossed) {
    tr->msc_r0 = -1.0; /* a new volume: the step limit starts again */
    tr->vol = newvol;
    if (newvol < 0) {
      t->escaped += tr->E;
      if (tr->type == 2) t->escaped += 2.0 * EMASS;
      return 0;
    }
    return 1;
  }
  if (sel >= 0) {
    tr->nil[sel] = -1.0;
    run_model(w, tr, sel, st, t);
    if (tr->E <= 0.0) return 0;
  }
  return 1;
}

/* test front ends of the multiple-scattering model */
void gxo_msc_cos_batch(double Z, double X0, int n, double *states, double t, double lam0, double lam1, double e0,
                       double e1, double *out)
{
  struct msc_mat m;
  msc_material(Z, X0, &m);
  for (int i = 0; i < n; ++i) {
    gxo_mrg_t r;
    memcpy(r.s, &states[6 * i], sizeof(r.s));
    out[i] = msc_cos_theta(&r, &m, t, lam0, lam1, e0, e1);
    memcpy(&states[6 * i], r.s, sizeof(r.s));
  }
}

double gxo_msc_lambda1(const gxo_data_t *d, int type, int mat, double e)
{
  world_t w;
  memset(&w, 0, sizeof(w));
  w.d = d;
  return msc_lambda1(&w, type, mat, e);
}

double gxo_msc_true_to_geom(double t, double lam) { return msc_true_to_geom(t, lam); }
double gxo_msc_geom_to_true(double z, double lam, double tmax) { return msc_geom_to_true(z, lam, tmax); }

/* ------------------------------------------------ tracks handed in or out */
static void track_in(const world_t *w, const gxo_tracks_t *a, int i, track_t *tr)
{
  memset(tr, 0, sizeof(*tr));
  tr->type = a->type[i];
  tr->E = a->ekin[i];
  for (int k = 0; k < 3; ++k) {
    tr->pos[k] = a->pos[3 * i + k];
    tr->dir[k] = a->dir[3 * i + k];
    tr->nil[k] = a->nil[3 * i + k];
  }
  tr->msc_r0 = a->msc ? a->msc[i] : -1.0;
  memcpy(tr->rng.s, &a->rng[6 * i], sizeof(tr->rng.s));
  tr->vol = a->volume[i];
  if (tr->vol < -1) tr->vol = locate(w, tr->pos, tr->dir);
  tr->event = a->event ? a->event[i] : 0;
  tr->primary = -1;
}

static void track_out(const track_t *tr, gxo_tracks_t *a, int i, int status)
{
  a->type[i] = tr->type;
  a->status[i] = status;
  if (a->event) a->event[i] = tr->event;
  if (a->primary) a->primary[i] = -1;
  a->volume[i] = tr->vol;
  a->ekin[i] = tr->E;
  for (int k = 0; k < 3; ++k) {
    a->pos[3 * i + k] = tr->pos[k];
    a->dir[3 * i + k] = tr->dir[k];
    a->nil[3 * i + k] = tr->nil[k];
  }
  if (a->msc) a->msc[i] = tr->msc_r0;
  memcpy(&a->rng[6 * i], tr->rng.s, sizeof(tr->rng.s));
}

static void world_init(world_t *w, const gxo_data_t *d, const gxo_config_t *cfg)
{
  memset(w, 0, sizeof(*w));
  w->d = d;
  w->c = cfg;
  w->pitch = cfg->t_abs + cfg->t_gap;
  gxo_material_make(1.0, 1.01, 1.e-25, &w->mat[0]);
  gxo_material_make(82.0, 207.2, 11.35, &w->mat[1]);
  gxo_material_make(18.0, 39.95, 1.396, &w->mat[2]);
  for (int m = 0; m < 3; ++m) msc_material(w->mat[m].Z, w->mat[m].radlen, &w->msc[m]);
}

/* One OneStep of every track of t with status 0 (alive), in order, single
 * thread: the step-by-step counterpart of the CUDA library's stage calls
 * (gx_gpil .. gx_post_step).  A track's secondaries go to sec entries 2i,
 * 2i+1 in the order they are made (status 0; unused entries status 1, type
 * -1); t's status becomes 0 alive, 1 finished, 3 left the world (its energy
 * kept).  counters: steps, substeps, secondaries (gamma, e-, e+), pairs,
 * annihilations, errors. */
int gxo_step_tracks(const gxo_data_t *d, const gxo_config_t *cfg, gxo_tracks_t *t, gxo_tracks_t *sec,
                    double *edep, int nvol, double *escaped, long long *counters)
{
  world_t w;
  world_init(&w, d, cfg);
  tally_t ta;
  memset(&ta, 0, sizeof(ta));
  ta.edep = edep;
  ta.nvol = nvol;
  stack_t st = {0, 0, 0};
  for (int i = 0; i < t->n; ++i) {
    int nsec = 0;
    if (t->status[i] == 0) {
      track_t tr;
      track_in(&w, t, i, &tr);
      st.n = 0;
      int alive = (tr.vol >= 0) ? one_step(&w, &tr, &st, &ta) : 0;
      track_out(&tr, t, i, alive ? 0 : (tr.vol < 0 ? 3 : 1));
      for (int k = 0; k < st.n && k < 2; ++k) {
        track_out(&st.a[k], sec, 2 * i + k, 0);
        nsec++;
      }
    }
    for (int k = nsec; k < 2; ++k) {
      sec->status[2 * i + k] = 1;
      sec->type[2 * i + k] = -1;
    }
  }
  sec->n = 2 * t->n;
  free(st.a);
  *escaped = ta.escaped;
  counters[0] = ta.steps;
  counters[1] = ta.substeps;
  counters[2] = ta.sec[0];
  counters[3] = ta.sec[1];
  counters[4] = ta.sec[2];
  counters[5] = ta.npair;
  counters[6] = ta.nannih;
  counters[7] = ta.errors;
  return 0;
}

/* -------------------------------------------------------------- runner */
typedef struct {
  world_t *w;
  int nprim;
  const gxo_primary_t *prims;
  const gxo_tracks_t *tracks; /* instead of prims: tracks handed in with their state */
  int tid, nthreads;
  tally_t t;
  double seedcopy[6];
} job_t;

static void *worker(void *arg)
{
  job_t *j = (job_t *)arg;
  world_t *w = j->w;
  stack_t st = {0, 0, 0};
  for (int i = j->tid; i < j->nprim; i += j->nthreads) {
    track_t tr;
    if (j->tracks) {
      if (j->tracks->status[i] != 0) continue;
      track_in(w, j->tracks, i, &tr);
    } else {
      const gxo_primary_t *pr = &j->prims[i];
      memset(&tr, 0, sizeof(tr));
      tr.type = pr->type;
      tr.E = pr->E;
      memcpy(tr.pos, pr->pos, sizeof(tr.pos));
      memcpy(tr.dir, pr->dir, sizeof(tr.dir));
      tr.vol = locate(w, tr.pos, tr.dir);
      tr.nil[0] = tr.nil[1] = tr.nil[2] = -1.0;
      tr.msc_r0 = -1.0;
      gxo_mrg_substreams(w->c->seed, w->c->first_substream + i, 1, tr.rng.s);
      tr.event = pr->event;
      tr.primary = i;
    }
    if (tr.vol < 0) {
      j->t.escaped += tr.E;
      continue;
    }
    push(&st, &tr);
    while (st.n > 0) {
      track_t cur = st.a[--st.n];
      j->t.tracks++;
      int nsteps = 0;
      while (one_step(w, &cur, &st, &j->t)) {
        if (++nsteps >= w->c->max_steps) {
          j->t.errors++;
          deposit(&j->t, cur.event, cur.vol, cur.E);
          break;
        }
      }
      if (cur.primary >= 0 && j->t.pstep) j->t.pstep[cur.primary] = nsteps + 1;
    }
  }
  free(st.a);
  return NULL;
}

static int transport_jobs(const gxo_data_t *d, const gxo_config_t *cfg, int nprim, const gxo_primary_t *prims,
                          const gxo_tracks_t *tracks, gxo_result_t *res)
{
  world_t w;
  world_init(&w, d, cfg);
  int nt = cfg->nthreads > 0 ? cfg->nthreads : 1;
  int nvol = res->nvol;
  if (cfg->geometry == 2 && (!cfg->csg || nvol != cfg->csg->nscore)) return -1;
  int nev = cfg->score_events > 0 ? cfg->score_events : 1;
  job_t *jobs = (job_t *)calloc(nt, sizeof(job_t));
  pthread_t *th = (pthread_t *)calloc(nt, sizeof(pthread_t));
  for (int k = 0; k < nt; ++k) {
    jobs[k].w = &w;
    jobs[k].nprim = nprim;
    jobs[k].prims = prims;
    jobs[k].tracks = tracks;
    jobs[k].tid = k;
    jobs[k].nthreads = nt;
    jobs[k].t.nvol = nvol;
    jobs[k].t.edep = (double *)calloc((size_t)nev * nvol, sizeof(double));
    jobs[k].t.pstep = res->primary_steps;
    jobs[k].t.csg = cfg->geometry == 2 ? cfg->csg : NULL;
    pthread_create(&th[k], NULL, worker, &jobs[k]);
  }
  memset(res->edep, 0, sizeof(double) * (size_t)nev * nvol);
  res->escaped = 0;
  res->steps = res->substeps = res->tracks = res->n_pair = res->n_annih = res->errors = 0;
  res->secondaries[0] = res->secondaries[1] = res->secondaries[2] = 0;
  for (int k = 0; k < nt; ++k) {
    pthread_join(th[k], NULL);
    for (long v = 0; v < (long)nev * nvol; ++v) res->edep[v] += jobs[k].t.edep[v];
    res->escaped += jobs[k].t.escaped;
    res->steps += jobs[k].t.steps;
    res->substeps += jobs[k].t.substeps;
    res->tracks += jobs[k].t.tracks;
    res->n_pair += jobs[k].t.npair;
    res->n_annih += jobs[k].t.nannih;
    res->errors += jobs[k].t.errors;
    for (int s = 0; s < 3; ++s) res->secondaries[s] += jobs[k].t.sec[s];
    free(jobs[k].t.edep);
  }
  free(jobs);
  free(th);
  return 0;
}

int gxo_transport(const gxo_data_t *d, const gxo_config_t *cfg, int nprim, const gxo_primary_t *prims,
                  gxo_result_t *res)
{
  return transport_jobs(d, cfg, nprim, prims, NULL, res);
}

/* The tracks of t with status 0, handed in with their state, transported to
 * completion with their secondaries (the oracle's side of the hand-over of
 * gx_transport_tracks); counters as gxo_transport_flat's. */
int gxo_transport_tracks(const gxo_data_t *d, const gxo_config_t *cfg, const gxo_tracks_t *t, double *edep, int nvol,
                         double *escaped, long long *counters)
{
  gxo_result_t r;
  memset(&r, 0, sizeof(r));
  r.edep = edep;
  r.nvol = nvol;
  int rc = transport_jobs(d, cfg, t->n, NULL, t, &r);
  *escaped = r.escaped;
  counters[0] = r.steps;
  counters[1] = r.substeps;
  counters[2] = r.tracks;
  counters[3] = r.secondaries[0];
  counters[4] = r.secondaries[1];
  counters[5] = r.secondaries[2];
  counters[6] = r.n_pair;
  counters[7] = r.n_annih;
  counters[8] = r.errors;
  return rc;
}

int gxo_transport_flat(const gxo_data_t *d, const gxo_config_t *cfg, int nprim, const int *type,
                       const double *E, const double *pos, const double *dir, const int *event,
                       double *edep, int nvol, double *escaped, long long *counters, int *primary_steps)
{
  gxo_primary_t *p = (gxo_primary_t *)malloc(sizeof(gxo_primary_t) * (nprim > 0 ? nprim : 1));
  for (int i = 0; i < nprim; ++i) {
    p[i].type = type[i];
    p[i].E = E[i];
    for (int k = 0; k < 3; ++k) {
      p[i].pos[k] = pos[3 * i + k];
      p[i].dir[k] = dir[3 * i + k];
    }
    p[i].event = event ? event[i] : 0;
  }
  gxo_result_t r;
  memset(&r, 0, sizeof(r));
  r.edep = edep;
  r.nvol = nvol;
  r.primary_steps = primary_steps;
  int rc = gxo_transport(d, cfg, nprim, p, &r);
  *escaped = r.escaped;
  counters[0] = r.steps;
  counters[1] = r.substeps;
  counters[2] = r.tracks;
  counters[3] = r.secondaries[0];
  counters[4] = r.secondaries[1];
  counters[5] = r.secondaries[2];
  counters[6] = r.n_pair;
  counters[7] = r.n_annih;
  counters[8] = r.errors;
  free(p);
  return rc;
}
