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

typedef struct {
  int type;
  double E, pos[3], dir[3];
  int vol;
  double nil[3];
  gxo_mrg_t rng;
  int event;
  int primary; /* index of the primary if this is the primary track, else -1 */
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
} world_t;

/* ---------------------------------------------------------------- geometry */
/* Volumes: calorimeter: vol = 2 * layer + slab (slab 0 absorber = material 1
 * (Pb), slab 1 gap = material 2 (LAr)); box: vol 0 = box material; -1 outside. */
static int vol_material(const world_t *w, int vol)
{
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
 * low axis plane, +1 high axis plane, 2 transverse wall. */
static double dist_to_out(const world_t *w, int vol, const double *p, const double *d, int *plane)
{
  const gxo_config_t *c = w->c;
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

/* ---------------------------------------------------------- one track step */
typedef struct {
  double *edep; /* [events][nvol] */
  int nvol;
  double escaped;
  long long steps, substeps, tracks, sec[3], npair, nannih, errors;
  int *pstep;
} tally_t;

static void deposit(tally_t *t, int event, int vol, double e)
{
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
  gxo_mrg_seed_child(&parent->rng, &s.rng);
  s.event = parent->event;
  s.primary = -1;
  t->sec[type]++;
  push(st, &s);
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
    double pt = p * sqrt(fmax(1.0 - tr->dir[2] * tr->dir[2], 0.0));
    double step_field = DBL_MAX;
    if (pt > 0.0) {
      double curv = 0.299792458 * fabs(Bz) / pt;
      step_field = fmax(2.0 * sqrt(eps / curv), saf);
    }
    double s = fmin(fmin(step_gp, step_field), remaining);
    double np[3], nd[3];
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
    if (tr->nil[i] <= 0.0) tr->nil[i] = -log(gxo_mrg_u01(&tr->rng));
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
  int vol0 = tr->vol, crossed = 0, newvol = tr->vol;
  double step;
  if (!charged || w->c->Bz == 0.0) {
    int plane;
    double d = dist_to_out(w, tr->vol, tr->pos, tr->dir, &plane);
    if (d < pstep) {
      step = d;
      crossed = 1;
      newvol = next_volume(w, tr->vol, plane);
      for (int k = 0; k < 3; ++k) tr->pos[k] += step * tr->dir[k];
      if (plane != 2) {
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
  }
  if (crossed) {
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

/* -------------------------------------------------------------- runner */
typedef struct {
  world_t *w;
  int nprim;
  const gxo_primary_t *prims;
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
    const gxo_primary_t *pr = &j->prims[i];
    track_t tr;
    memset(&tr, 0, sizeof(tr));
    tr.type = pr->type;
    tr.E = pr->E;
    memcpy(tr.pos, pr->pos, sizeof(tr.pos));
    memcpy(tr.dir, pr->dir, sizeof(tr.dir));
    tr.vol = locate(w, tr.pos, tr.dir);
    tr.nil[0] = tr.nil[1] = tr.nil[2] = -1.0;
    gxo_mrg_substreams(w->c->seed, w->c->first_substream + i, 1, tr.rng.s);
    tr.event = pr->event;
    tr.primary = i;
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

int gxo_transport(const gxo_data_t *d, const gxo_config_t *cfg, int nprim, const gxo_primary_t *prims,
                  gxo_result_t *res)
{
  world_t w;
  memset(&w, 0, sizeof(w));
  w.d = d;
  w.c = cfg;
  w.pitch = cfg->t_abs + cfg->t_gap;
  gxo_material_make(1.0, 1.01, 1.e-25, &w.mat[0]);
  gxo_material_make(82.0, 207.2, 11.35, &w.mat[1]);
  gxo_material_make(18.0, 39.95, 1.396, &w.mat[2]);
  int nt = cfg->nthreads > 0 ? cfg->nthreads : 1;
  int nvol = res->nvol;
  int nev = cfg->score_events > 0 ? cfg->score_events : 1;
  job_t *jobs = (job_t *)calloc(nt, sizeof(job_t));
  pthread_t *th = (pthread_t *)calloc(nt, sizeof(pthread_t));
  for (int k = 0; k < nt; ++k) {
    jobs[k].w = &w;
    jobs[k].nprim = nprim;
    jobs[k].prims = prims;
    jobs[k].tid = k;
    jobs[k].nthreads = nt;
    jobs[k].t.nvol = nvol;
    jobs[k].t.edep = (double *)calloc((size_t)nev * nvol, sizeof(double));
    jobs[k].t.pstep = res->primary_steps;
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
