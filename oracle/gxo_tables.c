/*
 * gxo_tables.c -- ORACLE (test infrastructure only): physics-table reader and
 * spline interpolation restated from the reference's
 * source/Geant/proxy/src/ProxyPhysicsVector.cu, ProxyPhysicsTable.cu,
 * ProxyDataManager.cu and Proxy2DVector.cpp, plus the Seltzer-Berger loader of
 * ProxySeltzerBerger.hpp:487-526 and the shell / Sandia data of
 * ProxySandiaData.hpp (read from the imported sandia.dat).
 */
#include "gxo.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static const char *kTableName[GXO_NTABLES] = {
    "DEDX.eBrem.e-.asc", "DEDX.eBrem.e+.asc", "DEDX.eIoni.e-.asc", "DEDX.eIoni.e+.asc",
    "InverseRange.eIoni.e-.asc", "InverseRange.eIoni.e+.asc", "Ionisation.eIoni.e-.asc",
    "Ionisation.eIoni.e+.asc", "Lambda.compt.gamma.asc", "Lambda.conv.gamma.asc",
    "Lambda.eBrem.e-.asc", "Lambda.eBrem.e+.asc", "Lambda.eIoni.e-.asc", "Lambda.eIoni.e+.asc",
    "LambdaMod1.msc.e-.asc", "LambdaMod1.msc.e+.asc", "LambdaPrim.compt.gamma.asc",
    "LambdaPrim.phot.gamma.asc", "Range.eIoni.e-.asc", "Range.eIoni.e+.asc"};

/* ComputeSecDerivatives, ProxyPhysicsVector.cu:211-238 (fewer than 5 nodes) */
static void compute_sec_derivatives(gxo_pvec_t *v)
{
  int n = v->n - 1;
  double *x = v->x, *y = v->y, *d = v->d2;
  for (int i = 0; i <= n; ++i) d[i] = 0.0;
  if (3 > v->n) return;
  for (int i = 1; i < n; ++i)
    d[i] = 3.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])) /
           (x[i + 1] - x[i - 1]);
  d[n] = d[n - 1];
  d[0] = d[1];
}

/* FillSecondDerivatives, not-a-knot end conditions, ProxyPhysicsVector.cu:308-386 */
static void fill_second_derivatives(gxo_pvec_t *v)
{
  if (5 > v->n) {
    compute_sec_derivatives(v);
    return;
  }
  double *x = v->x, *y = v->y, *d = v->d2;
  int n = v->n - 1;
  for (int i = 0; i <= n; ++i) d[i] = 0.0; /* SplinePossible, :188-209 */
  double *u = (double *)calloc((size_t)n, sizeof(double));
  double p, sig;
  u[1] = ((y[2] - y[1]) / (x[2] - x[1]) - (y[1] - y[0]) / (x[1] - x[0]));
  u[1] = 6.0 * u[1] * (x[2] - x[1]) / ((x[2] - x[0]) * (x[2] - x[0]));
  d[1] = (2.0 * x[1] - x[0] - x[2]) / (2.0 * x[2] - x[0] - x[1]);
  for (int i = 2; i < n - 1; ++i) {
    sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
    p = sig * d[i - 1] + 2.0;
    d[i] = (sig - 1.0) / p;
    u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
    u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1])) - sig * u[i - 1] / p;
  }
  sig = (x[n - 1] - x[n - 2]) / (x[n] - x[n - 2]);
  p = sig * d[n - 3] + 2.0;
  u[n - 1] = (y[n] - y[n - 1]) / (x[n] - x[n - 1]) - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
  u[n - 1] = 6.0 * sig * u[n - 1] / (x[n] - x[n - 2]) - (2.0 * sig - 1.0) * u[n - 2] / p;
  p = (1.0 + sig) + (2.0 * sig - 1.0) * d[n - 2];
  d[n - 1] = u[n - 1] / p;
  for (int k = n - 2; k > 1; --k)
    d[k] *= (d[k + 1] - u[k] * (x[k + 1] - x[k - 1]) / (x[k + 1] - x[k]));
  d[n] = (d[n - 1] - (1.0 - sig) * d[n - 2]) / sig;
  sig = 1.0 - ((x[2] - x[1]) / (x[2] - x[0]));
  d[1] *= (d[2] - u[1] / (1.0 - sig));
  d[0] = (d[1] - sig * d[2]) / (1.0 - sig);
  free(u);
}

/* Retrieve, ProxyPhysicsVector.cu:89-128; SetSpline(true), ProxyPhysicsTable.cu:75 */
static int retrieve_vector(FILE *f, gxo_pvec_t *v)
{
  int type, siz;
  if (fscanf(f, "%d", &type) != 1) return 0;
  if (fscanf(f, "%lf %lf %d", &v->emin, &v->emax, &v->n) != 3) return 0;
  if (fscanf(f, "%d", &siz) != 1 || siz <= 0) return 0;
  v->type = type;
  v->n = siz;
  v->x = (double *)malloc(sizeof(double) * siz);
  v->y = (double *)malloc(sizeof(double) * siz);
  v->d2 = (double *)calloc(siz, sizeof(double));
  for (int i = 0; i < siz; ++i)
    if (fscanf(f, "%lf %lf", &v->x[i], &v->y[i]) != 2) return 0;
  v->emin = v->x[0];
  v->emax = v->x[siz - 1];
  v->dbin = log(v->x[1] / v->emin);
  v->base = log(v->emin) / v->dbin;
  fill_second_derivatives(v);
  return 1;
}

/* FindBinLocation, ProxyPhysicsVector.cu:388-394 */
static int find_bin(const gxo_pvec_t *v, double e)
{
  int bin = (int)(gxo_log(e) / v->dbin - v->base);
  /* the reference reads outside the vector when the grid is not logarithmic
   * (InverseRange tables); the oracle keeps the bin inside it */
  if (bin > v->n - 2) bin = v->n - 2;
  if (bin > 0 && e < v->x[bin]) --bin;
  if (bin < 0) bin = 0;
  return bin;
}

/* SplineInterpolation, ProxyPhysicsVector.cu:396-429 */
static double spline(const gxo_pvec_t *v, double e, int b)
{
  double x1 = v->x[b], x2 = v->x[b + 1];
  double delta = x2 - x1;
  double a = (x2 - e) / delta;
  double bb = (e - x1) / delta;
  double y1 = v->y[b], y2 = v->y[b + 1];
  return a * y1 + bb * y2 +
         ((a * a * a - a) * v->d2[b] + (bb * bb * bb - bb) * v->d2[b + 1]) * delta * delta / 6.0;
}

/* Value, ProxyPhysicsVector.cu:469-483 */
double gxo_pvec_value(const gxo_pvec_t *v, double e)
{
  if (e <= v->emin) return v->y[0];
  if (e >= v->emax) return v->y[v->n - 1];
  return spline(v, e, find_bin(v, e));
}

/* InvRangeValue + InvRangeFindBinLocation, ProxyPhysicsVector.cu:491-524 */
double gxo_pvec_invrange_value(const gxo_pvec_t *v, double e)
{
  if (e <= v->emin) return v->y[0];
  if (e >= v->emax) return v->y[v->n - 1];
  int n1 = 0, n2 = v->n / 2, n3 = v->n - 1;
  while (n1 != n3 - 1) {
    if (e > v->x[n2])
      n1 = n2;
    else
      n3 = n2;
    n2 = n1 + (n3 - n1 + 1) / 2;
  }
  return spline(v, e, n1);
}

double gxo_table_value(const gxo_data_t *d, int table, int mat, double e)
{
  return gxo_pvec_value(&d->vec[table][mat], e);
}

double gxo_table_invrange(const gxo_data_t *d, int table, int mat, double r)
{
  return gxo_pvec_invrange_value(&d->vec[table][mat], r);
}

void gxo_table_value_batch(const gxo_data_t *d, int table, int mat, int n, const double *e, double *out)
{
  for (int i = 0; i < n; ++i) out[i] = gxo_table_value(d, table, mat, e[i]);
}

void gxo_table_invrange_batch(const gxo_data_t *d, int table, int mat, int n, const double *r, double *out)
{
  for (int i = 0; i < n; ++i) out[i] = gxo_table_invrange(d, table, mat, r[i]);
}

/* Proxy2DVector::FindBinLocationX/Y, Proxy2DVector.cpp:93-139 */
static size_t find_bin_2d(const double *v, size_t nn, double z)
{
  if (z < v[1]) return 0;
  if (z >= v[nn - 2]) return nn - 2;
  size_t lo = 0, hi = nn - 2;
  while (lo <= hi) {
    size_t mid = (lo + hi) / 2;
    if (z < v[mid])
      hi = mid - 1;
    else
      lo = mid + 1;
  }
  return hi;
}

/* Proxy2DVector::Value, Proxy2DVector.cpp:37-67 */
double gxo_sb_value(const gxo_sb_t *t, double x, double y)
{
  if (x < t->x[0])
    x = t->x[0];
  else if (x > t->x[31])
    x = t->x[31];
  if (y < t->y[0])
    y = t->y[0];
  else if (y > t->y[56])
    y = t->y[56];
  size_t ix = find_bin_2d(t->x, 32, x);
  size_t iy = find_bin_2d(t->y, 57, y);
  double x1 = t->x[ix], x2 = t->x[ix + 1], y1 = t->y[iy], y2 = t->y[iy + 1];
  double v11 = t->v[iy][ix], v12 = t->v[iy][ix + 1], v21 = t->v[iy + 1][ix], v22 = t->v[iy + 1][ix + 1];
  return ((y2 - y) * (v11 * (x2 - x) + v12 * (x - x1)) + ((y - y1) * (v21 * (x2 - x) + v22 * (x - x1)))) /
         ((x2 - x1) * (y2 - y1));
}

/* RetrieveSeltzerBergerData, ProxySeltzerBerger.hpp:487-526 */
static int load_sb(const char *dir, int Z, gxo_sb_t *t)
{
  char fn[1024];
  snprintf(fn, sizeof(fn), "%s/brem_SB/br%d", dir, Z);
  FILE *f = fopen(fn, "r");
  if (!f) return 0;
  int k, nx, ny, ok = 1;
  if (fscanf(f, "%d %d %d", &k, &nx, &ny) != 3) ok = 0;
  for (int i = 0; ok && i < 32; ++i) ok = fscanf(f, "%lf", &t->x[i]) == 1;
  for (int j = 0; ok && j < 57; ++j) ok = fscanf(f, "%lf", &t->y[j]) == 1;
  for (int j = 0; ok && j < 57; ++j)
    for (int i = 0; ok && i < 32; ++i) ok = fscanf(f, "%lf", &t->v[j][i]) == 1;
  fclose(f);
  return ok;
}

/* RetrieveCutsTable, ProxyDataManager.cu:83-122: the file holds, per particle,
 * (length mm, energy keV) for each material; the reference stores the energies
 * sequentially in file order. */
static int load_cuts(const char *dir, gxo_data_t *d)
{
  char fn[1024], version[64];
  snprintf(fn, sizeof(fn), "%s/table/cut.dat", dir);
  FILE *f = fopen(fn, "r");
  if (!f) return 0;
  int nmat;
  if (fscanf(f, "%63s %d", version, &nmat) != 2 || nmat != GXO_NMAT) {
    fclose(f);
    return 0;
  }
  for (int i = 0; i < 12; ++i) {
    double len, en;
    if (fscanf(f, "%lf %lf", &len, &en) != 2) {
      fclose(f);
      return 0;
    }
    d->cut_raw[i] = en;
    int ipart = i / GXO_NMAT, mat = i % GXO_NMAT;
    d->cut_energy[ipart][mat] = en * 1.0e-3; /* keV -> MeV */
    d->cut_length[ipart][mat] = len;
  }
  fclose(f);
  return 1;
}

/* ProxyDataManager::GetCutValue(index, ipart), ProxyDataManager.cuh:52-54: reads
 * entry 4*ipart + index of the sequential array (stride 4 over a 3-material file). */
double gxo_get_cut_value(const gxo_data_t *d, int index, int ipart)
{
  int k = 4 * ipart + index;
  return (k >= 0 && k < 12) ? d->cut_raw[k] : 0.0;
}

static int load_sandia(const char *dir, gxo_data_t *d)
{
  char fn[1024], line[512];
  snprintf(fn, sizeof(fn), "%s/sandia.dat", dir);
  FILE *f = fopen(fn, "r");
  if (!f) return 0;
  int ok = 1, n;
  /* skip comment lines */
  long pos;
  do {
    pos = ftell(f);
    if (!fgets(line, sizeof(line), f)) {
      fclose(f);
      return 0;
    }
  } while (line[0] == '#');
  fseek(f, pos, SEEK_SET);
  ok = fscanf(f, " SHELLS %d", &n) == 1 && n == 101;
  for (int i = 0; ok && i < 101; ++i) ok = fscanf(f, "%d", &d->nshell[i]) == 1;
  for (int i = 0; ok && i < 101; ++i) ok = fscanf(f, "%d", &d->ishell[i]) == 1;
  ok = ok && fscanf(f, " BINDING %d", &n) == 1 && n == 1540;
  for (int i = 0; ok && i < 1540; ++i) ok = fscanf(f, "%lf", &d->binding[i]) == 1;
  ok = ok && fscanf(f, " INTERVALS %d", &n) == 1 && n == 101;
  for (int i = 0; ok && i < 101; ++i) ok = fscanf(f, "%d", &d->nint[i]) == 1;
  ok = ok && fscanf(f, " SANDIA %d", &n) == 1 && n == 981;
  for (int i = 0; ok && i < 981; ++i)
    for (int j = 0; ok && j < 5; ++j) ok = fscanf(f, "%lf", &d->sandia[i][j]) == 1;
  fclose(f);
  d->cumint[0] = 1;
  for (int z = 1; z < 101; ++z) d->cumint[z] = d->cumint[z - 1] + d->nint[z - 1];
  return ok;
}

gxo_data_t *gxo_data_load(const char *dir)
{
  gxo_data_t *d = (gxo_data_t *)calloc(1, sizeof(gxo_data_t));
  char fn[1024];
  for (int t = 0; t < GXO_NTABLES; ++t) {
    snprintf(fn, sizeof(fn), "%s/table/%s", dir, kTableName[t]);
    FILE *f = fopen(fn, "r");
    if (!f) goto fail;
    int nv = 0;
    if (fscanf(f, "%d", &nv) != 1 || nv != GXO_NMAT) {
      fclose(f);
      goto fail;
    }
    for (int m = 0; m < GXO_NMAT; ++m)
      if (!retrieve_vector(f, &d->vec[t][m])) {
        fclose(f);
        goto fail;
      }
    fclose(f);
  }
  if (!load_cuts(dir, d)) goto fail;
  if (!load_sb(dir, 11, &d->sb_slot10) || !load_sb(dir, 18, &d->sb_ar) || !load_sb(dir, 82, &d->sb_pb))
    goto fail;
  if (!load_sandia(dir, d)) goto fail;
  return d;
fail:
  gxo_data_free(d);
  return NULL;
}

void gxo_data_free(gxo_data_t *d)
{
  if (!d) return;
  for (int t = 0; t < GXO_NTABLES; ++t)
    for (int m = 0; m < GXO_NMAT; ++m) {
      free(d->vec[t][m].x);
      free(d->vec[t][m].y);
      free(d->vec[t][m].d2);
    }
  free(d);
}
