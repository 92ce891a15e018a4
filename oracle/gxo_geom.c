/* gxo_geom.c -- CSG geometry and navigation for the oracle's step loop
 * (transport config geometry = 2).  Test infrastructure: the library's device
 * navigator is tested against it; never part of the product.
 *
 * The reference navigates a VecGeom volume tree (NavigationInterface::
 * FindNextBoundary, source/Geant/geometry/NavigationInterface.hpp:63-98, calls
 * VNavigator::FindNextBoundaryAndStepAndSafety; IsSameLocation :43-60
 * relocates), built from unplaced boxes, logical volumes and placed daughters
 * (source/Geant/proxy/test/BasicCpuTransport/ProxyDetectorConstruction.cpp:
 * 241-324).  VecGeom itself is an un-vendored submodule, absent here, so this
 * is a restatement of the published ray/solid algorithms, not of its code
 * (parity with VecGeom is unpinned; the CSG calorimeter is pinned to the
 * analytic layered navigator instead):
 *   - the tree is flattened into touchables (one per placed instance), each
 *     with its global transform x_global = R x_local + t, a padded global
 *     bounding box and its children;
 *   - the step: distance to leave the current solid, and to enter each child
 *     whose bounding box the ray meets closer than that;
 *   - after a crossing: into the child that was hit, then down into the child
 *     containing the point; or up through the parents until one contains it,
 *     then down;
 *   - "contains" on a surface (within a tolerance) is decided by the
 *     direction: a point on a face it moves out through is outside;
 *   - safety: to the current solid's surface and to each child (the larger of
 *     the distance to its bounding box and the solid's own lower bound).
 * Solids: box (half lengths), tube (rmin, rmax, half length in z; full phi or
 * a phi segment [s, s + dphi] between two half-planes),
 * sphere (rmin, rmax), convex polyhedron (intersection of half-spaces
 * n.x <= d; the ray clipped against each plane).  Quadratic roots are taken in
 * the cancellation-free form (near root c / (-b + sqrt(D)), far root
 * -c / (b + sqrt(D))). */
#include "gxo.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CSG_INF 1.7976931348623157e308
#define CSG_MAXDEPTH 64
#define CSG_MAXNODES (1 << 22)
#define CSG_PAD 1e-6 /* bounding boxes are padded by this (mm) */

static double dmin(double a, double b) { return a < b ? a : b; }
static double dmax(double a, double b) { return a > b ? a : b; }

/* ------------------------------------------------------------- building */
typedef struct {
  int nsolid, nlv, npv;
  const int *skind;
  const double *spar;
  const int *splane_off;
  double *slo, *shi; /* local bounding box per solid */
  int *smode;        /* tubes: phi segment mode (0 full) */
  const int *lv_solid, *lv_mat, *lv_scored;
  const int *pv_mother, *pv_lv;
  const double *pv_t, *pv_r;
  gxo_csg_t *g;
  int kcur, scur, err;
} build_t;

/* The bounding box of the convex polyhedron {x : n_k . x <= d_k} (unit
 * normals): the extent of the points where three planes meet inside all the
 * others.  0 when the planes bound no finite volume (no such point, or an
 * edge direction +-(n_i x n_j) that no plane closes). */
static int poly_bbox(const double *pl, int np, double lo[3], double hi[3])
{
  int nv = 0;
  for (int k = 0; k < 3; ++k) {
    lo[k] = CSG_INF;
    hi[k] = -CSG_INF;
  }
  for (int i = 0; i < np; ++i)
    for (int j = i + 1; j < np; ++j)
      for (int k = j + 1; k < np; ++k) {
        const double *a = pl + 4 * i, *b = pl + 4 * j, *c = pl + 4 * k;
        double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
        double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
        double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
        if (fabs(det) < 1e-12) continue;
        double x[3];
        for (int m = 0; m < 3; ++m) x[m] = (a[3] * bc[m] + b[3] * ca[m] + c[3] * ab[m]) / det;
        int in = 1;
        for (int l = 0; l < np && in; ++l) {
          const double *p = pl + 4 * l;
          in = p[0] * x[0] + p[1] * x[1] + p[2] * x[2] - p[3] <= 1e-9 * (1.0 + fabs(p[3]));
        }
        if (!in) continue;
        ++nv;
        for (int m = 0; m < 3; ++m) {
          lo[m] = dmin(lo[m], x[m]);
          hi[m] = dmax(hi[m], x[m]);
        }
      }
  if (nv == 0) return 0;
  for (int i = 0; i < np; ++i)
    for (int j = i + 1; j < np; ++j) {
      const double *a = pl + 4 * i, *b = pl + 4 * j;
      double v[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
      double len = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      if (len < 1e-12) continue;
      for (int sgn = -1; sgn <= 1; sgn += 2) {
        int open = 1;
        for (int l = 0; l < np && open; ++l) {
          const double *p = pl + 4 * l;
          open = sgn * (p[0] * v[0] + p[1] * v[1] + p[2] * v[2]) <= 1e-12 * len;
        }
        if (open) return 0;
      }
    }
  return 1;
}

static int visit(build_t *b, int lv, int parent, const double R[9], const double t[3], int depth)
{
  gxo_csg_t *g = b->g;
  if (depth > CSG_MAXDEPTH || g->n >= CSG_MAXNODES) {
    b->err = 1;
    return -1;
  }
  const int id = g->n++;
  gxo_csg_node_t *n = &g->node[id];
  const int s = b->lv_solid[lv];
  n->kind = b->skind[s];
  n->a = b->spar[3 * s];
  n->b = b->spar[3 * s + 1];
  n->c = b->spar[3 * s + 2];
  n->p0 = b->splane_off ? b->splane_off[s] : 0;
  n->np = (n->kind == GXO_CSG_POLY) ? b->splane_off[s + 1] - b->splane_off[s] : 0;
  if (n->kind == GXO_CSG_TUBE && b->splane_off && b->splane_off[s + 1] > b->splane_off[s])
    n->np = b->smode[s]; /* a phi segment: 1 (dphi <= pi) or 2 */
  memcpy(n->t, t, sizeof(n->t));
  memcpy(n->r, R, sizeof(n->r));
  n->rot = !(R[0] == 1.0 && R[1] == 0.0 && R[2] == 0.0 && R[3] == 0.0 && R[4] == 1.0 && R[5] == 0.0 &&
             R[6] == 0.0 && R[7] == 0.0 && R[8] == 1.0);
  n->mat = b->lv_mat[lv];
  n->parent = parent;
  n->lv = lv;
  n->score = b->lv_scored[lv] ? g->nscore++ : -1;
  /* global bounding box: the local one's eight corners */
  const double *slo = b->slo + 3 * s, *shi = b->shi + 3 * s;
  for (int k = 0; k < 3; ++k) {
    n->lo[k] = CSG_INF;
    n->hi[k] = -CSG_INF;
  }
  for (int corner = 0; corner < 8; ++corner) {
    double x[3] = {(corner & 1) ? shi[0] : slo[0], (corner & 2) ? shi[1] : slo[1], (corner & 4) ? shi[2] : slo[2]};
    for (int k = 0; k < 3; ++k) {
      double y = R[3 * k] * x[0] + R[3 * k + 1] * x[1] + R[3 * k + 2] * x[2] + t[k];
      n->lo[k] = dmin(n->lo[k], y);
      n->hi[k] = dmax(n->hi[k], y);
    }
  }
  for (int k = 0; k < 3; ++k) {
    n->lo[k] -= CSG_PAD;
    n->hi[k] += CSG_PAD;
  }
  /* children: a contiguous block of the kids array, reserved before recursing */
  int nk = 0;
  for (int p = 0; p < b->npv; ++p)
    if (b->pv_mother[p] == lv) ++nk;
  n->nkid = nk;
  n->kid0 = b->kcur;
  b->kcur += nk;
  int j = 0;
  for (int p = 0; p < b->npv && !b->err; ++p) {
    if (b->pv_mother[p] != lv) continue;
    const double *Rp = b->pv_r + 9 * p, *tp = b->pv_t + 3 * p;
    double Rc[9], tc[3];
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c)
        Rc[3 * r + c] = R[3 * r] * Rp[c] + R[3 * r + 1] * Rp[3 + c] + R[3 * r + 2] * Rp[6 + c];
      tc[r] = R[3 * r] * tp[0] + R[3 * r + 1] * tp[1] + R[3 * r + 2] * tp[2] + t[r];
    }
    int kid = visit(b, b->pv_lv[p], id, Rc, tc, depth + 1);
    g->kids[g->node[id].kid0 + j++] = kid;
  }
  return id;
}

/* count the touchables below lv (for the allocation); -1 when too many */
static long count_nodes(const build_t *b, int lv, int depth)
{
  if (depth > CSG_MAXDEPTH) return -1;
  long n = 1;
  for (int p = 0; p < b->npv; ++p)
    if (b->pv_mother[p] == lv) {
      long k = count_nodes(b, b->pv_lv[p], depth + 1);
      if (k < 0) return -1;
      n += k;
      if (n > CSG_MAXNODES) return -1;
    }
  return n;
}

gxo_csg_t *gxo_csg_build(int nsolid, const int *skind, const double *spar, const int *splane_off,
                         const double *splanes, int nlv, const int *lv_solid, const int *lv_mat, const int *lv_scored,
                         int npv, const int *pv_mother, const int *pv_lv, const double *pv_t, const double *pv_r,
                         int world)
{
  if (world < 0 || world >= nlv) return NULL;
  build_t b = {nsolid, nlv, npv, skind, spar, splane_off, NULL, NULL, NULL, lv_solid, lv_mat, lv_scored, pv_mother,
               pv_lv, pv_t, pv_r, NULL, 0, 0, 0};
  long total = count_nodes(&b, world, 0);
  if (total < 0) return NULL;
  gxo_csg_t *g = (gxo_csg_t *)calloc(1, sizeof(gxo_csg_t));
  /* solids' local bounding boxes; polyhedra's planes normalised */
  int nplanes = splane_off ? splane_off[nsolid] : 0;
  g->planes = (double *)calloc((size_t)(4 * nplanes + 4), sizeof(double));
  b.slo = (double *)calloc((size_t)(3 * nsolid + 3), sizeof(double));
  b.shi = (double *)calloc((size_t)(3 * nsolid + 3), sizeof(double));
  b.smode = (int *)calloc((size_t)(nsolid + 1), sizeof(int));
  int bad = 0;
  for (int s = 0; s < nsolid && !bad; ++s) {
    const double *p = spar + 3 * s;
    double *lo = b.slo + 3 * s, *hi = b.shi + 3 * s;
    if (skind[s] == GXO_CSG_POLY) {
      int p0 = splane_off[s], np = splane_off[s + 1] - p0;
      for (int k = p0; k < p0 + np; ++k) {
        const double *q = splanes + 4 * k;
        double len = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
        for (int m = 0; m < 4; ++m) g->planes[4 * k + m] = q[m] / len;
      }
      bad = np < 4 || !poly_bbox(g->planes + 4 * p0, np, lo, hi);
      continue;
    }
    if (skind[s] == GXO_CSG_TUBE && splane_off && splane_off[s + 1] > splane_off[s]) {
      /* a phi segment: the row holds (sphi, dphi); stored as the half-planes'
       * directions (cos s, sin s, cos e, sin e), e = sphi + dphi */
      const double *row = splanes + 4 * splane_off[s];
      double sphi = row[0], dphi = row[1], e = sphi + dphi;
      double *w = g->planes + 4 * splane_off[s];
      w[0] = cos(sphi);
      w[1] = sin(sphi);
      w[2] = cos(e);
      w[3] = sin(e);
      b.smode[s] = dphi <= 3.14159265358979323846 ? 1 : 2;
      bad = !(dphi > 0.0 && dphi < 2.0 * 3.14159265358979323846);
    }
    double h[3] = {p[0], p[1], p[2]};
    if (skind[s] == GXO_CSG_TUBE) h[0] = p[1];
    if (skind[s] == GXO_CSG_SPHERE) h[0] = h[2] = p[1];
    for (int k = 0; k < 3; ++k) {
      lo[k] = -h[k];
      hi[k] = h[k];
    }
  }
  g->node = (gxo_csg_node_t *)calloc((size_t)total, sizeof(gxo_csg_node_t));
  g->kids = (int *)calloc((size_t)total, sizeof(int));
  b.g = g;
  const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, z[3] = {0, 0, 0};
  if (!bad) visit(&b, world, -1, I, z, 0);
  free(b.slo);
  free(b.shi);
  free(b.smode);
  if (b.err || bad) {
    gxo_csg_free(g);
    return NULL;
  }
  return g;
}

void gxo_csg_free(gxo_csg_t *g)
{
  if (!g) return;
  free(g->node);
  free(g->kids);
  free(g->planes);
  free(g);
}

/* ---------------------------------------------------------------- solids */
static void to_local(const gxo_csg_node_t *n, const double *p, const double *d, double *q, double *e)
{
  double x[3] = {p[0] - n->t[0], p[1] - n->t[1], p[2] - n->t[2]};
  if (!n->rot) {
    for (int k = 0; k < 3; ++k) {
      q[k] = x[k];
      e[k] = d[k];
    }
    return;
  }
  for (int k = 0; k < 3; ++k) { /* R^T */
    q[k] = n->r[k] * x[0] + n->r[3 + k] * x[1] + n->r[6 + k] * x[2];
    e[k] = n->r[k] * d[0] + n->r[3 + k] * d[1] + n->r[6 + k] * d[2];
  }
}

/* inside, or on the surface and not moving out through it */
/* The phi segment of a tube: (cos s, sin s, cos e, sin e) at plane-table row
 * p0, np = 1 for dphi <= pi (the intersection of n1.q <= 0, n1 = (sin s,
 * -cos s), and n2.q <= 0, n2 = (-sin e, cos e)), 2 for dphi > pi (their union). */
typedef struct { double cs, ss, ce, se; int mode; } wedge_t;
static wedge_t wedge_of(const gxo_csg_node_t *n, const double *pl)
{
  const double *w = pl + 4 * n->p0;
  wedge_t x = {w[0], w[1], w[2], w[3], n->np};
  return x;
}
static double wh1(const wedge_t *w, double x, double y) { return w->ss * x - w->cs * y; }
static double wh2(const wedge_t *w, double x, double y) { return w->ce * y - w->se * x; }
static int win(double h, double ne, double tol) { return h < -tol || (h <= tol && ne <= 0.0); }
static int wedge_contains(const wedge_t *w, const double *q, const double *e, double tol)
{
  int a = win(wh1(w, q[0], q[1]), wh1(w, e[0], e[1]), tol), b = win(wh2(w, q[0], q[1]), wh2(w, e[0], e[1]), tol);
  return w->mode == 1 ? (a && b) : (a || b);
}
static int wedge_holds(const wedge_t *w, double x, double y, double tol)
{
  int a = wh1(w, x, y) <= tol, b = wh2(w, x, y) <= tol;
  return w->mode == 1 ? (a && b) : (a || b);
}
/* distance to leave the wedge from inside: the first plane left (dphi <= pi);
 * for the union, the end of the stretch of the ray inside either half-space */
static double wedge_out(const wedge_t *w, const double *q, const double *e, double tol)
{
  double a = wh1(w, q[0], q[1]), na = wh1(w, e[0], e[1]), b = wh2(w, q[0], q[1]), nb = wh2(w, e[0], e[1]);
  double ta = na > 0.0 ? -a / na : CSG_INF, tb = nb > 0.0 ? -b / nb : CSG_INF;
  if (w->mode == 1) return dmin(ta, tb);
  int ia = win(a, na, tol), ib = win(b, nb, tol);
  if (ia && ib) return dmax(ta, tb);
  if (ia) return (nb < 0.0 && -b / nb <= ta) ? CSG_INF : ta;
  if (ib) return (na < 0.0 && -a / na <= tb) ? CSG_INF : tb;
  return 0.0;
}
static double wedge_safety_out(const wedge_t *w, const double *q)
{
  double a = -wh1(w, q[0], q[1]), b = -wh2(w, q[0], q[1]);
  return w->mode == 1 ? dmin(a, b) : dmax(a, b);
}
static double wedge_safety_in(const wedge_t *w, const double *q)
{
  double a = wh1(w, q[0], q[1]), b = wh2(w, q[0], q[1]);
  return w->mode == 1 ? dmax(a, b) : dmin(a, b);
}

/* n.q - d and n.e of plane k */
static void plane_at(const double *pl, int k, const double *q, const double *e, double *h, double *ne)
{
  const double *p = pl + 4 * k;
  *h = p[0] * q[0] + p[1] * q[1] + p[2] * q[2] - p[3];
  *ne = p[0] * e[0] + p[1] * e[1] + p[2] * e[2];
}

static int contains_local(const gxo_csg_node_t *n, const double *q, const double *e, double tol, const double *pl)
{
  if (n->kind == GXO_CSG_POLY) {
    for (int k = n->p0; k < n->p0 + n->np; ++k) {
      double h, ne;
      plane_at(pl, k, q, e, &h, &ne);
      if (h > tol || (h >= -tol && ne > 0.0)) return 0;
    }
    return 1;
  }
  if (n->kind == GXO_CSG_BOX) {
    const double h[3] = {n->a, n->b, n->c};
    for (int k = 0; k < 3; ++k) {
      double a = fabs(q[k]);
      if (a > h[k] + tol) return 0;
      if (a >= h[k] - tol && q[k] * e[k] > 0.0) return 0;
    }
    return 1;
  }
  if (n->kind == GXO_CSG_TUBE) {
    double a = fabs(q[2]);
    if (a > n->c + tol) return 0;
    if (a >= n->c - tol && q[2] * e[2] > 0.0) return 0;
    if (n->np) {
      wedge_t w = wedge_of(n, pl);
      if (!wedge_contains(&w, q, e, tol)) return 0;
    }
    double r = sqrt(q[0] * q[0] + q[1] * q[1]), out = q[0] * e[0] + q[1] * e[1];
    if (r > n->b + tol) return 0;
    if (r >= n->b - tol && out > 0.0) return 0;
    if (n->a > 0.0) {
      if (r < n->a - tol) return 0;
      if (r <= n->a + tol && out < 0.0) return 0;
    }
    return 1;
  }
  double r = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]), out = q[0] * e[0] + q[1] * e[1] + q[2] * e[2];
  if (r > n->b + tol) return 0;
  if (r >= n->b - tol && out > 0.0) return 0;
  if (n->a > 0.0) {
    if (r < n->a - tol) return 0;
    if (r <= n->a + tol && out < 0.0) return 0;
  }
  return 1;
}

/* far root of a t^2 + 2 b t + c = 0 (D = b^2 - a c >= 0) */
static double far_root(double a, double b, double c, double sq) { return b > 0.0 ? -c / (b + sq) : (sq - b) / a; }
/* near root */
static double near_root(double a, double b, double c, double sq) { return b < 0.0 ? c / (sq - b) : -(b + sq) / a; }

/* distance to leave the solid from a point inside (or on its surface) */
static double dist_out_local(const gxo_csg_node_t *n, const double *q, const double *e, const double *pl)
{
  double s = CSG_INF;
  if (n->kind == GXO_CSG_POLY) {
    for (int k = n->p0; k < n->p0 + n->np; ++k) {
      double h, ne;
      plane_at(pl, k, q, e, &h, &ne);
      if (ne > 0.0) s = dmin(s, -h / ne);
    }
    return s < 0.0 ? 0.0 : s;
  }
  if (n->kind == GXO_CSG_BOX) {
    const double h[3] = {n->a, n->b, n->c};
    for (int k = 0; k < 3; ++k) {
      double t = CSG_INF;
      if (e[k] > 0.0)
        t = (h[k] - q[k]) / e[k];
      else if (e[k] < 0.0)
        t = (-h[k] - q[k]) / e[k];
      s = dmin(s, t);
    }
    return s < 0.0 ? 0.0 : s;
  }
  if (n->kind == GXO_CSG_TUBE) {
    if (e[2] > 0.0)
      s = (n->c - q[2]) / e[2];
    else if (e[2] < 0.0)
      s = (-n->c - q[2]) / e[2];
    double a = e[0] * e[0] + e[1] * e[1];
    if (a > 0.0) {
      double b = q[0] * e[0] + q[1] * e[1], r2 = q[0] * q[0] + q[1] * q[1];
      double c = r2 - n->b * n->b, D = b * b - a * c;
      s = dmin(s, far_root(a, b, c, sqrt(D > 0.0 ? D : 0.0)));
      if (n->a > 0.0 && b < 0.0) {
        double c2 = r2 - n->a * n->a, D2 = b * b - a * c2;
        if (D2 >= 0.0) s = dmin(s, near_root(a, b, c2, sqrt(D2)));
      }
    }
    if (n->np) {
      wedge_t w = wedge_of(n, pl);
      s = dmin(s, wedge_out(&w, q, e, GXO_CSG_TOL));
    }
    return s < 0.0 ? 0.0 : s;
  }
  double a = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
  double b = q[0] * e[0] + q[1] * e[1] + q[2] * e[2], r2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
  double c = r2 - n->b * n->b, D = b * b - a * c;
  s = far_root(a, b, c, sqrt(D > 0.0 ? D : 0.0));
  if (n->a > 0.0 && b < 0.0) {
    double c2 = r2 - n->a * n->a, D2 = b * b - a * c2;
    if (D2 >= 0.0) s = dmin(s, near_root(a, b, c2, sqrt(D2)));
  }
  return s < 0.0 ? 0.0 : s;
}

/* distance to enter the solid from a point outside it; CSG_INF if missed */
static double dist_in_local(const gxo_csg_node_t *n, const double *q, const double *e, double tol,
                            const double *pl)
{
  if (n->kind == GXO_CSG_POLY) { /* the ray clipped against every plane */
    double tmin = -CSG_INF, tmax = CSG_INF;
    for (int k = n->p0; k < n->p0 + n->np; ++k) {
      double h, ne;
      plane_at(pl, k, q, e, &h, &ne);
      if (ne == 0.0) {
        if (h > 0.0) return CSG_INF;
        continue;
      }
      double t = -h / ne;
      if (ne < 0.0)
        tmin = dmax(tmin, t);
      else
        tmax = dmin(tmax, t);
    }
    if (!(tmax > tmin) || tmax <= tol) return CSG_INF;
    return tmin < 0.0 ? 0.0 : tmin;
  }
  if (n->kind == GXO_CSG_BOX) {
    const double h[3] = {n->a, n->b, n->c};
    double tmin = -CSG_INF, tmax = CSG_INF;
    for (int k = 0; k < 3; ++k) {
      if (e[k] == 0.0) {
        if (fabs(q[k]) > h[k]) return CSG_INF;
        continue;
      }
      double t0 = (-h[k] - q[k]) / e[k], t1 = (h[k] - q[k]) / e[k];
      if (t0 > t1) {
        double x = t0;
        t0 = t1;
        t1 = x;
      }
      tmin = dmax(tmin, t0);
      tmax = dmin(tmax, t1);
    }
    if (!(tmax > tmin) || tmax <= tol) return CSG_INF;
    return tmin < 0.0 ? 0.0 : tmin;
  }
  double s = CSG_INF;
  if (n->kind == GXO_CSG_TUBE) {
    const double rmin = n->a, rmax = n->b, dz = n->c;
    const int seg = n->np != 0;
    wedge_t w = {0, 0, 0, 0, 0};
    if (seg) w = wedge_of(n, pl);
#define IN_PHI(t) (!seg || wedge_holds(&w, q[0] + (t) * e[0], q[1] + (t) * e[1], tol))
    /* the end planes */
    double tz = -1.0;
    if (q[2] >= dz && e[2] < 0.0)
      tz = (dz - q[2]) / e[2];
    else if (q[2] <= -dz && e[2] > 0.0)
      tz = (-dz - q[2]) / e[2];
    if (tz >= 0.0) {
      double x = q[0] + tz * e[0], y = q[1] + tz * e[1], r = sqrt(x * x + y * y);
      if (r <= rmax + tol && (rmin <= 0.0 || r >= rmin - tol) && IN_PHI(tz)) s = tz;
    }
    double a = e[0] * e[0] + e[1] * e[1];
    if (a > 0.0) {
      double b = q[0] * e[0] + q[1] * e[1], r2 = q[0] * q[0] + q[1] * q[1];
      double c = r2 - rmax * rmax, D = b * b - a * c;
      if (c >= 0.0 && b < 0.0 && D >= 0.0) { /* the outer surface from outside */
        double t = near_root(a, b, c, sqrt(D));
        if (t < s && fabs(q[2] + t * e[2]) <= dz + tol && IN_PHI(t)) s = t;
      }
      if (rmin > 0.0) { /* the inner surface from the bore */
        double c2 = r2 - rmin * rmin, D2 = b * b - a * c2;
        if (D2 >= 0.0) {
          double t = far_root(a, b, c2, sqrt(D2));
          if (t >= 0.0 && t < s && fabs(q[2] + t * e[2]) <= dz + tol && IN_PHI(t)) s = t;
        }
      }
    }
#undef IN_PHI
    if (seg) { /* the two half-planes, entered from their outer side */
      for (int k = 0; k < 2; ++k) {
        double h = k == 0 ? wh1(&w, q[0], q[1]) : wh2(&w, q[0], q[1]);
        double ne = k == 0 ? wh1(&w, e[0], e[1]) : wh2(&w, e[0], e[1]);
        if (!(ne < 0.0) || h < -tol) continue;
        double t = dmax(-h / ne, 0.0);
        if (!(t < s)) continue;
        double x = q[0] + t * e[0], y = q[1] + t * e[1];
        double along = k == 0 ? w.cs * x + w.ss * y : w.ce * x + w.se * y;
        double r = sqrt(x * x + y * y);
        if (along >= -tol && r <= rmax + tol && (rmin <= 0.0 || r >= rmin - tol) && fabs(q[2] + t * e[2]) <= dz + tol)
          s = t;
      }
    }
    return s;
  }
  const double rmin = n->a, rmax = n->b;
  double a = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
  double b = q[0] * e[0] + q[1] * e[1] + q[2] * e[2], r2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
  double c = r2 - rmax * rmax, D = b * b - a * c;
  if (c >= 0.0 && b < 0.0 && D >= 0.0) s = near_root(a, b, c, sqrt(D));
  if (rmin > 0.0) {
    double c2 = r2 - rmin * rmin, D2 = b * b - a * c2;
    if (D2 >= 0.0) {
      double t = far_root(a, b, c2, sqrt(D2));
      if (t >= 0.0 && t < s) s = t;
    }
  }
  return s;
}

static double safety_out_local(const gxo_csg_node_t *n, const double *q, const double *pl)
{
  if (n->kind == GXO_CSG_POLY) {
    double s = CSG_INF;
    for (int k = n->p0; k < n->p0 + n->np; ++k) {
      const double *p = pl + 4 * k;
      s = dmin(s, -(p[0] * q[0] + p[1] * q[1] + p[2] * q[2] - p[3]));
    }
    return s;
  }
  if (n->kind == GXO_CSG_BOX)
    return dmin(dmin(n->a - fabs(q[0]), n->b - fabs(q[1])), n->c - fabs(q[2]));
  if (n->kind == GXO_CSG_TUBE) {
    double r = sqrt(q[0] * q[0] + q[1] * q[1]);
    double s = dmin(n->c - fabs(q[2]), n->b - r);
    if (n->a > 0.0) s = dmin(s, r - n->a);
    if (n->np) {
      wedge_t w = wedge_of(n, pl);
      s = dmin(s, wedge_safety_out(&w, q));
    }
    return s;
  }
  double r = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  return n->a > 0.0 ? dmin(n->b - r, r - n->a) : n->b - r;
}

/* a lower bound of the distance to the solid from a point outside it */
static double safety_in_local(const gxo_csg_node_t *n, const double *q, const double *pl)
{
  if (n->kind == GXO_CSG_POLY) {
    double s = -CSG_INF;
    for (int k = n->p0; k < n->p0 + n->np; ++k) {
      const double *p = pl + 4 * k;
      s = dmax(s, p[0] * q[0] + p[1] * q[1] + p[2] * q[2] - p[3]);
    }
    return s;
  }
  if (n->kind == GXO_CSG_BOX)
    return dmax(dmax(fabs(q[0]) - n->a, fabs(q[1]) - n->b), fabs(q[2]) - n->c);
  if (n->kind == GXO_CSG_TUBE) {
    double r = sqrt(q[0] * q[0] + q[1] * q[1]);
    double s = dmax(dmax(fabs(q[2]) - n->c, r - n->b), n->a - r);
    if (n->np) {
      wedge_t w = wedge_of(n, pl);
      s = dmax(s, wedge_safety_in(&w, q));
    }
    return s;
  }
  double r = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  return dmax(r - n->b, n->a - r);
}

/* ------------------------------------------------------------ navigation */
static double bbox_gap(const gxo_csg_node_t *n, const double *p)
{
  double g = -CSG_INF;
  for (int k = 0; k < 3; ++k) g = dmax(g, dmax(n->lo[k] - p[k], p[k] - n->hi[k]));
  return g;
}

/* entry distance of the ray into the bounding box, CSG_INF if missed */
static double bbox_ray(const gxo_csg_node_t *n, const double *p, const double *d)
{
  double tmin = 0.0, tmax = CSG_INF;
  for (int k = 0; k < 3; ++k) {
    if (d[k] == 0.0) {
      if (p[k] < n->lo[k] || p[k] > n->hi[k]) return CSG_INF;
      continue;
    }
    double t0 = (n->lo[k] - p[k]) / d[k], t1 = (n->hi[k] - p[k]) / d[k];
    if (t0 > t1) {
      double x = t0;
      t0 = t1;
      t1 = x;
    }
    tmin = dmax(tmin, t0);
    tmax = dmin(tmax, t1);
  }
  return tmax < tmin ? CSG_INF : tmin;
}

int gxo_csg_contains(const gxo_csg_t *g, int v, const double *p, const double *d, double tol)
{
  const gxo_csg_node_t *n = &g->node[v];
  if (bbox_gap(n, p) > 0.0) return 0;
  double q[3], e[3];
  to_local(n, p, d, q, e);
  return contains_local(n, q, e, tol, g->planes);
}

/* the deepest touchable at or below v (which contains p) containing p */
static int descend(const gxo_csg_t *g, int v, const double *p, const double *d, double tol)
{
  for (int depth = 0; depth < CSG_MAXDEPTH; ++depth) {
    const gxo_csg_node_t *n = &g->node[v];
    int next = -1;
    for (int k = 0; k < n->nkid && next < 0; ++k) {
      int c = g->kids[n->kid0 + k];
      if (gxo_csg_contains(g, c, p, d, tol)) next = c;
    }
    if (next < 0) return v;
    v = next;
  }
  return v;
}

int gxo_csg_locate(const gxo_csg_t *g, int v, const double *p, const double *d, double tol)
{
  if (v < 0) v = 0;
  for (int depth = 0; v >= 0 && depth <= CSG_MAXDEPTH; ++depth) {
    if (gxo_csg_contains(g, v, p, d, tol)) return descend(g, v, p, d, tol);
    v = g->node[v].parent;
  }
  return -1;
}

double gxo_csg_step(const gxo_csg_t *g, int v, const double *p, const double *d, double limit, int *hit)
{
  const gxo_csg_node_t *n = &g->node[v];
  double q[3], e[3];
  to_local(n, p, d, q, e);
  double s = dist_out_local(n, q, e, g->planes);
  *hit = -1;
  for (int k = 0; k < n->nkid; ++k) {
    int c = g->kids[n->kid0 + k];
    const gxo_csg_node_t *m = &g->node[c];
    double tb = bbox_ray(m, p, d);
    if (!(tb < s && tb < limit)) continue;
    to_local(m, p, d, q, e);
    double t = dist_in_local(m, q, e, GXO_CSG_TOL, g->planes);
    if (t < s) {
      s = t;
      *hit = c;
    }
  }
  return s;
}

double gxo_csg_safety(const gxo_csg_t *g, int v, const double *p)
{
  const gxo_csg_node_t *n = &g->node[v];
  double q[3], e[3];
  const double zero[3] = {0, 0, 0};
  to_local(n, p, zero, q, e);
  double s = safety_out_local(n, q, g->planes);
  for (int k = 0; k < n->nkid; ++k) {
    const gxo_csg_node_t *m = &g->node[g->kids[n->kid0 + k]];
    double gap = bbox_gap(m, p);
    if (gap >= s) continue;
    to_local(m, p, zero, q, e);
    s = dmin(s, dmax(gap, safety_in_local(m, q, g->planes)));
  }
  return s < 0.0 ? 0.0 : s;
}

int gxo_csg_cross(const gxo_csg_t *g, int v, int hit, const double *p, const double *d)
{
  if (hit >= 0) return descend(g, hit, p, d, GXO_CSG_TOL);
  return gxo_csg_locate(g, g->node[v].parent, p, d, GXO_CSG_TOL);
}

void gxo_csg_probe(const gxo_csg_t *g, int n, const double *pos, const double *dir, const double *limit, int *vol,
                   double *snext, int *next, double *safety)
{
  for (int i = 0; i < n; ++i) {
    const double *p = pos + 3 * i, *d = dir + 3 * i;
    int v = gxo_csg_locate(g, 0, p, d, GXO_CSG_TOL);
    vol[i] = v;
    if (v < 0) {
      snext[i] = -1.0;
      next[i] = -1;
      safety[i] = -1.0;
      continue;
    }
    int hit;
    double s = gxo_csg_step(g, v, p, d, limit[i], &hit);
    snext[i] = s;
    safety[i] = gxo_csg_safety(g, v, p);
    if (s < limit[i]) {
      double x[3] = {p[0] + s * d[0], p[1] + s * d[1], p[2] + s * d[2]};
      next[i] = gxo_csg_cross(g, v, hit, x, d);
    } else {
      next[i] = v;
    }
  }
}

int gxo_csg_node_count(const gxo_csg_t *g, int *nscore) { if (nscore) *nscore = g->nscore; return g->n; }
void gxo_csg_node_info(const gxo_csg_t *g, int i, int *info, double *tr)
{
  const gxo_csg_node_t *n = &g->node[i];
  info[0] = n->lv;
  info[1] = n->parent;
  info[2] = n->score;
  info[3] = n->mat;
  info[4] = n->nkid;
  memcpy(tr, n->t, 3 * sizeof(double));
  memcpy(tr + 3, n->r, 9 * sizeof(double));
}
