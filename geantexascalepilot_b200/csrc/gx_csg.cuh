// gx_csg.cuh -- CSG geometry on the device: a volume tree of placed solids,
// flattened into touchables (transport geometry 2).
//
// The reference's navigation is VecGeom's (NavigationInterface::
// FindNextBoundary, source/Geant/geometry/NavigationInterface.hpp:63-98:
// FindNextBoundaryAndStepAndSafety, then the snext / safety / boundary
// bookkeeping; IsSameLocation :43-60 relocates after a step), over a tree
// built from unplaced solids, logical volumes and placed daughters
// (source/Geant/proxy/test/BasicCpuTransport/ProxyDetectorConstruction.cpp:
// 241-324).  VecGeom is not part of the reference sources; this is a
// restatement of the standard ray/solid algorithms for the solids that
// calorimeters are built from:
//   - each touchable (one placed instance; the whole tree unrolled, as
//     VecGeom's navigation-state index does) carries its global transform
//     x_global = R x_local + t, its solid, material, parent and a contiguous
//     run of children; a track's volume is one int, like the layered
//     navigator's;
//   - step: the distance to leave the current solid, and to enter each child
//     whose padded bounding box the ray meets before that (and before the
//     physics step);
//   - after a crossing: into the child that was hit, then down into the child
//     containing the point; or up through the parents until one contains it,
//     then down;
//   - on a surface (within a tolerance) "contains" is decided by the
//     direction: a point on a face it moves out through is outside;
//   - safety: to the current solid's surface and, for each child, the larger
//     of the distance to its bounding box and the solid's own lower bound.
// Solids: box (half lengths), tube (rmin, rmax, half length; full phi or a
// phi segment), sphere (rmin, rmax), convex polyhedron (the intersection of half-spaces
// n.x <= d, unit outward normals: trapezoids such as VecGeom's UnplacedTrd,
// prisms, wedges).  Quadratic roots in the cancellation-free form; the
// polyhedron's ray distances by clipping the ray against each plane.
// A touchable with many children also carries a one-dimensional grid along
// the axis that separates its children best: equal slabs of its bounding box,
// each listing (in child order) the children whose bounding box overlaps it.
// Locating looks only at the point's slab; the step walks the slabs the ray
// crosses before the nearest boundary found so far; the safety looks at the
// slabs within the current safety.  Every child that can matter is in a slab
// looked at, and ties go to the lowest child index, so the results are those
// of the plain loop over all children.
// Products and sums are rounded separately (__dmul_rn / __dadd_rn), so that
// the results do not depend on FMA contraction.
#pragma once

#include <cstdint>

namespace gx {

enum { kCsgBox = 0, kCsgTube = 1, kCsgSphere = 2, kCsgPoly = 3 };
// Sets of solids (bit k: solid kind k).  The navigation routines take the set
// a tree can hold as a template argument: a kernel for trees of boxes only
// (the calorimeters') carries none of the other solids' code.
constexpr int kSolidsAll = 0xF, kSolidsBox = 1 << kCsgBox;
// whether node n is of kind k, for a tree of solids S (constant when S decides)
template <int S> __host__ __device__ __forceinline__ bool csg_is(int kind, int k)
{
  if ((S & (1 << k)) == 0) return false;
  if (S == (1 << k)) return true;
  return kind == k;
}
constexpr int kCsgMaxPlanes = 32;   // planes of one polyhedron, at most
constexpr double kCsgTol = 1e-9;    // surface tolerance (mm)
constexpr double kCsgPad = 1e-6;    // bounding-box padding (mm)
constexpr int kCsgMaxDepth = 64;    // tree depth, at most
constexpr int kCsgMaxNodes = 1 << 22;
constexpr int kCsgGridMin = 8;      // children from which a touchable gets a grid
constexpr double kCsgInf = 1.7976931348623157e308;

struct CsgNode {
  double t[3];         // global translation
  double r[9];         // global rotation, row-major (x_global = R x_local + t)
  double lo[3], hi[3]; // global bounding box, padded
  double a, b, c;      // box: half lengths; tube: rmin, rmax, half length in z; sphere: rmin, rmax
  double glo, ginv, gw; // grid: start along the axis, slabs per mm, slab width
  int kind, rot;       // rot 0: R is the identity
  int mat, parent, kid0, nkid;
  int gaxis, gn, g0;   // grid axis (-1: none), slabs, first slab's entry in the slab table
  int p0, np;          // polyhedron: first plane in the plane table, planes
};

struct CsgView {
  const CsgNode *node; // node 0 is the world
  const int *kids;
  const int *slab;     // per slab: first candidate, candidates (pairs)
  const int *cand;     // candidates (touchable indices)
  const double *planes; // polyhedra: (nx, ny, nz, d) per plane
  int solids;           // the solid kinds present (bit k: kind k)
};

// Slab of coordinate x in a touchable's grid (host and device alike).
__host__ __device__ __forceinline__ int csg_slab(const CsgNode &n, double x)
{
  const double u = (x - n.glo) * n.ginv;
  return u >= 0.0 ? (u < (double)n.gn ? (int)u : n.gn - 1) : 0;
}
template <class T> __host__ __device__ __forceinline__ T csg_comp(const T *p, int a)
{
  return a == 0 ? p[0] : (a == 1 ? p[1] : p[2]);
}

__device__ __forceinline__ double cmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double cadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double csub(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ void csg_local(const CsgNode &n, const double *p, const double *d, double *q, double *e)
{
  const double x0 = p[0] - n.t[0], x1 = p[1] - n.t[1], x2 = p[2] - n.t[2];
  if (!n.rot) {
    q[0] = x0;
    q[1] = x1;
    q[2] = x2;
    e[0] = d[0];
    e[1] = d[1];
    e[2] = d[2];
    return;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) { // R^T
    q[k] = cadd(cadd(cmul(n.r[k], x0), cmul(n.r[3 + k], x1)), cmul(n.r[6 + k], x2));
    e[k] = cadd(cadd(cmul(n.r[k], d[0]), cmul(n.r[3 + k], d[1])), cmul(n.r[6 + k], d[2]));
  }
}
__device__ __forceinline__ void csg_local_point(const CsgNode &n, const double *p, double *q)
{
  const double x0 = p[0] - n.t[0], x1 = p[1] - n.t[1], x2 = p[2] - n.t[2];
  if (!n.rot) {
    q[0] = x0;
    q[1] = x1;
    q[2] = x2;
    return;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) q[k] = cadd(cadd(cmul(n.r[k], x0), cmul(n.r[3 + k], x1)), cmul(n.r[6 + k], x2));
}

__device__ __forceinline__ double dot2(const double *a, const double *b) { return cadd(cmul(a[0], b[0]), cmul(a[1], b[1])); }
__device__ __forceinline__ double dot3(const double *a, const double *b)
{
  return cadd(cadd(cmul(a[0], b[0]), cmul(a[1], b[1])), cmul(a[2], b[2]));
}

// The phi segment of a tube: phi in [s, s + dphi], bounded by the half-planes
// at s and at e = s + dphi; (cos s, sin s, cos e, sin e) in the plane table at
// p0, np = 1 for dphi <= pi (the wedge is the intersection of the half-spaces
// n1.q <= 0, n1 = (sin s, -cos s), and n2.q <= 0, n2 = (-sin e, cos e)), 2 for
// dphi > pi (their union).  h_k = n_k.q, ne_k = n_k.e.
struct Wedge {
  double cs, ss, ce, se;
  int mode;
  __device__ __forceinline__ double h1(double x, double y) const { return csub(cmul(ss, x), cmul(cs, y)); }
  __device__ __forceinline__ double h2(double x, double y) const { return csub(cmul(ce, y), cmul(se, x)); }
  // inside the half-space, or on its plane and not moving out
  __device__ __forceinline__ static bool in(double h, double ne, double tol)
  {
    return h < -tol || (h <= tol && ne <= 0.0);
  }
  __device__ __forceinline__ bool contains(const double *q, const double *e, double tol) const
  {
    const bool a = in(h1(q[0], q[1]), h1(e[0], e[1]), tol), b = in(h2(q[0], q[1]), h2(e[0], e[1]), tol);
    return mode == 1 ? (a && b) : (a || b);
  }
  // a point (no direction) within tol of the wedge
  __device__ __forceinline__ bool holds(double x, double y, double tol) const
  {
    const bool a = h1(x, y) <= tol, b = h2(x, y) <= tol;
    return mode == 1 ? (a && b) : (a || b);
  }
  // distance to leave the wedge from a point inside it
  __device__ __forceinline__ double out(const double *q, const double *e, double tol) const
  {
    const double a = h1(q[0], q[1]), na = h1(e[0], e[1]), b = h2(q[0], q[1]), nb = h2(e[0], e[1]);
    const double ta = na > 0.0 ? -a / na : kCsgInf, tb = nb > 0.0 ? -b / nb : kCsgInf;
    if (mode == 1) return fmin(ta, tb);
    const bool ia = in(a, na, tol), ib = in(b, nb, tol);
    if (ia && ib) return fmax(ta, tb);
    // inside one half-space only: out when it is left, unless the other is
    // entered first (moving into it, it is never left again)
    if (ia) return (nb < 0.0 && -b / nb <= ta) ? kCsgInf : ta;
    if (ib) return (na < 0.0 && -a / na <= tb) ? kCsgInf : tb;
    return 0.0;
  }
  __device__ __forceinline__ double safety_out(const double *q) const
  {
    const double a = -h1(q[0], q[1]), b = -h2(q[0], q[1]);
    return mode == 1 ? fmin(a, b) : fmax(a, b);
  }
  __device__ __forceinline__ double safety_in(const double *q) const
  {
    const double a = h1(q[0], q[1]), b = h2(q[0], q[1]);
    return mode == 1 ? fmax(a, b) : fmin(a, b);
  }
};
__device__ __forceinline__ Wedge csg_wedge(const CsgNode &n, const double *pl)
{
  const double *w = pl + 4 * n.p0;
  return Wedge{w[0], w[1], w[2], w[3], n.np};
}

// The convex polyhedron's queries: op 0 contains (1 or 0), 1 distance out,
// 2 distance in, 3 safety out, 4 safety in (a constant at every call site).
enum { kPolyContains = 0, kPolyOut = 1, kPolyIn = 2, kPolySafeOut = 3, kPolySafeIn = 4 };
__device__ __forceinline__ double csg_poly(const double *__restrict__ pl, int p0, int np, double q0, double q1,
                                        double q2, double e0, double e1, double e2, int op, double tol)
{
  double tmin = -kCsgInf, tmax = kCsgInf, s = (op == kPolySafeIn) ? -kCsgInf : kCsgInf;
  for (int k = p0; k < p0 + np; ++k) {
    const double *p = pl + 4 * k;
    // n.q - d and n.e
    const double h = csub(cadd(cadd(cmul(p[0], q0), cmul(p[1], q1)), cmul(p[2], q2)), p[3]);
    const double ne = cadd(cadd(cmul(p[0], e0), cmul(p[1], e1)), cmul(p[2], e2));
    if (op == kPolyContains) {
      if (h > tol || (h >= -tol && ne > 0.0)) return 0.0;
    } else if (op == kPolyOut) {
      if (ne > 0.0) s = fmin(s, -h / ne);
    } else if (op == kPolyIn) {
      if (ne == 0.0) {
        if (h > 0.0) return kCsgInf;
        continue;
      }
      const double t = -h / ne;
      if (ne < 0.0)
        tmin = fmax(tmin, t);
      else
        tmax = fmin(tmax, t);
    } else if (op == kPolySafeOut) {
      s = fmin(s, -h);
    } else {
      s = fmax(s, h);
    }
  }
  if (op == kPolyContains) return 1.0;
  if (op == kPolyOut) return s < 0.0 ? 0.0 : s;
  if (op == kPolyIn) {
    if (!(tmax > tmin) || tmax <= tol) return kCsgInf;
    return tmin < 0.0 ? 0.0 : tmin;
  }
  return s;
}

// inside, or on the surface and not moving out through it
template <int S = kSolidsAll>
__device__ __forceinline__ bool csg_contains_local(const CsgNode &n, const double *q, const double *e, double tol,
                                                   const double *pl)
{
  if (csg_is<S>(n.kind, kCsgPoly)) return csg_poly(pl, n.p0, n.np, q[0], q[1], q[2], e[0], e[1], e[2], kPolyContains, tol) != 0.0;
  if (csg_is<S>(n.kind, kCsgBox)) {
    const double h0 = n.a, h1 = n.b, h2 = n.c;
    const double a0 = fabs(q[0]), a1 = fabs(q[1]), a2 = fabs(q[2]);
    if (a0 > h0 + tol || a1 > h1 + tol || a2 > h2 + tol) return false;
    if (a0 >= h0 - tol && cmul(q[0], e[0]) > 0.0) return false;
    if (a1 >= h1 - tol && cmul(q[1], e[1]) > 0.0) return false;
    if (a2 >= h2 - tol && cmul(q[2], e[2]) > 0.0) return false;
    return true;
  }
  double r, out;
  if (csg_is<S>(n.kind, kCsgTube)) {
    const double az = fabs(q[2]);
    if (az > n.c + tol) return false;
    if (az >= n.c - tol && cmul(q[2], e[2]) > 0.0) return false;
    if (n.np && !csg_wedge(n, pl).contains(q, e, tol)) return false;
    r = sqrt(dot2(q, q));
    out = dot2(q, e);
  } else {
    r = sqrt(dot3(q, q));
    out = dot3(q, e);
  }
  if (r > n.b + tol) return false;
  if (r >= n.b - tol && out > 0.0) return false;
  if (n.a > 0.0) {
    if (r < n.a - tol) return false;
    if (r <= n.a + tol && out < 0.0) return false;
  }
  return true;
}

// roots of a t^2 + 2 b t + c = 0 with sq = sqrt(b^2 - a c)
__device__ __forceinline__ double far_root(double a, double b, double c, double sq)
{
  return b > 0.0 ? -c / cadd(b, sq) : csub(sq, b) / a;
}
__device__ __forceinline__ double near_root(double a, double b, double c, double sq)
{
  return b < 0.0 ? c / csub(sq, b) : -cadd(b, sq) / a;
}

// distance to leave the solid from a point inside it (or on its surface)
template <int S = kSolidsAll>
__device__ __forceinline__ double csg_dist_out_local(const CsgNode &n, const double *q, const double *e,
                                                     const double *pl)
{
  double s = kCsgInf;
  if (csg_is<S>(n.kind, kCsgPoly)) return csg_poly(pl, n.p0, n.np, q[0], q[1], q[2], e[0], e[1], e[2], kPolyOut, 0.0);
  if (csg_is<S>(n.kind, kCsgBox)) {
    const double h[3] = {n.a, n.b, n.c};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double t = kCsgInf;
      if (e[k] > 0.0)
        t = (h[k] - q[k]) / e[k];
      else if (e[k] < 0.0)
        t = (-h[k] - q[k]) / e[k];
      s = fmin(s, t);
    }
    return s < 0.0 ? 0.0 : s;
  }
  double a, b, r2;
  if (csg_is<S>(n.kind, kCsgTube)) {
    if (e[2] > 0.0)
      s = (n.c - q[2]) / e[2];
    else if (e[2] < 0.0)
      s = (-n.c - q[2]) / e[2];
    a = dot2(e, e);
    b = dot2(q, e);
    r2 = dot2(q, q);
  } else {
    a = dot3(e, e);
    b = dot3(q, e);
    r2 = dot3(q, q);
  }
  if (a > 0.0) {
    const double c = csub(r2, cmul(n.b, n.b)), D = csub(cmul(b, b), cmul(a, c));
    s = fmin(s, far_root(a, b, c, sqrt(D > 0.0 ? D : 0.0)));
    if (n.a > 0.0 && b < 0.0) {
      const double c2 = csub(r2, cmul(n.a, n.a)), D2 = csub(cmul(b, b), cmul(a, c2));
      if (D2 >= 0.0) s = fmin(s, near_root(a, b, c2, sqrt(D2)));
    }
  }
  if (csg_is<S>(n.kind, kCsgTube) && n.np) s = fmin(s, csg_wedge(n, pl).out(q, e, kCsgTol));
  return s < 0.0 ? 0.0 : s;
}

// distance to enter the solid from a point outside it; kCsgInf if missed
template <int S = kSolidsAll>
__device__ __forceinline__ double csg_dist_in_local(const CsgNode &n, const double *q, const double *e,
                                                    const double *pl)
{
  const double tol = kCsgTol;
  if (csg_is<S>(n.kind, kCsgPoly)) return csg_poly(pl, n.p0, n.np, q[0], q[1], q[2], e[0], e[1], e[2], kPolyIn, tol);
  if (csg_is<S>(n.kind, kCsgBox)) {
    const double h[3] = {n.a, n.b, n.c};
    double tmin = -kCsgInf, tmax = kCsgInf;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (e[k] == 0.0) {
        if (fabs(q[k]) > h[k]) return kCsgInf;
        continue;
      }
      double t0 = (-h[k] - q[k]) / e[k], t1 = (h[k] - q[k]) / e[k];
      if (t0 > t1) {
        const double x = t0;
        t0 = t1;
        t1 = x;
      }
      tmin = fmax(tmin, t0);
      tmax = fmin(tmax, t1);
    }
    if (!(tmax > tmin) || tmax <= tol) return kCsgInf;
    return tmin < 0.0 ? 0.0 : tmin;
  }
  double s = kCsgInf;
  const double rmin = n.a, rmax = n.b;
  double a, b, r2;
  if (csg_is<S>(n.kind, kCsgTube)) {
    const double dz = n.c;
    const bool seg = n.np != 0;
    Wedge w{0.0, 0.0, 0.0, 0.0, 0};
    if (seg) w = csg_wedge(n, pl);
    // the hit point at t is in the phi segment
    auto in_phi = [&](double t) {
      return !seg || w.holds(cadd(q[0], cmul(t, e[0])), cadd(q[1], cmul(t, e[1])), tol);
    };
    double tz = -1.0;
    if (q[2] >= dz && e[2] < 0.0)
      tz = (dz - q[2]) / e[2];
    else if (q[2] <= -dz && e[2] > 0.0)
      tz = (-dz - q[2]) / e[2];
    if (tz >= 0.0) {
      const double x = cadd(q[0], cmul(tz, e[0])), y = cadd(q[1], cmul(tz, e[1]));
      const double r = sqrt(cadd(cmul(x, x), cmul(y, y)));
      if (r <= rmax + tol && (rmin <= 0.0 || r >= rmin - tol) && in_phi(tz)) s = tz;
    }
    a = dot2(e, e);
    b = dot2(q, e);
    r2 = dot2(q, q);
    if (a > 0.0) {
      const double c = csub(r2, cmul(rmax, rmax)), D = csub(cmul(b, b), cmul(a, c));
      if (c >= 0.0 && b < 0.0 && D >= 0.0) { // the outer surface from outside
        const double t = near_root(a, b, c, sqrt(D));
        if (t < s && fabs(cadd(q[2], cmul(t, e[2]))) <= dz + tol && in_phi(t)) s = t;
      }
      if (rmin > 0.0) { // the inner surface from the bore
        const double c2 = csub(r2, cmul(rmin, rmin)), D2 = csub(cmul(b, b), cmul(a, c2));
        if (D2 >= 0.0) {
          const double t = far_root(a, b, c2, sqrt(D2));
          if (t >= 0.0 && t < s && fabs(cadd(q[2], cmul(t, e[2]))) <= dz + tol && in_phi(t)) s = t;
        }
      }
    }
    if (seg) { // the two half-planes, entered from their outer side
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const double h = k == 0 ? w.h1(q[0], q[1]) : w.h2(q[0], q[1]);
        const double ne = k == 0 ? w.h1(e[0], e[1]) : w.h2(e[0], e[1]);
        if (!(ne < 0.0) || h < -tol) continue;
        const double t = fmax(-h / ne, 0.0);
        if (!(t < s)) continue;
        const double x = cadd(q[0], cmul(t, e[0])), y = cadd(q[1], cmul(t, e[1]));
        const double along = k == 0 ? cadd(cmul(w.cs, x), cmul(w.ss, y)) : cadd(cmul(w.ce, x), cmul(w.se, y));
        const double r = sqrt(cadd(cmul(x, x), cmul(y, y)));
        if (along >= -tol && r <= rmax + tol && (rmin <= 0.0 || r >= rmin - tol) &&
            fabs(cadd(q[2], cmul(t, e[2]))) <= dz + tol)
          s = t;
      }
    }
    return s;
  }
  a = dot3(e, e);
  b = dot3(q, e);
  r2 = dot3(q, q);
  const double c = csub(r2, cmul(rmax, rmax)), D = csub(cmul(b, b), cmul(a, c));
  if (c >= 0.0 && b < 0.0 && D >= 0.0) s = near_root(a, b, c, sqrt(D));
  if (rmin > 0.0) {
    const double c2 = csub(r2, cmul(rmin, rmin)), D2 = csub(cmul(b, b), cmul(a, c2));
    if (D2 >= 0.0) {
      const double t = far_root(a, b, c2, sqrt(D2));
      if (t >= 0.0 && t < s) s = t;
    }
  }
  return s;
}

template <int S = kSolidsAll>
__device__ __forceinline__ double csg_safety_out_local(const CsgNode &n, const double *q, const double *pl)
{
  if (csg_is<S>(n.kind, kCsgPoly)) return csg_poly(pl, n.p0, n.np, q[0], q[1], q[2], 0.0, 0.0, 0.0, kPolySafeOut, 0.0);
  if (csg_is<S>(n.kind, kCsgBox)) return fmin(fmin(n.a - fabs(q[0]), n.b - fabs(q[1])), n.c - fabs(q[2]));
  if (csg_is<S>(n.kind, kCsgTube)) {
    const double r = sqrt(dot2(q, q));
    double s = fmin(n.c - fabs(q[2]), n.b - r);
    if (n.a > 0.0) s = fmin(s, r - n.a);
    return n.np ? fmin(s, csg_wedge(n, pl).safety_out(q)) : s;
  }
  const double r = sqrt(dot3(q, q));
  return n.a > 0.0 ? fmin(n.b - r, r - n.a) : n.b - r;
}

// a lower bound of the distance to the solid from a point outside it
template <int S = kSolidsAll>
__device__ __forceinline__ double csg_safety_in_local(const CsgNode &n, const double *q, const double *pl)
{
  if (csg_is<S>(n.kind, kCsgPoly)) return csg_poly(pl, n.p0, n.np, q[0], q[1], q[2], 0.0, 0.0, 0.0, kPolySafeIn, 0.0);
  if (csg_is<S>(n.kind, kCsgBox)) return fmax(fmax(fabs(q[0]) - n.a, fabs(q[1]) - n.b), fabs(q[2]) - n.c);
  if (csg_is<S>(n.kind, kCsgTube)) {
    const double r = sqrt(dot2(q, q));
    const double s = fmax(fmax(fabs(q[2]) - n.c, r - n.b), n.a - r);
    return n.np ? fmax(s, csg_wedge(n, pl).safety_in(q)) : s;
  }
  const double r = sqrt(dot3(q, q));
  return fmax(r - n.b, n.a - r);
}

__device__ __forceinline__ double csg_bbox_gap(const CsgNode &n, const double *p)
{
  double g = -kCsgInf;
#pragma unroll
  for (int k = 0; k < 3; ++k) g = fmax(g, fmax(n.lo[k] - p[k], p[k] - n.hi[k]));
  return g;
}

// entry distance of the ray into the bounding box, kCsgInf if missed
__device__ __forceinline__ double csg_bbox_ray(const CsgNode &n, const double *p, const double *d)
{
  double tmin = 0.0, tmax = kCsgInf;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (d[k] == 0.0) {
      if (p[k] < n.lo[k] || p[k] > n.hi[k]) return kCsgInf;
      continue;
    }
    double t0 = (n.lo[k] - p[k]) / d[k], t1 = (n.hi[k] - p[k]) / d[k];
    if (t0 > t1) {
      const double x = t0;
      t0 = t1;
      t1 = x;
    }
    tmin = fmax(tmin, t0);
    tmax = fmin(tmax, t1);
  }
  return tmax < tmin ? kCsgInf : tmin;
}

template <int S = kSolidsAll>
__device__ __forceinline__ bool csg_contains(const CsgView &g, int v, const double *p, const double *d, double tol)
{
  const CsgNode &n = g.node[v];
  if (csg_bbox_gap(n, p) > 0.0) return false;
  double q[3], e[3];
  csg_local(n, p, d, q, e);
  return csg_contains_local<S>(n, q, e, tol, g.planes);
}

// the deepest touchable at or below v (which contains p) that contains p
template <int S = kSolidsAll>
__device__ __forceinline__ int csg_descend(const CsgView &g, int v, const double *p, const double *d, double tol)
{
  for (int depth = 0; depth < kCsgMaxDepth; ++depth) {
    const CsgNode &n = g.node[v];
    int next = -1;
    if (n.gaxis >= 0) {
      const int sl = n.g0 + csg_slab(n, csg_comp(p, n.gaxis));
      const int j0 = g.slab[2 * sl], nj = g.slab[2 * sl + 1];
      for (int j = 0; j < nj && next < 0; ++j) {
        const int c = g.cand[j0 + j];
        if (csg_contains<S>(g, c, p, d, tol)) next = c;
      }
    } else {
      const int k0 = n.kid0, nk = n.nkid;
      for (int k = 0; k < nk && next < 0; ++k) {
        const int c = g.kids[k0 + k];
        if (csg_contains<S>(g, c, p, d, tol)) next = c;
      }
    }
    if (next < 0) return v;
    v = next;
  }
  return v;
}

// from touchable v up until one contains p, then down; -1 outside the world
template <int S = kSolidsAll>
__device__ __forceinline__ int csg_locate(const CsgView &g, int v, const double *p, const double *d, double tol)
{
  if (v < 0) v = 0;
  for (int depth = 0; v >= 0 && depth <= kCsgMaxDepth; ++depth) {
    if (csg_contains<S>(g, v, p, d, tol)) return csg_descend<S>(g, v, p, d, tol);
    v = g.node[v].parent;
  }
  return -1;
}

// distance to the next boundary from p in v; children whose bounding box the
// ray reaches only beyond `limit` are skipped (the result is then >= limit);
// hit = the child entered, -1 when leaving v
template <int S = kSolidsAll>
__device__ __forceinline__ double csg_step(const CsgView &g, int v, const double *p, const double *d, double limit,
                                           int &hit)
{
  double q[3], e[3];
  const CsgNode &n = g.node[v];
  csg_local(n, p, d, q, e);
  double s = csg_dist_out_local<S>(n, q, e, g.planes);
  hit = -1;
  auto child = [&](int c) {
    const double tb = csg_bbox_ray(g.node[c], p, d);
    if (!(tb < s && tb < limit)) return;
    csg_local(g.node[c], p, d, q, e);
    const double t = csg_dist_in_local<S>(g.node[c], q, e, g.planes);
    if (t < s || (t == s && hit >= 0 && c < hit)) {
      s = t;
      hit = c;
    }
  };
  if (n.gaxis >= 0) {
    // the slabs in the order the ray crosses them, while their entry (moved
    // back by the bounding-box padding) comes before the nearest boundary
    const double pa = csg_comp(p, n.gaxis), da = csg_comp(d, n.gaxis);
    const int step = da > 0.0 ? 1 : (da < 0.0 ? -1 : 0);
    int sl = csg_slab(n, pa);
    for (int it = 0; it < n.gn; ++it) {
      const int row = n.g0 + sl;
      const int j0 = g.slab[2 * row], nj = g.slab[2 * row + 1];
      for (int j = 0; j < nj; ++j) child(g.cand[j0 + j]);
      sl += step;
      if (step == 0 || sl < 0 || sl >= n.gn) break;
      const double xb = n.glo + (step > 0 ? sl : sl + 1) * n.gw - step * kCsgPad;
      const double tb = (xb - pa) / da;
      if (!(tb < s && tb < limit)) break;
    }
  } else {
    const int k0 = n.kid0, nk = n.nkid;
    for (int k = 0; k < nk; ++k) child(g.kids[k0 + k]);
  }
  return s;
}

template <int S = kSolidsAll>
__device__ __forceinline__ double csg_safety(const CsgView &g, int v, const double *p)
{
  double q[3];
  const CsgNode &n = g.node[v];
  csg_local_point(n, p, q);
  double s = csg_safety_out_local<S>(n, q, g.planes);
  auto child = [&](int c) {
    const CsgNode &m = g.node[c];
    const double gap = csg_bbox_gap(m, p);
    if (gap >= s) return;
    csg_local_point(m, p, q);
    s = fmin(s, fmax(gap, csg_safety_in_local<S>(m, q, g.planes)));
  };
  if (n.gaxis >= 0) {
    // children farther than the safety along the axis cannot lower it
    const double pa = csg_comp(p, n.gaxis), r = fmax(s, 0.0) + kCsgPad;
    const int s0 = csg_slab(n, pa - r), s1 = csg_slab(n, pa + r);
    for (int sl = s0; sl <= s1; ++sl) {
      const int row = n.g0 + sl;
      const int j0 = g.slab[2 * row], nj = g.slab[2 * row + 1];
      for (int j = 0; j < nj; ++j) child(g.cand[j0 + j]);
    }
  } else {
    const int k0 = n.kid0, nk = n.nkid;
    for (int k = 0; k < nk; ++k) child(g.kids[k0 + k]);
  }
  return s < 0.0 ? 0.0 : s;
}

// the touchable entered at p after csg_step's crossing out of v
template <int S = kSolidsAll>
__device__ __forceinline__ int csg_cross(const CsgView &g, int v, int hit, const double *p, const double *d)
{
  if (hit >= 0) return csg_descend<S>(g, hit, p, d, kCsgTol);
  return csg_locate<S>(g, g.node[v].parent, p, d, kCsgTol);
}

} // namespace gx
