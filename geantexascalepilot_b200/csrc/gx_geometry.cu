// gx_geometry.cu -- the CSG volume tree (transport geometry 2): the host
// builder behind gx_geom_*, its upload into a context and the navigation
// probe kernel.
//
// The builder takes the calls a VecGeom detector construction makes
// (UnplacedBox / LogicalVolume / PlaceDaughter with a Transformation3D /
// SetWorld / CloseGeometry, as in the reference's
// source/Geant/proxy/test/BasicCpuTransport/ProxyDetectorConstruction.cpp:
// 241-324), plus a material and a scoring flag per logical volume.  Closing
// unrolls the tree depth-first into touchables (one per placed instance) with
// global transforms and padded bounding boxes; scored touchables get
// consecutive tally columns in that order.  Navigation itself is in gx_csg.cuh.
#include "gx_csg.cuh"
#include "gx_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

struct gx_geom {
  struct Solid {
    int kind;
    double p[3];
    int p0, np;  // polyhedron: its planes in `planes`
    double lo[3], hi[3]; // local bounding box
  };
  struct Lv {
    int solid, mat, scored;
  };
  struct Pv {
    int mother, lv;
    double t[3], r[9];
  };
  std::vector<Solid> solids;
  std::vector<Lv> lvs;
  std::vector<Pv> pvs;
  std::vector<double> planes; // polyhedra: unit outward normal and offset per plane
  // after gx_geom_close
  int world = -1, nscore = 0;
  std::vector<gx::CsgNode> nodes;
  std::vector<int> kids, score, lv_of;
  std::vector<int> slab, cand; // the children's grids (gx_csg.cuh)
};

namespace gx {

namespace {

struct Flattener {
  gx_geom &g;
  std::vector<std::vector<int>> daughters; // placements per logical volume, in placement order
  int kcur = 0;
  bool err = false;

  long count(int lv, int depth)
  {
    if (depth > kCsgMaxDepth) return -1;
    long n = 1;
    for (int p : daughters[lv]) {
      long k = count(g.pvs[p].lv, depth + 1);
      if (k < 0) return -1;
      n += k;
      if (n > kCsgMaxNodes) return -1;
    }
    return n;
  }

  int visit(int lv, int parent, const double R[9], const double t[3], int depth)
  {
    const int id = (int)g.nodes.size();
    g.nodes.emplace_back();
    g.score.push_back(-1);
    g.lv_of.push_back(lv);
    {
      CsgNode &n = g.nodes[id];
      const gx_geom::Solid &s = g.solids[g.lvs[lv].solid];
      n.kind = s.kind;
      n.a = s.p[0];
      n.b = s.p[1];
      n.c = s.p[2];
      n.p0 = s.p0;
      n.np = s.np;
      std::memcpy(n.t, t, sizeof(n.t));
      std::memcpy(n.r, R, sizeof(n.r));
      n.rot = !(R[0] == 1.0 && R[1] == 0.0 && R[2] == 0.0 && R[3] == 0.0 && R[4] == 1.0 && R[5] == 0.0 &&
                R[6] == 0.0 && R[7] == 0.0 && R[8] == 1.0);
      n.mat = g.lvs[lv].mat;
      n.parent = parent;
      if (g.lvs[lv].scored) g.score[id] = g.nscore++;
      for (int k = 0; k < 3; ++k) {
        n.lo[k] = kCsgInf;
        n.hi[k] = -kCsgInf;
      }
      for (int corner = 0; corner < 8; ++corner) {
        const double x[3] = {(corner & 1) ? s.hi[0] : s.lo[0], (corner & 2) ? s.hi[1] : s.lo[1],
                             (corner & 4) ? s.hi[2] : s.lo[2]};
        for (int k = 0; k < 3; ++k) {
          const double y = R[3 * k] * x[0] + R[3 * k + 1] * x[1] + R[3 * k + 2] * x[2] + t[k];
          n.lo[k] = std::min(n.lo[k], y);
          n.hi[k] = std::max(n.hi[k], y);
        }
      }
      for (int k = 0; k < 3; ++k) {
        n.lo[k] -= kCsgPad;
        n.hi[k] += kCsgPad;
      }
      n.nkid = (int)daughters[lv].size();
      n.kid0 = kcur; // the children's block, reserved before recursing
      kcur += n.nkid;
      n.gaxis = -1;
      n.gn = n.g0 = 0;
      n.glo = n.ginv = n.gw = 0.0;
    }
    int j = 0;
    for (int p : daughters[lv]) {
      const double *Rp = g.pvs[p].r, *tp = g.pvs[p].t;
      double Rc[9], tc[3];
      for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c)
          Rc[3 * r + c] = R[3 * r] * Rp[c] + R[3 * r + 1] * Rp[3 + c] + R[3 * r + 2] * Rp[6 + c];
        tc[r] = R[3 * r] * tp[0] + R[3 * r + 1] * tp[1] + R[3 * r + 2] * tp[2] + t[r];
      }
      const int kid = visit(g.pvs[p].lv, id, Rc, tc, depth + 1);
      g.kids[g.nodes[id].kid0 + j++] = kid;
    }
    return id;
  }
};

// The slab grid of a touchable with many children: along each axis, slabs
// of equal width over its bounding box, twice as many as children (at most
// 4096); each child listed in the slabs its bounding box overlaps; the axis
// with the fewest listings wins.
void build_grid(gx_geom &g, int v)
{
  CsgNode &n = g.nodes[v];
  if (n.nkid < kCsgGridMin) return;
  const int gn = std::min(2 * n.nkid, 4096);
  long best = -1;
  int best_axis = -1;
  for (int a = 0; a < 3; ++a) {
    CsgNode t = n;
    t.gn = gn;
    t.glo = n.lo[a];
    t.ginv = gn / (n.hi[a] - n.lo[a]);
    long entries = 0;
    for (int k = 0; k < n.nkid; ++k) {
      const CsgNode &c = g.nodes[g.kids[n.kid0 + k]];
      entries += csg_slab(t, c.hi[a]) - csg_slab(t, c.lo[a]) + 1;
    }
    if (best < 0 || entries < best) {
      best = entries;
      best_axis = a;
    }
  }
  n.gaxis = best_axis;
  n.gn = gn;
  n.glo = n.lo[best_axis];
  n.gw = (n.hi[best_axis] - n.lo[best_axis]) / gn;
  n.ginv = gn / (n.hi[best_axis] - n.lo[best_axis]);
  n.g0 = (int)(g.slab.size() / 2);
  std::vector<std::vector<int>> lists(gn);
  for (int k = 0; k < n.nkid; ++k) { // child order within every slab
    const int c = g.kids[n.kid0 + k];
    const int s0 = csg_slab(n, g.nodes[c].lo[best_axis]), s1 = csg_slab(n, g.nodes[c].hi[best_axis]);
    for (int s = s0; s <= s1; ++s) lists[s].push_back(c);
  }
  for (int s = 0; s < gn; ++s) {
    g.slab.push_back((int)g.cand.size());
    g.slab.push_back((int)lists[s].size());
    g.cand.insert(g.cand.end(), lists[s].begin(), lists[s].end());
  }
}

// The bounding box of the convex polyhedron {x : n_k . x <= d_k} (unit
// normals): the extent of its vertices, the points where three planes meet
// inside all the others.  False when the planes bound no finite volume: no
// vertex, or an edge direction +-(n_i x n_j) along which no plane closes it.
bool poly_bbox(const double *pl, int np, double lo[3], double hi[3])
{
  int nv = 0;
  for (int k = 0; k < 3; ++k) {
    lo[k] = kCsgInf;
    hi[k] = -kCsgInf;
  }
  for (int i = 0; i < np; ++i)
    for (int j = i + 1; j < np; ++j)
      for (int k = j + 1; k < np; ++k) {
        const double *a = pl + 4 * i, *b = pl + 4 * j, *c = pl + 4 * k;
        const double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
        const double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
        const double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        const double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
        if (std::fabs(det) < 1e-12) continue;
        double x[3];
        for (int m = 0; m < 3; ++m) x[m] = (a[3] * bc[m] + b[3] * ca[m] + c[3] * ab[m]) / det;
        bool in = true;
        for (int l = 0; l < np && in; ++l) {
          const double *p = pl + 4 * l;
          in = p[0] * x[0] + p[1] * x[1] + p[2] * x[2] - p[3] <= 1e-9 * (1.0 + std::fabs(p[3]));
        }
        if (!in) continue;
        ++nv;
        for (int m = 0; m < 3; ++m) {
          lo[m] = std::min(lo[m], x[m]);
          hi[m] = std::max(hi[m], x[m]);
        }
      }
  if (nv == 0) return false;
  for (int i = 0; i < np; ++i)
    for (int j = i + 1; j < np; ++j) {
      const double *a = pl + 4 * i, *b = pl + 4 * j;
      const double v[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
      const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      if (len < 1e-12) continue;
      for (int sgn = -1; sgn <= 1; sgn += 2) {
        bool open = true;
        for (int l = 0; l < np && open; ++l) {
          const double *p = pl + 4 * l;
          open = sgn * (p[0] * v[0] + p[1] * v[1] + p[2] * v[2]) <= 1e-12 * len;
        }
        if (open) return false;
      }
    }
  return true;
}

bool orthonormal(const double *R)
{
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double d = R[3 * i] * R[3 * j] + R[3 * i + 1] * R[3 * j + 1] + R[3 * i + 2] * R[3 * j + 2];
      if (std::fabs(d - (i == j ? 1.0 : 0.0)) > 1e-9) return false;
    }
  return true;
}

// S: the solids the tree holds (the box-only instantiation for trees of boxes,
// as the transport kernels use it)
template <int S>
__global__ void k_geom_probe(CsgView g, int n, const double *__restrict__ pos, const double *__restrict__ dir,
                             const double *__restrict__ limit, int *__restrict__ vol, double *__restrict__ snext,
                             int *__restrict__ next, double *__restrict__ safety)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  const double d[3] = {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
  const int v = csg_locate<S>(g, 0, p, d, kCsgTol);
  vol[i] = v;
  if (v < 0) {
    snext[i] = -1.0;
    next[i] = -1;
    safety[i] = -1.0;
    return;
  }
  int hit;
  const double s = csg_step<S>(g, v, p, d, limit[i], hit);
  snext[i] = s;
  safety[i] = csg_safety<S>(g, v, p);
  if (s < limit[i]) {
    const double x[3] = {cadd(p[0], cmul(s, d[0])), cadd(p[1], cmul(s, d[1])), cadd(p[2], cmul(s, d[2]))};
    next[i] = csg_cross<S>(g, v, hit, x, d);
  } else {
    next[i] = v;
  }
}

} // namespace

} // namespace gx

using namespace gx;

extern "C" {

int gx_geom_create(gx_geom **out)
{
  if (!out) return set_error(GX_ERR_ARG, "gx_geom_create: null argument");
  *out = new gx_geom();
  return GX_OK;
}

void gx_geom_destroy(gx_geom *g) { delete g; }

static int add_solid(gx_geom *g, int kind, double a, double b, double c, int *solid)
{
  if (!g || !solid) return set_error(GX_ERR_ARG, "gx_geom: null argument");
  if (g->world >= 0) return set_error(GX_ERR_ARG, "gx_geom: the geometry is closed");
  gx_geom::Solid s{kind, {a, b, c}, 0, 0, {0, 0, 0}, {0, 0, 0}};
  // local bounding box half lengths: box (a, b, c), tube (b, b, c), sphere (b, b, b)
  double h[3] = {a, b, c};
  if (kind == kCsgTube) h[0] = b;
  if (kind == kCsgSphere) h[0] = h[2] = b;
  for (int k = 0; k < 3; ++k) {
    s.lo[k] = -h[k];
    s.hi[k] = h[k];
  }
  g->solids.push_back(s);
  *solid = (int)g->solids.size() - 1;
  return GX_OK;
}

int gx_geom_box(gx_geom *g, double hx, double hy, double hz, int *solid)
{
  if (!(hx > 0.0 && hy > 0.0 && hz > 0.0)) return set_error(GX_ERR_ARG, "gx_geom_box: half lengths must be > 0");
  return add_solid(g, kCsgBox, hx, hy, hz, solid);
}

int gx_geom_tube(gx_geom *g, double rmin, double rmax, double dz, int *solid)
{
  if (!(rmin >= 0.0 && rmax > rmin && dz > 0.0))
    return set_error(GX_ERR_ARG, "gx_geom_tube: need 0 <= rmin < rmax and dz > 0");
  return add_solid(g, kCsgTube, rmin, rmax, dz, solid);
}

int gx_geom_tube_segment(gx_geom *g, double rmin, double rmax, double dz, double sphi, double dphi, int *solid)
{
  const double pi = 3.14159265358979323846;
  if (!(dphi > 0.0) || !std::isfinite(sphi))
    return set_error(GX_ERR_ARG, "gx_geom_tube_segment: need dphi > 0 and a finite sphi");
  if (dphi >= 2.0 * pi) return gx_geom_tube(g, rmin, rmax, dz, solid);
  int rc = gx_geom_tube(g, rmin, rmax, dz, solid);
  if (rc) return rc;
  // the half-planes' directions (cos s, sin s, cos e, sin e), e = sphi + dphi,
  // as one row of the plane table; np = 1 (dphi <= pi: the wedge is convex)
  // or 2 (the union of the two half-spaces)
  gx_geom::Solid &s = g->solids[*solid];
  const double e = sphi + dphi;
  s.p0 = (int)(g->planes.size() / 4);
  s.np = dphi <= pi ? 1 : 2;
  g->planes.insert(g->planes.end(), {std::cos(sphi), std::sin(sphi), std::cos(e), std::sin(e)});
  return GX_OK;
}

int gx_geom_sphere(gx_geom *g, double rmin, double rmax, int *solid)
{
  if (!(rmin >= 0.0 && rmax > rmin)) return set_error(GX_ERR_ARG, "gx_geom_sphere: need 0 <= rmin < rmax");
  return add_solid(g, kCsgSphere, rmin, rmax, 0.0, solid);
}

int gx_geom_polyhedron(gx_geom *g, int nplanes, const double *planes, int *solid)
{
  if (!g || !solid || !planes) return set_error(GX_ERR_ARG, "gx_geom_polyhedron: null argument");
  if (g->world >= 0) return set_error(GX_ERR_ARG, "gx_geom: the geometry is closed");
  if (nplanes < 4 || nplanes > kCsgMaxPlanes)
    return set_error(GX_ERR_ARG, "gx_geom_polyhedron: %d planes (4 to %d)", nplanes, kCsgMaxPlanes);
  std::vector<double> pl(4 * nplanes);
  for (int k = 0; k < nplanes; ++k) {
    const double *p = planes + 4 * k;
    const double len = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    if (!(len > 0.0) || !std::isfinite(len) || !std::isfinite(p[3]))
      return set_error(GX_ERR_ARG, "gx_geom_polyhedron: plane %d has no normal", k);
    for (int m = 0; m < 4; ++m) pl[4 * k + m] = p[m] / len;
  }
  gx_geom::Solid s{kCsgPoly, {0, 0, 0}, (int)(g->planes.size() / 4), nplanes, {0, 0, 0}, {0, 0, 0}};
  if (!poly_bbox(pl.data(), nplanes, s.lo, s.hi))
    return set_error(GX_ERR_ARG, "gx_geom_polyhedron: the planes bound no finite volume");
  g->planes.insert(g->planes.end(), pl.begin(), pl.end());
  g->solids.push_back(s);
  *solid = (int)g->solids.size() - 1;
  return GX_OK;
}

int gx_geom_logical_volume(gx_geom *g, int solid, int material, int scored, int *lv)
{
  if (!g || !lv) return set_error(GX_ERR_ARG, "gx_geom_logical_volume: null argument");
  if (g->world >= 0) return set_error(GX_ERR_ARG, "gx_geom: the geometry is closed");
  if (solid < 0 || solid >= (int)g->solids.size()) return set_error(GX_ERR_ARG, "gx_geom_logical_volume: bad solid");
  if (material < 0 || material >= kNMat) return set_error(GX_ERR_ARG, "gx_geom_logical_volume: bad material");
  g->lvs.push_back({solid, material, scored ? 1 : 0});
  *lv = (int)g->lvs.size() - 1;
  return GX_OK;
}

int gx_geom_place_daughter(gx_geom *g, int mother, int daughter, const double translation[3],
                           const double rotation[9], int *pv)
{
  if (!g || !translation) return set_error(GX_ERR_ARG, "gx_geom_place_daughter: null argument");
  if (g->world >= 0) return set_error(GX_ERR_ARG, "gx_geom: the geometry is closed");
  const int nlv = (int)g->lvs.size();
  if (mother < 0 || mother >= nlv || daughter < 0 || daughter >= nlv)
    return set_error(GX_ERR_ARG, "gx_geom_place_daughter: bad logical volume");
  gx_geom::Pv p;
  p.mother = mother;
  p.lv = daughter;
  std::memcpy(p.t, translation, sizeof(p.t));
  const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::memcpy(p.r, rotation ? rotation : I, sizeof(p.r));
  if (!orthonormal(p.r)) return set_error(GX_ERR_ARG, "gx_geom_place_daughter: rotation is not orthonormal");
  g->pvs.push_back(p);
  if (pv) *pv = (int)g->pvs.size() - 1;
  return GX_OK;
}

int gx_geom_close(gx_geom *g, int world, int *ntouchables, int *nscore)
{
  if (!g) return set_error(GX_ERR_ARG, "gx_geom_close: null argument");
  if (g->world >= 0) return set_error(GX_ERR_ARG, "gx_geom: the geometry is closed");
  if (world < 0 || world >= (int)g->lvs.size()) return set_error(GX_ERR_ARG, "gx_geom_close: bad world volume");
  Flattener f{*g, std::vector<std::vector<int>>(g->lvs.size())};
  for (int p = 0; p < (int)g->pvs.size(); ++p) f.daughters[g->pvs[p].mother].push_back(p);
  const long total = f.count(world, 0);
  if (total < 0)
    return set_error(GX_ERR_ARG, "gx_geom_close: more than %d touchables or deeper than %d levels (a volume placed "
                                 "inside itself?)",
                     kCsgMaxNodes, kCsgMaxDepth);
  g->nodes.clear();
  g->nodes.reserve(total);
  g->kids.assign(total, 0);
  g->nscore = 0;
  const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, z[3] = {0, 0, 0};
  f.visit(world, -1, I, z, 0);
  g->slab.clear();
  g->cand.clear();
  for (int v = 0; v < (int)g->nodes.size(); ++v) build_grid(*g, v);
  g->world = world;
  if (ntouchables) *ntouchables = (int)g->nodes.size();
  if (nscore) *nscore = g->nscore;
  return GX_OK;
}

int gx_geom_touchable(const gx_geom *g, int i, int *lv, int *parent, int *score, double translation[3],
                      double rotation[9])
{
  if (!g || g->world < 0) return set_error(GX_ERR_ARG, "gx_geom_touchable: geometry not closed");
  if (i < 0 || i >= (int)g->nodes.size()) return set_error(GX_ERR_ARG, "gx_geom_touchable: bad index");
  const CsgNode &n = g->nodes[i];
  if (lv) *lv = g->lv_of[i];
  if (parent) *parent = n.parent;
  if (score) *score = g->score[i];
  if (translation) std::memcpy(translation, n.t, sizeof(n.t));
  if (rotation) std::memcpy(rotation, n.r, sizeof(n.r));
  return GX_OK;
}

int gx_ctx_load_geometry(gx_ctx *ctx, const gx_geom *g)
{
  if (!ctx || !g) return set_error(GX_ERR_ARG, "gx_ctx_load_geometry: null argument");
  if (g->world < 0) return set_error(GX_ERR_ARG, "gx_ctx_load_geometry: geometry not closed (gx_geom_close)");
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_error(e, "gx_ctx_load_geometry: cudaSetDevice");
  const size_t nn = g->nodes.size();
  CsgNode *dn = nullptr;
  int *dk = nullptr, *ds = nullptr, *dsl = nullptr, *dc = nullptr;
  double *dp = nullptr;
  auto upload = [&](int **dst, const std::vector<int> &src) {
    const size_t bytes = std::max<size_t>(src.size(), 1) * sizeof(int);
    cudaError_t r = cudaMalloc((void **)dst, bytes);
    if (r == cudaSuccess && !src.empty()) r = cudaMemcpy(*dst, src.data(), src.size() * sizeof(int), cudaMemcpyHostToDevice);
    return r;
  };
  if ((e = cudaMalloc((void **)&dn, nn * sizeof(CsgNode))) != cudaSuccess ||
      (e = cudaMemcpy(dn, g->nodes.data(), nn * sizeof(CsgNode), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = upload(&dk, g->kids)) != cudaSuccess || (e = upload(&ds, g->score)) != cudaSuccess ||
      (e = upload(&dsl, g->slab)) != cudaSuccess || (e = upload(&dc, g->cand)) != cudaSuccess ||
      (e = cudaMalloc((void **)&dp, std::max<size_t>(g->planes.size(), 1) * sizeof(double))) != cudaSuccess ||
      (!g->planes.empty() && (e = cudaMemcpy(dp, g->planes.data(), g->planes.size() * sizeof(double),
                                             cudaMemcpyHostToDevice)) != cudaSuccess)) {
    for (void *q : {(void *)dn, (void *)dk, (void *)ds, (void *)dsl, (void *)dc, (void *)dp}) cudaFree(q);
    return cuda_error(e, "gx_ctx_load_geometry: upload");
  }
  // the previous tree (if any) stays allocated until the context goes: a
  // captured transport graph may still refer to it
  for (void *q : {(void *)dn, (void *)dk, (void *)ds, (void *)dsl, (void *)dc, (void *)dp}) c->owned.push_back(q);
  c->csg_node = dn;
  c->csg_kids = dk;
  c->csg_score = ds;
  c->csg_slab = dsl;
  c->csg_cand = dc;
  c->csg_planes = dp;
  c->csg_n = (int)nn;
  c->csg_nscore = g->nscore;
  int solids = 0;
  for (const CsgNode &n : g->nodes) solids |= 1 << n.kind;
  c->csg_solids = solids;
  return GX_OK;
}

int gx_geom_probe(gx_ctx *ctx, int n, const double *d_pos, const double *d_dir, const double *d_limit, int *d_vol,
                  double *d_snext, int *d_next, double *d_safety, gx_stream_t s)
{
  if (!ctx || n < 0 || (n > 0 && (!d_pos || !d_dir || !d_limit || !d_vol || !d_snext || !d_next || !d_safety)))
    return set_error(GX_ERR_ARG, "gx_geom_probe: bad arguments");
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->csg_node) return set_error(GX_ERR_ARG, "gx_geom_probe: no geometry loaded (gx_ctx_load_geometry)");
  if (n == 0) return GX_OK;
  CsgView v{c->csg_node, c->csg_kids, c->csg_slab, c->csg_cand, c->csg_planes, c->csg_solids};
  (c->csg_solids == kSolidsBox ? k_geom_probe<kSolidsBox> : k_geom_probe<kSolidsAll>)<<<(n + 127) / 128, 128, 0,
                                                                                      stream_of(s)>>>(
      v, n, d_pos, d_dir, d_limit, d_vol, d_snext, d_next, d_safety);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GX_OK : cuda_error(e, "k_geom_probe");
}

} // extern "C"
