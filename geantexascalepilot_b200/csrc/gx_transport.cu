// gx_transport.cu -- the transport engine: every alive track takes one step
// per iteration, in FP64 or FP32-mixed arithmetic.
//
// Layout in HBM: per particle type (gamma, e-, e+) two SoA track stores of
// `capacity` slots (current / next) and one overflow stack.  A step kernel
// reads the current store of its type, runs one OneStep per track and writes
// the survivor and its secondaries to the next stores through warp-aggregated
// slot reservations (prefix sums over the warp, one atomic per warp and type),
// so the stores stay compact and particle-pure without a separate compaction
// pass.  Tracks that do not fit go to the stack and are re-injected when the
// stores drain; primaries are injected on the device, with per-primary
// MRG32k3a substreams by skip-ahead, whenever fewer than `refill_below`
// tracks are in flight.  The per-iteration launch sequence (refill, three
// step kernels, finish) is captured once in a CUDA graph and replayed.
//
// The "plain" engine runs the same step code as one kernel over one mixed
// store, launched and synchronised from the host every iteration, in FP64: the
// straightforward GPU loop the batched engine is measured against.
//
// The FP64 parity variant: gx_transport_parity.cu compiles this file a second
// time with GX_PARITY defined and without floating-point contraction, into
// namespace gx::parity (FP64 only).  There the step takes the reference's
// spline form for every table lookup, the reference's ionisation GPIL/DoIt,
// the general helix step (ConstFieldHelixStepper::DoStep) with the
// oracle's sub-step length, and the elementary functions of gx_math.h: the
// same operations, in the same order and rounding, as the oracle's step loop,
// so that the two agree track by track (gx_transport_config.fp64_parity).
#include "gx_internal.cuh"

#include <algorithm>
#include <mutex>
#include <type_traits>
#include <cmath>
#include <cstring>

namespace gx {
#ifdef GX_PARITY
namespace parity {
#define GX_ENGINE_OF(c) ((c)->parity_engine)
#define GX_RELEASE_ENGINE(c) ::gx::parity::release_engine(c)
#else
#define GX_ENGINE_OF(c) ((c)->engine)
#define GX_RELEASE_ENGINE(c) ::gx::release_engine(c)
#endif

// ------------------------------------------------------------------ layout
template <class R> struct Store {
  double *x, *y, *z;
  R *dx, *dy, *dz, *E, *n0, *n1, *n2;
  R *r0; // multiple scattering: range scale of the step limit in the current volume (<= 0: unset)
  uint32_t *rng; // 6 planes of cap words
  int *vol, *event, *prim, *type;
  long long cap;
};

struct Geom {
  int geometry, axis, nlayers, box_mat, charged_local, nvol, nevents;
  int msc;       // multiple scattering of e-/e+
  int field_map; // 1: the context's field map with Runge-Kutta sub-steps, 0: uniform Bz
  double t_abs, pitch, x0, total, half_trans, Bz;
  double box_half[3], box_centre[3];
  CsgView csg; // geometry 2: the context's volume tree
};

constexpr int kNStat = 28;
// S_READ/S_WRITE: track records read and written by the step kernels of a
// type other than its transport kernel (the interaction kernels, the plain
// loop's fused kernel); S_TREAD/S_TWRITE: by its transport kernel (the host
// reports the sums as the type's records read and written); S_TQUEUE: of the
// transport kernel's writes, the records put in an interaction buffer (added
// up by k_finish from the buffers' counters); S_TSTEP: steps completed in the
// transport kernel of a type.
enum { S_STEPS, S_SUBSTEPS, S_TRACKS, S_SEC0, S_SEC1, S_SEC2, S_PAIR, S_ANNIH, S_ERR, S_OVERFLOW,
       S_READ0, S_READ1, S_READ2, S_WRITE0, S_WRITE1, S_WRITE2, S_TREAD0, S_TREAD1, S_TREAD2,
       S_TWRITE0, S_TWRITE1, S_TWRITE2, S_TQUEUE0, S_TQUEUE1, S_TQUEUE2, S_TSTEP0, S_TSTEP1, S_TSTEP2 };

struct Ctl {
  int parity;
  int err_flags;
  long long count[2][3];
  long long stack_count[3];
  long long prim_next, nprim;
  long long take_stack[3], take_prim; // refill plan
  long long stack_dst[3], stack_src[3];
  long long in_flight, pending, peak, iterations;
  unsigned long long stat[kNStat];
  double escaped;
  double retired;     // energy deposited or escaped so far (the rest is still carried by tracks)
  long long extracted; // tracks written out by gx_transport_tracks
  const double *cumE; // inclusive prefix sum of the primary energies
  double wave_energy; // energy carried by live tracks before more primaries are injected, at most
  long long refill_below, stack_cap;
  long long qcount[3][3]; // records in the interaction buffers [particle][process]
  long long take[3];      // tracks of the current stores handed out to the transport kernels
};

// Tracks handed in as a gx_track_soa (gx_transport_tracks) instead of
// primaries: injected with their state as it is.
struct SoaIn {
  const int *type, *status, *event, *primary, *volume;
  const double *x, *y, *z, *dx, *dy, *dz, *ekin, *nil0, *nil1, *nil2, *msc;
  const uint32_t *rng;
  long long cap;
};

struct Prims {
  const int *type, *event;
  const double *E, *pos, *dir;
  double seed[6];
  long long first_substream;
  const uint64_t *jump;
  int from_soa; // 1: inject the tracks of soa
  SoaIn soa;
};

template <class R> struct Args {
  const Data *d;
  Ctl *ctl;
  Store<R> st[2][3];
  Store<R> stack[3];
  Geom g;
  Prims p;
  double *edep;
  int *pstep;
  int nstores;
  long long refill_below;
  // tracks waiting for an interaction, per particle type and process, stored
  // compactly so the interaction kernels read them coalesced (batched engine)
  Store<R> ibuf[3][3];
  long long qcap;
  int step_budget[3]; // steps of one track per transport launch, at most, per particle type
  int fetch_min[3];   // idle lanes of a warp before it takes new records, per particle type
};

// ---------------------------------------------------------------- geometry
// Component a (the run-time layer axis) of a 3-vector.  Selects instead of an
// indexed access keep the vectors in registers: an array indexed by a run-time
// value lives in local memory.
template <class T> __device__ __forceinline__ T comp(const T *p, int a) { return a == 0 ? p[0] : (a == 1 ? p[1] : p[2]); }
template <class T> __device__ __forceinline__ void set_comp(T *p, int a, T v)
{
  if (a == 0)
    p[0] = v;
  else if (a == 1)
    p[1] = v;
  else
    p[2] = v;
}

// The layered calorimeter along axis a: layer k occupies [x0 + k pitch,
// x0 + (k+1) pitch), absorber first.  vol = 2 layer + slab; -1 outside.
__device__ __forceinline__ int vol_material(const Geom &g, int vol)
{
  if (g.geometry == 2) return g.csg.node[vol].mat;
  return g.geometry == 0 ? g.box_mat : ((vol & 1) ? 2 : 1);
}
__device__ __forceinline__ void slab_bounds(const Geom &g, int vol, double &lo, double &hi)
{
  if (g.geometry == 0) {
    const double c = comp(g.box_centre, g.axis), h = comp(g.box_half, g.axis);
    lo = c - h;
    hi = c + h;
    return;
  }
  double base = g.x0 + (vol >> 1) * g.pitch;
  lo = (vol & 1) ? base + g.t_abs : base;
  hi = (vol & 1) ? base + g.pitch : base + g.t_abs;
}
__device__ __forceinline__ double thalf(const Geom &g, int b) { return g.geometry == 0 ? g.box_half[b] : g.half_trans; }
__device__ __forceinline__ double tcentre(const Geom &g, int b) { return g.geometry == 0 ? g.box_centre[b] : 0.0; }

__device__ __forceinline__ int locate(const Geom &g, const double *p, const double *d)
{
  const double tol = 1e-12;
  int a = g.axis;
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    double h = thalf(g, b), q = p[b] - tcentre(g, b);
    if (q > h || q < -h) return -1;
    if ((q > h - tol && d[b] > 0) || (q < -h + tol && d[b] < 0)) return -1;
  }
  const double pa = comp(p, a), da = comp(d, a);
  if (g.geometry == 0) {
    double q = pa - comp(g.box_centre, a), h = comp(g.box_half, a);
    if (q > h || q < -h) return -1;
    if ((q > h - tol && da > 0) || (q < -h + tol && da < 0)) return -1;
    return 0;
  }
  double u = pa - g.x0;
  if (u < -tol || u > g.total + tol) return -1;
  if ((u < tol && da < 0) || (u > g.total - tol && da > 0)) return -1;
  int layer = (int)floor(u / g.pitch);
  layer = min(max(layer, 0), g.nlayers - 1);
  double q = u - layer * g.pitch;
  if (q < tol && da < 0 && layer > 0) return 2 * (layer - 1) + 1;
  if (q > g.pitch - tol && da > 0 && layer + 1 < g.nlayers) return 2 * (layer + 1);
  if (fabs(q - g.t_abs) < tol) return 2 * layer + (da > 0 ? 1 : 0);
  return 2 * layer + (q < g.t_abs ? 0 : 1);
}

__device__ __forceinline__ double dist_to_out(const Geom &g, int vol, const double *p, const double *d, int &plane)
{
  int a = g.axis;
  double lo, hi, dist = 1.7976931348623157e308;
  slab_bounds(g, vol, lo, hi);
  plane = 0;
  const double pa = comp(p, a), da = comp(d, a);
  if (da > 0) {
    dist = (hi - pa) / da;
    plane = 1;
  } else if (da < 0) {
    dist = (lo - pa) / da;
    plane = -1;
  }
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    double h = thalf(g, b), q = p[b] - tcentre(g, b), t = 1.7976931348623157e308;
    if (d[b] > 0)
      t = (h - q) / d[b];
    else if (d[b] < 0)
      t = (-h - q) / d[b];
    if (t < dist) {
      dist = t;
      plane = 2;
    }
  }
  return dist < 0 ? 0 : dist;
}

// The same distance with one division (the FP32-mixed engine): each plane's
// candidate kept as a fraction num / den with den > 0, candidates compared by
// cross-multiplication in the order the loop above takes them (axis planes
// first, ties to the earlier), and only the nearest divided out.
__device__ __forceinline__ double dist_to_out_1div(const Geom &g, int vol, const double *p, const double *d,
                                                   int &plane)
{
  int a = g.axis;
  double lo, hi;
  slab_bounds(g, vol, lo, hi);
  plane = 0;
  double num = 1.7976931348623157e308, den = 1.0;
  const double pa = comp(p, a), da = comp(d, a);
  if (da > 0) {
    num = hi - pa;
    den = da;
    plane = 1;
  } else if (da < 0) {
    num = pa - lo;
    den = -da;
    plane = -1;
  }
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    const double h = thalf(g, b), q = p[b] - tcentre(g, b);
    double n = 0.0, m = 0.0;
    if (d[b] > 0) {
      n = h - q;
      m = d[b];
    } else if (d[b] < 0) {
      n = h + q;
      m = -d[b];
    }
    if (m > 0 && n * den < num * m) {
      num = n;
      den = m;
      plane = 2;
    }
  }
  const double dist = num / den;
  return dist < 0 ? 0 : dist;
}

__device__ __forceinline__ double safety(const Geom &g, int vol, const double *p)
{
  int a = g.axis;
  double lo, hi;
  slab_bounds(g, vol, lo, hi);
  const double pa = comp(p, a);
  double s = fmin(pa - lo, hi - pa);
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    s = fmin(s, thalf(g, b) - fabs(p[b] - tcentre(g, b)));
  }
  return s < 0 ? 0 : s;
}

__device__ __forceinline__ int next_volume(const Geom &g, int vol, int plane)
{
  if (plane == 2 || g.geometry == 0) return -1;
  int nv = vol + (plane > 0 ? 1 : -1);
  return (nv < 0 || nv >= 2 * g.nlayers) ? -1 : nv;
}

// Volume after a helix sub-step that started in vol.  An end point within
// kSnap of a face it is moving out through (or past it) is put on that face
// and enters the neighbour; otherwise the point is located.  The reference
// pushes 2e-9 mm past the straight-line boundary and locates the helix end
// point, which lands within rounding of the plane often enough for ulp-level
// differences to decide the crossing; the snap distance is far from both.
constexpr double kSnap = 1e-6;
__device__ __forceinline__ int relocate(const Geom &g, int vol, double *p, const double *d)
{
  int a = g.axis;
  double lo, hi;
  slab_bounds(g, vol, lo, hi);
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    if (b == a) continue;
    double h = thalf(g, b), q = p[b] - tcentre(g, b);
    if ((d[b] > 0 && h - q < kSnap) || (d[b] < 0 && q + h < kSnap)) return -1;
  }
  const double pa = comp(p, a), da = comp(d, a);
  if (da > 0 && hi - pa < kSnap) {
    set_comp(p, a, hi);
    return next_volume(g, vol, 1);
  }
  if (da < 0 && pa - lo < kSnap) {
    set_comp(p, a, lo);
    return next_volume(g, vol, -1);
  }
  return locate(g, p, d);
}

// Kernel variants, template parameters so that each kernel carries only the
// code it runs: bit 0 follows the field map (Runge-Kutta sub-steps) instead of
// the uniform field's helix, bit 1 navigates the CSG tree (gx_csg.cuh) instead
// of the analytic volumes above, bit 2 applies multiple scattering, bit 3
// (with bit 1, FP32-mixed kernels) navigates a tree of boxes only: the
// navigator's code for the other solids is left out of those kernels.
enum { kKindFieldMap = 1, kKindCsg = 2, kKindMsc = 4, kKindBoxes = 8 };
template <int K> constexpr int kSolidsOf = (K & kKindBoxes) != 0 ? kSolidsBox : kSolidsAll;

template <int K> __device__ __forceinline__ double nav_safety(const Geom &g, int vol, const double *p)
{
  if constexpr ((K & kKindCsg) != 0)
    return csg_safety<kSolidsOf<K>>(g.csg, vol, p);
  else
    return safety(g, vol, p);
}
// Straight-line distance to the next boundary.  plane: the analytic
// navigator's face code, or the CSG child entered (-1: leaving the volume);
// the CSG navigator skips children met only beyond limit.  ONE_DIV (the
// FP32-mixed engine): the analytic navigator's distance with one division.
template <int K, bool ONE_DIV = false>
__device__ __forceinline__ double nav_distance(const Geom &g, int vol, const double *p, const double *d, double limit,
                                               int &plane)
{
  if constexpr ((K & kKindCsg) != 0)
    return csg_step<kSolidsOf<K>>(g.csg, vol, p, d, limit, plane);
  else if constexpr (ONE_DIV)
    return dist_to_out_1div(g, vol, p, d, plane);
  else
    return dist_to_out(g, vol, p, d, plane);
}
template <int K> __device__ __forceinline__ int nav_relocate(const Geom &g, int vol, double *p, const double *d)
{
  if constexpr ((K & kKindCsg) != 0)
    return csg_locate<kSolidsOf<K>>(g.csg, vol, p, d, kSnap);
  else
    return relocate(g, vol, p, d);
}

// ---------------------------------------------------------- cross sections
// A table lookup of the step: the polynomial form (one record per bin); in
// the parity variant the reference's spline form, as the oracle evaluates it.
template <class R> __device__ __forceinline__ R tab_value(const Data &d, const VecDesc &v, R e)
{
#ifdef GX_PARITY
  static_assert(sizeof(R) == 8, "the parity variant is FP64");
  return vec_value_ref(d, v, e);
#else
  return vec_value_fast<R>(d, v, e);
#endif
}

template <class R> __device__ __forceinline__ R lambda_tab(const Data &d, int t, int mat, R e)
{
  const VecDesc &v = d.vec[t][mat];
  if ((double)e <= v.emin) return R(0);
  return tab_value<R>(d, v, e);
}

// Macroscopic cross sections (1/mm): gamma {Compton, conversion, photo-electric},
// e- {ionisation, brems}, e+ {ionisation, brems, annihilation}.
template <class R> __device__ __forceinline__ void cross_sections(const Data &d, int type, int mat, R e, R xs[3])
{
  xs[0] = xs[1] = xs[2] = R(0);
  if (type == 0) {
    xs[0] = (e < R(1)) ? tab_value<R>(d, d.vec[GX_Lambda_compt][mat], e)
                       : tab_value<R>(d, d.vec[GX_LambdaPrim_compt][mat], e) / e;
    xs[1] = lambda_tab<R>(d, GX_Lambda_conv, mat, e);
    if (e >= R(0.2))
      xs[2] = tab_value<R>(d, d.vec[GX_LambdaPrim_phot][mat], e) / e;
    else if constexpr (sizeof(R) == 4)
      xs[2] = pe_xs_sandia_f(d, (int)d.mat_Z[mat], (float)d.mat_density[mat], e);
    else
      xs[2] = (R)pe_xs_sandia(d, (int)d.mat_Z[mat], d.mat_density[mat], (double)e);
  } else if (type == 1) {
    xs[0] = lambda_tab<R>(d, GX_Lambda_eIoni_em, mat, e);
    xs[1] = lambda_tab<R>(d, GX_Lambda_eBrem_em, mat, e);
  } else {
    xs[0] = lambda_tab<R>(d, GX_Lambda_eIoni_ep, mat, e);
    xs[1] = lambda_tab<R>(d, GX_Lambda_eBrem_ep, mat, e);
    xs[2] = annih_xs<R>(d, mat, e);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (!(xs[i] > R(0))) xs[i] = R(0);
}

// ProxyIonization::AlongStepGPIL in physics mode (Geant4 step function, length
// cut); raw: the range table's value at e, which the step's continuous loss
// reuses (the energy does not change before it)
template <class R> __device__ __forceinline__ R range_limit(const Data &d, int type, int mat, R e, R &raw)
{
#ifdef GX_PARITY
  raw = R(-1);
  return ioni_along_gpil_ref(d, 1, type == 2 ? 1 : -1, mat, e);
#endif
  const R dR = R(0.2), finalRange = R(10.0);
  R range = vec_value_fast<R>(d, d.vec[type == 2 ? GX_Range_ep : GX_Range_em][mat], e);
  raw = range;
  if (e < R(kMinE)) range *= e / R(kMinE);
  R cut = (R)d.cut_length[1][mat];
  R finR = (finalRange < cut) ? finalRange : cut;
  if (range <= finR) return range;
  return range * dR + finR * (R(1) - dR) * (R(2) - finR / range);
}

// ProxyIonization::AlongStepDoIt in physics mode; the inverse range (used when
// the loss exceeds 1%, i.e. near the end of the range) is evaluated in FP64.
// range0 >= 0: the range table's value at e, taken at the start of the step.
template <class R>
__device__ __forceinline__ R along_loss(const Data &d, int type, int mat, double step, R &e, R range0 = R(-1))
{
#ifdef GX_PARITY
  double edep = 0.0, ee = e;
  ioni_along_doit_ref(d, 1, type == 2 ? 1 : -1, mat, step, ee, edep);
  e = ee;
  return edep;
#endif
  bool ep = type == 2;
  R energy = e;
  R range = range0 >= R(0) ? range0 : vec_value_fast<R>(d, d.vec[ep ? GX_Range_ep : GX_Range_em][mat], energy);
  if (step >= (double)range || energy <= R(kMinE)) {
    e = R(0);
    return energy;
  }
  R dedx = vec_value_fast<R>(d, d.vec[ep ? GX_DEDX_eIoni_ep : GX_DEDX_eIoni_em][mat], energy);
  if (energy < R(kMinE)) dedx *= M<R>::sqrt(energy / R(kMinE));
  R eloss = (R)step * dedx;
  if (eloss > energy * R(0.01)) {
    const VecDesc &vr = d.vec[ep ? GX_Range_ep : GX_Range_em][mat];
    const VecDesc &vi = d.vec[ep ? GX_InverseRange_ep : GX_InverseRange_em][mat];
    if constexpr (sizeof(R) == 4) {
      // the FP32-mixed engine: bin from the FP32 logarithm, one reciprocal
      const double r64 = vec_value_f64_f32bin(d, vr, (double)energy) - step;
      eloss = (R)((double)energy - vec_invrange_fast(d, vi, r64));
    } else {
      const double r64 = vec_value_fast<double>(d, vr, (double)energy) - step;
      eloss = (R)((double)energy - vec_invrange_ref(d, vi, r64));
    }
  }
  R finalE = energy - eloss;
  if (finalE < R(kMinE)) {
    eloss += finalE;
    finalE = R(0);
  }
  e = finalE;
  return eloss > R(0) ? eloss : R(0);
}

// ---------------------------------------------------------------- one step
template <class R> struct Track {
  int type, vol, event, prim;
  double pos[3];
  R dir[3], E, nil[3];
  R msc_r0;       // multiple scattering: range scale of the step limit in this volume (<= 0: unset)
  uint32_t rs[6]; // MRG32k3a state words; draws go through a Mrg made from them (rng / set_rng)
  __device__ __forceinline__ Mrg rng() const
  {
    Mrg m;
    m.from_words(rs);
    return m;
  }
  __device__ __forceinline__ void set_rng(const Mrg &m) { m.to_words(rs); }
  __device__ __forceinline__ void load_rng(const uint32_t *st, long long n, long long i)
  {
#pragma unroll
    for (int k = 0; k < 6; ++k) rs[k] = __ldg(&st[k * n + i]);
  }
  __device__ __forceinline__ void store_rng(uint32_t *st, long long n, long long i) const
  {
#pragma unroll
    for (int k = 0; k < 6; ++k) st[k * n + i] = rs[k];
  }
};

struct Local {
  // deposits go to a shared-memory tally when it fits, else to global memory
  double *sm_edep;
  double *g_edep;
  double *sm_esc; // this block's [escaped, retired] energy sums (shared memory)
  int nvol, nevents, sm_bins;
  double retired; // energy this thread took out of the live tracks (deposited or escaped)
  unsigned int st[kNStat];
  int err;
  __device__ __forceinline__ void escape(double e)
  {
    retired += e;
    atomicAdd(sm_esc, e);
  }
  __device__ __forceinline__ void deposit(int event, int vol, double e)
  {
    retired += e;
    if (vol < 0 || vol >= nvol || e == 0.0) return;
    if (event < 0 || event >= nevents) { // a primary with an event index outside the tally
      err |= kErrEvent;
      return;
    }
    int bin = event * nvol + vol;
    if (bin < sm_bins)
      atomicAdd(&sm_edep[bin], e);
    else
      atomicAdd(&g_edep[bin], e);
  }
};

template <class R> struct Secs {
  int n;
  int type[2];
  R E[2], dir[2][3];
  // slot chosen by a branch, not an index, so the record stays in registers
  __device__ __forceinline__ void add(int ty, R e, const R *u)
  {
    if (n == 0) {
      type[0] = ty;
      E[0] = e;
      dir[0][0] = u[0];
      dir[0][1] = u[1];
      dir[0][2] = u[2];
    } else {
      type[1] = ty;
      E[1] = e;
      dir[1][0] = u[0];
      dir[1][1] = u[1];
      dir[1][2] = u[2];
    }
    ++n;
  }
};

// One helix sub-step of length s in a uniform field along z: the reference's
// ConstFieldHelixStepper::DoStep (magneticfield/ConstFieldHelixStepper.hpp:164-239)
// with B = (0, 0, Bz) substituted, where the field-direction terms vanish.
// With rn = p / (kB2C q |Bz|) (signed), phi = -s / rn and sB = sign(Bz):
//   x' = x + rn ((cos phi - 1) dy sB - sin phi dx),   dx' = cos phi dx + sin phi dy sB
//   y' = y + rn (-(cos phi - 1) dx sB - sin phi dy),  dy' = cos phi dy - sin phi dx sB
//   z' = z + s dz,                                     dz' = dz
// (the reference's R v equals rn (dx, dy) since sinVB = |(dx, dy)|), with
// cos phi - 1 = -2 sin^2(phi / 2), free of cancellation at small bending
// angles.  The rotation and the transverse displacement are computed in T, the
// displacement is added to the FP64 position.
__device__ __forceinline__ void sincos_t(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void sincos_t(double x, double *s, double *c) { ::sincos(x, s, c); }

template <class T>
__device__ __forceinline__ void helix_bz(T rn, T sB, double s, const double pos[3], const T dir[3], double np[3],
                                         T nd[3])
{
  const T phi = -(T)s / rn;
  T sh, ch;
  sincos_t(T(0.5) * phi, &sh, &ch);
  const T sinp = T(2) * sh * ch, cm1 = T(-2) * sh * sh, cosp = T(1) + cm1;
  np[0] = pos[0] + (double)(rn * (cm1 * dir[1] * sB - sinp * dir[0]));
  np[1] = pos[1] + (double)(rn * (-cm1 * dir[0] * sB - sinp * dir[1]));
  np[2] = pos[2] + s * (double)dir[2];
  nd[0] = cosp * dir[0] + sinp * dir[1] * sB;
  nd[1] = cosp * dir[1] - sinp * dir[0] * sB;
  nd[2] = dir[2];
}

template <class R>
__device__ __forceinline__ void run_model(const Data &d, const Geom &g, Track<R> &t, int proc, Secs<R> &sec,
                                          Local &L)
{
  int mat = vol_material(g, t.vol);
  ModelParams mp;
  mp.mode = 1;
  mp.Z = (int)d.mat_Z[mat];
  mp.cut = 0.0;
  mp.density_factor = d.mat_dfactor[mat];
  mp.sb = d.sb + ((mat == 1) ? 2 : 1);
  Inter<R> io;
  io.E = t.E;
  io.dir[0] = t.dir[0];
  io.dir[1] = t.dir[1];
  io.dir[2] = t.dir[2];
  io.edep = R(0);
  io.status = 0;
  io.nsec = 0;
  int err = 0;
  Mrg rng = t.rng();
  if (t.type == 0) {
    if (proc == 0)
      kn_sample(rng, mp, io, &err);
    else if (proc == 1) {
      bh_sample(rng, mp, io, &err);
      if (io.nsec == 2) L.st[S_PAIR]++;
    } else
      sg_sample(rng, d, mp, io, &err);
  } else if (proc == 0) {
    mp.cut = d.cut_energy[1][mat];
    if (t.type == 1)
      mb_sample(rng, mp, io, &err);
    else
      bhabha_sample(rng, mp, io, &err);
  } else if (proc == 1) {
    mp.cut = d.cut_energy[0][mat];
    sb_sample(rng, mp, io, &err);
  } else {
    annih_sample(rng, io, &err);
    L.st[S_ANNIH]++;
  }
  t.set_rng(rng);
  if (err) {
    L.err |= err;
    L.st[S_ERR]++;
  }
  L.deposit(t.event, t.vol, (double)io.edep);
  t.E = io.E;
  t.dir[0] = io.dir[0];
  t.dir[1] = io.dir[1];
  t.dir[2] = io.dir[2];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    if (s >= io.nsec) break;
    if (g.charged_local && io.sec_type[s] != 0) {
      L.deposit(t.event, t.vol, (double)io.sec_E[s]);
      continue;
    }
    sec.add(io.sec_type[s], io.sec_E[s], io.sec_dir[s]);
  }
  if (io.status == 1) t.E = R(0);
}

// ------------------------------------------------------- multiple scattering
// Multiple scattering of e-/e+ (config msc = 1, or 2 with lateral
// displacement): the Urban model as published
// (L. Urban, CERN-OPEN-2006-077); the reference has only a placeholder
// (proxy/ProxyScattering.hpp:53-71) and ships the transport mean free path
// tables (LambdaMod1.msc: E^2 / lambda1).  The oracle restates the same model
// in the same order of random draws.
//   step limit: t <= max(0.04 r0, 0.6 safety, 1e-5 mm), r0 = max(range,
//     lambda1) at the first step in each volume;
//   paths: geometric z = lambda1 (1 - exp(-t / lambda1)) from the true length t,
//     and back when a boundary stops the step;
//   deflection after the along-step loss: cos(theta) from the model's mixture
//     of a central exponential part (Highland-type width theta0), a power tail
//     and a uniform part, weighted so that <cos theta> = exp(-tau); where the
//     published weights would need a uniform part above 1 it is dropped and
//     the central / tail split keeps that mean; phi uniform;
//   lateral displacement (msc = 2), after a step that ends inside its volume:
//     r = 0.73 r_max, r_max = sqrt(t^2 - z^2) the largest displacement the
//     true and geometric lengths allow (the fixed fraction of early versions
//     of the model), perpendicular to the direction at the start of the step,
//     at the azimuth of the deflection (the displacement follows the turn),
//     cut to 0.99 of the safety at the end point so that it never crosses a
//     boundary, and none within 1e-5 mm of one.
// Not modelled: the e+ correction of theta0.
constexpr double kMscFr = 0.04, kMscFs = 0.6, kMscTmin = 1.0e-5;
constexpr double kMscTauBig = 8.0, kMscTauSmall = 1.0e-16, kMscTauLim = 1.0e-6;

// transport mean free path lambda1 (mm); 0 when the table has nothing
template <class R> __device__ __forceinline__ R msc_lambda1(const Data &d, int type, int mat, R e)
{
  const R v = tab_value<R>(d, d.vec[type == 2 ? GX_LambdaMod1_msc_ep : GX_LambdaMod1_msc_em][mat], e);
  return v > R(0) ? e * e / v : R(0);
}

template <class R> __device__ __forceinline__ R msc_expm1(R x);
template <> __device__ __forceinline__ float msc_expm1(float x) { return expm1f(x); }
template <> __device__ __forceinline__ double msc_expm1(double x) { return dexpm1(x); }
template <class R> __device__ __forceinline__ R msc_log1p(R x);
template <> __device__ __forceinline__ float msc_log1p(float x) { return log1pf(x); }
template <> __device__ __forceinline__ double msc_log1p(double x) { return dlog1p(x); }

template <class R> __device__ __forceinline__ double msc_true_to_geom(double t, R lam)
{
  const R tau = (R)t / lam;
  return tau < R(kMscTauLim) ? t : -(double)lam * (double)msc_expm1<R>(-tau);
}

template <class R> __device__ __forceinline__ double msc_geom_to_true(double z, R lam, double tmax)
{
  const R x = (R)z / lam;
  if (x < R(kMscTauLim)) return z;
  const double t = x < R(1) ? -(double)lam * (double)msc_log1p<R>(-x) : tmax;
  return t < tmax ? t : tmax;
}

// the model's two-function form for large angles: exact first and second moments
template <class R> __device__ __forceinline__ R msc_simple(Mrg &rng, R xm, R x2m)
{
  const R a = (R(2) * xm + R(9) * x2m - R(3)) / (R(2) * xm - R(3) * x2m + R(1));
  const R prob = (a + R(2)) * xm / a;
  const R r0 = rng.template u<R>(), r1 = rng.template u<R>();
  if (r0 < prob) return R(-1) + R(2) * M<R>::exp(M<R>::log(r1) / (a + R(1)));
  return R(-1) + R(2) * r1;
}

// cos(theta) after a true path t; lam0 / lam1 and e0 / e1 at the start and
// the end of the step; c = the material's constants {X0, th1, th2, ca..cd}
template <class R>
__device__ __forceinline__ R msc_cos_theta(Mrg &rng, const double *c, R t, R lam0, R lam1, R e0, R e1)
{
  R tau = t / lam0;
  if (lam1 > R(0) && fabs(lam1 - lam0) > R(0.01) * lam0) tau = t * M<R>::log(lam0 / lam1) / (lam0 - lam1);
  if (tau >= R(kMscTauBig)) return R(-1) + R(2) * rng.template u<R>();
  if (tau < R(kMscTauSmall)) return R(1);
  R xm, x2m;
  if (tau < R(0.01)) {
    xm = R(1) - tau * (R(1) - R(0.5) * tau);
    x2m = R(1) - tau * (R(5) - R(6.25) * tau) / R(3);
  } else {
    xm = M<R>::exp(-tau);
    x2m = (R(1) + R(2) * M<R>::exp(R(-2.5) * tau)) / R(3);
  }
  if (R(1) - e1 / e0 > R(0.5)) return msc_simple<R>(rng, xm, x2m);
  const R m = R(kEMass);
  const R inv0 = (e0 + m) / (e0 * (e0 + R(2) * m)), inv1 = (e1 + m) / (e1 * (e1 + R(2) * m));
  const R X0 = (R)c[0], y = t / X0;
  const R th0 = R(13.6) * M<R>::sqrt(y) * M<R>::sqrt(inv0 * inv1) * ((R)c[1] + (R)c[2] * M<R>::log(y));
  const R th2 = th0 * th0;
  if (th2 < R(kMscTauSmall)) return R(1);
  if (th0 > R(kPi / 6)) return msc_simple<R>(rng, xm, x2m);
  R x = th2 * (R(1) - th2 / R(12));
  if (th2 > R(0.01)) {
    const R s = R(2) * M<R>::sinr(R(0.5) * th0);
    x = s * s;
  }
  const R u = M<R>::exp(M<R>::log(tau) / R(6));
  R xsi = (R)c[3] + u * ((R)c[4] + (R)c[5] * u) + (R)c[6] * M<R>::log((t / tau) / X0);
  if (xsi < R(1.9)) xsi = R(1.9);
  R cc = xsi;
  if (fabs(cc - R(3)) < R(0.001))
    cc = R(3.001);
  else if (fabs(cc - R(2)) < R(0.001))
    cc = R(2.001);
  const R c1 = cc - R(1);
  const R ea = M<R>::exp(-xsi), eaa = R(1) - ea;
  const R xmean1 = R(1) - (R(1) - (R(1) + xsi) * ea) * x / eaa;
  if (xmean1 <= R(0.999) * xm) return msc_simple<R>(rng, xm, x2m);
  const R x0 = R(1) - xsi * x;
  const R b = R(1) + (cc - xsi) * x, b1 = b + R(1), bx = cc * x;
  const R dd = M<R>::exp(c1 * M<R>::log(bx)) / M<R>::exp(c1 * M<R>::log(b1));
  const R xmean2 = (x0 + dd - (bx - b1 * dd) / (cc - R(2))) / (R(1) - dd);
  const R f1x0 = ea / eaa, f2x0 = c1 / (cc * (R(1) - dd));
  R prob = f2x0 / (f1x0 + f2x0);
  R qprob = xm / (prob * xmean1 + (R(1) - prob) * xmean2);
  if (qprob > R(1)) {
    qprob = R(1);
    prob = (xm - xmean2) / (xmean1 - xmean2);
  }
  const R r0 = rng.template u<R>(), r1 = rng.template u<R>();
  if (r0 < qprob) {
    if (r1 < prob) return R(1) + M<R>::log(ea + rng.template u<R>() * eaa) * x;
    R var = (R(1) - dd) * rng.template u<R>();
    if (var < R(0.01) * dd) {
      var /= dd * c1;
      return R(-1) + var * (R(1) - R(0.5) * var * cc) * (R(2) + (cc - xsi) * x);
    }
    return R(1) + x * (cc - xsi - cc * M<R>::exp(-M<R>::log(var + dd) / c1));
  }
  return R(-1) + R(2) * r1;
}

// deflect the direction by the sampled angle (no draw for phi when it is 0)
template <class R>
// Returns false when the direction is kept (no azimuth drawn); sp, cp: the
// azimuth of the deflection.
__device__ __forceinline__ bool msc_deflect(const Data &d, Track<R> &t, int mat, R step, R lam0, R e0, R &sp, R &cp)
{
  const R lam1 = msc_lambda1<R>(d, t.type, mat, t.E);
  Mrg rng = t.rng();
  R ct = msc_cos_theta<R>(rng, d.mat_msc[mat], step, lam0, lam1, e0, t.E);
  if (!(ct < R(1))) {
    t.set_rng(rng);
    return false;
  }
  if (ct < R(-1)) ct = R(-1);
  const R st = M<R>::sqrt((R(1) - ct) * (R(1) + ct));
  M<R>::sincos2pi(rng.template u<R>(), &sp, &cp);
  t.set_rng(rng);
  R u = st * cp, v = st * sp, w = ct;
  rotate_to_lab(u, v, w, t.dir[0], t.dir[1], t.dir[2]);
  t.dir[0] = u;
  t.dir[1] = v;
  t.dir[2] = w;
  return true;
}

// The lateral displacement of a multiple-scattering step that ended inside
// its volume (config msc = 2): 0.73 sqrt(t^2 - z^2) perpendicular to the
// step's starting direction (d0, d1, d2) at the deflection's azimuth, cut to
// 0.99 of the safety at the end point, none within kMscTmin of a boundary.
// Out of line: the common path (msc 0 or 1) carries only the call.
template <class R, int K>
__device__ __noinline__ double3 msc_displacement(const Geom &g, int vol, double x, double y, double z, double t,
                                                 double zg, R cp, R sp, R d0, R d1, R d2)
{
  double3 out = make_double3(0.0, 0.0, 0.0);
  const double rmax2 = (t - zg) * (t + zg);
  if (!(rmax2 > 0.0)) return out;
  const double p[3] = {x, y, z};
  const double saf = nav_safety<K>(g, vol, p);
  if (!(saf > kMscTmin)) return out;
  const double r = fmin(0.73 * sqrt(rmax2), 0.99 * saf);
  R u = cp, v = sp, w = R(0);
  rotate_to_lab(u, v, w, d0, d1, d2);
  out.x = r * (double)u;
  out.y = r * (double)v;
  out.z = r * (double)w;
  return out;
}

enum { kDone = 0, kAlive = 1, kInteract = 2 };

// One OneStep (test_BasicCpuTransport.cpp:408-497 / InnerStep :358-403) in
// physics mode, up to the choice of the post-step interaction, in three
// phases so that a kernel can interleave tracks at different points of their
// steps: step_begin (GPIL and the step limit; a straight-line move completes
// here), field_substep (one helix sub-step, repeated until the step ends) and
// step_end (NIL update, continuous loss, outcome).  The state carried from one
// phase to the next:
template <class R> struct StepCtx {
  // macroscopic cross sections at the start of the step (scalars: an array
  // member of a structure that lives across loop passes ends up in local
  // memory)
  R xs0, xs1, xs2;
  double remaining; // helix: length of the step still to go
  double total;     // length travelled in this step
  int sel;          // process that limits the step (-1: none)
  int vol0;         // volume at the start of the step
  int newvol;       // volume entered (-2: sub-step cap hit)
  int nsub;         // helix sub-steps taken
  bool crossed;     // the step ended on a boundary
  // multiple scattering (lam0 > 0 when it applies to this step): transport
  // mean free path and energy at the start, the step's true length
  R lam0, e0;
  double ttrue;
  R range0; // charged: the range table's value at the step's energy (-1: none)
  __device__ __forceinline__ R xs(int i) const { return i == 0 ? xs0 : (i == 1 ? xs1 : xs2); }
};

// A photon's cross sections in the two calorimeter materials while its energy
// does not change (it stays in a transport kernel until it interacts):
// computed at its first step in each material, reused after.
template <class R> struct GammaXs {
  R pb0, pb1, pb2, ar0, ar1, ar2;
  int have; // bit 0: lead (material 1), bit 1: argon (material 2)
};

// GPIL and step limit (PostStepGPIL of the discrete processes, the range and
// multiple-scattering limits): returns the step to move (geometric length),
// and sets the step context.  gx, when given, caches a photon's cross
// sections per material.
template <class R, int K>
__device__ __forceinline__ R step_gpil(const Data &d, const Geom &g, Track<R> &t, StepCtx<R> &c,
                                       GammaXs<R> *gx = nullptr)
{
  const int mat = vol_material(g, t.vol);
  const int np = (t.type == 1) ? 2 : 3;
  const bool charged = t.type != 0;
  R xs[3];
  if (gx && mat == 1 && (gx->have & 1)) {
    xs[0] = gx->pb0;
    xs[1] = gx->pb1;
    xs[2] = gx->pb2;
  } else if (gx && mat == 2 && (gx->have & 2)) {
    xs[0] = gx->ar0;
    xs[1] = gx->ar1;
    xs[2] = gx->ar2;
  } else {
    cross_sections<R>(d, t.type, mat, t.E, xs);
    if (gx && mat == 1) {
      gx->pb0 = xs[0];
      gx->pb1 = xs[1];
      gx->pb2 = xs[2];
      gx->have |= 1;
    } else if (gx && mat == 2) {
      gx->ar0 = xs[0];
      gx->ar1 = xs[1];
      gx->ar2 = xs[2];
      gx->have |= 2;
    }
  }
  c.xs0 = xs[0];
  c.xs1 = xs[1];
  c.xs2 = xs[2];
  // loops over the three process slots are unrolled with the bound as a guard,
  // so xs[] and nil[] are indexed by constants and stay in registers
  bool draw = false;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (i < np && t.nil[i] <= R(0)) draw = true;
  if (draw) {
    Mrg rng = t.rng();
#pragma unroll
    for (int i = 0; i < 3; ++i)
      if (i < np && t.nil[i] <= R(0)) t.nil[i] = -M<R>::log(rng.template u<R>());
    t.set_rng(rng);
  }
  R pstep = R(3.0e38);
  int sel = -1;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (i < np && xs[i] > R(0)) {
      R s = t.nil[i] / xs[i];
      if (s < pstep) {
        pstep = s;
        sel = i;
      }
    }
  c.range0 = R(-1);
  if (charged) {
    R slim = range_limit<R>(d, t.type, mat, t.E, c.range0);
    if (slim < pstep) {
      pstep = slim;
      sel = -1;
    }
  }
  // multiple scattering: its step limit, then the true step becomes the
  // geometric length to move
  c.lam0 = R(0);
  c.e0 = t.E;
  if ((K & kKindMsc) != 0 && charged) {
    const R lam0 = msc_lambda1<R>(d, t.type, mat, t.E);
    if (t.msc_r0 <= R(0)) {
      R range = tab_value<R>(d, d.vec[t.type == 2 ? GX_Range_ep : GX_Range_em][mat], t.E);
      if (t.E < R(kMinE)) range *= t.E / R(kMinE);
      t.msc_r0 = range > lam0 ? range : lam0;
    }
    const double tlim = fmax(fmax(kMscFr * (double)t.msc_r0, kMscFs * nav_safety<K>(g, t.vol, t.pos)), kMscTmin);
    if (tlim < (double)pstep) {
      pstep = (R)tlim;
      sel = -1;
    }
    c.ttrue = (double)pstep;
    if (lam0 > R(0)) {
      c.lam0 = lam0;
      pstep = (R)msc_true_to_geom<R>((double)pstep, lam0);
    }
  }
  c.sel = sel;
  c.vol0 = t.vol;
  c.newvol = t.vol;
  c.crossed = false;
  c.nsub = 0;
  return pstep;
}

// The start of the move by pstep: true when the step continues with helix
// sub-steps (a charged track in a field); otherwise the straight move to pstep
// or the first boundary is made here and false returned.
template <class R, int K>
__device__ __forceinline__ bool step_move_begin(const Geom &g, Track<R> &t, StepCtx<R> &c, R pstep)
{
  if (t.type != 0 && (g.Bz != 0.0 || g.field_map)) {
    c.remaining = (double)pstep;
    c.total = 0.0;
    return true;
  }
  int plane;
  double dir[3] = {(double)t.dir[0], (double)t.dir[1], (double)t.dir[2]};
  double ps = (double)pstep;
  double dd = nav_distance<K, sizeof(R) == 4>(g, t.vol, t.pos, dir, ps, plane);
  if (dd < ps) {
    c.total = dd;
    c.crossed = true;
    if constexpr ((K & kKindCsg) != 0) {
      for (int k = 0; k < 3; ++k) t.pos[k] += dd * dir[k];
      c.newvol = csg_cross<kSolidsOf<K>>(g.csg, t.vol, plane, t.pos, dir);
    } else {
      c.newvol = next_volume(g, t.vol, plane);
      for (int k = 0; k < 3; ++k) t.pos[k] += dd * dir[k];
      if (plane != 2) {
        double lo, hi;
        slab_bounds(g, t.vol, lo, hi);
        set_comp(t.pos, g.axis, plane > 0 ? hi : lo);
      }
    }
  } else {
    c.total = ps;
    for (int k = 0; k < 3; ++k) t.pos[k] += ps * dir[k];
  }
  return false;
}

// GPIL, step limit and the start of the move.  Returns true when the step
// continues with helix sub-steps (a charged track in a field), false when it
// is complete.
template <class R, int K>
__device__ __forceinline__ bool step_begin(const Data &d, const Geom &g, Track<R> &t, StepCtx<R> &c,
                                           GammaXs<R> *gx = nullptr)
{
  const R pstep = step_gpil<R, K>(d, g, t, c, gx);
  return step_move_begin<R, K>(g, t, c, pstep);
}

// One helix sub-step in Bz (FieldPropagationHandler::Propagate /
// PropagateInVolume, magneticfield/src/FieldPropagationHandler.cpp:87-360).
// Positions, the geometry and the step bookkeeping are FP64; the direction,
// the momentum and the sub-step length heuristic are in R (FP32 in the mixed
// build).  Returns true when the step is complete (boundary reached, length
// used up, or the cap of 10000 sub-steps hit: then newvol = -2).
// One classical fourth-order Runge-Kutta step of length s through the field
// map (FP64): position x and unit direction u with du/ds = k u x B(x),
// k = 0.299792458 q / p (MeV, T, mm); four map lookups, direction renormalised.
__device__ __forceinline__ void rk4_map_step(const float4 *__restrict__ fmap, double k, double s, double x[3],
                                             double u[3], const double B0[3])
{
  double xs[3], us[3], B[3], kx[4][3], ku[4][3];
  const double h[3] = {0.5 * s, 0.5 * s, s};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    kx[0][j] = u[j];
  }
  ku[0][0] = k * (u[1] * B0[2] - u[2] * B0[1]);
  ku[0][1] = k * (u[2] * B0[0] - u[0] * B0[2]);
  ku[0][2] = k * (u[0] * B0[1] - u[1] * B0[0]);
#pragma unroll
  for (int st = 1; st < 4; ++st) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      xs[j] = x[j] + h[st - 1] * kx[st - 1][j];
      us[j] = u[j] + h[st - 1] * ku[st - 1][j];
    }
    field_map_value(fmap, xs, B);
#pragma unroll
    for (int j = 0; j < 3; ++j) kx[st][j] = us[j];
    ku[st][0] = k * (us[1] * B[2] - us[2] * B[1]);
    ku[st][1] = k * (us[2] * B[0] - us[0] * B[2]);
    ku[st][2] = k * (us[0] * B[1] - us[1] * B[0]);
  }
  double m = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    x[j] += s / 6.0 * (kx[0][j] + 2.0 * kx[1][j] + 2.0 * kx[2][j] + kx[3][j]);
    u[j] += s / 6.0 * (ku[0][j] + 2.0 * ku[1][j] + 2.0 * ku[2][j] + ku[3][j]);
    m += u[j] * u[j];
  }
  m = 1.0 / ::sqrt(m);
  u[0] *= m;
  u[1] *= m;
  u[2] *= m;
}

// One sub-step through the field map: the sub-step length from the same
// geometry and sagitta limits as the helix (with the field at the start
// point), then a Runge-Kutta step.  Returns the length moved.
template <class R>
__device__ __forceinline__ double field_map_substep(const Data &d, const Geom &g, Track<R> &t, double remaining,
                                                    double saf, double snext)
{
  const double eps = 0.1, charge = (t.type == 1) ? -1.0 : 1.0;
  const double E = (double)t.E, p = ::sqrt(E * (E + 2.0 * kEMass));
  double B0[3], u[3] = {(double)t.dir[0], (double)t.dir[1], (double)t.dir[2]};
  field_map_value(d.fmap, t.pos, B0);
  const double cx = u[1] * B0[2] - u[2] * B0[1], cy = u[2] * B0[0] - u[0] * B0[2], cz = u[0] * B0[1] - u[1] * B0[0];
  const double bperp = ::sqrt(cx * cx + cy * cy + cz * cz); // |u x B|
  double step_field = 1.7976931348623157e308;
  if (bperp > 0.0) step_field = fmax(2.0 * ::sqrt(eps * p / (0.299792458 * bperp)), saf);
  const double step_gp = fmax(fmin(remaining, 1e-4), snext);
  const double s = fmin(fmin(step_gp, step_field), remaining);
  if (bperp > 0.0) {
    rk4_map_step(d.fmap, 0.299792458 * charge / p, s, t.pos, u, B0);
    for (int k = 0; k < 3; ++k) t.dir[k] = (R)u[k];
  } else {
    for (int k = 0; k < 3; ++k) t.pos[k] += s * u[k];
  }
  return s;
}

// K: the kernel variant (kKindFieldMap, kKindCsg, kKindMsc bits).
template <class R, int K>
__device__ __forceinline__ bool field_substep(const Data &d, const Geom &g, Track<R> &t, StepCtx<R> &c, Local &L)
{
  const R eps = R(0.1); // gEpsDeflection = 1e-2 cm
  const R charge = (t.type == 1) ? R(-1) : R(1);
  const R p = M<R>::sqrt(t.E * (t.E + R(2.0 * kEMass)));
  const R absB = (R)fabs(g.Bz), sB = g.Bz >= 0.0 ? R(1) : R(-1);
  const R curv_per_pt = R(0.299792458) * absB; // 1 / radius = curv_per_pt / pt
  int plane;
  double dd[3] = {(double)t.dir[0], (double)t.dir[1], (double)t.dir[2]};
  const double remaining = c.remaining;
  double saf = nav_safety<K>(g, t.vol, t.pos);
  double snext = (saf > remaining)
                     ? remaining
                     : fmax(2e-9, fmin(nav_distance<K, sizeof(R) == 4>(g, t.vol, t.pos, dd, remaining, plane),
                                       remaining) + 2e-9);
  double s;
  if constexpr ((K & kKindFieldMap) != 0) {
    s = field_map_substep<R>(d, g, t, remaining, saf, snext);
  } else {
  double step_gp = fmax(fmin(remaining, 1e-4), snext);
  R pt = p * M<R>::sqrt(fmax(R(1) - t.dir[2] * t.dir[2], R(0)));
  double step_field = 1.7976931348623157e308;
#ifdef GX_PARITY
  // the oracle's form: the sagitta length from the curvature, the general
  // helix step, the direction renormalised by division
  if (pt > 0.0) {
    const double curv = 0.299792458 * fabs(g.Bz) / pt;
    step_field = fmax(2.0 * ::sqrt(eps / curv), saf);
  }
  s = fmin(fmin(step_gp, step_field), remaining);
  if (pt > 0.0) {
    const double B[3] = {0.0, 0.0, g.Bz};
    double np[3], nd[3];
    helix_dostep(kB2C_mm, B, t.pos, t.dir, (double)charge, p, s, np, nd);
    const double m = ::sqrt(nd[0] * nd[0] + nd[1] * nd[1] + nd[2] * nd[2]);
    for (int k = 0; k < 3; ++k) {
      t.pos[k] = np[k];
      t.dir[k] = nd[k] / m;
    }
  } else {
    for (int k = 0; k < 3; ++k) t.pos[k] += s * dd[k];
  }
#else
  if (pt > R(0)) step_field = fmax(2.0 * (double)M<R>::sqrt(eps * pt / curv_per_pt), saf);
  s = fmin(fmin(step_gp, step_field), remaining);
  if (pt > R(0)) {
    const R rn = p / (R(kB2C_mm) * charge * absB);
    double np[3];
    R nd[3];
    helix_bz<R>(rn, sB, s, t.pos, t.dir, np, nd);
    const R inv = R(1) / M<R>::sqrt(nd[0] * nd[0] + nd[1] * nd[1] + nd[2] * nd[2]);
    for (int k = 0; k < 3; ++k) {
      t.pos[k] = np[k];
      t.dir[k] = nd[k] * inv;
    }
  } else {
    for (int k = 0; k < 3; ++k) t.pos[k] += s * dd[k];
  }
#endif
  }
  c.total += s;
  c.remaining = remaining - s;
  L.st[S_SUBSTEPS]++;
  dd[0] = (double)t.dir[0];
  dd[1] = (double)t.dir[1];
  dd[2] = (double)t.dir[2];
  int v = nav_relocate<K>(g, t.vol, t.pos, dd);
  if (v != t.vol || c.remaining <= 1e-10) {
    if (v != t.vol) {
      c.crossed = true;
      c.newvol = v;
    }
    return true;
  }
  if (++c.nsub >= 10000) {
    L.err |= kErrFieldCap;
    L.st[S_ERR]++;
    c.crossed = true;
    c.newvol = -2;
    return true;
  }
  return false;
}

// NIL update, continuous loss and the outcome of the step: kDone (track
// finished), kAlive (no interaction this step) or kInteract with *proc set
// (for a stopped e+, proc 2 = annihilation at rest, at E = 0).
template <class R, int K>
__device__ __forceinline__ int step_end(const Data &d, const Geom &g, Track<R> &t, const StepCtx<R> &c, Local &L,
                                        int *proc)
{
  const int np = (t.type == 1) ? 2 : 3;
  // the true length of the step: all of it, or back from where a boundary
  // stopped it
  const bool msc = (K & kKindMsc) != 0 && c.lam0 > R(0); // multiple scattering applied to this step
  const double step = msc ? (c.crossed ? msc_geom_to_true<R>(c.total, c.lam0, c.ttrue) : c.ttrue) : c.total;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (i < np) t.nil[i] -= (R)step * c.xs(i);
  L.st[S_STEPS]++;
  if (c.newvol == -2) {
    L.deposit(t.event, c.vol0, (double)t.E);
    return kDone;
  }
  if (t.type != 0) {
    R eloss = along_loss<R>(d, t.type, vol_material(g, c.vol0), step, t.E, c.range0);
    L.deposit(t.event, c.vol0, (double)eloss);
    if (t.E <= R(0)) {
      if (t.type == 2) {
        int v = c.crossed ? c.newvol : c.vol0;
        if (v >= 0) {
          t.vol = v;
          t.E = R(0);
          *proc = 2;
          return kInteract;
        }
        L.escape(2.0 * kEMass);
      }
      return kDone;
    }
    if (msc) {
      const R d0 = t.dir[0], d1 = t.dir[1], d2 = t.dir[2]; // the direction the step started in
      R sp, cp;
      const bool turned = msc_deflect<R>(d, t, vol_material(g, c.vol0), (R)step, c.lam0, c.e0, sp, cp);
      if (g.msc == 2 && turned && !c.crossed) {
        const double3 dx =
            msc_displacement<R, K>(g, t.vol, t.pos[0], t.pos[1], t.pos[2], step, c.total, cp, sp, d0, d1, d2);
        t.pos[0] += dx.x;
        t.pos[1] += dx.y;
        t.pos[2] += dx.z;
      }
    }
  }
  if (c.crossed) {
    t.msc_r0 = R(-1); // a new volume: the step limit starts again
    t.vol = c.newvol;
    if (c.newvol < 0) {
      L.escape((double)t.E + ((t.type == 2) ? 2.0 * kEMass : 0.0));
      return kDone;
    }
    return kAlive;
  }
  if (c.sel >= 0) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
      if (i == c.sel) t.nil[i] = R(-1);
    *proc = c.sel;
    return kInteract;
  }
  return kAlive;
}

// The three phases in sequence: one whole step up to the interaction.
template <class R, int K>
__device__ __forceinline__ int transport_part(const Data &d, const Geom &g, Track<R> &t, Local &L,
                                                                 int *proc)
{
  StepCtx<R> c;
  if (step_begin<R, K>(d, g, t, c))
    while (!field_substep<R, K>(d, g, t, c, L)) {
    }
  return step_end<R, K>(d, g, t, c, L, proc);
}

// The whole OneStep, interaction included (the fused form the plain loop
// runs); the oracle's one_step is the same algorithm in the same order of
// random draws.  Returns false when the track is finished.
template <class R, int K>
__device__ bool one_step(const Data &d, const Geom &g, Track<R> &t, Secs<R> &sec, Local &L)
{
  sec.n = 0;
  int proc = -1;
  int r = transport_part<R, K>(d, g, t, L, &proc);
  if (r == kInteract) {
    run_model(d, g, t, proc, sec, L);
    return t.E > R(0);
  }
  return r == kAlive;
}

// ------------------------------------------------------------- load / store
template <class R> __device__ __forceinline__ void load_track(const Store<R> &s, long long i, int ptype, Track<R> &t)
{
  t.type = (ptype < 3) ? ptype : s.type[i];
  t.pos[0] = s.x[i];
  t.pos[1] = s.y[i];
  t.pos[2] = s.z[i];
  t.dir[0] = s.dx[i];
  t.dir[1] = s.dy[i];
  t.dir[2] = s.dz[i];
  t.E = s.E[i];
  t.nil[0] = s.n0[i];
  t.nil[1] = s.n1[i];
  t.nil[2] = s.n2[i];
  t.msc_r0 = s.r0[i];
  t.load_rng(s.rng, s.cap, i);
  t.vol = s.vol[i];
  t.event = s.event[i];
  t.prim = s.prim[i];
}

template <class R> __device__ __forceinline__ void store_track(const Store<R> &s, long long i, const Track<R> &t)
{
  s.x[i] = t.pos[0];
  s.y[i] = t.pos[1];
  s.z[i] = t.pos[2];
  s.dx[i] = t.dir[0];
  s.dy[i] = t.dir[1];
  s.dz[i] = t.dir[2];
  s.E[i] = t.E;
  s.n0[i] = t.nil[0];
  s.n1[i] = t.nil[1];
  s.n2[i] = t.nil[2];
  s.r0[i] = t.msc_r0;
  t.store_rng(s.rng, s.cap, i);
  s.vol[i] = t.vol;
  s.event[i] = t.event;
  s.prim[i] = t.prim;
  if (s.type) s.type[i] = t.type;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

// Reserve `cnt` consecutive slots per lane (0 <= cnt <= 3: a survivor and up
// to two secondaries) in counter *ctr: one atomic per warp, returns this
// lane's first slot.  The lanes' counts go in as two ballots (their bits 0
// and 1), so the exclusive prefix is two popcounts instead of a shuffle scan;
// the slots are those of the scan, in lane order.
__device__ __forceinline__ long long warp_reserve(unsigned long long *ctr, int cnt)
{
  const unsigned b0 = __ballot_sync(0xffffffffu, cnt & 1), b1 = __ballot_sync(0xffffffffu, cnt & 2);
  const int total = __popc(b0) + 2 * __popc(b1);
  if (total == 0) return 0;
  const unsigned lt = lanemask_lt();
  const int leader = __ffs(b0 | b1) - 1;
  unsigned long long base = 0;
  if ((int)lane_id() == leader) base = atomicAdd(ctr, (unsigned long long)total);
  base = __shfl_sync(0xffffffffu, base, leader);
  return (long long)base + __popc(b0 & lt) + 2 * __popc(b1 & lt);
}

// Write a track to store q, or to q's overflow stack when the store is full.
template <class R> __device__ __forceinline__ void put_track(const Args<R> &a, int q, long long idx, const Track<R> &t, Local &L)
{
  const Store<R> &s = a.st[a.ctl->parity ^ 1][q];
  if (idx < s.cap) {
    store_track(s, idx, t);
    return;
  }
  unsigned long long j = atomicAdd((unsigned long long *)&a.ctl->stack_count[q], 1ULL);
  if ((long long)j < a.stack[q].cap) {
    store_track(a.stack[q], (long long)j, t);
  } else {
    // no room anywhere: the track is retired and its energy scored where it is
    L.err |= kErrOverflow;
    L.st[S_OVERFLOW]++;
    L.deposit(t.event, t.vol, (double)t.E);
  }
}

// ----------------------------------------------------------------- kernels
// Shared-memory tally and block statistics of one step kernel.
__device__ __forceinline__ void tally_begin(Local &L, const Geom &g, double *edep, double *sm_edep,
                                            unsigned long long *sm_stat, double *sm_esc, int *sm_err)
{
  L.nvol = g.nvol;
  L.nevents = g.nevents;
  L.g_edep = edep;
  L.sm_edep = sm_edep;
  L.sm_esc = sm_esc;
  // event row 0 of the tally lives in shared memory when it fits in 6 KB
  L.sm_bins = (g.nvol <= 768) ? g.nvol : 0;
  for (int k = threadIdx.x; k < L.sm_bins; k += blockDim.x) sm_edep[k] = 0.0;
  for (int k = threadIdx.x; k < kNStat; k += blockDim.x) sm_stat[k] = 0;
  if (threadIdx.x == 0) {
    sm_esc[0] = sm_esc[1] = 0.0;
    *sm_err = 0;
  }
  __syncthreads();
  L.retired = 0.0;
  L.err = 0;
#pragma unroll
  for (int k = 0; k < kNStat; ++k) L.st[k] = 0;
}

// steps_slot >= 0: the stat that also receives this kernel's step count
__device__ __forceinline__ void tally_end(Local &L, Ctl *ctl, double *edep, double *sm_edep,
                                          unsigned long long *sm_stat, double *sm_esc, int *sm_err,
                                          int steps_slot = -1)
{
#pragma unroll
  for (int k = 0; k < kNStat; ++k)
    if (L.st[k]) atomicAdd(&sm_stat[k], (unsigned long long)L.st[k]);
  if (steps_slot >= 0 && L.st[S_STEPS]) atomicAdd(&sm_stat[steps_slot], (unsigned long long)L.st[S_STEPS]);
  if (L.retired != 0.0) atomicAdd(&sm_esc[1], L.retired);
  if (L.err) atomicOr(sm_err, L.err);
  __syncthreads();
  for (int k = threadIdx.x; k < L.sm_bins; k += blockDim.x)
    if (sm_edep[k] != 0.0) atomicAdd(&edep[k], sm_edep[k]);
  for (int k = threadIdx.x; k < kNStat; k += blockDim.x)
    if (sm_stat[k]) atomicAdd(&ctl->stat[k], sm_stat[k]);
  if (threadIdx.x == 0) {
    if (sm_esc[0] != 0.0) atomicAdd(&ctl->escaped, sm_esc[0]);
    if (sm_esc[1] != 0.0) atomicAdd(&ctl->retired, sm_esc[1]);
    if (*sm_err) atomicOr(&ctl->err_flags, *sm_err);
  }
}

// Element q of a 3-array by unrolled compare, so the array stays in registers.
template <class T> __device__ __forceinline__ T take3(T (&v)[3], int q, T inc)
{
  T r = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if (j == q) {
      r = v[j];
      v[j] += inc;
    }
  return r;
}

// The NIL of every discrete process of track t that has none (<= 0), drawn
// from the track's stream in process order -- the draws its next GPIL would
// make first.  Drawn where a track is created or survives an interaction,
// right after the stream's other draws there, they are the same numbers in
// the same order on the same stream, and the transport kernels' GPIL then
// finds them set: the draws run convergently in the kernel that makes the
// tracks instead of for one or two lanes in most passes of a transport warp.
template <class R> __device__ __forceinline__ void draw_nils(Track<R> &t, Mrg &rng)
{
  const int np = (t.type == 1) ? 2 : 3;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (i < np && t.nil[i] <= R(0)) t.nil[i] = -M<R>::log(rng.template u<R>());
}

// After a track's interaction: its secondaries (streams seeded from the
// parent, in order, their NILs drawn) and the survivor (its spent NIL drawn
// anew) go to the next stores, destination =
// particle type, or store 0 with one mixed store.  Every lane of the warp
// calls this (the slot reservations are warp-wide); `active` lanes write.
// SRC is the store the tracks were read from (for the write statistics).
template <class R, int SRC>
__device__ __forceinline__ void emit_tracks(const Args<R> &a, Ctl *ctl, int par, bool active, bool alive, Track<R> &t,
                                            const Secs<R> &sec, Local &L)
{
  const bool mixed = a.nstores == 1;
  int cnt[3] = {0, 0, 0};
  if (alive) take3(cnt, mixed ? 0 : t.type, 1);
#pragma unroll
  for (int k = 0; k < 2; ++k)
    if (k < sec.n) take3(cnt, mixed ? 0 : sec.type[k], 1);
  long long next[3];
#pragma unroll
  for (int q = 0; q < 3; ++q)
    next[q] = (q < a.nstores) ? warp_reserve((unsigned long long *)&ctl->count[par ^ 1][q], cnt[q]) : 0;
  if (!active) return;
  Mrg rng = t.rng();
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    if (k >= sec.n) break;
    Track<R> c;
    c.type = sec.type[k];
    c.pos[0] = t.pos[0];
    c.pos[1] = t.pos[1];
    c.pos[2] = t.pos[2];
    c.dir[0] = sec.dir[k][0];
    c.dir[1] = sec.dir[k][1];
    c.dir[2] = sec.dir[k][2];
    c.E = sec.E[k];
    c.nil[0] = c.nil[1] = c.nil[2] = R(-1);
    c.msc_r0 = R(-1);
    Mrg cr;
    rng.seed_child(cr);
    draw_nils(c, cr);
    c.set_rng(cr);
    c.vol = t.vol;
    c.event = t.event;
    c.prim = -1;
    const int q = mixed ? 0 : c.type;
    put_track(a, q, take3(next, q, 1LL), c, L);
    unsigned int sc[3] = {L.st[S_SEC0], L.st[S_SEC1], L.st[S_SEC2]};
    take3(sc, c.type, 1u);
    L.st[S_SEC0] = sc[0];
    L.st[S_SEC1] = sc[1];
    L.st[S_SEC2] = sc[2];
    L.st[S_WRITE0 + SRC]++;
  }
  if (alive) draw_nils(t, rng);
  t.set_rng(rng);
  if (alive) {
    const int q = mixed ? 0 : t.type;
    put_track(a, q, take3(next, q, 1LL), t, L);
    L.st[S_WRITE0 + SRC]++;
  }
}

// PT: particle type of the store (0, 1, 2), or 3 for the single mixed store.
// The fused step (transport and interaction in one kernel) of the plain loop.
template <class R, int PT, int K> __device__ __forceinline__ void step_body(const Args<R> &a)
{
  extern __shared__ double sm_edep[];
  __shared__ unsigned long long sm_stat[kNStat];
  __shared__ double sm_esc[2];
  __shared__ int sm_err;
  const Data &d = *a.d;
  Ctl *ctl = a.ctl;
  const int par = ctl->parity;
  constexpr int SRC = (PT < 3) ? PT : 0;
  const Store<R> &cur = a.st[par][SRC];
  const long long n = min(ctl->count[par][SRC], cur.cap);
  Local L;
  tally_begin(L, a.g, a.edep, sm_edep, sm_stat, sm_esc, &sm_err);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += stride) {
    long long i = base + threadIdx.x;
    bool active = i < n;
    Track<R> t;
    Secs<R> sec;
    sec.n = 0;
    bool alive = false;
    if (active) {
      load_track(cur, i, PT, t);
      L.st[S_READ0 + SRC]++;
      alive = one_step<R, K>(d, a.g, t, sec, L);
      if (t.prim >= 0 && a.pstep) atomicAdd(&a.pstep[t.prim], 1);
    }
    emit_tracks<R, SRC>(a, ctl, par, active, alive, t, sec, L);
  }
  tally_end(L, ctl, a.edep, sm_edep, sm_stat, sm_esc, &sm_err);
}

// Arguments by value (the allocation-free entry point) or from a device copy.
// Two resident blocks per SM: the fused step needs ~190 registers per thread
// unconstrained, which would leave one 256-thread block (8 warps) per SM.
template <class R, int PT, int K> __global__ void __launch_bounds__(256, 2) k_step(Args<R> a)
{
  step_body<R, PT, K>(a);
}
template <class R, int PT, int K> __global__ void __launch_bounds__(256, 2) k_step_p(const Args<R> *__restrict__ A)
{
  step_body<R, PT, K>(*A);
}

// ------------------------------------------------- batched engine: split step
// Resident 256-thread blocks per SM the step kernels are compiled for: the FP64
// kernels would take 160-180 registers unbounded (12 warps per SM); bounded to
// 128 they keep 16 warps at the cost of a few spills.  The FP32-mixed kernels
// take 110-126 registers unbounded.  Held to 96 (kMaxRegs: the interaction
// kernels and the transport kernels of the uniform field, layered geometry and
// no multiple scattering) five 128-thread blocks fit on an SM instead of four,
// and C3 and C4 run 7-8% faster although the kernels spill 0-30 words; the
// field-map and multiple-scattering variants would spill 50-270 bytes there
// and stay unbounded (255).
template <class R> constexpr int kMinBlocks = sizeof(R) == 8 ? 2 : 0; // 0: no minimum
template <class R, int K> constexpr int kMaxRegs = sizeof(R) == 8 ? 128 : (K == 0 ? 96 : 255);

// One slot per flagged lane in counter *ctr (ballot and popcount, one atomic
// per warp when any lane is flagged); returns this lane's slot, 0 for lanes
// not flagged.  Every lane of the warp calls it.
__device__ __forceinline__ long long warp_take1(unsigned long long *ctr, bool flag)
{
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  if (!m) return 0;
  const int leader = __ffs(m) - 1;
  unsigned long long base = 0;
  if ((int)lane_id() == leader) base = atomicAdd(ctr, (unsigned long long)__popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  return flag ? (long long)base + __popc(m & lanemask_lt()) : 0;
}

// Timeline tracing (the library built with GX_TIMELINE, a separate build of
// this file): per iteration and step kernel, the global timer when the first
// block of the kernel starts and when the last one ends, so that a run shows
// how the kernels of an iteration follow or overlap one another.  Kernel ids:
// 0 refill, 1 refill bookkeeping, 2-4 transport of gamma, e-, e+, 5 + 3 type +
// process the interaction kernels, 14 end of iteration; 512 iterations kept
// (iteration i in row (i + 1) mod 512; row 0 holds the planning launch).
// Without GX_TIMELINE the marks compile to nothing.
#if defined(GX_TIMELINE) && !defined(GX_PARITY)
constexpr int kTimelineRows = 512, kTimelineKernels = 16;
__device__ unsigned long long g_timeline[kTimelineRows * kTimelineKernels][2];
__device__ __forceinline__ int timeline_slot(const Ctl *ctl, int id)
{
  const long long it = ((volatile const Ctl *)ctl)->iterations + 1;
  return (int)((it & (kTimelineRows - 1)) * kTimelineKernels + id);
}
__device__ __forceinline__ void timeline_mark(int slot, int end)
{
  if (threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (end)
      atomicMax(&g_timeline[slot][1], t);
    else
      atomicMin(&g_timeline[slot][0], t);
  }
}
#define GX_TL_BEGIN(ctl, id)                                                                                          \
  const int gx_tl_slot = timeline_slot(ctl, id);                                                                     \
  timeline_mark(gx_tl_slot, 0)
#define GX_TL_END() timeline_mark(gx_tl_slot, 1)
#else
#define GX_TL_BEGIN(ctl, id)
#define GX_TL_END()
#endif

// Transport of the tracks of type PT: each lane keeps its track in registers
// and steps it until the track interacts (it then goes to the interaction
// buffer of its process), dies, leaves the world, or has taken step_budget
// steps in this launch (it then goes to the next store).  A lane without a
// track takes the next one of the current store from a work counter shared by
// the whole grid (one atomic per warp for all its idle lanes), so the lanes
// of a warp stay busy while their tracks take different numbers of steps.
// One pass of the loop advances every lane by one helix sub-step (charged
// tracks in a field), with the start and the end of a step attached to it, so
// a lane whose step needs several sub-steps does not hold up the others.
// All stores and buffers are written at slots reserved per warp, contiguous.
template <class R, int PT, int K> __device__ __forceinline__ void transport_body(const Args<R> *__restrict__ A)
{
  extern __shared__ double sm_edep[];
  __shared__ unsigned long long sm_stat[kNStat];
  __shared__ double sm_esc[2];
  __shared__ int sm_err;
  const Args<R> &a = *A;
  const Data &d = *a.d;
  Ctl *ctl = a.ctl;
  const int par = ctl->parity;
  const Store<R> &cur = a.st[par][PT];
  GX_TL_BEGIN(ctl, 2 + PT);
  const long long n = min(ctl->count[par][PT], cur.cap);
  if ((long long)blockIdx.x * blockDim.x >= n) { // no work for this block (uniform exit)
    GX_TL_END();
    return;
  }
  Local L;
  tally_begin(L, a.g, a.edep, sm_edep, sm_stat, sm_esc, &sm_err);
  const int budget = a.step_budget[PT], fetch_min = a.fetch_min[PT];
  Track<R> t;
  StepCtx<R> c;
  GammaXs<R> gxs;
  gxs.have = 0;
  bool have = false, more = true; // `more` is warp-uniform: the work counter is not exhausted
  bool infield = false;           // in the middle of a step (helix sub-steps)
  int nst = 0;
  for (;;) {
    // new records once fetch_min lanes are idle (or all are: the last ones)
    const unsigned need = __ballot_sync(0xffffffffu, !have);
    if (need && more && (__popc(need) >= fetch_min || need == 0xffffffffu)) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if ((int)lane_id() == leader) base = atomicAdd((unsigned long long *)&ctl->take[PT], (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (!have) {
        const long long i = (long long)base + __popc(need & lanemask_lt());
        if (i < n) {
          load_track(cur, i, PT, t);
          have = true;
          infield = false;
          nst = 0;
          gxs.have = 0; // a new photon energy
        }
      }
      // records read: counted per warp (no per-thread counters held across
      // the loop; the host adds them to the type's total of records read)
      if ((int)lane_id() == leader) {
        const long long got = min((long long)__popc(need), n - (long long)base);
        if (got > 0) atomicAdd(&sm_stat[S_TREAD0 + PT], (unsigned long long)got);
      }
      if ((long long)base + __popc(need) >= n) more = false;
    }
    if (!__any_sync(0xffffffffu, have)) break;
    int r = kDone, proc = -1;
    bool done = false; // a step ends in this pass
    if (have && !infield) {
      infield = step_begin<R, K>(d, a.g, t, c, PT == 0 ? &gxs : nullptr);
      done = !infield;
    }
    if (PT != 0 && have && infield && field_substep<R, K>(d, a.g, t, c, L)) {
      infield = false;
      done = true;
    }
    if (done) {
      r = step_end<R, K>(d, a.g, t, c, L, &proc);
      ++nst;
      if (t.prim >= 0 && a.pstep) atomicAdd(&a.pstep[t.prim], 1);
    }
    const bool w_alive = done && r == kAlive && nst >= budget;
    const bool w_int = done && r == kInteract;
    const long long slot = warp_take1((unsigned long long *)&ctl->count[par ^ 1][PT], w_alive);
    long long q = 0;
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      if (PT == 1 && p == 2) continue; // e- has two processes
      const long long v = warp_take1((unsigned long long *)&ctl->qcount[PT][p], w_int && proc == p);
      if (p == proc) q = v;
    }
    bool queued = false;
    if (w_alive) {
      put_track(a, PT, slot, t, L);
    } else if (w_int) {
      if (q < a.qcap) {
        store_track(a.ibuf[PT][proc], q, t);
        queued = true;
      } else {
        L.err |= kErrOverflow;
        L.st[S_OVERFLOW]++;
        L.deposit(t.event, t.vol, (double)t.E);
      }
    }
    // records written (to the next store or an interaction buffer), per warp;
    // those queued for interactions are counted by k_finish from the buffers'
    // counters, and the host adds these to the type's total of records written
    const unsigned wr = __ballot_sync(0xffffffffu, w_alive || queued);
    if (lane_id() == 0 && wr) atomicAdd(&sm_stat[S_TWRITE0 + PT], (unsigned long long)__popc(wr));
    if (done && (r != kAlive || nst >= budget)) have = false;
  }
  tally_end(L, ctl, a.edep, sm_edep, sm_stat, sm_esc, &sm_err, S_TSTEP0 + PT);
  GX_TL_END();
}

template <class R, int PT, int K>
__global__ void __launch_bounds__(256, kMinBlocks<R>) __maxnreg__((kMaxRegs<R, K>)) k_transport(const Args<R> *__restrict__ A)
{
  transport_body<R, PT, K>(A);
}
// The FP32 CSG variants: held to the 128 registers of the others they spill
// 100-300 bytes; at 168 (three 128-thread blocks per SM) nearly none.
template <class R, int PT, int K> __global__ void __maxnreg__(168) k_transport_csg(const Args<R> *__restrict__ A)
{
  transport_body<R, PT, K>(A);
}
// Variants for 512- and 1024-thread blocks (the launch-setting sweep): held
// to the 64 registers per thread a 1024-thread block leaves, they spill.
template <class R, int PT, int K> __global__ void __launch_bounds__(1024, 1) k_transport_wide(const Args<R> *__restrict__ A)
{
  transport_body<R, PT, K>(A);
}

// Post-step interaction of process PROC for the buffered tracks of type PT:
// one model per kernel, so a warp runs one sampling algorithm; survivor and
// secondaries go to the next stores.
template <class R, int PT, int PROC> __device__ __forceinline__ void interact_body(const Args<R> *__restrict__ A)
{
  extern __shared__ double sm_edep[];
  __shared__ unsigned long long sm_stat[kNStat];
  __shared__ double sm_esc[2];
  __shared__ int sm_err;
  const Args<R> &a = *A;
  const Data &d = *a.d;
  Ctl *ctl = a.ctl;
  const int par = ctl->parity;
  const Store<R> &buf = a.ibuf[PT][PROC];
  GX_TL_BEGIN(ctl, 5 + 3 * PT + PROC);
  const long long n = min(ctl->qcount[PT][PROC], a.qcap);
  if ((long long)blockIdx.x * blockDim.x >= n) { // no work for this block (uniform exit)
    GX_TL_END();
    return;
  }
  Local L;
  tally_begin(L, a.g, a.edep, sm_edep, sm_stat, sm_esc, &sm_err);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += stride) {
    long long j = base + threadIdx.x;
    bool active = j < n;
    Track<R> t;
    Secs<R> sec;
    sec.n = 0;
    bool alive = false;
    if (active) {
      load_track(buf, j, PT, t);
      L.st[S_READ0 + PT]++;
      run_model(d, a.g, t, PROC, sec, L);
      alive = t.E > R(0);
    }
    emit_tracks<R, PT>(a, ctl, par, active, alive, t, sec, L);
  }
  tally_end(L, ctl, a.edep, sm_edep, sm_stat, sm_esc, &sm_err);
  GX_TL_END();
}

template <class R, int PT, int PROC>
__global__ void __launch_bounds__(256, kMinBlocks<R>) __maxnreg__((kMaxRegs<R, 0>)) k_interact(const Args<R> *__restrict__ A)
{
  interact_body<R, PT, PROC>(A);
}
template <class R, int PT, int PROC>
__global__ void __launch_bounds__(1024, 1) k_interact_wide(const Args<R> *__restrict__ A)
{
  interact_body<R, PT, PROC>(A);
}

// End of an iteration: the next stores become current, the refill plan for
// the following iteration is made.  One thread.  interacted: the interaction
// kernels ran in this iteration (their buffers are emptied); otherwise the
// tracks waiting in them count as pending.
__global__ void k_finish(Ctl *ctl, long long cap0, long long cap1, long long cap2, int nstores, int interacted)
{
  GX_TL_BEGIN(ctl, 14);
  int par = ctl->parity, np = par ^ 1;
  const long long cap[3] = {cap0, cap1, cap2};
  const long long refill_below = ctl->refill_below, stack_cap = ctl->stack_cap;
  long long buffered = 0;
  for (int q = 0; q < 3; ++q) {
    for (int p = 0; p < 3; ++p) {
      if (interacted) {
        // the records the transport kernels queued for this interaction
        ctl->stat[S_TQUEUE0 + q] += (unsigned long long)ctl->qcount[q][p];
        ctl->qcount[q][p] = 0;
      } else {
        buffered += ctl->qcount[q][p];
      }
    }
    ctl->take[q] = 0;
  }
  long long fl = 0;
  for (int q = 0; q < nstores; ++q) {
    // pushes past the end of a full stack were not written (and were counted as errors)
    ctl->stack_count[q] = min(ctl->stack_count[q], stack_cap);
    ctl->count[np][q] = min(ctl->count[np][q], cap[q]);
    ctl->count[par][q] = 0;
    fl += ctl->count[np][q];
  }
  ctl->parity = np;
  ctl->iterations++;
  // refill plan: deferred tracks first (most recent first), then primaries
  long long budget = refill_below - fl;
  long long pend = ctl->nprim - ctl->prim_next + buffered;
  for (int q = 0; q < nstores; ++q) {
    long long room = cap[q] - ctl->count[np][q];
    long long take = 0;
    if (budget > 0) take = min(min(ctl->stack_count[q], room), budget);
    // reserve the slots now: deferred tracks land at the end of the store,
    // primaries are appended after them by the refill kernel
    ctl->take_stack[q] = take;
    ctl->stack_dst[q] = ctl->count[np][q];
    ctl->count[np][q] += take;
    ctl->stack_count[q] -= take;
    ctl->stack_src[q] = ctl->stack_count[q];
    budget -= take;
    pend += ctl->stack_count[q];
  }
  // primaries: a shower's population peaks in proportion to its energy, long
  // after it is injected, so primaries are injected only while the energy the
  // live tracks carry (injected minus deposited or escaped) stays within
  // wave_energy; one primary at least once nothing is left in flight
  long long tp = 0;
  if (budget > 0 && ctl->prim_next < ctl->nprim) {
    long long lo = ctl->prim_next, hi = min(ctl->nprim, ctl->prim_next + budget);
    double e0 = lo > 0 ? ctl->cumE[lo - 1] : 0.0;
    const double room = ctl->wave_energy - (e0 - ctl->retired);
    // largest k in [lo, hi] with cumE[k - 1] - e0 <= room
    long long a = lo, b = hi;
    while (a < b) {
      long long m = (a + b + 1) / 2;
      if (ctl->cumE[m - 1] - e0 <= room)
        a = m;
      else
        b = m - 1;
    }
    long long live = 0;
    for (int q = 0; q < nstores; ++q) live += ctl->count[np][q] + ctl->stack_count[q];
    if (a == lo && live == 0) a = lo + 1;
    tp = a - lo;
  }
  ctl->take_prim = tp;
  ctl->in_flight = fl;
  ctl->pending = pend;
  if (fl > ctl->peak) ctl->peak = fl;
  GX_TL_END();
}

// Inclusive prefix sum of the primary energies, one block: each thread scans a
// contiguous chunk, the chunk totals are scanned in shared memory.
// status (optional): only the entries with status GX_TRACK_ALIVE count.
__global__ void __launch_bounds__(1024) k_prefix_energy(const double *__restrict__ E, long long n,
                                                        double *__restrict__ out, const int *__restrict__ status)
{
  __shared__ double part[1024];
  int t = threadIdx.x, nt = blockDim.x;
  long long chunk = (n + nt - 1) / nt;
  long long b = t * chunk, e = min(n, b + chunk);
  double s = 0.0;
  for (long long i = b; i < e; ++i) s += (!status || status[i] == GX_TRACK_ALIVE) ? E[i] : 0.0;
  part[t] = s;
  __syncthreads();
  if (t == 0)
    for (int k = 1; k < nt; ++k) part[k] += part[k - 1];
  __syncthreads();
  double run = t > 0 ? part[t - 1] : 0.0;
  for (long long i = b; i < e; ++i) {
    run += (!status || status[i] == GX_TRACK_ALIVE) ? E[i] : 0.0;
    out[i] = run;
  }
}

__device__ __forceinline__ void jump_matvec(const uint64_t *A, uint64_t v[3], uint64_t m)
{
  uint64_t r[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) acc = ((A[3 * i + k] * v[k]) % m + acc) % m;
    r[i] = acc;
  }
  v[0] = r[0];
  v[1] = r[1];
  v[2] = r[2];
}

// Execute the refill plan: move deferred tracks back from the stacks, then
// inject primaries (MRG32k3a substream first_substream + primary index).
template <class R> __device__ __forceinline__ void refill_body(const Args<R> &a)
{
  Ctl *ctl = a.ctl;
  int par = ctl->parity;
  long long ts[3] = {ctl->take_stack[0], ctl->take_stack[1], ctl->take_stack[2]};
  long long tp = ctl->take_prim;
  long long total = ts[0] + ts[1] + ts[2] + tp;
  long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    long long j = i;
    int q = 0;
    while (q < 3 && j >= ts[q]) {
      j -= ts[q];
      ++q;
    }
    if (q < 3) {
      Track<R> t;
      load_track(a.stack[q], ctl->stack_src[q] + j, (a.nstores == 1) ? 3 : q, t);
      store_track(a.st[par][q], ctl->stack_dst[q] + j, t);
      continue;
    }
    long long pi = ctl->prim_next + j;
    Track<R> t;
    if (a.p.from_soa) {
      // a track handed in with its state
      const SoaIn &q = a.p.soa;
      if (q.status[pi] != GX_TRACK_ALIVE) continue;
      t.type = q.type[pi];
      t.E = (R)q.ekin[pi];
      t.pos[0] = q.x[pi];
      t.pos[1] = q.y[pi];
      t.pos[2] = q.z[pi];
      t.dir[0] = (R)q.dx[pi];
      t.dir[1] = (R)q.dy[pi];
      t.dir[2] = (R)q.dz[pi];
      t.nil[0] = (R)q.nil0[pi];
      t.nil[1] = (R)q.nil1[pi];
      t.nil[2] = (R)q.nil2[pi];
      t.msc_r0 = q.msc ? (R)q.msc[pi] : R(-1);
      t.load_rng(q.rng, q.cap, pi);
      t.vol = q.volume[pi];
      if (t.vol < -1) {
        double dd[3] = {q.dx[pi], q.dy[pi], q.dz[pi]};
        t.vol = a.g.geometry == 2 ? csg_locate(a.g.csg, 0, t.pos, dd, kCsgTol) : locate(a.g, t.pos, dd);
      }
      t.event = q.event ? q.event[pi] : 0;
      t.prim = q.primary ? q.primary[pi] : -1;
    } else {
      t.type = a.p.type[pi];
      t.E = (R)a.p.E[pi];
      for (int k = 0; k < 3; ++k) {
        t.pos[k] = a.p.pos[3 * pi + k];
        t.dir[k] = (R)a.p.dir[3 * pi + k];
      }
      double dd[3] = {a.p.dir[3 * pi], a.p.dir[3 * pi + 1], a.p.dir[3 * pi + 2]};
      t.vol = a.g.geometry == 2 ? csg_locate(a.g.csg, 0, t.pos, dd, kCsgTol) : locate(a.g, t.pos, dd);
      t.nil[0] = t.nil[1] = t.nil[2] = R(-1);
      t.msc_r0 = R(-1);
      t.event = a.p.event ? a.p.event[pi] : 0;
      t.prim = (int)pi;
      unsigned long long kk = (unsigned long long)(a.p.first_substream + pi);
      uint64_t v1[3] = {(uint64_t)a.p.seed[0], (uint64_t)a.p.seed[1], (uint64_t)a.p.seed[2]};
      uint64_t v2[3] = {(uint64_t)a.p.seed[3], (uint64_t)a.p.seed[4], (uint64_t)a.p.seed[5]};
      for (int b = 0; kk != 0 && b < 64; ++b, kk >>= 1)
        if (kk & 1ULL) {
          jump_matvec(a.p.jump + 9 * b, v1, 4294967087ULL);
          jump_matvec(a.p.jump + 9 * (64 + b), v2, 4294944443ULL);
        }
      for (int k = 0; k < 3; ++k) {
        t.rs[k] = (uint32_t)v1[k];
        t.rs[3 + k] = (uint32_t)v2[k];
      }
    }
    atomicAdd(&ctl->stat[S_TRACKS], 1ULL);
    if (t.vol < 0) {
      atomicAdd(&ctl->escaped, (double)t.E);
      atomicAdd(&ctl->retired, (double)t.E);
      continue;
    }
    int qs = (a.nstores == 1) ? 0 : t.type;
    unsigned long long slot = atomicAdd((unsigned long long *)&ctl->count[par][qs], 1ULL);
    if ((long long)slot < a.st[par][qs].cap) {
      store_track(a.st[par][qs], (long long)slot, t);
    } else {
      atomicOr(&ctl->err_flags, (int)kErrOverflow);
      atomicAdd(&ctl->stat[S_OVERFLOW], 1ULL);
    }
  }
}

// launched with the step kernels' block size, up to 1024 threads
template <class R> __global__ void __launch_bounds__(1024) k_refill(Args<R> a) { refill_body(a); }
template <class R> __global__ void __launch_bounds__(1024) k_refill_p(const Args<R> *__restrict__ A)
{
  GX_TL_BEGIN(A->ctl, 0);
  refill_body(*A);
  GX_TL_END();
}

// Bookkeeping after a refill: the primary cursor.  One thread.
__global__ void k_refill_done(Ctl *ctl)
{
  GX_TL_BEGIN(ctl, 1);
  GX_TL_END();
  for (int q = 0; q < 3; ++q) ctl->take_stack[q] = 0;
  ctl->prim_next += ctl->take_prim;
  ctl->take_prim = 0;
}

__global__ void k_count_new_tracks(Ctl *ctl)
{
  // every secondary becomes a track exactly once
  ctl->stat[S_TRACKS] += ctl->stat[S_SEC0] + ctl->stat[S_SEC1] + ctl->stat[S_SEC2];
}

// ------------------------------------------------------------------ engine
struct Engine {
  int precision = -1, engine = -1;
  long long cap = 0, stack_cap = 0;
  void *pool = nullptr;
  size_t pool_bytes = 0;
  Ctl *ctl = nullptr;
  Ctl *h_ctl = nullptr; // pinned mirror
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  std::vector<char> graph_args; // launch arguments the graph was captured with
  double *cumE = nullptr;
  long long cumE_cap = 0;
  double *vtally = nullptr; // geometry 2: deposits per (event, touchable), folded into the caller's columns
  long long vtally_cap = 0;
  void *dargs = nullptr; // device copy of the launch arguments (batched engine)
  cudaStream_t s1 = nullptr, s2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_j1 = nullptr, ev_j2 = nullptr;
};

// Lay the SoA planes of one store out from `base + off` (256-byte aligned);
// with base == 0 it only measures.
template <class R> static Store<R> carve(uintptr_t base, size_t &off, long long cap, bool with_type)
{
  Store<R> s;
  auto take = [&](size_t bytes) {
    uintptr_t q = base + off;
    off += (bytes + 255) & ~size_t(255);
    return q;
  };
  s.cap = cap;
  s.x = (double *)take(cap * sizeof(double));
  s.y = (double *)take(cap * sizeof(double));
  s.z = (double *)take(cap * sizeof(double));
  s.dx = (R *)take(cap * sizeof(R));
  s.dy = (R *)take(cap * sizeof(R));
  s.dz = (R *)take(cap * sizeof(R));
  s.E = (R *)take(cap * sizeof(R));
  s.n0 = (R *)take(cap * sizeof(R));
  s.n1 = (R *)take(cap * sizeof(R));
  s.n2 = (R *)take(cap * sizeof(R));
  s.r0 = (R *)take(cap * sizeof(R));
  s.rng = (uint32_t *)take(6 * cap * sizeof(uint32_t));
  s.vol = (int *)take(cap * sizeof(int));
  s.event = (int *)take(cap * sizeof(int));
  s.prim = (int *)take(cap * sizeof(int));
  s.type = with_type ? (int *)take(cap * sizeof(int)) : nullptr;
  return s;
}

void release_engine(Ctx *c)
{
  Engine *e = GX_ENGINE_OF(c);
  if (!e) return;
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->pool) cudaFree(e->pool);
  if (e->ctl) cudaFree(e->ctl);
  if (e->cumE) cudaFree(e->cumE);
  if (e->vtally) cudaFree(e->vtally);
  if (e->dargs) cudaFree(e->dargs);
  if (e->h_ctl) cudaFreeHost(e->h_ctl);
  if (e->s1) cudaStreamDestroy(e->s1);
  if (e->s2) cudaStreamDestroy(e->s2);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->ev_j1) cudaEventDestroy(e->ev_j1);
  if (e->ev_j2) cudaEventDestroy(e->ev_j2);
  delete e;
  GX_ENGINE_OF(c) = nullptr;
}


template <class R> struct Launch {
  Args<R> a;
  int block, grid, smem;
};

// Geometry 2: the deposits per (event, touchable) added to the caller's
// tally columns (touchables without a column are dropped).
__global__ void k_fold_touchables(const double *__restrict__ vt, const int *__restrict__ score, int ntouch,
                                  int nscore, long long n, double *__restrict__ edep)
{
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double e = vt[i];
    const long long ev = i / ntouch;
    const int c = score[i - ev * ntouch];
    if (e != 0.0 && c >= 0) edep[ev * nscore + c] += e;
  }
}

// The variant of the step kernels for a geometry and field (kKind* bits).
template <class R> static int kernel_kind(const Geom &g)
{
  const bool boxes = sizeof(R) == 4 && g.geometry == 2 && g.csg.solids == kSolidsBox;
  return (g.field_map ? kKindFieldMap : 0) | (g.geometry == 2 ? kKindCsg : 0) | (g.msc ? kKindMsc : 0) |
         (boxes ? kKindBoxes : 0);
}
template <class R, int PT, int K> static void (*transport_variant())(const Args<R> *)
{
  if constexpr (sizeof(R) == 4 && (K & kKindCsg) != 0)
    return k_transport_csg<R, PT, K>;
  else
    return k_transport<R, PT, K>;
}
template <class R, int PT> static void (*transport_kernel(int kind))(const Args<R> *)
{
  if constexpr (sizeof(R) == 4) {
    switch (kind) {
    case 10: return transport_variant<R, PT, 10>();
    case 11: return transport_variant<R, PT, 11>();
    case 14: return transport_variant<R, PT, 14>();
    case 15: return transport_variant<R, PT, 15>();
    default: break;
    }
  }
  switch (kind & 7) {
  case 1: return transport_variant<R, PT, 1>();
  case 2: return transport_variant<R, PT, 2>();
  case 3: return transport_variant<R, PT, 3>();
  case 4: return transport_variant<R, PT, 4>();
  case 5: return transport_variant<R, PT, 5>();
  case 6: return transport_variant<R, PT, 6>();
  case 7: return transport_variant<R, PT, 7>();
  default: return transport_variant<R, PT, 0>();
  }
}
template <class R> static void (*step_kernel_p(int kind))(const Args<R> *)
{
  if constexpr (sizeof(R) == 4) {
    switch (kind) {
    case 10: return k_step_p<R, 3, 10>;
    case 11: return k_step_p<R, 3, 11>;
    case 14: return k_step_p<R, 3, 14>;
    case 15: return k_step_p<R, 3, 15>;
    default: break;
    }
  }
  switch (kind & 7) {
  case 1: return k_step_p<R, 3, 1>;
  case 2: return k_step_p<R, 3, 2>;
  case 3: return k_step_p<R, 3, 3>;
  case 4: return k_step_p<R, 3, 4>;
  case 5: return k_step_p<R, 3, 5>;
  case 6: return k_step_p<R, 3, 6>;
  case 7: return k_step_p<R, 3, 7>;
  default: return k_step_p<R, 3, 0>;
  }
}

// The step kernels of one type for a launch: blocks above 256 threads take the
// wide variants (kernel kind 0 only, FP32 and FP64 library kernels).
template <class R, int PT> static void (*transport_for(const Launch<R> &L))(const Args<R> *)
{
#ifndef GX_PARITY
  if (L.block > 256) return k_transport_wide<R, PT, 0>;
#endif
  return transport_kernel<R, PT>(kernel_kind<R>(L.a.g));
}
template <class R, int PT, int PROC> static void (*interact_for(const Launch<R> &L))(const Args<R> *)
{
#ifndef GX_PARITY
  if (L.block > 256) return k_interact_wide<R, PT, PROC>;
#endif
  return k_interact<R, PT, PROC>;
}

// One type's interaction kernels (gamma 3 processes, e- 2, e+ 3).
template <class R, int PT> static void enqueue_interactions(const Launch<R> &L, const Args<R> *A, cudaStream_t s)
{
  interact_for<R, PT, 0>(L)<<<L.grid, L.block, L.smem, s>>>(A);
  interact_for<R, PT, 1>(L)<<<L.grid, L.block, L.smem, s>>>(A);
  if constexpr (PT != 1) interact_for<R, PT, 2>(L)<<<L.grid, L.block, L.smem, s>>>(A);
}

// One iteration.  interact: this iteration runs the interaction kernels (the
// compaction interval: otherwise the interacting tracks wait in their buffers).
template <class R>
static void enqueue_iteration(const Launch<R> &L, Engine *e, cudaStream_t s, bool concurrent, bool interact = true)
{
  const Args<R> *A = (const Args<R> *)e->dargs;
  if (L.a.nstores == 1) {
    // plain loop: one fused step kernel over the mixed store
    k_refill_p<R><<<L.grid, L.block, 0, s>>>(A);
    k_refill_done<<<1, 1, 0, s>>>(L.a.ctl);
    step_kernel_p<R>(kernel_kind<R>(L.a.g))<<<L.grid, L.block, L.smem, s>>>(A);
    k_finish<<<1, 1, 0, s>>>(L.a.ctl, L.a.st[0][0].cap, L.a.st[0][1].cap, L.a.st[0][2].cap, L.a.nstores, 1);
    return;
  }
  k_refill_p<R><<<L.grid, L.block, 0, s>>>(A);
  k_refill_done<<<1, 1, 0, s>>>(L.a.ctl);
  cudaStream_t sg = s, se = s, sp = s;
  if (concurrent) {
    // gamma on s, e- on s1, e+ on s2
    cudaEventRecord(e->ev_fork, s);
    cudaStreamWaitEvent(e->s1, e->ev_fork, 0);
    cudaStreamWaitEvent(e->s2, e->ev_fork, 0);
    se = e->s1;
    sp = e->s2;
  }
  // Each type's transport kernel fills every SM, so the three run nearly one
  // after another, the next one's blocks taking the SMs the previous one's
  // blocks leave.  Positrons go first: their chain (a transport kernel with
  // about one record per lane, then three interaction kernels) is the one
  // that ends an iteration most often when it is dispatched last.
  transport_for<R, 2>(L)<<<L.grid, L.block, L.smem, sp>>>(A);
  if (interact) enqueue_interactions<R, 2>(L, A, sp);
  transport_for<R, 1>(L)<<<L.grid, L.block, L.smem, se>>>(A);
  if (interact) enqueue_interactions<R, 1>(L, A, se);
  transport_for<R, 0>(L)<<<L.grid, L.block, L.smem, sg>>>(A);
  if (interact) enqueue_interactions<R, 0>(L, A, sg);
  if (concurrent) {
    cudaEventRecord(e->ev_j1, e->s1);
    cudaEventRecord(e->ev_j2, e->s2);
    cudaStreamWaitEvent(s, e->ev_j1, 0);
    cudaStreamWaitEvent(s, e->ev_j2, 0);
  }
  k_finish<<<1, 1, 0, s>>>(L.a.ctl, L.a.st[0][0].cap, L.a.st[0][1].cap, L.a.st[0][2].cap, L.a.nstores,
                           interact ? 1 : 0);
}

// One particle type's step (transport + its interactions), for the profiling
// pass; `mid` is recorded between the transport kernel and the interactions.
template <class R>
static void enqueue_type(const Launch<R> &L, Engine *e, cudaStream_t s, int q, cudaEvent_t mid, bool interact = true)
{
  const Args<R> *A = (const Args<R> *)e->dargs;
  if (q == 0) {
    transport_for<R, 0>(L)<<<L.grid, L.block, L.smem, s>>>(A);
    cudaEventRecord(mid, s);
    if (interact) enqueue_interactions<R, 0>(L, A, s);
  } else if (q == 1) {
    transport_for<R, 1>(L)<<<L.grid, L.block, L.smem, s>>>(A);
    cudaEventRecord(mid, s);
    if (interact) enqueue_interactions<R, 1>(L, A, s);
  } else {
    transport_for<R, 2>(L)<<<L.grid, L.block, L.smem, s>>>(A);
    cudaEventRecord(mid, s);
    if (interact) enqueue_interactions<R, 2>(L, A, s);
  }
}

// Copy the tracks of a store (or stack), or the not yet injected tracks of a
// handed-in batch, into a caller's gx_track_soa at slots taken from a counter.
template <class R>
__global__ void k_extract(Store<R> src, long long n, int ptype, Ctl *ctl, gx_track_soa out)
{
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    Track<R> t;
    load_track(src, i, ptype, t);
    const long long j = (long long)atomicAdd((unsigned long long *)&ctl->extracted, 1ULL);
    if (j >= out.capacity) continue;
    out.type[j] = t.type;
    out.status[j] = GX_TRACK_ALIVE;
    if (out.event) out.event[j] = t.event;
    if (out.primary) out.primary[j] = t.prim;
    out.volume[j] = t.vol;
    out.next_volume[j] = t.vol;
    out.process[j] = -1;
    out.boundary[j] = 0;
    out.x[j] = t.pos[0];
    out.y[j] = t.pos[1];
    out.z[j] = t.pos[2];
    out.dx[j] = (double)t.dir[0];
    out.dy[j] = (double)t.dir[1];
    out.dz[j] = (double)t.dir[2];
    out.ekin[j] = (double)t.E;
    out.nil0[j] = (double)t.nil[0];
    out.nil1[j] = (double)t.nil[1];
    out.nil2[j] = (double)t.nil[2];
    out.lambda_inv0[j] = out.lambda_inv1[j] = out.lambda_inv2[j] = 0.0;
    out.pstep[j] = out.step[j] = out.snext[j] = out.safety[j] = 0.0;
    if (out.msc_range) out.msc_range[j] = (double)t.msc_r0;
    t.store_rng(out.rng, out.capacity, j);
  }
}

__global__ void k_extract_pending(SoaIn in, long long first, long long n, Ctl *ctl, gx_track_soa out)
{
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const long long i = first + k;
    if (in.status[i] != GX_TRACK_ALIVE) continue;
    const long long j = (long long)atomicAdd((unsigned long long *)&ctl->extracted, 1ULL);
    if (j >= out.capacity) continue;
    out.type[j] = in.type[i];
    out.status[j] = GX_TRACK_ALIVE;
    if (out.event) out.event[j] = in.event ? in.event[i] : 0;
    if (out.primary) out.primary[j] = in.primary ? in.primary[i] : -1;
    out.volume[j] = in.volume[i];
    out.next_volume[j] = in.volume[i];
    out.process[j] = -1;
    out.boundary[j] = 0;
    out.x[j] = in.x[i];
    out.y[j] = in.y[i];
    out.z[j] = in.z[i];
    out.dx[j] = in.dx[i];
    out.dy[j] = in.dy[i];
    out.dz[j] = in.dz[i];
    out.ekin[j] = in.ekin[i];
    out.nil0[j] = in.nil0[i];
    out.nil1[j] = in.nil1[i];
    out.nil2[j] = in.nil2[i];
    out.lambda_inv0[j] = out.lambda_inv1[j] = out.lambda_inv2[j] = 0.0;
    out.pstep[j] = out.step[j] = out.snext[j] = out.safety[j] = 0.0;
    if (out.msc_range) out.msc_range[j] = in.msc ? in.msc[i] : -1.0;
#pragma unroll
    for (int w = 0; w < 6; ++w) out.rng[w * out.capacity + j] = in.rng[w * in.cap + i];
  }
}

// The transport loop.  tin (optional): transport these tracks instead of the
// primaries; max_iter > 0: stop after that many iterations and write every
// track still alive to tout.
template <class R>
static int run(Ctx *C, const gx_transport_config *cfg, int nprim, const int *d_type, const double *d_E,
               const double *d_pos, const double *d_dir, const int *d_event, double *d_edep, int nvol,
               int *d_pstep, gx_transport_stats *stats, cudaStream_t s, const gx_track_soa *tin = nullptr,
               int max_iter = 0, gx_track_soa *tout = nullptr)
{
  const int prec = std::is_same<R, float>::value ? 1 : 0;
  const bool batched = cfg->engine == 1;
  const int nstores = batched ? 3 : 1;
  long long cap = cfg->capacity > 0 ? cfg->capacity : (batched ? (1LL << 24) : (3LL << 24));
  long long stack_cap = std::max(cap, 1LL << 20);
  Engine *&E = GX_ENGINE_OF(C);
  if (E && (E->precision != prec || E->engine != cfg->engine || E->cap != cap)) GX_RELEASE_ENGINE(C);
  cudaError_t err;
  if (!E) {
    E = new Engine();
    E->precision = prec;
    E->engine = cfg->engine;
    E->cap = cap;
    E->stack_cap = stack_cap;
    size_t bytes = 0;
    for (int b = 0; b < 2; ++b)
      for (int q = 0; q < nstores; ++q) carve<R>(0, bytes, cap, !batched);
    for (int q = 0; q < nstores; ++q) carve<R>(0, bytes, stack_cap, !batched);
    if (batched) // interaction buffers: gamma 3 processes, e- 2, e+ 3
      for (int k = 0; k < 8; ++k) carve<R>(0, bytes, cap, false);
    err = cudaMalloc(&E->pool, bytes);
    if (err != cudaSuccess) {
      GX_RELEASE_ENGINE(C);
      return cuda_error(err, "transport track stores");
    }
    E->pool_bytes = bytes;
    if ((err = cudaMalloc((void **)&E->ctl, sizeof(Ctl))) != cudaSuccess ||
        (err = cudaMallocHost((void **)&E->h_ctl, sizeof(Ctl))) != cudaSuccess) {
      GX_RELEASE_ENGINE(C);
      return cuda_error(err, "transport control block");
    }
    cudaStreamCreateWithFlags(&E->s1, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&E->s2, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&E->ev_fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&E->ev_j1, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&E->ev_j2, cudaEventDisableTiming);
  }
  Launch<R> L;
  std::memset(&L.a, 0, sizeof(L.a));
  size_t off = 0;
  uintptr_t base = (uintptr_t)E->pool;
  for (int b = 0; b < 2; ++b)
    for (int q = 0; q < nstores; ++q) L.a.st[b][q] = carve<R>(base, off, cap, !batched);
  for (int q = 0; q < nstores; ++q) L.a.stack[q] = carve<R>(base, off, stack_cap, !batched);
  for (int q = nstores; q < 3; ++q) {
    L.a.st[0][q] = L.a.st[0][0];
    L.a.st[1][q] = L.a.st[1][0];
    L.a.stack[q] = L.a.stack[0];
  }
  if (batched) {
    for (int q = 0; q < 3; ++q)
      for (int pr = 0; pr < 3; ++pr)
        if (q != 1 || pr != 2) L.a.ibuf[q][pr] = carve<R>(base, off, cap, false);
    L.a.qcap = cap;
  }
  {
    // positrons are few and long-lived: a shorter budget keeps their kernel
    // (on its own stream) off the iteration's critical path
    const int spl = cfg->steps_per_launch > 0 ? cfg->steps_per_launch : kDefaultStepsPerLaunch;
    for (int q = 0; q < 3; ++q)
      L.a.step_budget[q] = cfg->steps_per_launch_by_type[q] > 0 ? cfg->steps_per_launch_by_type[q]
                                                                : (q == 2 ? std::max(1, spl / 4) : spl);
    // a warp refills when this many of its lanes are idle: a photon takes a
    // few cheap boundary-crossing steps, so the new-track work (record load,
    // NIL draws, cross sections) would otherwise run for one or two lanes in
    // most passes of the photon kernel
    for (int q = 0; q < 3; ++q)
      L.a.fetch_min[q] = cfg->fetch_min_by_type[q] > 0 ? cfg->fetch_min_by_type[q] : default_fetch_min(*cfg, q);
  }
  if (off > E->pool_bytes) return set_error(GX_ERR_OVERFLOW, "transport pool layout");
  L.a.d = C->dev;
  L.a.ctl = E->ctl;
  Geom &g = L.a.g;
  g.geometry = cfg->geometry;
  g.axis = cfg->axis;
  g.nlayers = cfg->nlayers;
  g.box_mat = cfg->box_mat;
  g.charged_local = cfg->charged_local;
  g.nvol = nvol;
  g.nevents = cfg->nevents;
  g.t_abs = cfg->t_abs;
  g.pitch = cfg->t_abs + cfg->t_gap;
  g.x0 = -0.5 * cfg->nlayers * g.pitch;
  g.total = cfg->nlayers * g.pitch;
  g.half_trans = cfg->half_trans;
  g.Bz = cfg->Bz;
  g.msc = cfg->msc;
  g.field_map = cfg->field_map;
  for (int k = 0; k < 3; ++k) {
    g.box_half[k] = cfg->box_half[k];
    g.box_centre[k] = cfg->box_centre[k];
  }
  uint64_t *jt;
  int rc = get_jump_table(&jt);
  if (rc) return rc;
  L.a.p.type = d_type;
  L.a.p.event = d_event;
  L.a.p.E = d_E;
  L.a.p.pos = d_pos;
  L.a.p.dir = d_dir;
  for (int k = 0; k < 6; ++k) L.a.p.seed[k] = cfg->seed[k];
  L.a.p.first_substream = cfg->first_substream;
  L.a.p.jump = jt;
  if (tin) {
    L.a.p.from_soa = 1;
    L.a.p.soa = SoaIn{tin->type, tin->status, tin->event, tin->primary, tin->volume, tin->x, tin->y, tin->z,
                      tin->dx, tin->dy, tin->dz, tin->ekin, tin->nil0, tin->nil1, tin->nil2, tin->msc_range,
                      tin->rng, (long long)tin->capacity};
  }
  L.a.edep = d_edep;
  L.a.pstep = d_pstep;
  if (cfg->geometry == 2) {
    // the kernels score per (event, touchable); folded into d_edep at the end
    g.csg = CsgView{C->csg_node, C->csg_kids, C->csg_slab, C->csg_cand, C->csg_planes, C->csg_solids};
    g.nvol = C->csg_n;
    const long long nt = (long long)cfg->nevents * C->csg_n;
    if (nt > E->vtally_cap) {
      if (E->vtally) cudaFree(E->vtally);
      E->vtally = nullptr;
      E->vtally_cap = 0;
      if ((err = cudaMalloc((void **)&E->vtally, sizeof(double) * nt)) != cudaSuccess)
        return cuda_error(err, "transport touchable tally");
      E->vtally_cap = nt;
    }
    if ((err = cudaMemsetAsync(E->vtally, 0, sizeof(double) * nt, s)) != cudaSuccess)
      return cuda_error(err, "transport touchable tally");
    L.a.edep = E->vtally;
  }
  L.a.nstores = nstores;
  L.a.refill_below = cfg->refill_below > 0 ? std::min(cfg->refill_below, cap) : cap / 2;
  L.block = cfg->block_size > 0 ? cfg->block_size : default_block(cfg->engine);
  int bpsm = cfg->blocks_per_sm > 0 ? cfg->blocks_per_sm : default_blocks_per_sm(*cfg);
  L.grid = C->num_sms * bpsm;
  L.smem = 768 * sizeof(double);

  if (nprim > E->cumE_cap) {
    if (E->cumE) cudaFree(E->cumE);
    E->cumE = nullptr;
    E->cumE_cap = 0;
    if ((err = cudaMalloc((void **)&E->cumE, sizeof(double) * nprim)) != cudaSuccess)
      return cuda_error(err, "transport primary energies");
    E->cumE_cap = nprim;
  }
  if (nprim > 0) k_prefix_energy<<<1, 1024, 0, s>>>(tin ? tin->ekin : d_E, nprim, E->cumE, tin ? tin->status : nullptr);
  Ctl h;
  std::memset(&h, 0, sizeof(h));
  h.nprim = nprim;
  h.iterations = -1; // the planning launch below is not an iteration
  h.cumE = E->cumE;
  h.wave_energy = cfg->wave_energy > 0 ? cfg->wave_energy : default_wave_energy(cap, batched ? kWaveFillBatched : kWaveFillPlain);
  h.refill_below = L.a.refill_below;
  h.stack_cap = stack_cap;
  err = cudaMemcpyAsync(E->ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, s);
  if (err != cudaSuccess) return cuda_error(err, "transport control init");
  // first refill plan
  k_finish<<<1, 1, 0, s>>>(E->ctl, cap, cap, cap, nstores, 1);
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, s);
  const long long kMaxIter = 2000000LL;
  long long iters = 0;
  // the kernels read their arguments from a device copy (indexing a kernel
  // parameter by a run-time value would copy the whole block to local memory)
  if (!E->dargs && (err = cudaMalloc(&E->dargs, sizeof(Args<double>))) != cudaSuccess)
    return cuda_error(err, "transport arguments");
  if ((err = cudaMemcpyAsync(E->dargs, &L.a, sizeof(Args<R>), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_error(err, "transport arguments upload");
  double step_ms[3] = {0, 0, 0}, transport_ms[3] = {0, 0, 0};
  long long step_launches[3] = {0, 0, 0};
  // the compaction interval: the interaction kernels run (and their buffers
  // are emptied into the stores) every `every` iterations; one iteration for
  // the plain loop and for runs that hand their tracks over at the end
  const int every = (batched && !tout && cfg->interaction_interval > 1) ? cfg->interaction_interval : 1;
  if (!batched || cfg->profile || max_iter > 0) {
    // plain loop (and the profiling pass, and runs stopped after a number of
    // iterations): launch, synchronise, look at the counters, every iteration
    cudaEvent_t ea[3], em[3], eb[3];
    for (int q = 0; q < 3; ++q) {
      cudaEventCreate(&ea[q]);
      cudaEventCreate(&em[q]);
      cudaEventCreate(&eb[q]);
    }
    for (;;) {
      if (cfg->profile) {
        k_refill_p<R><<<L.grid, L.block, 0, s>>>((const Args<R> *)E->dargs);
        k_refill_done<<<1, 1, 0, s>>>(L.a.ctl);
        for (int q = 0; q < nstores; ++q) {
          cudaEventRecord(ea[q], s);
          if (!batched) {
            step_kernel_p<R>(kernel_kind<R>(L.a.g))<<<L.grid, L.block, L.smem, s>>>(
                (const Args<R> *)E->dargs);
            cudaEventRecord(em[q], s);
          } else {
            enqueue_type(L, E, s, q, em[q], (iters + 1) % every == 0);
          }
          cudaEventRecord(eb[q], s);
        }
        k_finish<<<1, 1, 0, s>>>(L.a.ctl, L.a.st[0][0].cap, L.a.st[0][1].cap, L.a.st[0][2].cap, L.a.nstores,
                                 (iters + 1) % every == 0 ? 1 : 0);
      } else {
        enqueue_iteration(L, E, s, false, (iters + 1) % every == 0);
      }
      cudaMemcpyAsync(E->h_ctl, E->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
      if ((err = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(err, "transport iteration");
      if (cfg->profile)
        for (int q = 0; q < nstores; ++q) {
          float t = 0, tt = 0;
          cudaEventElapsedTime(&t, ea[q], eb[q]);
          cudaEventElapsedTime(&tt, ea[q], em[q]);
          step_ms[q] += t;
          transport_ms[q] += tt;
          step_launches[q]++;
        }
      ++iters;
      if (E->h_ctl->in_flight == 0 && E->h_ctl->pending == 0) break;
      if (max_iter > 0 && iters >= max_iter) break;
      if (iters > kMaxIter) return set_error(GX_ERR_ITERCAP, "transport: iteration cap");
    }
    for (int q = 0; q < 3; ++q) {
      cudaEventDestroy(ea[q]);
      cudaEventDestroy(em[q]);
      cudaEventDestroy(eb[q]);
    }
  } else {
    int G = cfg->graph_iters > 0 ? cfg->graph_iters : 16;
    G = ((G + every - 1) / every) * every; // whole compaction intervals
    // (re)capture the iteration graph when its launch shape or its kernels
    // (field kind, geometry kind) change; the arguments themselves are read
    // from the device copy uploaded above
    int shape[6] = {G, L.block, L.grid, L.smem, kernel_kind<R>(L.a.g), every};
    std::vector<char> key(sizeof(shape) + 2 * sizeof(void *));
    const void *ptrs[2] = {E->dargs, E->ctl};
    std::memcpy(key.data(), shape, sizeof(shape));
    std::memcpy(key.data() + sizeof(shape), ptrs, sizeof(ptrs));
    if (!E->graph || E->graph_args != key) {
      if (E->graph) {
        cudaGraphExecDestroy(E->graph);
        E->graph = nullptr;
      }
      cudaStream_t cs;
      cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
      cudaGraph_t graph;
      if ((err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return cuda_error(err, "graph capture");
      for (int k = 0; k < G; ++k) enqueue_iteration(L, E, cs, true, (k + 1) % every == 0);
      cudaMemcpyAsync(E->h_ctl, E->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, cs);
      if ((err = cudaStreamEndCapture(cs, &graph)) != cudaSuccess) return cuda_error(err, "graph capture end");
      err = cudaGraphInstantiate(&E->graph, graph, 0);
      cudaGraphDestroy(graph);
      cudaStreamDestroy(cs);
      if (err != cudaSuccess) return cuda_error(err, "graph instantiate");
      E->graph_iters = G;
      E->graph_args = key;
    }
    for (;;) {
      if ((err = cudaGraphLaunch(E->graph, s)) != cudaSuccess) return cuda_error(err, "graph launch");
      if ((err = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(err, "transport graph");
      iters += G;
      if (E->h_ctl->in_flight == 0 && E->h_ctl->pending == 0) break;
      if (iters > kMaxIter) return set_error(GX_ERR_ITERCAP, "transport: iteration cap");
    }
  }
  if (cfg->geometry == 2) {
    const long long nt = (long long)cfg->nevents * C->csg_n;
    k_fold_touchables<<<(int)std::min<long long>((nt + 255) / 256, 4096), 256, 0, s>>>(
        E->vtally, C->csg_score, C->csg_n, C->csg_nscore, nt, d_edep);
  }
  k_count_new_tracks<<<1, 1, 0, s>>>(E->ctl);
  if (tout) {
    // the tracks still alive: carry out the refill plan the last iteration
    // made (deferred tracks back into the stores, the next primaries in), then
    // write out the stores, the stacks and what was never injected
    const Args<R> *A = (const Args<R> *)E->dargs;
    k_refill_p<R><<<L.grid, L.block, 0, s>>>(A);
    k_refill_done<<<1, 1, 0, s>>>(L.a.ctl);
    cudaMemcpyAsync(E->h_ctl, E->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
    if ((err = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(err, "transport hand-over");
    const Ctl hc = *E->h_ctl;
    const int par = hc.parity;
    const int ptype_of[3] = {batched ? 0 : 3, batched ? 1 : 3, batched ? 2 : 3};
    for (int q = 0; q < nstores; ++q) {
      const long long nc = std::min(hc.count[par][q], cap), ns = std::min(hc.stack_count[q], stack_cap);
      if (nc > 0) k_extract<R><<<(int)std::min<long long>((nc + 255) / 256, 4096), 256, 0, s>>>(
          L.a.st[par][q], nc, ptype_of[q], E->ctl, *tout);
      if (ns > 0) k_extract<R><<<(int)std::min<long long>((ns + 255) / 256, 4096), 256, 0, s>>>(
          L.a.stack[q], ns, ptype_of[q], E->ctl, *tout);
    }
    if (tin && hc.prim_next < hc.nprim) {
      const long long np = hc.nprim - hc.prim_next;
      k_extract_pending<<<(int)std::min<long long>((np + 255) / 256, 4096), 256, 0, s>>>(L.a.p.soa, hc.prim_next,
                                                                                        np, E->ctl, *tout);
    }
  }
  cudaEventRecord(t1, s);
  cudaMemcpyAsync(E->h_ctl, E->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
  if ((err = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(err, "transport end");
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  const Ctl &c = *E->h_ctl;
  if (stats) {
    stats->steps = (long long)c.stat[S_STEPS];
    stats->substeps = (long long)c.stat[S_SUBSTEPS];
    stats->tracks = (long long)c.stat[S_TRACKS];
    for (int q = 0; q < 3; ++q) stats->secondaries[q] = (long long)c.stat[S_SEC0 + q];
    stats->n_pair = (long long)c.stat[S_PAIR];
    stats->n_annih = (long long)c.stat[S_ANNIH];
    stats->errors = (long long)(c.stat[S_ERR] + c.stat[S_OVERFLOW]);
    stats->escaped = c.escaped;
    stats->iterations = c.iterations;
    stats->peak_in_flight = c.peak;
    stats->kernel_ms = ms;
    for (int q = 0; q < 3; ++q) {
      stats->step_ms[q] = step_ms[q];
      stats->step_launches[q] = step_launches[q];
      // the transport kernels count their records in the transport entries only
      stats->tracks_read[q] = (long long)(c.stat[S_READ0 + q] + c.stat[S_TREAD0 + q]);
      stats->tracks_written[q] = (long long)(c.stat[S_WRITE0 + q] + c.stat[S_TWRITE0 + q]);
      stats->transport_ms[q] = transport_ms[q];
      stats->transport_read[q] = (long long)c.stat[S_TREAD0 + q];
      stats->transport_written[q] = (long long)c.stat[S_TWRITE0 + q];
      stats->transport_queued[q] = (long long)c.stat[S_TQUEUE0 + q];
      stats->transport_steps[q] = (long long)c.stat[S_TSTEP0 + q];
    }
    stats->bytes_per_track = (long long)(3 * sizeof(double) + 8 * sizeof(R) + 6 * sizeof(uint32_t) +
                                         3 * sizeof(int) + (batched ? 0 : sizeof(int)));
  }
  if (tout) tout->n = (int)std::min<long long>(c.extracted, INT32_MAX);
  if (c.err_flags & kErrEvent)
    return set_error(GX_ERR_ARG, "transport: a primary's event index is outside [0, nevents = %d)", cfg->nevents);
  if (c.err_flags & kErrOverflow) return set_error(GX_ERR_OVERFLOW, "transport: track stores and stacks full");
  if (tout && c.extracted > tout->capacity)
    return set_error(GX_ERR_OVERFLOW, "gx_transport_tracks: %lld tracks alive, the output holds %d", c.extracted,
                     tout->capacity);
  if (c.err_flags) return set_error(GX_ERR_ITERCAP, "transport: an iteration cap was hit (flags %d)", c.err_flags);
  return GX_OK;
}


// ------------------------------------------------- the stages of one step
// gx_gpil, gx_propagate, gx_along_step, gx_post_step: OneStep cut at the
// points where the reference's process interface hands over (GPIL, the move,
// the along-step DoIt, the post-step DoIt), one thread per track of a
// caller's gx_track_soa, FP64; the state carried from one stage to the next
// is the SoA's (lambda_inv*, pstep, process, step, boundary, next_volume).
// Multiple scattering is not offered stage by stage (its along-step state is
// not part of the SoA); K: kKindFieldMap or 0.
struct StageArgs {
  const Data *d;
  Geom g;
  gx_track_soa t, sec;
  double *edep;
  double *escaped;
};

__device__ __forceinline__ void soa_load(const gx_track_soa &s, int i, Track<double> &t)
{
  t.type = s.type[i];
  t.pos[0] = s.x[i];
  t.pos[1] = s.y[i];
  t.pos[2] = s.z[i];
  t.dir[0] = s.dx[i];
  t.dir[1] = s.dy[i];
  t.dir[2] = s.dz[i];
  t.E = s.ekin[i];
  t.nil[0] = s.nil0[i];
  t.nil[1] = s.nil1[i];
  t.nil[2] = s.nil2[i];
  t.msc_r0 = s.msc_range ? s.msc_range[i] : -1.0;
  t.load_rng(s.rng, s.capacity, i);
  t.vol = s.volume[i];
  t.event = s.event ? s.event[i] : 0;
  t.prim = s.primary ? s.primary[i] : -1;
}

// the state a stage may change
__device__ __forceinline__ void soa_store(const gx_track_soa &s, int i, const Track<double> &t)
{
  s.x[i] = t.pos[0];
  s.y[i] = t.pos[1];
  s.z[i] = t.pos[2];
  s.dx[i] = t.dir[0];
  s.dy[i] = t.dir[1];
  s.dz[i] = t.dir[2];
  s.ekin[i] = t.E;
  s.nil0[i] = t.nil[0];
  s.nil1[i] = t.nil[1];
  s.nil2[i] = t.nil[2];
  if (s.msc_range) s.msc_range[i] = t.msc_r0;
  t.store_rng(s.rng, s.capacity, i);
  s.volume[i] = t.vol;
}

// the step context of a track from its SoA fields (after gx_gpil)
__device__ __forceinline__ void soa_ctx(const gx_track_soa &s, int i, const Track<double> &t, StepCtx<double> &c)
{
  c.xs0 = s.lambda_inv0[i];
  c.xs1 = s.lambda_inv1[i];
  c.xs2 = s.lambda_inv2[i];
  c.sel = s.process[i];
  c.vol0 = t.vol;
  c.newvol = t.vol;
  c.crossed = false;
  c.nsub = 0;
  c.remaining = 0.0;
  c.total = 0.0;
  c.lam0 = 0.0;
  c.e0 = t.E;
  c.ttrue = 0.0;
  c.range0 = -1.0;
}

__device__ __forceinline__ void stage_local(Local &L, const StageArgs &a)
{
  L.sm_edep = nullptr;
  L.g_edep = a.edep;
  L.sm_esc = a.escaped;
  L.nvol = a.g.nvol;
  L.nevents = a.g.nevents;
  L.sm_bins = 0;
  L.retired = 0.0;
  L.err = 0;
#pragma unroll
  for (int k = 0; k < kNStat; ++k) L.st[k] = 0;
}

template <int K> __global__ void __launch_bounds__(128) k_stage_gpil(StageArgs a)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.t.n || a.t.status[i] != GX_TRACK_ALIVE) return;
  Track<double> t;
  soa_load(a.t, i, t);
  if (t.vol < -1) t.vol = locate(a.g, t.pos, t.dir);
  if (t.vol < 0) { // outside the world
    a.t.volume[i] = t.vol;
    a.t.status[i] = GX_TRACK_EXITED;
    return;
  }
  StepCtx<double> c;
  const double ps = step_gpil<double, K>(*a.d, a.g, t, c);
  soa_store(a.t, i, t);
  a.t.pstep[i] = ps;
  a.t.process[i] = c.sel;
  a.t.lambda_inv0[i] = c.xs0;
  a.t.lambda_inv1[i] = c.xs1;
  a.t.lambda_inv2[i] = c.xs2;
  a.t.safety[i] = nav_safety<K>(a.g, t.vol, t.pos);
  int plane;
  a.t.snext[i] = fmin(nav_distance<K>(a.g, t.vol, t.pos, t.dir, ps, plane), ps);
}

template <int K> __global__ void __launch_bounds__(128) k_stage_propagate(StageArgs a)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.t.n || a.t.status[i] != GX_TRACK_ALIVE) return;
  Track<double> t;
  soa_load(a.t, i, t);
  StepCtx<double> c;
  soa_ctx(a.t, i, t, c);
  Local L;
  stage_local(L, a);
  if (step_move_begin<double, K>(a.g, t, c, a.t.pstep[i]))
    while (!field_substep<double, K>(*a.d, a.g, t, c, L)) {
    }
  soa_store(a.t, i, t);
  a.t.step[i] = c.total;
  a.t.boundary[i] = c.crossed ? 1 : 0;
  a.t.next_volume[i] = c.crossed ? c.newvol : t.vol;
}

template <int K> __global__ void __launch_bounds__(128) k_stage_along(StageArgs a)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.t.n || a.t.status[i] != GX_TRACK_ALIVE) return;
  Track<double> t;
  soa_load(a.t, i, t);
  StepCtx<double> c;
  soa_ctx(a.t, i, t, c);
  c.crossed = a.t.boundary[i] != 0;
  c.newvol = a.t.next_volume[i];
  c.total = a.t.step[i];
  Local L;
  stage_local(L, a);
  int proc = -1;
  const int r = step_end<double, K>(*a.d, a.g, t, c, L, &proc);
  soa_store(a.t, i, t);
  a.t.process[i] = (r == kInteract) ? proc : -1;
  a.t.status[i] = (r == kInteract) ? GX_TRACK_INTERACT
                  : (r == kAlive)  ? GX_TRACK_ALIVE
                  : (c.crossed && c.newvol == -1) ? GX_TRACK_EXITED
                                                  : GX_TRACK_KILLED;
}

template <int K> __global__ void __launch_bounds__(128) k_stage_post(StageArgs a)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.t.n) return;
  int nsec = 0;
  if (a.t.status[i] == GX_TRACK_INTERACT) {
    Track<double> t;
    soa_load(a.t, i, t);
    Secs<double> sec;
    sec.n = 0;
    Local L;
    stage_local(L, a);
    run_model(*a.d, a.g, t, a.t.process[i], sec, L);
    Mrg rng = t.rng();
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (k >= sec.n) break;
      Track<double> ch;
      ch.type = sec.type[k];
      ch.pos[0] = t.pos[0];
      ch.pos[1] = t.pos[1];
      ch.pos[2] = t.pos[2];
      ch.dir[0] = sec.dir[k][0];
      ch.dir[1] = sec.dir[k][1];
      ch.dir[2] = sec.dir[k][2];
      ch.E = sec.E[k];
      ch.nil[0] = ch.nil[1] = ch.nil[2] = -1.0;
      ch.msc_r0 = -1.0;
      Mrg cr;
      rng.seed_child(cr);
      ch.set_rng(cr);
      ch.vol = t.vol;
      ch.event = t.event;
      ch.prim = -1;
      const int j = 2 * i + k;
      soa_store(a.sec, j, ch);
      a.sec.type[j] = ch.type;
      a.sec.status[j] = GX_TRACK_ALIVE;
      if (a.sec.event) a.sec.event[j] = ch.event;
      if (a.sec.primary) a.sec.primary[j] = -1;
      a.sec.next_volume[j] = ch.vol;
      a.sec.process[j] = -1;
      a.sec.boundary[j] = 0;
      a.sec.lambda_inv0[j] = a.sec.lambda_inv1[j] = a.sec.lambda_inv2[j] = 0.0;
      a.sec.pstep[j] = a.sec.step[j] = a.sec.snext[j] = a.sec.safety[j] = 0.0;
      ++nsec;
    }
    t.set_rng(rng);
    soa_store(a.t, i, t);
    a.t.process[i] = -1;
    a.t.status[i] = t.E > 0.0 ? GX_TRACK_ALIVE : GX_TRACK_KILLED;
  }
  for (int k = nsec; k < 2; ++k) {
    a.sec.status[2 * i + k] = GX_TRACK_KILLED;
    a.sec.type[2 * i + k] = -1;
  }
}

// Geometry and options of a transport configuration, for the kernels.
static void make_geom(const Ctx *C, const gx_transport_config *cfg, int nvol, Geom &g)
{
  std::memset(&g, 0, sizeof(g));
  g.geometry = cfg->geometry;
  g.axis = cfg->axis;
  g.nlayers = cfg->nlayers;
  g.box_mat = cfg->box_mat;
  g.charged_local = cfg->charged_local;
  g.nvol = nvol;
  g.nevents = cfg->nevents;
  g.t_abs = cfg->t_abs;
  g.pitch = cfg->t_abs + cfg->t_gap;
  g.x0 = -0.5 * cfg->nlayers * g.pitch;
  g.total = cfg->nlayers * g.pitch;
  g.half_trans = cfg->half_trans;
  g.Bz = cfg->Bz;
  g.msc = cfg->msc;
  g.field_map = cfg->field_map;
  for (int k = 0; k < 3; ++k) {
    g.box_half[k] = cfg->box_half[k];
    g.box_centre[k] = cfg->box_centre[k];
  }
}

// One stage (0 gpil, 1 propagate, 2 along, 3 post) over a track SoA.
int run_stage(int stage, Ctx *C, const gx_transport_config *cfg, gx_track_soa *t, gx_track_soa *sec, double *d_edep,
              int nvol, cudaStream_t s)
{
  StageArgs a;
  std::memset(&a, 0, sizeof(a));
  a.d = C->dev;
  make_geom(C, cfg, nvol, a.g);
  a.t = *t;
  if (sec) a.sec = *sec;
  a.edep = d_edep;
  a.escaped = C->stage_scratch;
  if (t->n <= 0) return GX_OK;
  const int grid = (t->n + 127) / 128;
  const bool fm = cfg->field_map != 0;
  switch (stage) {
  case 0: (fm ? k_stage_gpil<kKindFieldMap> : k_stage_gpil<0>)<<<grid, 128, 0, s>>>(a); break;
  case 1: (fm ? k_stage_propagate<kKindFieldMap> : k_stage_propagate<0>)<<<grid, 128, 0, s>>>(a); break;
  case 2: (fm ? k_stage_along<kKindFieldMap> : k_stage_along<0>)<<<grid, 128, 0, s>>>(a); break;
  default: (fm ? k_stage_post<kKindFieldMap> : k_stage_post<0>)<<<grid, 128, 0, s>>>(a); break;
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GX_OK : cuda_error(e, "gx stage launch");
}

// gx_transport_tracks in this variant (FP64 here, or FP32-mixed)
int run_tracks(Ctx *C, const gx_transport_config *cfg, const gx_track_soa *in, int max_iter, gx_track_soa *out,
               double *d_edep, int nvol, gx_transport_stats *stats, cudaStream_t s)
{
#ifndef GX_PARITY
  if (cfg->precision == 1)
    return run<float>(C, cfg, in->n, nullptr, nullptr, nullptr, nullptr, nullptr, d_edep, nvol, nullptr, stats, s, in,
                      max_iter, out);
#endif
  return run<double>(C, cfg, in->n, nullptr, nullptr, nullptr, nullptr, nullptr, d_edep, nvol, nullptr, stats, s, in,
                     max_iter, out);
}

#ifdef GX_PARITY
// The FP64 transport of gx_transport_run with gx_transport_config.fp64_parity
int run_transport(Ctx *C, const gx_transport_config *cfg, int nprim, const int *d_type, const double *d_E,
                  const double *d_pos, const double *d_dir, const int *d_event, double *d_edep, int nvol,
                  int *d_pstep, gx_transport_stats *stats, cudaStream_t s)
{
  return run<double>(C, cfg, nprim, d_type, d_E, d_pos, d_dir, d_event, d_edep, nvol, d_pstep, stats, s);
}
} // namespace parity
#endif
} // namespace gx

#ifndef GX_PARITY
using namespace gx;

extern "C" {

void gx_transport_config_default(gx_transport_config *c)
{
  std::memset(c, 0, sizeof(*c));
  c->geometry = 1;
  c->axis = 2;
  c->nlayers = 50;
  c->t_abs = 2.3;
  c->t_gap = 5.7;
  c->half_trans = 200.0;
  c->box_mat = 1;
  c->max_steps = 1000000;
  for (int k = 0; k < 6; ++k) c->seed[k] = 12345.0;
  c->nevents = 1;
  c->precision = 0;
  c->engine = 1;
}

int gx_timeline_reset(gx_ctx *ctx)
{
#ifdef GX_TIMELINE
  if (!ctx) return set_error(GX_ERR_ARG, "gx_timeline_reset: null context");
  cudaError_t e = cudaSetDevice(reinterpret_cast<Ctx *>(ctx)->device);
  if (e != cudaSuccess) return cuda_error(e, "gx_timeline_reset: cudaSetDevice");
  static unsigned long long h[kTimelineRows * kTimelineKernels][2];
  for (int i = 0; i < kTimelineRows * kTimelineKernels; ++i) {
    h[i][0] = ~0ULL; // first start: a minimum
    h[i][1] = 0ULL;  // last end: a maximum
  }
  if ((e = cudaMemcpyToSymbol(g_timeline, h, sizeof(h))) != cudaSuccess) return cuda_error(e, "gx_timeline_reset");
  return GX_OK;
#else
  (void)ctx;
  return set_error(GX_ERR_ARG, "gx_timeline_reset: the library was built without GX_TIMELINE "
                               "(python geantexascalepilot_b200/build.py --timeline builds libgxb200_timeline.so)");
#endif
}

int gx_timeline_read(gx_ctx *ctx, unsigned long long *h_out, long long n)
{
#ifdef GX_TIMELINE
  if (!ctx || !h_out) return set_error(GX_ERR_ARG, "gx_timeline_read: null argument");
  if (n != (long long)kTimelineRows * kTimelineKernels * 2)
    return set_error(GX_ERR_ARG, "gx_timeline_read: n must be %d", kTimelineRows * kTimelineKernels * 2);
  cudaError_t e = cudaSetDevice(reinterpret_cast<Ctx *>(ctx)->device);
  if (e != cudaSuccess) return cuda_error(e, "gx_timeline_read: cudaSetDevice");
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cuda_error(e, "gx_timeline_read: synchronize");
  if ((e = cudaMemcpyFromSymbol(h_out, g_timeline, sizeof(g_timeline))) != cudaSuccess)
    return cuda_error(e, "gx_timeline_read");
  return GX_OK;
#else
  (void)ctx;
  (void)h_out;
  (void)n;
  return set_error(GX_ERR_ARG, "gx_timeline_read: the library was built without GX_TIMELINE "
                               "(python geantexascalepilot_b200/build.py --timeline builds libgxb200_timeline.so)");
#endif
}

// The checks of a transport configuration shared by the entry points.
static int check_config(const Ctx *C, const gx_transport_config *cfg, int nvol, const char *who)
{
  if (cfg->geometry == 1 && (cfg->nlayers <= 0 || cfg->t_abs <= 0 || cfg->t_gap <= 0 || cfg->half_trans <= 0 ||
                             nvol < 2 * cfg->nlayers))
    return set_error(GX_ERR_ARG, "%s: bad calorimeter (nvol must be >= 2 nlayers)", who);
  if (cfg->axis < 0 || cfg->axis > 2 || cfg->precision < 0 || cfg->precision > 1 || cfg->engine < 0 ||
      cfg->engine > 1 || cfg->nevents < 1)
    return set_error(GX_ERR_ARG, "%s: bad config", who);
  if (cfg->box_mat < 0 || cfg->box_mat > 2) return set_error(GX_ERR_ARG, "%s: bad box material", who);
  if (cfg->block_size && (cfg->block_size % 32 || cfg->block_size > 1024))
    return set_error(GX_ERR_ARG, "%s: block_size must be a multiple of 32, at most 1024", who);
  if (cfg->block_size > 256 && (cfg->engine != 1 || cfg->fp64_parity || cfg->geometry == 2 || cfg->msc ||
                                cfg->field_map))
    return set_error(GX_ERR_ARG, "%s: blocks above 256 threads are for the batched engine with the uniform field, "
                                 "layered geometry and no multiple scattering", who);
  if (cfg->interaction_interval < 0 || cfg->interaction_interval > 64)
    return set_error(GX_ERR_ARG, "%s: interaction_interval must be 0 .. 64", who);
  for (int q = 0; q < 3; ++q)
    if (cfg->fetch_min_by_type[q] < 0 || cfg->fetch_min_by_type[q] > 32)
      return set_error(GX_ERR_ARG, "%s: fetch_min_by_type must be 0 .. 32", who);
  if (cfg->field_map && !C->host.fmap)
    return set_error(GX_ERR_ARG, "%s: field_map = 1 without a field map (gx_ctx_load_field_map)", who);
  if (cfg->geometry < 0 || cfg->geometry > 2) return set_error(GX_ERR_ARG, "%s: bad geometry", who);
  if (cfg->msc < 0 || cfg->msc > 2) return set_error(GX_ERR_ARG, "%s: msc must be 0, 1 or 2", who);
  if (cfg->geometry == 2 && !C->csg_node)
    return set_error(GX_ERR_ARG, "%s: geometry 2 without a volume tree (gx_ctx_load_geometry)", who);
  if (cfg->geometry == 2 && nvol != C->csg_nscore)
    return set_error(GX_ERR_ARG, "%s: nvol %d, the volume tree has %d scored touchables", who, nvol, C->csg_nscore);
  if (cfg->fp64_parity < 0 || cfg->fp64_parity > 1 || (cfg->fp64_parity && cfg->precision != 0))
    return set_error(GX_ERR_ARG, "%s: fp64_parity must be 0 or 1, and 1 needs precision 0", who);
  return GX_OK;
}

// The arrays every stage and the hand-over read or write.
static bool soa_complete(const gx_track_soa *t)
{
  return t && t->n >= 0 && t->capacity >= t->n && t->type && t->status && t->volume && t->next_volume && t->process &&
         t->boundary && t->x && t->y && t->z && t->dx && t->dy && t->dz && t->ekin && t->nil0 && t->nil1 && t->nil2 &&
         t->lambda_inv0 && t->lambda_inv1 && t->lambda_inv2 && t->pstep && t->step && t->snext && t->safety && t->rng;
}

int gx_transport_run(gx_ctx *ctx, const gx_transport_config *cfg, int nprim, const int *d_type, const double *d_E,
                     const double *d_pos, const double *d_dir, const int *d_event, double *d_edep, int nvol,
                     int *d_primary_steps, gx_transport_stats *stats, gx_stream_t s)
{
  if (!ctx || !cfg) return set_error(GX_ERR_ARG, "gx_transport_run: null argument");
  if (nprim < 0 || (nprim > 0 && (!d_type || !d_E || !d_pos || !d_dir)) || !d_edep || nvol <= 0)
    return set_error(GX_ERR_ARG, "gx_transport_run: bad arguments");
  Ctx *C = reinterpret_cast<Ctx *>(ctx);
  int rc = check_config(C, cfg, nvol, "gx_transport_run");
  if (rc) return rc;
  cudaSetDevice(C->device);
  if (cfg->fp64_parity)
    return parity::run_transport(C, cfg, nprim, d_type, d_E, d_pos, d_dir, d_event, d_edep, nvol, d_primary_steps,
                                 stats, stream_of(s));
  if (cfg->precision == 1)
    return run<float>(C, cfg, nprim, d_type, d_E, d_pos, d_dir, d_event, d_edep, nvol, d_primary_steps, stats,
                      stream_of(s));
  return run<double>(C, cfg, nprim, d_type, d_E, d_pos, d_dir, d_event, d_edep, nvol, d_primary_steps, stats,
                     stream_of(s));
}

static int stage_entry(int stage, gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *t, gx_track_soa *sec,
                       double *d_edep, int nvol, gx_stream_t s, const char *who)
{
  if (!ctx || !cfg || !soa_complete(t)) return set_error(GX_ERR_ARG, "%s: null argument or incomplete track SoA", who);
  if (stage >= 2 && (!d_edep || nvol <= 0)) return set_error(GX_ERR_ARG, "%s: no tally", who);
  if (stage == 3 && (!soa_complete(sec) || sec->capacity < 2 * t->n))
    return set_error(GX_ERR_ARG, "%s: the secondaries' SoA needs capacity 2 n", who);
  Ctx *C = reinterpret_cast<Ctx *>(ctx);
  int rc = check_config(C, cfg, nvol > 0 ? nvol : 2 * cfg->nlayers, who);
  if (rc) return rc;
  if (cfg->msc || cfg->geometry == 2)
    return set_error(GX_ERR_ARG, "%s: the stage calls take msc = 0 and geometry 0 or 1 (use gx_transport_tracks)", who);
  cudaSetDevice(C->device);
  if (!C->stage_scratch) {
    cudaError_t e = cudaMalloc((void **)&C->stage_scratch, 8 * sizeof(double));
    if (e != cudaSuccess) return cuda_error(e, "stage scratch");
    C->owned.push_back(C->stage_scratch);
    cudaMemset(C->stage_scratch, 0, 8 * sizeof(double));
  }
  if (stage == 3) sec->n = 2 * t->n;
  if (cfg->fp64_parity) return parity::run_stage(stage, C, cfg, t, sec, d_edep, nvol, stream_of(s));
  return run_stage(stage, C, cfg, t, sec, d_edep, nvol, stream_of(s));
}

int gx_gpil(gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *tracks, gx_stream_t s)
{
  return stage_entry(0, ctx, cfg, tracks, nullptr, nullptr, 0, s, "gx_gpil");
}

int gx_propagate(gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *tracks, gx_stream_t s)
{
  return stage_entry(1, ctx, cfg, tracks, nullptr, nullptr, 0, s, "gx_propagate");
}

int gx_along_step(gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *tracks, double *d_edep, int nvol,
                  gx_stream_t s)
{
  return stage_entry(2, ctx, cfg, tracks, nullptr, d_edep, nvol, s, "gx_along_step");
}

int gx_post_step(gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *tracks, gx_track_soa *secondaries,
                 double *d_edep, int nvol, gx_stream_t s)
{
  return stage_entry(3, ctx, cfg, tracks, secondaries, d_edep, nvol, s, "gx_post_step");
}

int gx_transport_tracks(gx_ctx *ctx, const gx_transport_config *cfg, const gx_track_soa *in, int max_iterations,
                        gx_track_soa *out, double *d_edep, int nvol, gx_transport_stats *stats, gx_stream_t s)
{
  if (!ctx || !cfg || !soa_complete(in) || !soa_complete(out) || !d_edep || nvol <= 0 || max_iterations < 0)
    return set_error(GX_ERR_ARG, "gx_transport_tracks: bad arguments");
  if (in->rng == out->rng || in->x == out->x || in->status == out->status)
    return set_error(GX_ERR_ARG, "gx_transport_tracks: in and out share arrays");
  Ctx *C = reinterpret_cast<Ctx *>(ctx);
  int rc = check_config(C, cfg, nvol, "gx_transport_tracks");
  if (rc) return rc;
  cudaSetDevice(C->device);
  out->n = 0;
  if (cfg->fp64_parity) return parity::run_tracks(C, cfg, in, max_iterations, out, d_edep, nvol, stats, stream_of(s));
  return run_tracks(C, cfg, in, max_iterations, out, d_edep, nvol, stats, stream_of(s));
}

int gx_transport_run_host(gx_ctx *ctx, const gx_transport_config *cfg, int nprim, const int *h_type,
                          const double *h_E, const double *h_pos, const double *h_dir, const int *h_event,
                          double *h_edep, int nvol, int *h_primary_steps, gx_transport_stats *stats)
{
  if (!ctx || !cfg || nprim < 0 || !h_edep || nvol <= 0 || (nprim > 0 && (!h_type || !h_E || !h_pos || !h_dir)))
    return set_error(GX_ERR_ARG, "gx_transport_run_host: bad arguments");
  Ctx *C = reinterpret_cast<Ctx *>(ctx);
  cudaSetDevice(C->device);
  const size_t n = (size_t)(nprim > 0 ? nprim : 1), nt = (size_t)cfg->nevents * nvol;
  // one staging buffer and one stream kept by the context, grown when a call
  // needs more: no allocation, no stream creation per call
  auto pad = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t b_int = pad(n * sizeof(int)), b_dbl = pad(n * sizeof(double)), b_vec = pad(3 * n * sizeof(double));
  const size_t need = 3 * b_int + 2 * b_vec + b_dbl + pad(nt * sizeof(double));
  cudaError_t e;
  if (!C->host_stream && (e = cudaStreamCreateWithFlags(&C->host_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_error(e, "gx_transport_run_host: stream");
  if (need > C->host_buf_bytes) {
    if (C->host_buf) cudaFree(C->host_buf);
    C->host_buf = nullptr;
    C->host_buf_bytes = 0;
    if ((e = cudaMalloc(&C->host_buf, need)) != cudaSuccess) return cuda_error(e, "gx_transport_run_host: staging");
    C->host_buf_bytes = need;
  }
  cudaStream_t s = C->host_stream;
  char *b = (char *)C->host_buf;
  int *dt = (int *)b, *dev = (int *)(b + b_int), *dps = (int *)(b + 2 * b_int);
  double *dp = (double *)(b + 3 * b_int), *dd = (double *)(b + 3 * b_int + b_vec);
  double *dE = (double *)(b + 3 * b_int + 2 * b_vec), *ded = (double *)(b + 3 * b_int + 2 * b_vec + b_dbl);
  if (nprim > 0) {
    cudaMemcpyAsync(dt, h_type, nprim * sizeof(int), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dE, h_E, nprim * sizeof(double), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dp, h_pos, 3 * nprim * sizeof(double), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dd, h_dir, 3 * nprim * sizeof(double), cudaMemcpyHostToDevice, s);
    if (h_event) cudaMemcpyAsync(dev, h_event, nprim * sizeof(int), cudaMemcpyHostToDevice, s);
  }
  cudaMemsetAsync(ded, 0, nt * sizeof(double), s);
  if (h_primary_steps) cudaMemsetAsync(dps, 0, n * sizeof(int), s);
  int rc = gx_transport_run(ctx, cfg, nprim, dt, dE, dp, dd, h_event ? dev : nullptr, ded, nvol,
                            h_primary_steps ? dps : nullptr, stats, reinterpret_cast<gx_stream_t>(s));
  if (!rc) {
    cudaMemcpyAsync(h_edep, ded, nt * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (h_primary_steps) cudaMemcpyAsync(h_primary_steps, dps, nprim * sizeof(int), cudaMemcpyDeviceToHost, s);
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess && !rc) rc = cuda_error(e, "gx_transport_run_host copy back");
  return rc;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free transport (gx_transport_run_noalloc).
//
// For callers that must not allocate device memory while they run -- a host
// framework whose caching allocator owns the device memory, a process under a
// fixed memory budget, a time-critical loop that cannot absorb the implicit
// device synchronisation of cudaMalloc/cudaFree -- this entry point runs the
// plain FP64 loop on one static device array owned by the library instead of
// allocating track stores, the control block, the primary-energy prefix sums
// and the skip-ahead table.  Limits: at most kNoallocCapacity tracks in
// flight (mixed store), as many deferred on the stack, at most
// kNoallocMaxPrimaries primaries per call.  The array is shared by every call
// on a device and keeps the last call's contents; each call rewrites the parts
// that must start from zero (the control block) before its first launch.
// Calls that overlap on the GPU (two streams, two host threads) race on it.
// The first call on a device sets up that device (cudaGetSymbolAddress and
// the skip-ahead table upload).
// Every call synchronises its stream after each iteration (the host reads the
// control block to decide whether to go on).  The set-up is kept for the life
// of the process: a cudaDeviceReset while the library is loaded is not
// supported (the array would come back zeroed without its skip-ahead table).
namespace gx {

constexpr long long kNoallocCapacity = 16384;
constexpr int kNoallocMaxPrimaries = 4096;
static_assert(kNoallocCapacity == GX_NOALLOC_CAPACITY && kNoallocMaxPrimaries == GX_NOALLOC_MAX_PRIMARIES,
              "the limits of the allocation-free entry point must match gx_abi.h");
constexpr size_t kNoallocStoreBytes = 128 * (size_t)kNoallocCapacity; // FP64 record with type field
constexpr size_t kNoallocCtlBytes = 4096;
constexpr size_t kNoallocCumEBytes = sizeof(double) * kNoallocMaxPrimaries;
constexpr size_t kNoallocJumpBytes = sizeof(uint64_t) * 2 * 64 * 9;
constexpr size_t kNoallocBytes = 3 * kNoallocStoreBytes + kNoallocCtlBytes + kNoallocCumEBytes + kNoallocJumpBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[64] = {nullptr};

// Once per device, with that device current: the device address of the
// static array, and the skip-ahead table written into it.
static int noalloc_setup(int dev, unsigned char **out)
{
  static_assert(sizeof(Ctl) <= kNoallocCtlBytes, "control block does not fit");
  if (dev < 0 || dev >= 64) return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: device index %d", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "gx_transport_run_noalloc: cudaGetSymbolAddress");
    uint64_t h[2][64][9];
    build_jump_host(h);
    unsigned char *base = (unsigned char *)p;
    e = cudaMemcpy(base + 3 * kNoallocStoreBytes + kNoallocCtlBytes + kNoallocCumEBytes, h, sizeof(h),
                   cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(e, "gx_transport_run_noalloc: skip-ahead table");
    g_noalloc_ptr[dev] = base;
  }
  *out = g_noalloc_ptr[dev];
  return GX_OK;
}

} // namespace gx

extern "C" int gx_transport_run_noalloc(gx_ctx *ctx, const gx_transport_config *cfg, int nprim, const int *d_type,
                                        const double *d_E, const double *d_pos, const double *d_dir,
                                        const int *d_event, double *d_edep, int nvol, gx_transport_stats *stats,
                                        gx_stream_t stream)
{
  using namespace gx;
  if (!ctx || !cfg) return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: null argument");
  if (nprim < 0 || (nprim > 0 && (!d_type || !d_E || !d_pos || !d_dir)) || !d_edep || nvol <= 0)
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: bad arguments");
  if (nprim > kNoallocMaxPrimaries)
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: %d primaries exceed the static limit of %d", nprim,
                     kNoallocMaxPrimaries);
  if (cfg->precision != 0)
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: FP64 only (precision must be 0)");
  if (cfg->geometry != 0 && cfg->geometry != 1)
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: geometry 0 or 1 only (the volume tree's per-touchable "
                                 "tally is allocated: use gx_transport_run)");
  if (cfg->geometry == 1 && (cfg->nlayers <= 0 || cfg->t_abs <= 0 || cfg->t_gap <= 0 || cfg->half_trans <= 0 ||
                             nvol < 2 * cfg->nlayers))
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: bad calorimeter (nvol must be >= 2 nlayers)");
  if (cfg->axis < 0 || cfg->axis > 2 || cfg->nevents < 1 || cfg->box_mat < 0 || cfg->box_mat > 2)
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: bad config");
  if (cfg->block_size && (cfg->block_size % 32 || cfg->block_size > 256))
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: block_size must be a multiple of 32, at most 256");
  Ctx *C = reinterpret_cast<Ctx *>(ctx);
  if (cfg->field_map && !C->host.fmap)
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: field_map = 1 without a field map");
  cudaError_t err = cudaSetDevice(C->device);
  if (err != cudaSuccess) return cuda_error(err, "gx_transport_run_noalloc: cudaSetDevice");
  unsigned char *base = nullptr;
  int rc = noalloc_setup(C->device, &base);
  if (rc) return rc;
  cudaStream_t s = stream_of(stream);
  const long long cap = kNoallocCapacity;

  Launch<double> L;
  std::memset(&L.a, 0, sizeof(L.a));
  size_t off = 0;
  uintptr_t b = (uintptr_t)base;
  L.a.st[0][0] = carve<double>(b, off, cap, true);
  L.a.st[1][0] = carve<double>(b, off, cap, true);
  L.a.stack[0] = carve<double>(b, off, cap, true);
  if (off != 3 * kNoallocStoreBytes) return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: layout");
  for (int q = 1; q < 3; ++q) {
    L.a.st[0][q] = L.a.st[0][0];
    L.a.st[1][q] = L.a.st[1][0];
    L.a.stack[q] = L.a.stack[0];
  }
  Ctl *ctl = (Ctl *)(base + 3 * kNoallocStoreBytes);
  double *cumE = (double *)(base + 3 * kNoallocStoreBytes + kNoallocCtlBytes);
  const uint64_t *jump = (const uint64_t *)(base + 3 * kNoallocStoreBytes + kNoallocCtlBytes + kNoallocCumEBytes);
  L.a.d = C->dev;
  L.a.ctl = ctl;
  Geom &g = L.a.g;
  g.geometry = cfg->geometry;
  g.axis = cfg->axis;
  g.nlayers = cfg->nlayers;
  g.box_mat = cfg->box_mat;
  g.charged_local = cfg->charged_local;
  g.nvol = nvol;
  g.nevents = cfg->nevents;
  g.t_abs = cfg->t_abs;
  g.pitch = cfg->t_abs + cfg->t_gap;
  g.x0 = -0.5 * cfg->nlayers * g.pitch;
  g.total = cfg->nlayers * g.pitch;
  g.half_trans = cfg->half_trans;
  g.Bz = cfg->Bz;
  g.msc = cfg->msc;
  g.field_map = cfg->field_map;
  for (int k = 0; k < 3; ++k) {
    g.box_half[k] = cfg->box_half[k];
    g.box_centre[k] = cfg->box_centre[k];
  }
  L.a.p.type = d_type;
  L.a.p.event = d_event;
  L.a.p.E = d_E;
  L.a.p.pos = d_pos;
  L.a.p.dir = d_dir;
  for (int k = 0; k < 6; ++k) L.a.p.seed[k] = cfg->seed[k];
  L.a.p.first_substream = cfg->first_substream;
  L.a.p.jump = jump;
  L.a.edep = d_edep;
  L.a.pstep = nullptr;
  L.a.nstores = 1;
  L.a.refill_below = cfg->refill_below > 0 ? std::min(cfg->refill_below, cap) : cap / 2;
  L.block = cfg->block_size > 0 ? cfg->block_size : 256;
  L.grid = C->num_sms * (cfg->blocks_per_sm > 0 ? cfg->blocks_per_sm : 4);
  L.smem = 768 * sizeof(double);

  // the control block starts from zero on every call
  Ctl h;
  std::memset(&h, 0, sizeof(h));
  h.nprim = nprim;
  h.iterations = -1;
  h.cumE = cumE;
  h.wave_energy = cfg->wave_energy > 0 ? cfg->wave_energy : default_wave_energy(cap, kWaveFillPlain);
  h.refill_below = L.a.refill_below;
  h.stack_cap = cap;
  if ((err = cudaMemcpyAsync(ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (err = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_error(err, "gx_transport_run_noalloc: control block");
  if (nprim > 0) k_prefix_energy<<<1, 1024, 0, s>>>(d_E, nprim, cumE, nullptr);
  k_finish<<<1, 1, 0, s>>>(ctl, cap, cap, cap, 1, 1);
  Ctl hc;
  long long iters = 0;
  for (;;) {
    k_refill<double><<<L.grid, L.block, 0, s>>>(L.a);
    k_refill_done<<<1, 1, 0, s>>>(ctl);
    (cfg->msc ? (cfg->field_map ? k_step<double, 3, 5> : k_step<double, 3, 4>)
              : (cfg->field_map ? k_step<double, 3, 1> : k_step<double, 3, 0>))<<<L.grid, L.block, L.smem, s>>>(L.a);
    k_finish<<<1, 1, 0, s>>>(ctl, cap, cap, cap, 1, 1);
    if ((err = cudaGetLastError()) != cudaSuccess) return cuda_error(err, "gx_transport_run_noalloc: launch");
    if ((err = cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (err = cudaStreamSynchronize(s)) != cudaSuccess)
      return cuda_error(err, "gx_transport_run_noalloc: iteration");
    ++iters;
    if (hc.in_flight == 0 && hc.pending == 0) break;
    if (iters > 2000000LL) return set_error(GX_ERR_ITERCAP, "gx_transport_run_noalloc: iteration cap");
  }
  k_count_new_tracks<<<1, 1, 0, s>>>(ctl);
  if ((err = cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (err = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_error(err, "gx_transport_run_noalloc: end");
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->steps = (long long)hc.stat[S_STEPS];
    stats->substeps = (long long)hc.stat[S_SUBSTEPS];
    stats->tracks = (long long)hc.stat[S_TRACKS];
    for (int q = 0; q < 3; ++q) stats->secondaries[q] = (long long)hc.stat[S_SEC0 + q];
    stats->n_pair = (long long)hc.stat[S_PAIR];
    stats->n_annih = (long long)hc.stat[S_ANNIH];
    stats->errors = (long long)(hc.stat[S_ERR] + hc.stat[S_OVERFLOW]);
    stats->escaped = hc.escaped;
    stats->iterations = hc.iterations;
    stats->peak_in_flight = hc.peak;
    stats->tracks_read[0] = (long long)hc.stat[S_READ0];
    stats->tracks_written[0] = (long long)hc.stat[S_WRITE0];
    stats->bytes_per_track = 128;
  }
  if (hc.err_flags & kErrEvent)
    return set_error(GX_ERR_ARG, "gx_transport_run_noalloc: a primary's event index is outside [0, nevents = %d)",
                     cfg->nevents);
  if (hc.err_flags & kErrOverflow)
    return set_error(GX_ERR_OVERFLOW, "gx_transport_run_noalloc: more than %lld tracks in flight and deferred",
                     2 * kNoallocCapacity);
  if (hc.err_flags) return set_error(GX_ERR_ITERCAP, "gx_transport_run_noalloc: an iteration cap was hit");
  return GX_OK;
}
#endif // GX_PARITY
