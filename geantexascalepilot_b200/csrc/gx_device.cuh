// gx_device.cuh -- device building blocks of the B200 EM transport step path:
// MRG32k3a streams, spline tables, the interaction models, and the
// layered-box navigator.  Everything is templated on the arithmetic type R of
// the bulk of the step (double for the FP64 path, float for FP32-mixed); the
// RNG recurrence, global positions, boundary distances, low-energy range
// inversion and the helix stay FP64 in both.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gx_math.h"

namespace gx {

// Elementary functions of the FP64 arithmetic: CUDA's in the library's
// kernels; in the FP64 parity variant of the transport (the translation unit
// compiled with GX_PARITY, without contraction) those of gx_math.h, which the
// oracle's parity build compiles too, so that the two take the same path
// track by track.
#ifdef GX_PARITY
__device__ __forceinline__ double dlog(double x) { return gxm_log(x); }
__device__ __forceinline__ double dexp(double x) { return gxm_exp(x); }
__device__ __forceinline__ double dpow(double x, double y) { return gxm_pow(x, y); }
__device__ __forceinline__ double dexpm1(double x) { return gxm_expm1(x); }
__device__ __forceinline__ double dlog1p(double x) { return gxm_log1p(x); }
__device__ __forceinline__ void dsincos(double x, double *s, double *c) { gxm_sincos(x, s, c); }
#else
__device__ __forceinline__ double dlog(double x) { return ::log(x); }
__device__ __forceinline__ double dexp(double x) { return ::exp(x); }
__device__ __forceinline__ double dpow(double x, double y) { return ::pow(x, y); }
__device__ __forceinline__ double dexpm1(double x) { return ::expm1(x); }
__device__ __forceinline__ double dlog1p(double x) { return ::log1p(x); }
__device__ __forceinline__ void dsincos(double x, double *s, double *c)
{
  *s = ::sin(x);
  *c = ::cos(x);
}
#endif

// ------------------------------------------------------------------ constants
// CLHEP units (mm, MeV, ns) as in source/Geant/proxy/ProxySystemOfUnits.hpp.
constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2 * kPi;
constexpr double kEMass = 0.510998910;  // ProxyPhysicalConstants.hpp:51
constexpr double keV = 1.e-3, eV = 1.e-6, TeV = 1.e+6;
constexpr double kMinE = 100.0 * eV;    // the models' low-energy limit, used as minE
constexpr double kB2C_mm = -0.299792458; // MeV / (T mm)

// MRG32k3a parameters (L'Ecuyer's published constants; the reference keeps
// them in source/Geant/random/MRG.hpp:39-48,84-90).
constexpr double kM1 = 4294967087.0;
constexpr double kM2 = 4294944443.0;
constexpr double kNorm = 1.0 / (4294967087.0 + 1.0);
constexpr double kA12 = 1403580.0, kA13n = 810728.0, kA21 = 527612.0, kA23n = 1370589.0;

// ------------------------------------------------------------------- errors
enum : int {
  kErrNone = 0,
  kErrRejectCap = 1,   // a rejection loop exceeded its iteration cap
  kErrStepCap = 2,     // a track exceeded max_steps
  kErrFieldCap = 4,    // field propagation sub-step cap
  kErrOverflow = 8,    // track store / stack full
  kErrEvent = 16,      // a primary's event index outside the tally
};

// --------------------------------------------------------------- math policy
template <class R> struct M;
template <> struct M<double> {
  static __device__ __forceinline__ double log(double x) { return dlog(x); }
  static __device__ __forceinline__ double exp(double x) { return dexp(x); }
  static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
  static __device__ __forceinline__ double pow(double x, double y) { return dpow(x, y); }
  static __device__ __forceinline__ double cbrt(double x) { return dpow(x, 1.0 / 3.0); }
  static __device__ __forceinline__ void sincos(double x, double *s, double *c) { dsincos(x, s, c); }
  // sin/cos of 2 pi u
  static __device__ __forceinline__ void sincos2pi(double u, double *s, double *c) { dsincos(kTwoPi * u, s, c); }
  static __device__ __forceinline__ double cosr(double x)
  {
    double s, c;
    dsincos(x, &s, &c);
    return c;
  }
  static __device__ __forceinline__ double sinr(double x)
  {
    double s, c;
    dsincos(x, &s, &c);
    return s;
  }
};
template <> struct M<float> {
  static __device__ __forceinline__ float log(float x) { return __logf(x); }
  static __device__ __forceinline__ float exp(float x) { return __expf(x); }
  static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
  static __device__ __forceinline__ float pow(float x, float y) { return __powf(x, y); }
  static __device__ __forceinline__ float cbrt(float x) { return cbrtf(x); }
  static __device__ __forceinline__ void sincos(float x, float *s, float *c) { sincosf(x, s, c); }
  static __device__ __forceinline__ void sincos2pi(float u, float *s, float *c) { sincospif(2.0f * u, s, c); }
  static __device__ __forceinline__ float cosr(float x) { return __cosf(x); }
  static __device__ __forceinline__ float sinr(float x) { return sinf(x); }
};

// ------------------------------------------------------------------ MRG32k3a
// The state as six 32-bit words in registers.  The recurrence of
// MRG32k3a::Kernel (source/Geant/random/src/MRG32k3a.cpp:124-163) is done in
// exact integer arithmetic: a12 s1 - a13n s0 = a12 s1 + a13n (m1 - s0)
// (mod m1), every term non-negative and the sum below 2^54, reduced modulo
// m = 2^32 - c (c = 209 for m1, 22853 for m2) by folding the high word twice,
// h 2^32 + l = h c + l (mod m), and one conditional subtraction.  The
// reference's FP64 form (a quotient from 1/m as two doubles) is exact as
// well, so both give the same residues and the same draws; the integer form
// keeps the state in 6 registers instead of 12 and needs no conversions
// between the words and FP64.
struct Mrg {
  uint32_t s[6];
  static constexpr uint32_t kM1u = 4294967087u, kM2u = 4294944443u;
  static constexpr uint32_t kC1 = 209u, kC2 = 22853u; // 2^32 - m
  static constexpr uint32_t kA12u = 1403580u, kA13nu = 810728u, kA21u = 527612u, kA23nu = 1370589u;
  // x mod (2^32 - c) for x < 2^54
  static __device__ __forceinline__ uint32_t mod_m(uint64_t x, uint32_t c, uint32_t m)
  {
    x = (x >> 32) * c + (x & 0xffffffffull); // < 2^22 c + 2^32
    x = (x >> 32) * c + (x & 0xffffffffull); // < 2^32 + 64 c
    return (x >= m) ? (uint32_t)(x - m) : (uint32_t)x;
  }

  __device__ __forceinline__ void load(const uint32_t *st, long long n, long long i)
  {
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = __ldg(&st[k * n + i]);
  }
  __device__ __forceinline__ void store(uint32_t *st, long long n, long long i) const
  {
#pragma unroll
    for (int k = 0; k < 6; ++k) st[k * n + i] = s[k];
  }
  __device__ __forceinline__ void from_words(const uint32_t w[6])
  {
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = w[k];
  }
  __device__ __forceinline__ void to_words(uint32_t w[6]) const
  {
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = s[k];
  }
  // draw numerator z in [1, m1]
  __device__ __forceinline__ uint32_t next_u32()
  {
    const uint32_t p1 = mod_m((uint64_t)kA12u * s[1] + (uint64_t)kA13nu * (kM1u - s[0]), kC1, kM1u);
    s[0] = s[1];
    s[1] = s[2];
    s[2] = p1;
    const uint32_t p2 = mod_m((uint64_t)kA21u * s[5] + (uint64_t)kA23nu * (kM2u - s[3]), kC2, kM2u);
    s[3] = s[4];
    s[4] = s[5];
    s[5] = p2;
    return (p1 > p2) ? (p1 - p2) : (p1 + (kM1u - p2));
  }
  __device__ __forceinline__ double next() { return (double)next_u32(); }
  __device__ __forceinline__ double u01() { return (double)next_u32() * kNorm; }
  template <class R> __device__ __forceinline__ R u();
  // Stream of a secondary track: six draw numerators of this stream reduced
  // mod m1 (words 0-2) and m2 (words 3-5); an all-zero component becomes 1.
  __device__ __forceinline__ void seed_child(Mrg &c)
  {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const uint32_t z = next_u32(), m = (k < 3) ? kM1u : kM2u;
      c.s[k] = (z >= m) ? z - m : z;
    }
    if ((c.s[0] | c.s[1] | c.s[2]) == 0u) c.s[0] = 1u;
    if ((c.s[3] | c.s[4] | c.s[5]) == 0u) c.s[3] = 1u;
  }
};
template <> __device__ __forceinline__ double Mrg::u<double>() { return u01(); }
// a draw rounded to float, kept strictly below 1
template <> __device__ __forceinline__ float Mrg::u<float>() { return fminf((float)u01(), 0x1.fffffep-1f); }

// ------------------------------------------------------------------- tables
// One physics vector: n nodes starting at `off` in the node arrays.
struct VecDesc {
  int n, off;
  double emin, emax, dbin, base, invdbin;
  float eminf, emaxf, invdbinf, basef;
};

struct SBTable {
  double x[32], y[57], v[57][32];
};

constexpr int kNTables = 20, kNMat = 3;

// Device-resident physics data (one per context).
struct Data {
  VecDesc vec[kNTables][kNMat];
  const double *x, *y, *d2;  // nodes, FP64 (reference spline form)
  const double *c64;         // per bin: x1, 1/delta, c0, c1, c2, c3 (polynomial form)
  const float *c32;          // the same in FP32
  const SBTable *sb;         // [0] br11, [1] br18, [2] br82
  const double *binding;     // 1540 shell binding energies (eV)
  const double *sandia;      // 981 x 5
  double cut_raw[12];
  double cut_energy[4][kNMat];
  double cut_length[4][kNMat];
  int nshell[101], ishell[101], nint[101], cumint[101];
  double mat_Z[kNMat], mat_density[kNMat], mat_nel[kNMat], mat_dfactor[kNMat];
  double mat_I[kNMat], mat_A[kNMat]; // mean excitation energy (MeV), atomic mass (g/mol)
  // multiple scattering, per material: radiation length (mm) and the Urban
  // model's Z-dependent constants {X0, th1, th2, ca, cb, cc, cd}
  double mat_msc[kNMat][7];
  double pi_rcl2; // pi r_e^2, mm^2
  double alpha;   // the fine-structure constant
  // field map (optional, gx_ctx_load_field_map): (Br, Bphi, Bz) on an r-z
  // lattice, r outer, each premultiplied by 1 / (dr dz) as the reference's
  // reader stores them; null when no map is loaded
  const float4 *fmap;
};

// Field of the map at pos (tesla): ScalarCMSmagField::GetFieldValue /
// GetFieldValueRZ (examples/magneticfield/simplifiedCMS/inc/Geant/
// ScalarCMSmagField.h:207-331) restated: r and z clamped to the lattice,
// bilinear weights from the areas to the four corners (the stored values
// carry the 1 / (dr dz)), the cell found with the reference's single-
// precision inverse spacings; (Br, Bphi) rotated by the azimuth.  181 x 161
// points, dr = 50 mm up to 9 m, dz = 200 mm over +-16 m.
constexpr int kFmapNr = 181, kFmapNz = 161;
__device__ __forceinline__ void field_map_value(const float4 *__restrict__ fmap, const double pos[3], double B[3])
{
  const float kRDiff = 9000.0f / (kFmapNr - 1), kZDiff = 2 * 16000.0f / (kFmapNz - 1);
  const float kRDiffInv = 1.0f / kRDiff, kZDiffInv = 1.0f / kZDiff;
  const double r0 = ::sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  const double radius = fmin(r0, 9000.0), z = fmax(fmin(pos[2], 16000.0), -16000.0);
  double rFloor = floor(radius * kRDiffInv), zInd = floor((z - (-16000.0)) * kZDiffInv);
  rFloor = fmin(rFloor, (double)(kFmapNr - 2)); // the reference relies on rounding to stay inside
  zInd = fmin(zInd, (double)(kFmapNz - 2));
  const int i1 = (int)(rFloor * kFmapNz + zInd), i2 = i1 + 1;
  const double zLow = (zInd - (kFmapNz - 1) / 2) * kZDiff, zHigh = zLow + kZDiff;
  const double rLow = rFloor * kRDiff, rHigh = rLow + kRDiff;
  const double a1 = (rHigh - radius) * (zHigh - z), a2 = (rHigh - radius) * (z - zLow);
  const double a3 = (radius - rLow) * (zHigh - z), a4 = (radius - rLow) * (z - zLow);
  const float4 b1 = __ldg(&fmap[i1]), b3 = __ldg(&fmap[i1 + kFmapNz]);
  const float4 b2 = __ldg(&fmap[i2]), b4 = __ldg(&fmap[i2 + kFmapNz]);
  const double br = b1.x * a1 + b2.x * a2 + b3.x * a3 + b4.x * a4;
  const double bphi = b1.y * a1 + b2.y * a2 + b3.y * a3 + b4.y * a4;
  const double bz = b1.z * a1 + b2.z * a2 + b3.z * a3 + b4.z * a4;
  double s = 0.0, c = 1.0;
  if (r0 != 0.0) {
    const float rinv = (float)(1.0 / r0); // a float member in the reference
    s = pos[1] * rinv;
    c = pos[0] * rinv;
  }
  B[0] = br * c - bphi * s;
  B[1] = br * s + bphi * c;
  B[2] = bz;
}

// ProxyPhysicsVector::Value (ProxyPhysicsVector.cu:469-483) with the reference's
// bin search (:388-394) and spline (:396-429); bin kept inside the vector.
__device__ __forceinline__ double vec_value_ref(const Data &d, const VecDesc &v, double e)
{
  if (e <= v.emin) return __ldg(&d.y[v.off]);
  if (e >= v.emax) return __ldg(&d.y[v.off + v.n - 1]);
  int bin = (int)(dlog(e) / v.dbin - v.base);
  if (bin > v.n - 2) bin = v.n - 2;
  const double *x = d.x + v.off, *y = d.y + v.off, *d2 = d.d2 + v.off;
  if (bin > 0 && e < __ldg(&x[bin])) --bin;
  if (bin < 0) bin = 0;
  double x1 = __ldg(&x[bin]), x2 = __ldg(&x[bin + 1]);
  double delta = x2 - x1;
  double a = (x2 - e) / delta, b = (e - x1) / delta;
  return a * __ldg(&y[bin]) + b * __ldg(&y[bin + 1]) +
         ((a * a * a - a) * __ldg(&d2[bin]) + (b * b * b - b) * __ldg(&d2[bin + 1])) * delta * delta / 6.0;
}

// ProxyPhysicsVector::InvRangeValue (ProxyPhysicsVector.cu:491-524).
__device__ __forceinline__ double vec_invrange_ref(const Data &d, const VecDesc &v, double e)
{
  const double *x = d.x + v.off, *y = d.y + v.off, *d2 = d.d2 + v.off;
  if (e <= v.emin) return __ldg(&y[0]);
  if (e >= v.emax) return __ldg(&y[v.n - 1]);
  int n1 = 0, n2 = v.n / 2, n3 = v.n - 1;
  while (n1 != n3 - 1) {
    if (e > __ldg(&x[n2]))
      n1 = n2;
    else
      n3 = n2;
    n2 = n1 + (n3 - n1 + 1) / 2;
  }
  double x1 = __ldg(&x[n1]), x2 = __ldg(&x[n1 + 1]);
  double delta = x2 - x1;
  double a = (x2 - e) / delta, b = (e - x1) / delta;
  return a * __ldg(&y[n1]) + b * __ldg(&y[n1 + 1]) +
         ((a * a * a - a) * __ldg(&d2[n1]) + (b * b * b - b) * __ldg(&d2[n1 + 1])) * delta * delta / 6.0;
}

// The FP64 value of the polynomial form at e with the bin found from the FP32
// logarithm and checked against the two nodes around it (the FP32 log is off
// by far less than one bin, so one step down or up gives the interval that
// holds e): the FP32-mixed engine's range at the start of a step that loses
// more than 1% of its energy, without an FP64 logarithm.
__device__ __forceinline__ double vec_value_f64_f32bin(const Data &d, const VecDesc &v, double e)
{
  if (e <= v.emin) return __ldg(&d.c64[6 * v.off + 2]);
  if (e >= v.emax) return __ldg(&d.y[v.off + v.n - 1]);
  int bin = (int)(__logf((float)e) * v.invdbinf - v.basef);
  bin = min(max(bin, 0), v.n - 2);
  const double *c = d.c64 + 6 * (v.off + bin);
  double x1 = __ldg(&c[0]);
  if (bin > 0 && e < x1) {
    c -= 6;
    x1 = __ldg(&c[0]);
  } else if (bin < v.n - 2 && e >= __ldg(&c[6])) {
    c += 6;
    x1 = __ldg(&c[0]);
  }
  double u = (e - x1) * __ldg(&c[1]);
  return __ldg(&c[2]) + u * (__ldg(&c[3]) + u * (__ldg(&c[4]) + u * __ldg(&c[5])));
}
// InvRangeValue in FP64 with one reciprocal of the interval instead of three
// divisions (the FP32-mixed engine; the reference form is vec_invrange_ref).
__device__ __forceinline__ double vec_invrange_fast(const Data &d, const VecDesc &v, double e)
{
  const double *x = d.x + v.off, *y = d.y + v.off, *d2 = d.d2 + v.off;
  if (e <= v.emin) return __ldg(&y[0]);
  if (e >= v.emax) return __ldg(&y[v.n - 1]);
  int n1 = 0, n2 = v.n / 2, n3 = v.n - 1;
  while (n1 != n3 - 1) {
    if (e > __ldg(&x[n2]))
      n1 = n2;
    else
      n3 = n2;
    n2 = n1 + (n3 - n1 + 1) / 2;
  }
  const double x1 = __ldg(&x[n1]), x2 = __ldg(&x[n1 + 1]);
  const double delta = x2 - x1, inv = 1.0 / delta;
  const double a = (x2 - e) * inv, b = (e - x1) * inv;
  return a * __ldg(&y[n1]) + b * __ldg(&y[n1 + 1]) +
         ((a * a * a - a) * __ldg(&d2[n1]) + (b * b * b - b) * __ldg(&d2[n1 + 1])) * (delta * delta * (1.0 / 6.0));
}

// Value() in the polynomial form y = c0 + u (c1 + u (c2 + u c3)), u = (E - x1)/delta:
// one 24/48-byte record per bin.  Same spline, same bin choice.
template <class R> __device__ __forceinline__ R vec_value_fast(const Data &d, const VecDesc &v, R e);
template <> __device__ __forceinline__ double vec_value_fast<double>(const Data &d, const VecDesc &v, double e)
{
  if (e <= v.emin) return __ldg(&d.c64[6 * v.off + 2]);
  if (e >= v.emax) return __ldg(&d.y[v.off + v.n - 1]);
  int bin = (int)(::log(e) * v.invdbin - v.base);
  bin = min(max(bin, 0), v.n - 2);
  const double *c = d.c64 + 6 * (v.off + bin);
  double x1 = __ldg(&c[0]);
  if (bin > 0 && e < x1) {
    c -= 6;
    x1 = __ldg(&c[0]);
  }
  double u = (e - x1) * __ldg(&c[1]);
  return __ldg(&c[2]) + u * (__ldg(&c[3]) + u * (__ldg(&c[4]) + u * __ldg(&c[5])));
}
template <> __device__ __forceinline__ float vec_value_fast<float>(const Data &d, const VecDesc &v, float e)
{
  if (e <= v.eminf) return __ldg(&d.c32[6 * v.off + 2]);
  if (e >= v.emaxf) return (float)__ldg(&d.y[v.off + v.n - 1]);
  int bin = (int)(__logf(e) * v.invdbinf - v.basef);
  bin = min(max(bin, 0), v.n - 2);
  const float2 *c = reinterpret_cast<const float2 *>(d.c32 + 6 * (v.off + bin));
  float2 h = __ldg(&c[0]);
  if (bin > 0 && e < h.x) {
    c -= 3;
    h = __ldg(&c[0]);
  }
  float2 p = __ldg(&c[1]), q = __ldg(&c[2]);
  float u = (e - h.x) * h.y;
  return p.x + u * (p.y + u * (q.x + u * q.y));
}

// Proxy2DVector::FindBinLocationX/Y and Value (Proxy2DVector.cpp:37-67,93-139).
__device__ __forceinline__ int bin2d(const double *v, int nn, double z)
{
  if (z < v[1]) return 0;
  if (z >= v[nn - 2]) return nn - 2;
  int lo = 0, hi = nn - 2;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    if (z < v[mid])
      hi = mid - 1;
    else
      lo = mid + 1;
  }
  return hi;
}
// The y part of a lookup (y = ln T fixed while a sampler tries several x):
// the row, and the weights' factors, found once.
struct SBRow {
  int iy;
  double wy2, wy1, dy; // y2 - y, y - y1, y2 - y1
};
__device__ __forceinline__ SBRow sb_row(const SBTable &t, double y)
{
  if (y < t.y[0])
    y = t.y[0];
  else if (y > t.y[56])
    y = t.y[56];
  SBRow r;
  r.iy = bin2d(t.y, 57, y);
  const double y1 = t.y[r.iy], y2 = t.y[r.iy + 1];
  r.wy2 = y2 - y;
  r.wy1 = y - y1;
  r.dy = y2 - y1;
  return r;
}
template <class R> __device__ __forceinline__ R sb_value_row(const SBTable &t, const SBRow &w, R xr)
{
  double x = xr;
  if (x < t.x[0])
    x = t.x[0];
  else if (x > t.x[31])
    x = t.x[31];
  const int ix = bin2d(t.x, 32, x), iy = w.iy;
  double x1 = t.x[ix], x2 = t.x[ix + 1];
  double v11 = t.v[iy][ix], v12 = t.v[iy][ix + 1], v21 = t.v[iy + 1][ix], v22 = t.v[iy + 1][ix + 1];
  return (R)((w.wy2 * (v11 * (x2 - x) + v12 * (x - x1)) + (w.wy1 * (v21 * (x2 - x) + v22 * (x - x1)))) /
             ((x2 - x1) * w.dy));
}
template <class R> __device__ __forceinline__ R sb_value(const SBTable &t, R xr, R yr)
{
  return sb_value_row<R>(t, sb_row(t, (double)yr), xr);
}

// ------------------------------------------------------- cross sections per atom
// ProxyKleinNishina::CrossSectionPerAtom (ProxyKleinNishina.hpp:62-93); the
// reference's low-energy threshold is 15 * geantx::units::keV, a GeV-based
// unit, i.e. 1.5e-5 in this MeV-based arithmetic.
__device__ __forceinline__ double kn_xs_per_atom(double Z, double e)
{
  double Z2 = Z * Z;
  double p1 = 2.7965e-1 + 1.9756e-5 * Z + -3.9178e-7 * Z2;
  double p2 = -1.8300e-1 + -1.0205e-2 * Z + 6.8241e-5 * Z2;
  double p3 = 6.7527 + -7.3913e-2 * Z + 6.0480e-5 * Z2;
  double p4 = -1.9798e+1 + 2.7079e-2 * Z + 3.0274e-4 * Z2;
  double T0 = (Z < 1.5) ? 40.0 * keV : 15.0 * 1.e-6;
  double X = fmax(e, T0) / kEMass, X2 = X * X;
  double xs = p1 * ::log(1. + 2. * X) / X + (p2 + p3 * X + p4 * X2) / (1. + 20. * X + 230. * X2 + 440. * X2 * X);
  if (e < T0) {
    const double dT0 = keV;
    X = (T0 + dT0) / kEMass;
    X2 = X * X;
    double sigma = p1 * ::log(1. + 2. * X) / X + (p2 + p3 * X + p4 * X2) / (1. + 20. * X + 230. * X2 + 440. * X2 * X);
    double c1 = -T0 * (sigma - xs) / (xs * dT0);
    double c2 = (Z > 1.5) ? 0.375 - 0.0556 * ::log(Z) : 0.150;
    double y = ::log(e / T0);
    xs *= ::exp(-y * (c1 + c2 * y));
  }
  return Z * xs * (1.e-28 * (1000. * 1000.));
}

// ProxyMollerScattering::CrossSectionPerAtom (ProxyMollerScattering.hpp:61-89)
// with the delta-ray threshold as an argument (the reference fixes it at 10 eV)
__device__ __forceinline__ double mb_xs_per_atom(double Z, double kin, double twopi_mc2_rcl2, double cutEnergy)
{
  double tmax = fmin(100.0 * TeV, 0.5 * kin);
  if (cutEnergy > tmax) return 0.0;
  double xmin = cutEnergy / kin, xmax = tmax / kin;
  double tau = kin / kEMass, gam = tau + 1.0, gamma2 = gam * gam;
  double beta2 = tau * (tau + 2) / gamma2;
  double gg = (2.0 * gam - 1.0) / gamma2;
  double xs = ((xmax - xmin) * (1.0 - gg + 1.0 / (xmin * xmax) + 1.0 / ((1.0 - xmin) * (1.0 - xmax))) -
               gg * ::log(xmax * (1.0 - xmin) / (xmin * (1.0 - xmax)))) /
              beta2;
  return Z * xs * twopi_mc2_rcl2 / kin;
}

// ------------------------------------------------------------ interaction I/O
template <class R> struct Inter {
  R E, dir[3], edep;
  int status, nsec;
  int sec_type[2];
  R sec_E[2], sec_dir[2][3];
  // slot chosen by a branch, not an index, so the record stays in registers
  __device__ __forceinline__ void add(int type, R e, R x, R y, R z)
  {
    if (nsec == 0) {
      sec_type[0] = type;
      sec_E[0] = e;
      sec_dir[0][0] = x;
      sec_dir[0][1] = y;
      sec_dir[0][2] = z;
    } else {
      sec_type[1] = type;
      sec_E[1] = e;
      sec_dir[1][0] = x;
      sec_dir[1][1] = y;
      sec_dir[1][2] = z;
    }
    ++nsec;
  }
};

struct ModelParams {
  int mode; // 0 quirk, 1 physics
  int Z;
  double cut;
  double density_factor;
  const SBTable *sb;
};

constexpr int kRejectCap = 1 << 16; // rejection-loop iteration cap

// Math::RotateToLabFrame, source/Geant/core/math_wrappers.hpp:194-212
template <class R> __device__ __forceinline__ void rotate_to_lab(R &u, R &v, R &w, R u1, R u2, R u3)
{
  R up = u1 * u1 + u2 * u2;
  if (up > R(0)) {
    up = M<R>::sqrt(up);
    R px = u, py = v, pz = w;
    R inv = R(1) / up;
    u = (u3 * px * u1 - u2 * py) * inv + u1 * pz;
    v = (u3 * px * u2 + u1 * py) * inv + u2 * pz;
    w = -up * px + u3 * pz;
  } else if (u3 < R(0)) {
    u = -u;
    w = -w;
  }
}

template <class R> __device__ __forceinline__ void unit3(R &x, R &y, R &z)
{
  R m = M<R>::sqrt(x * x + y * y + z * z);
  if (m > R(0)) {
    x /= m;
    y /= m;
    z /= m;
  }
}

// ---------------------------------------------------------------- models
// Klein-Nishina Compton, ProxyKleinNishina.hpp:96-166
template <class R> __device__ int kn_sample(Mrg &r, const ModelParams &p, Inter<R> &io, int *err)
{
  const R low = R(100.0 * eV);
  R E0 = io.E;
  io.nsec = 0;
  if (E0 < low) return 0;
  R d0x = io.dir[0], d0y = io.dir[1], d0z = io.dir[2];
  R epsilon, epsilonsq, onecost, sint2, greject;
  R E0_m = E0 / R(kEMass);
  R eps0 = R(1) / (R(1) + R(2) * E0_m);
  R epsilon0sq = eps0 * eps0;
  R alpha1 = -M<R>::log(eps0);
  R alpha2 = R(0.5) * (R(1) - epsilon0sq);
  int it = 0;
  do {
    if (alpha1 / (alpha1 + alpha2) > r.u<R>()) {
      epsilon = M<R>::exp(-alpha1 * r.u<R>());
      epsilonsq = epsilon * epsilon;
    } else {
      epsilonsq = epsilon0sq + (R(1) - epsilon0sq) * r.u<R>();
      epsilon = M<R>::sqrt(epsilonsq);
    }
    onecost = (R(1) - epsilon) / (epsilon * E0_m);
    sint2 = onecost * (R(2) - onecost);
    greject = R(1) - epsilon * sint2 / (R(1) + epsilonsq);
    if (++it > kRejectCap) {
      *err |= kErrRejectCap;
      break;
    }
  } while (greject < r.u<R>());
  R sinTheta = (sint2 < R(0)) ? R(0) : M<R>::sqrt(sint2);
  R sphi, cphi;
  M<R>::sincos2pi(r.u<R>(), &sphi, &cphi);
  R gE = epsilon * E0;
  R gx = sinTheta * cphi, gy = sinTheta * sphi, gz = R(1) - onecost;
  rotate_to_lab(gx, gy, gz, d0x, d0y, d0z);
  if (gE > low) {
    io.dir[0] = gx;
    io.dir[1] = gy;
    io.dir[2] = gz;
    io.E = gE;
  } else {
    io.status = 1;
    io.edep += gE;
  }
  R eKin = E0 - gE;
  bool make_e = (p.mode == 0) ? (gE > low) : (eKin > low);
  if (make_e) {
    R ex = E0 * d0x - gE * gx, ey = E0 * d0y - gE * gy, ez = E0 * d0z - gE * gz;
    unit3(ex, ey, ez);
    io.add(1, eKin, ex, ey, ez);
  } else {
    io.edep += eKin;
  }
  return io.nsec;
}

// ProxySauterGavrila::GetPhotoElectronEnergy, ProxySauterGavrila.hpp:132-145
// (quirk); physics: the innermost shell with B <= E, 0 if none.
__device__ __forceinline__ double photo_electron_energy(const Data &d, int Z, double e, int mode)
{
  int n = d.nshell[Z];
  const double *b = d.binding + d.ishell[Z];
  int i = 0;
  if (mode == 0) {
    while (i < n && e >= __ldg(&b[i]) * eV) i++;
    return e - __ldg(&b[i]) * eV;
  }
  while (i < n && e < __ldg(&b[i]) * eV) i++;
  return (i < n) ? e - __ldg(&b[i]) * eV : 0.0;
}

// Sauter-Gavrila photo-electric, ProxySauterGavrila.hpp:67-130
template <class R>
__device__ int sg_sample(Mrg &r, const Data &d, const ModelParams &p, Inter<R> &io, int *err)
{
  R gE = io.E;
  io.nsec = 0;
  int Z = (p.mode == 0) ? 10 : p.Z;
  R eE = (R)photo_electron_energy(d, Z, (double)gE, p.mode);
  if (p.mode != 0 && eE <= R(0)) {
    io.edep += gE;
    io.E = R(0);
    io.status = 1;
    return 0;
  }
  R tau = gE / R(kEMass);
  R cost = R(-1);
  if (tau > R(50)) {
    cost = R(1);
  } else {
    R gam = tau + R(1);
    R beta = M<R>::sqrt(tau * (tau + R(2))) / gam;
    R A = (R(1) - beta) / beta;
    R Ap2 = A + R(2);
    R B = R(0.5) * beta * gam * (gam - R(1)) * (gam - R(2));
    R grej = R(2) * (R(1) + A * B) / A;
    R z, g;
    int it = 0;
    do {
      R q = r.u<R>();
      z = R(2) * A * (R(2) * q + Ap2 * M<R>::sqrt(q)) / (Ap2 * Ap2 - R(4) * q);
      g = (R(2) - z) * (R(1) / (A + z) + B);
      if (++it > kRejectCap) {
        *err |= kErrRejectCap;
        break;
      }
    } while (g < r.u<R>() * grej);
    cost = R(1) - z;
  }
  R sint = M<R>::sqrt((R(1) + cost) * (R(1) - cost));
  R sphi, cphi;
  M<R>::sincos2pi(r.u<R>(), &sphi, &cphi);
  R xh = sint * cphi, yh = sint * sphi, zh = cost;
  rotate_to_lab(xh, yh, zh, io.dir[0], io.dir[1], io.dir[2]);
  io.add(1, eE, xh, yh, zh);
  if (p.mode != 0) io.edep += gE - eE;
  io.E = R(0);
  io.status = 1;
  return io.nsec;
}

// ProxyEmModel::ComputeCoulombFactor, ProxyEmModel.hpp:114-128
__device__ __forceinline__ double coulomb_factor(double Zeff)
{
  double az1 = (1.0 / 137) * Zeff;
  double az2 = az1 * az1, az4 = az2 * az2;
  return (0.0083 * az4 + 0.20206 + 1. / (1. + az2)) * az2 - (0.0020 * az4 + 0.0369) * az4;
}
template <class R> __device__ __forceinline__ R screen1(R s)
{
  return (s > R(1)) ? R(42.24) - R(8.368) * M<R>::log(s + R(0.952)) : R(42.392) - s * (R(7.796) - R(1.961) * s);
}
template <class R> __device__ __forceinline__ R screen2(R s)
{
  return (s > R(1)) ? R(42.24) - R(8.368) * M<R>::log(s + R(0.952)) : R(41.405) - s * (R(5.828) - R(0.8945) * s);
}

// Bethe-Heitler pair production, ProxyBetheHeitler.hpp:64-182
template <class R> __device__ int bh_sample(Mrg &r, const ModelParams &p, Inter<R> &io, int *err)
{
  R gE = io.E;
  io.nsec = 0;
  R epsil0 = R(kEMass) / gE;
  if (epsil0 > R(0.5)) return 0;
  int Z = (p.mode == 0) ? 10 : p.Z;
  R epsil;
  if (gE < R(2.0)) {
    epsil = epsil0 + (R(0.5) - epsil0) * r.u<R>();
  } else {
    double zi = (double)(int)(Z + 0.5);
    R logZ3 = (R)(dlog(zi) / 3.0);
    R FZ = R(8) * logZ3;
    if (gE > R(50.0)) FZ += R(8) * (R)coulomb_factor((double)Z);
    R Z3 = (R)dpow(zi, 1 / 3.0);
    R screenfac = R(136) * epsil0 / Z3;
    R screenmax = M<R>::exp((R(42.24) - FZ) / R(8.368)) - R(0.952);
    R screenmin = fmin(R(4) * screenfac, screenmax);
    R epsil1 = R(0.5) - R(0.5) * M<R>::sqrt(R(1) - screenmin / screenmax);
    R epsilmin = fmax(epsil0, epsil1);
    R epsilrange = R(0.5) - epsilmin;
    R screenvar, greject;
    R F10 = screen1(screenmin) - FZ;
    R F20 = screen2(screenmin) - FZ;
    R NormF1 = fmax(F10 * epsilrange * epsilrange, R(0));
    R NormF2 = fmax(R(1.5) * F20, R(0));
    int it = 0;
    do {
      if (NormF1 / (NormF1 + NormF2) > r.u<R>()) {
        epsil = R(0.5) - epsilrange * M<R>::pow(r.u<R>(), R(0.333333));
        screenvar = screenfac / (epsil * (R(1) - epsil));
        greject = (screen1(screenvar) - FZ) / F10;
      } else {
        epsil = epsilmin + epsilrange * r.u<R>();
        screenvar = screenfac / (epsil * (R(1) - epsil));
        greject = (screen2(screenvar) - FZ) / F20;
      }
      if (++it > kRejectCap) {
        *err |= kErrRejectCap;
        break;
      }
    } while (greject < r.u<R>());
  }
  R eTot = (r.u<R>() > R(0.5)) ? (R(1) - epsil) * gE : epsil * gE;
  R pTot = gE - eTot;
  R u1 = r.u<R>();
  R u2 = r.u<R>();
  R aa0 = -M<R>::log(u1 * u2);
  R u = (R(0.25) > r.u<R>()) ? aa0 / R(0.625) : aa0 / R(1.875);
  R sinp, cosp;
  M<R>::sincos2pi(r.u<R>(), &sinp, &cosp);
  R cost = u * R(kEMass) / eTot;
  if (p.mode != 0) cost = M<R>::cosr(cost);
  R sint = M<R>::sqrt((R(1) - cost) * (R(1) + cost));
  R xh = sint * cosp, yh = sint * sinp, zh = cost;
  rotate_to_lab(xh, yh, zh, io.dir[0], io.dir[1], io.dir[2]);
  io.add(1, eTot - R(kEMass), xh, yh, zh);
  cost = u * R(kEMass) / pTot;
  if (p.mode != 0) cost = M<R>::cosr(cost);
  sint = M<R>::sqrt((R(1) - cost) * (R(1) + cost));
  xh = -sint * cosp;
  yh = -sint * sinp;
  zh = cost;
  rotate_to_lab(xh, yh, zh, io.dir[0], io.dir[1], io.dir[2]);
  io.add(2, pTot - R(kEMass), xh, yh, zh);
  io.E = R(0);
  io.status = 1;
  return io.nsec;
}

// Seltzer-Berger bremsstrahlung, ProxySeltzerBerger.hpp:204-315
template <class R> __device__ int sb_sample(Mrg &r, const ModelParams &p, Inter<R> &io, int *err)
{
  R kin = io.E;
  io.nsec = 0;
  bool quirk = p.mode == 0;
  R cut = fmin(quirk ? R(1.0 * keV) : (R)p.cut, kin);
  R emax = fmin(R(1.0 * TeV), kin);
  if (cut >= emax) return 0;
  const SBTable &T = *p.sb;
  R totalEnergy = kin + R(kEMass);
  R densityCorr = (R)p.density_factor * totalEnergy * totalEnergy;
  R xmin = M<R>::log(cut * cut + densityCorr);
  R xmax = M<R>::log(emax * emax + densityCorr);
  R y = M<R>::log(kin);
  R x0 = cut / kin;
  const SBRow row = sb_row(T, (double)y); // y is the same for every lookup below but one
  R vmax = sb_value_row<R>(T, row, x0) * R(1.02);
  if (x0 < R(0.97) && ((kin > R(300.0)) || (kin < R(10 * keV)))) {
    R ylim = fmin(sb_value<R>(T, R(0.97), R(4 * 2.302585092994046)), R(1.1) * sb_value_row<R>(T, row, R(0.97)));
    if (ylim > vmax) vmax = ylim;
  }
  if (x0 < R(0.05)) vmax *= R(1.2);
  R gE = R(0), v;
  int it = 0;
  do {
    R auxrand = r.u<R>();
    R x = M<R>::exp(xmin + auxrand * (xmax - xmin)) - densityCorr;
    if (x < R(0)) x = R(0);
    gE = M<R>::sqrt(x);
    R x1 = gE / kin;
    v = sb_value_row<R>(T, row, x1);
    if (++it > kRejectCap) {
      *err |= kErrRejectCap;
      break;
    }
  } while (v < vmax * r.u<R>());
  // dipole-boosted photon direction (SamplePhotonDirection, :288-315); the
  // reference passes the photon energy, physics mode the electron's
  R c = R(4) - R(8) * r.u<R>();
  R signc = (c < R(0)) ? R(-1) : R(1);
  R a = fabs(c);
  R delta = R(0.5) * (M<R>::sqrt(R(4) + a * a) + a);
  R cofA = -signc * M<R>::cbrt(delta);
  R cosTheta = cofA - R(1) / cofA;
  R tau = (quirk ? gE : kin) / R(kEMass);
  R beta = M<R>::sqrt(tau * (tau + R(2))) / (tau + R(1));
  cosTheta = (cosTheta + beta) / (R(1) + cosTheta * beta);
  R sinTheta = M<R>::sqrt((R(1) - cosTheta) * (R(1) + cosTheta));
  R sphi, cphi;
  M<R>::sincos2pi(r.u<R>(), &sphi, &cphi);
  R gx = sinTheta * cphi, gy = sinTheta * sphi, gz = cosTheta;
  rotate_to_lab(gx, gy, gz, io.dir[0], io.dir[1], io.dir[2]);
  io.add(0, gE, gx, gy, gz);
  R totalMomentum = M<R>::sqrt(kin * (totalEnergy + R(kEMass)));
  io.E -= gE;
  R nx = totalMomentum * io.dir[0] - gE * gx;
  R ny = totalMomentum * io.dir[1] - gE * gy;
  R nz = totalMomentum * io.dir[2] - gE * gz;
  unit3(nx, ny, nz);
  io.dir[0] = nx;
  io.dir[1] = ny;
  io.dir[2] = nz;
  return io.nsec;
}

// delta-ray kinematics shared by Moller and Bhabha, ProxyMollerScattering.hpp:128-156
template <class R> __device__ __forceinline__ void delta_ray(Mrg &r, Inter<R> &io, R kin, R x)
{
  R energy = kin + R(kEMass);
  R deltaKin = x * kin;
  R totalMomentum = M<R>::sqrt(kin * (kin + R(2) * R(kEMass)));
  R deltaMomentum = M<R>::sqrt(deltaKin * (deltaKin + R(2) * R(kEMass)));
  R cost = deltaKin * (energy + R(kEMass)) / (deltaMomentum * totalMomentum);
  if (cost > R(1)) cost = R(1);
  R sint = M<R>::sqrt((R(1) - cost) * (R(1) + cost));
  R sphi, cphi;
  M<R>::sincos2pi(r.u<R>(), &sphi, &cphi);
  R xh = sint * cphi, yh = sint * sphi, zh = cost;
  rotate_to_lab(xh, yh, zh, io.dir[0], io.dir[1], io.dir[2]);
  io.add(1, deltaKin, xh, yh, zh);
  io.E -= deltaKin;
  R nx = totalMomentum * io.dir[0] - deltaMomentum * xh;
  R ny = totalMomentum * io.dir[1] - deltaMomentum * yh;
  R nz = totalMomentum * io.dir[2] - deltaMomentum * zh;
  unit3(nx, ny, nz);
  io.dir[0] = nx;
  io.dir[1] = ny;
  io.dir[2] = nz;
}

// Moller scattering, ProxyMollerScattering.hpp:92-159
template <class R> __device__ int mb_sample(Mrg &r, const ModelParams &p, Inter<R> &io, int *err)
{
  R kin = io.E;
  io.nsec = 0;
  R tmin = (p.mode == 0) ? R(1.0 * keV) : (R)p.cut;
  R tmax = R(0.5) * kin;
  if (R(1.0 * TeV) < tmax) tmax = R(1.0 * TeV);
  if (tmin >= tmax) return 0;
  R energy = kin + R(kEMass);
  R xmin = tmin / kin, xmax = tmax / kin;
  R gam = energy / R(kEMass), gamma2 = gam * gam;
  R x, z;
  R gg = (R(2) * gam - R(1)) / gamma2;
  R y = R(1) - xmax;
  R grej = R(1) - gg * xmax + xmax * xmax * (R(1) - gg + (R(1) - gg * y) / (y * y));
  int it = 0;
  do {
    R rndm = r.u<R>();
    x = xmin * xmax / (xmin * (R(1) - rndm) + xmax * rndm);
    y = R(1) - x;
    z = R(1) - gg * x + x * x * (R(1) - gg + (R(1) - gg * y) / (y * y));
    if (++it > kRejectCap) {
      *err |= kErrRejectCap;
      break;
    }
  } while (grej * r.u<R>() > z);
  delta_ray(r, io, kin, x);
  return io.nsec;
}

// Bhabha scattering (published Geant4 Moller-Bhabha sampling; the reference
// has no positron model).
template <class R> __device__ int bhabha_sample(Mrg &r, const ModelParams &p, Inter<R> &io, int *err)
{
  R kin = io.E;
  io.nsec = 0;
  R tmin = (R)p.cut, tmax = kin;
  if (tmin >= tmax) return 0;
  R energy = kin + R(kEMass);
  R xmin = tmin / kin, xmax = tmax / kin;
  R gam = energy / R(kEMass), gamma2 = gam * gam;
  R beta2 = R(1) - R(1) / gamma2;
  R y = R(1) / (R(1) + gam);
  R y2 = y * y;
  R y12 = R(1) - R(2) * y;
  R b1 = R(2) - y2;
  R b2 = y12 * (R(3) + y2);
  R y122 = y12 * y12;
  R b4 = y122 * y12;
  R b3 = b4 + y122;
  y = xmax * xmax;
  R grej = R(1) + (y * y * b4 - xmin * xmin * xmin * b3 + y * b2 - xmin * b1) * beta2;
  R x, z;
  int it = 0;
  do {
    R rndm = r.u<R>();
    x = xmin * xmax / (xmin * (R(1) - rndm) + xmax * rndm);
    y = x * x;
    z = R(1) + (y * y * b4 - x * y * b3 + y * b2 - x * b1) * beta2;
    if (++it > kRejectCap) {
      *err |= kErrRejectCap;
      break;
    }
  } while (grej * r.u<R>() > z);
  delta_ray(r, io, kin, x);
  return io.nsec;
}

// Two-photon annihilation (published Geant4 eeToTwoGamma sampling); at rest
// (E == 0) two back-to-back m_e c^2 photons, isotropic.
template <class R> __device__ int annih_sample(Mrg &r, Inter<R> &io, int *err)
{
  R kin = io.E;
  io.nsec = 0;
  if (kin <= R(0)) {
    R cost = R(2) * r.u<R>() - R(1);
    R sint = M<R>::sqrt((R(1) - cost) * (R(1) + cost));
    R sphi, cphi;
    M<R>::sincos2pi(r.u<R>(), &sphi, &cphi);
    R dx = sint * cphi, dy = sint * sphi, dz = cost;
    io.add(0, R(kEMass), dx, dy, dz);
    io.add(0, R(kEMass), -dx, -dy, -dz);
  } else {
    R tau = kin / R(kEMass);
    R gam = tau + R(1);
    R tau2 = tau + R(2);
    R sqgrate = M<R>::sqrt(tau / tau2) * R(0.5);
    R sqg2m1 = M<R>::sqrt(tau * tau2);
    R epsilmin = R(0.5) - sqgrate;
    R epsilmax = R(0.5) + sqgrate;
    R lq = M<R>::log(epsilmax / epsilmin);
    R epsil, greject;
    int it = 0;
    do {
      epsil = epsilmin * M<R>::exp(lq * r.u<R>());
      greject = R(1) - epsil + (R(2) * gam * epsil - R(1)) / (epsil * tau2 * tau2);
      if (++it > kRejectCap) {
        *err |= kErrRejectCap;
        break;
      }
    } while (greject < r.u<R>());
    R cost = (epsil * tau2 - R(1)) / (epsil * sqg2m1);
    cost = fmin(fmax(cost, R(-1)), R(1));
    R sint = M<R>::sqrt((R(1) + cost) * (R(1) - cost));
    R sphi, cphi;
    M<R>::sincos2pi(r.u<R>(), &sphi, &cphi);
    R tot = kin + R(2) * R(kEMass);
    R e1 = epsil * tot, e2 = (R(1) - epsil) * tot;
    R dx = sint * cphi, dy = sint * sphi, dz = cost;
    rotate_to_lab(dx, dy, dz, io.dir[0], io.dir[1], io.dir[2]);
    R pp = M<R>::sqrt(kin * (kin + R(2) * R(kEMass)));
    R ex = pp * io.dir[0] - e1 * dx, ey = pp * io.dir[1] - e1 * dy, ez = pp * io.dir[2] - e1 * dz;
    unit3(ex, ey, ez);
    io.add(0, e1, dx, dy, dz);
    io.add(0, e2, ex, ey, ez);
  }
  io.E = R(0);
  io.status = 1;
  return io.nsec;
}

// Heitler e+ e- -> 2 gamma cross section per target electron, mm^2
__device__ __forceinline__ double annih_xs_per_electron(double pi_rcl2, double kin)
{
  double ekin = fmax(eV, kin);
  double tau = ekin / kEMass, gam = tau + 1.0, gamma2 = gam * gam;
  double bg2 = tau * (tau + 2.0), bg = ::sqrt(bg2);
  return pi_rcl2 * ((gamma2 + 4 * gam + 1.) * dlog(gam + bg) - (gam + 3.) * bg) / (bg2 * (gam + 1.));
}

// The same cross section times the material's electron density (1/mm), in
// the working precision: FP64 as above; in the FP32-mixed build the Heitler
// formula in FP32 (single-precision log and square root instead of the FP64
// ones on every positron step; relative error ~1e-6).
template <class R> __device__ __forceinline__ R annih_xs(const Data &d, int mat, R kin)
{
  if constexpr (sizeof(R) == 8) {
    return d.mat_nel[mat] * annih_xs_per_electron(d.pi_rcl2, kin);
  } else {
    const float ekin = fmaxf(kin, (float)eV), tau = ekin / (float)kEMass, gam = tau + 1.0f;
    const float bg2 = tau * (tau + 2.0f), bg = sqrtf(bg2);
    const float f = ((gam * gam + 4.0f * gam + 1.0f) * logf(gam + bg) - (gam + 3.0f) * bg) / (bg2 * (gam + 1.0f));
    return (float)(d.mat_nel[mat] * d.pi_rcl2) * f;
  }
}

// Sandia photo-absorption below 200 keV (Geant4 photo-electric cross section
// below the reference's LambdaPrim.phot table), 1/mm.
__device__ __forceinline__ double pe_xs_sandia(const Data &d, int Z, double density, double e)
{
  double ekev = e / keV;
  int first = d.cumint[Z - 1], n = d.nint[Z];
  int row = first + n - 1;
  while (row > first && ekev < __ldg(&d.sandia[5 * row])) --row;
  if (ekev < __ldg(&d.sandia[5 * row])) return 0.0;
  const double *a = d.sandia + 5 * row;
  double i1 = 1.0 / ekev;
  double s = i1 * (__ldg(&a[1]) + i1 * (__ldg(&a[2]) + i1 * (__ldg(&a[3]) + i1 * __ldg(&a[4]))));
  return fmax(s, 0.0) * density * 0.1;
}
// The same for the FP32-mixed engine: the energy scaled by a multiplication,
// the interval found in FP64 as above, the polynomial in 1/E in FP32 (its
// reciprocal from the FP32 unit) instead of two FP64 divisions.
__device__ __forceinline__ float pe_xs_sandia_f(const Data &d, int Z, float density, float e)
{
  const double ekev = (double)e * (1.0 / keV);
  int first = d.cumint[Z - 1], n = d.nint[Z];
  int row = first + n - 1;
  while (row > first && ekev < __ldg(&d.sandia[5 * row])) --row;
  if (ekev < __ldg(&d.sandia[5 * row])) return 0.0f;
  const double *a = d.sandia + 5 * row;
  const float i1 = __frcp_rn((float)ekev);
  const float s = i1 * ((float)__ldg(&a[1]) +
                        i1 * ((float)__ldg(&a[2]) + i1 * ((float)__ldg(&a[3]) + i1 * (float)__ldg(&a[4]))));
  return fmaxf(s, 0.0f) * density * 0.1f;
}

// ------------------------------------------------------------------ helix
// ConstFieldHelixStepper::DoStep, ConstFieldHelixStepper.hpp:164-239 (FP64)
__device__ __forceinline__ void helix_dostep(double kB2C, const double B[3], const double pos[3],
                                             const double dir[3], double charge, double momentum, double step,
                                             double np[3], double nd[3])
{
  const double kSmall = 1.E-30;
  double Bmag = ::sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
  double ux = B[0], uy = B[1], uz = B[2];
  if (Bmag > 0) {
    ux /= Bmag;
    uy /= Bmag;
    uz /= Bmag;
  }
  double UVdotUB = dir[0] * ux + dir[1] * uy + dir[2] * uz;
  double dt2 = fmax(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2] - UVdotUB * UVdotUB, 0.0);
  double sinVB = ::sqrt(dt2) + kSmall;
  double R = momentum * sinVB / (kB2C * charge * Bmag);
  double vx = dir[0] - UVdotUB * ux, vy = dir[1] - UVdotUB * uy, vz = dir[2] - UVdotUB * uz;
  unit3(vx, vy, vz);
  double cx = vy * uz - vz * uy, cy = vz * ux - vx * uz, cz = vx * uy - vy * ux;
  double phi = -step * charge * Bmag * kB2C / momentum;
  double sinphi, cosphi;
  dsincos(phi, &sinphi, &cosphi);
  np[0] = pos[0] + R * (cosphi - 1) * cx - R * sinphi * vx + step * UVdotUB * ux;
  np[1] = pos[1] + R * (cosphi - 1) * cy - R * sinphi * vy + step * UVdotUB * uy;
  np[2] = pos[2] + R * (cosphi - 1) * cz - R * sinphi * vz + step * UVdotUB * uz;
  nd[0] = UVdotUB * ux + cosphi * sinVB * vx + sinphi * sinVB * cx;
  nd[1] = UVdotUB * uy + cosphi * sinVB * vy + sinphi * sinVB * cy;
  nd[2] = UVdotUB * uz + cosphi * sinVB * vz + sinphi * sinVB * cz;
}

// ------------------------------------------------------------ processes
// ProxyIonization::AlongStepGPIL, ProxyIonization.hpp:108-128 (quirk: energy
// cut with stride 4 used as a length and 2 finR/range; physics: length cut,
// Geant4 step function).
__device__ __forceinline__ double ioni_along_gpil_ref(const Data &d, int mode, int charge, int mat, double e)
{
  const double dR = 0.2, finalRange = 10.0;
  int rt = (mode == 1 && charge > 0) ? 19 : 18;
  double range = vec_value_ref(d, d.vec[rt][mat], e);
  if (e < kMinE) range *= e / kMinE;
  double cut;
  if (mode == 0) {
    int k = 4 * 1 + mat;
    cut = (k < 12) ? d.cut_raw[k] : 0.0;
  } else {
    cut = d.cut_length[1][mat];
  }
  double finR = (finalRange < cut) ? finalRange : cut;
  if (range <= finR) return range;
  if (mode == 0) return range * dR + finR * (1.0 - dR) * (2.0 * finR / range);
  return range * dR + finR * (1.0 - dR) * (2.0 - finR / range);
}

// ProxyIonization::AlongStepDoIt, ProxyIonization.hpp:130-168 (quirk: the
// inverse range through Value(), bin kept inside the vector; physics:
// InvRangeValue).
__device__ __forceinline__ void ioni_along_doit_ref(const Data &d, int mode, int charge, int mat, double step,
                                                    double &e, double &edep)
{
  bool ep = (mode == 1 && charge > 0);
  double energy = e;
  double range = vec_value_ref(d, d.vec[ep ? 19 : 18][mat], energy);
  if (step >= range || energy <= kMinE) {
    e = 0.0;
    edep += energy;
    return;
  }
  double dedx = vec_value_ref(d, d.vec[ep ? 3 : 2][mat], energy);
  if (energy < kMinE) dedx *= ::sqrt(energy / kMinE);
  double eloss = step * dedx;
  if (eloss > energy * 0.01) {
    range -= step;
    const VecDesc &iv = d.vec[ep ? 5 : 4][mat];
    double einv = (mode == 0) ? vec_value_ref(d, iv, range) : vec_invrange_ref(d, iv, range);
    eloss = energy - einv;
  }
  double finalE = energy - eloss;
  if (finalE < kMinE) {
    eloss += finalE;
    finalE = 0.0;
  }
  eloss = fmax(eloss, 0.0);
  e = finalE;
  edep += eloss;
}

} // namespace gx
