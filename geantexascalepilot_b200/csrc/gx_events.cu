// gx_events.cu -- primary generation feeding the transport's device arrays:
// the e/gamma particle gun on the device, the HEPEVT ASCII event reader on the
// host.
//
// The reference's ProxyEgammaGun draws four uniforms per particle from one
// MRG32k3a stream, particle after particle and event after event
// (proxy/src/ProxyEgammaGun.cpp:43-85).  Here every thread produces a chunk of
// consecutive particles: it jumps the stream ahead to its chunk's first draw
// (A^n applied to the seed, n = 4 x particle index, by binary powers of A) and
// then draws in the reference's order, so the device output equals the
// reference's sequential output particle for particle.
#include "gx_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

namespace gx {

namespace {

constexpr uint64_t kMod1 = 4294967087ULL, kMod2 = 4294944443ULL;
constexpr int kGunChunk = 16; // particles per thread

std::mutex g_step_mu;
uint64_t *g_step_jump[64]; // per device: A^(2^j) for j = 0..63, [component][j][3x3]

// A^(2^j), j = 0..63, of both MRG32k3a components, on the current device.
int get_step_jump_table(uint64_t **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return set_error(GX_ERR_ARG, "device index %d", dev);
  std::lock_guard<std::mutex> lk(g_step_mu);
  if (!g_step_jump[dev]) {
    static uint64_t h[2][64][9];
    const uint64_t m[2] = {kMod1, kMod2};
    for (int c = 0; c < 2; ++c) {
      uint64_t P[9];
      jump_matrix(c, 0, 1, P); // A
      for (int j = 0; j < 64; ++j) {
        std::memcpy(h[c][j], P, sizeof(P));
        mat_mul(P, P, P, m[c]);
      }
    }
    uint64_t *d = nullptr;
    if ((e = cudaMalloc((void **)&d, sizeof(h))) != cudaSuccess) return cuda_error(e, "cudaMalloc step jump table");
    if ((e = cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_error(e, "cudaMemcpy step jump table");
    g_step_jump[dev] = d;
  }
  *out = g_step_jump[dev];
  return GX_OK;
}

__device__ __forceinline__ void matvec_mod(const uint64_t *A, uint64_t v[3], uint64_t m)
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

struct Gun {
  long long n, first_draw;
  int nparticles, first_event;
  double gamma_fraction, minp, maxp, mineta, maxeta, minphi, maxphi;
  double vertex[3];
  uint64_t s[6];
};

__global__ void __launch_bounds__(256) k_egamma_gun(const uint64_t *__restrict__ J, Gun g, int *__restrict__ type,
                                                    double *__restrict__ E, double *__restrict__ pos,
                                                    double *__restrict__ dir, int *__restrict__ event,
                                                    int *__restrict__ pdg)
{
  const long long first = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kGunChunk;
  if (first >= g.n) return;
  const long long last = min(first + (long long)kGunChunk, g.n);
  uint64_t v1[3] = {g.s[0], g.s[1], g.s[2]}, v2[3] = {g.s[3], g.s[4], g.s[5]};
  unsigned long long k = (unsigned long long)g.first_draw + 4ULL * (unsigned long long)first;
  for (int b = 0; k != 0 && b < 64; ++b, k >>= 1)
    if (k & 1ULL) {
      matvec_mod(J + 9 * b, v1, kMod1);
      matvec_mod(J + 9 * (64 + b), v2, kMod2);
    }
  Mrg r;
  for (int c = 0; c < 3; ++c) {
    r.s[c] = (uint32_t)v1[c];
    r.s[3 + c] = (uint32_t)v2[c];
  }
  for (long long i = first; i < last; ++i) {
    const bool gamma = r.u01() < g.gamma_fraction;
    const double charge = gamma ? 0.0 : -1.0;
    const double p = g.minp + (g.maxp - g.minp) * r.u01();
    const double mass = kEMass * charge * charge;
    const double eta = g.mineta + (g.maxeta - g.mineta) * r.u01();
    const double phi = g.minphi + (g.maxphi - g.minphi) * r.u01();
    const double theta = 2. * ::atan(::exp(-eta));
    type[i] = gamma ? 0 : 1;
    if (pdg) pdg[i] = gamma ? 22 : 11;
    E[i] = p * p / (::sqrt(p * p + mass * mass) + mass);
    const double st = ::sin(theta);
    dir[3 * i + 0] = st * ::cos(phi);
    dir[3 * i + 1] = st * ::sin(phi);
    dir[3 * i + 2] = ::cos(theta);
    pos[3 * i + 0] = g.vertex[0];
    pos[3 * i + 1] = g.vertex[1];
    pos[3 * i + 2] = g.vertex[2];
    if (event) event[i] = g.first_event + (int)(i / g.nparticles);
  }
}

// The beam-spot gun (gx_spot_gun): one primary from its five uniforms.
struct Spot {
  long long n, first;
  int ntypes, types[3], axis;
  double emin, emax, cos_cone, centre[3], half[2];
};

__host__ __device__ __forceinline__ void spot_primary(const Spot &g, long long i, const double u[5], int *type,
                                                      double *E, double *pos, double *dir)
{
  *type = g.types[i % g.ntypes];
  *E = g.emin * ::exp(u[0] * ::log(g.emax / g.emin));
  const double ct = 1.0 - u[1] * (1.0 - g.cos_cone), st = ::sqrt((1.0 - ct) * (1.0 + ct));
  const double phi = 2.0 * kPi * u[2];
  const int a = g.axis, b = (a + 1) % 3, c = (a + 2) % 3;
  double d[3], p[3];
  d[a] = ct;
  d[b] = st * ::cos(phi);
  d[c] = st * ::sin(phi);
  p[a] = g.centre[a];
  p[b] = g.centre[b] + g.half[0] * (2.0 * u[3] - 1.0);
  p[c] = g.centre[c] + g.half[1] * (2.0 * u[4] - 1.0);
  for (int k = 0; k < 3; ++k) {
    dir[k] = d[k];
    pos[k] = p[k];
  }
}

// the stream's state (seed advanced by stream x 2^127, then by 5 first draws)
void spot_start(const gx_spot_gun_params &p, uint64_t v1[3], uint64_t v2[3])
{
  const uint64_t m[2] = {kMod1, kMod2};
  for (int k = 0; k < 3; ++k) {
    v1[k] = (uint64_t)p.seed[k];
    v2[k] = (uint64_t)p.seed[3 + k];
  }
  uint64_t J[9];
  for (int c = 0; c < 2; ++c) {
    jump_matrix(c, 127, 0, J);
    for (long long s = 0; s < p.stream; ++s) mat_vec(J, c ? v2 : v1, m[c]);
  }
}

__global__ void __launch_bounds__(256) k_spot_gun(const uint64_t *__restrict__ J, Spot g, uint64_t s0, uint64_t s1,
                                                  uint64_t s2, uint64_t s3, uint64_t s4, uint64_t s5,
                                                  int *__restrict__ type, double *__restrict__ E,
                                                  double *__restrict__ pos, double *__restrict__ dir)
{
  const long long first = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kGunChunk;
  if (first >= g.n) return;
  const long long last = min(first + (long long)kGunChunk, g.n);
  uint64_t v1[3] = {s0, s1, s2}, v2[3] = {s3, s4, s5};
  unsigned long long k = 5ULL * (unsigned long long)(g.first + first);
  for (int b = 0; k != 0 && b < 64; ++b, k >>= 1)
    if (k & 1ULL) {
      matvec_mod(J + 9 * b, v1, kMod1);
      matvec_mod(J + 9 * (64 + b), v2, kMod2);
    }
  Mrg r;
  for (int c = 0; c < 3; ++c) {
    r.s[c] = (uint32_t)v1[c];
    r.s[3 + c] = (uint32_t)v2[c];
  }
  for (long long i = first; i < last; ++i) {
    double u[5];
    for (int j = 0; j < 5; ++j) u[j] = r.u01();
    spot_primary(g, g.first + i, u, &type[i], &E[i], &pos[3 * i], &dir[3 * i]);
  }
}

// MRG32k3a on the host in exact integer arithmetic (the same numbers as the
// device's FP64 recurrence)
struct HostMrg {
  int64_t s[6];
  double u01()
  {
    const int64_t m1 = (int64_t)kMod1, m2 = (int64_t)kMod2;
    int64_t p1 = ((int64_t)kA12 * s[1] - (int64_t)kA13n * s[0]) % m1;
    if (p1 < 0) p1 += m1;
    s[0] = s[1];
    s[1] = s[2];
    s[2] = p1;
    int64_t p2 = ((int64_t)kA21 * s[5] - (int64_t)kA23n * s[3]) % m2;
    if (p2 < 0) p2 += m2;
    s[3] = s[4];
    s[4] = s[5];
    s[5] = p2;
    return (double)(p1 > p2 ? p1 - p2 : p1 - p2 + m1) * kNorm;
  }
};

int spot_check(const gx_spot_gun_params *p, long long n, Spot &g)
{
  if (!p || n < 0) return set_error(GX_ERR_ARG, "gx_spot_gun: bad arguments");
  if (p->ntypes < 1 || p->ntypes > 3 || p->axis < 0 || p->axis > 2 || p->stream < 0 || p->first < 0 ||
      !(p->emin > 0.0 && p->emax >= p->emin) || !(p->cone_deg >= 0.0 && p->cone_deg <= 180.0))
    return set_error(GX_ERR_ARG, "gx_spot_gun: bad parameters");
  for (int k = 0; k < p->ntypes; ++k)
    if (p->types[k] < 0 || p->types[k] > 2) return set_error(GX_ERR_ARG, "gx_spot_gun: bad particle type");
  g.n = n;
  g.first = p->first;
  g.ntypes = p->ntypes;
  for (int k = 0; k < 3; ++k) g.types[k] = p->types[k];
  g.axis = p->axis;
  g.emin = p->emin;
  g.emax = p->emax;
  g.cos_cone = ::cos(p->cone_deg * kPi / 180.0);
  for (int k = 0; k < 3; ++k) g.centre[k] = p->centre[k];
  g.half[0] = p->half[0];
  g.half[1] = p->half[1];
  return GX_OK;
}

// One HEPEVT event entry (G4HEPEvtInterface layout, as the reference reads
// it, proxy/ProxyHepEvtGenerator.hpp:40-49).
struct HepEntry {
  int ist, id, jda1, jda2;
  double p[4]; // px, py, pz (GeV), mass (GeV)
};

} // namespace

int pdg_to_type(int pdg) { return pdg == 22 ? 0 : (pdg == 11 ? 1 : (pdg == -11 ? 2 : -1)); }

} // namespace gx

using namespace gx;

extern "C" {

int gx_egamma_gun(const gx_egamma_gun_params *p, int *d_type, double *d_E, double *d_pos, double *d_dir,
                  int *d_event, int *d_pdg, gx_stream_t stream)
{
  if (!p || p->nevents < 0 || p->nparticles < 0 || p->first_draw < 0)
    return set_error(GX_ERR_ARG, "gx_egamma_gun: bad arguments");
  const long long n = (long long)p->nevents * p->nparticles;
  if (n > 0x7fffffffLL) return set_error(GX_ERR_ARG, "gx_egamma_gun: %lld particles exceed 2^31 - 1", n);
  if (n == 0) return GX_OK;
  if (!d_type || !d_E || !d_pos || !d_dir) return set_error(GX_ERR_ARG, "gx_egamma_gun: null output");
  if (!(p->min_p >= 0.0 && p->max_p >= p->min_p))
    return set_error(GX_ERR_ARG, "gx_egamma_gun: momentum range [%g, %g]", p->min_p, p->max_p);
  if (p->first_draw > (long long)(0x3fffffffffffffffLL - 4 * n))
    return set_error(GX_ERR_ARG, "gx_egamma_gun: first_draw too large");
  Gun g;
  g.n = n;
  g.first_draw = p->first_draw;
  g.nparticles = p->nparticles;
  g.first_event = p->first_event;
  g.gamma_fraction = p->gamma_fraction;
  g.minp = p->min_p;
  g.maxp = p->max_p;
  g.mineta = p->min_eta;
  g.maxeta = p->max_eta;
  g.minphi = p->min_phi;
  g.maxphi = p->max_phi;
  for (int k = 0; k < 3; ++k) g.vertex[k] = p->vertex[k];
  for (int k = 0; k < 6; ++k) {
    const double v = p->seed[k];
    const uint64_t m = k < 3 ? kMod1 : kMod2;
    if (!(v >= 0.0 && v < (double)m && v == std::floor(v)))
      return set_error(GX_ERR_ARG, "gx_egamma_gun: seed word %d = %g is not an integer in [0, m)", k, v);
    g.s[k] = (uint64_t)v;
  }
  uint64_t *J;
  int rc = get_step_jump_table(&J);
  if (rc) return rc;
  const long long threads = (n + kGunChunk - 1) / kGunChunk;
  const int block = 256;
  k_egamma_gun<<<(unsigned)((threads + block - 1) / block), block, 0, stream_of(stream)>>>(J, g, d_type, d_E, d_pos,
                                                                                          d_dir, d_event, d_pdg);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GX_OK : cuda_error(e, "k_egamma_gun");
}

int gx_spot_gun(const gx_spot_gun_params *p, long long n, int *d_type, double *d_E, double *d_pos, double *d_dir,
                gx_stream_t s)
{
  Spot g;
  int rc = spot_check(p, n, g);
  if (rc) return rc;
  if (n > 0 && (!d_type || !d_E || !d_pos || !d_dir)) return set_error(GX_ERR_ARG, "gx_spot_gun: null output");
  if (n == 0) return GX_OK;
  uint64_t *J;
  if ((rc = get_step_jump_table(&J))) return rc;
  uint64_t v1[3], v2[3];
  spot_start(*p, v1, v2);
  const long long threads = (n + kGunChunk - 1) / kGunChunk;
  k_spot_gun<<<(unsigned)((threads + 255) / 256), 256, 0, stream_of(s)>>>(J, g, v1[0], v1[1], v1[2], v2[0], v2[1],
                                                                          v2[2], d_type, d_E, d_pos, d_dir);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GX_OK : cuda_error(e, "k_spot_gun");
}

int gx_spot_gun_host(const gx_spot_gun_params *p, long long n, int *type, double *E, double *pos, double *dir)
{
  Spot g;
  int rc = spot_check(p, n, g);
  if (rc) return rc;
  if (n > 0 && (!type || !E || !pos || !dir)) return set_error(GX_ERR_ARG, "gx_spot_gun_host: null output");
  uint64_t v1[3], v2[3];
  spot_start(*p, v1, v2);
  if (p->first > 0) {
    uint64_t J[9];
    const uint64_t m[2] = {kMod1, kMod2};
    for (int c = 0; c < 2; ++c) {
      jump_matrix(c, 0, 5 * p->first, J);
      mat_vec(J, c ? v2 : v1, m[c]);
    }
  }
  HostMrg r;
  for (int k = 0; k < 3; ++k) {
    r.s[k] = (int64_t)v1[k];
    r.s[3 + k] = (int64_t)v2[k];
  }
  for (long long i = 0; i < n; ++i) {
    double u[5];
    for (int j = 0; j < 5; ++j) u[j] = r.u01();
    spot_primary(g, p->first + i, u, &type[i], &E[i], &pos[3 * i], &dir[3 * i]);
  }
  return GX_OK;
}

int gx_pdg_to_type(int pdg) { return pdg_to_type(pdg); }

int gx_hepevt_read(const char *path, int mode, int max_events, int cap, int *h_event, int *h_pdg, double *h_E,
                   double *h_dir, int *n_out, int *nev_out, int *bad_out)
{
  if (!path || !n_out || max_events < 0 || cap < 0 || (cap > 0 && (!h_event || !h_pdg || !h_E || !h_dir)))
    return set_error(GX_ERR_ARG, "gx_hepevt_read: bad arguments");
  if (mode != GX_MODE_QUIRK && mode != GX_MODE_PHYSICS) return set_error(GX_ERR_ARG, "gx_hepevt_read: bad mode");
  FILE *f = std::fopen(path, "r");
  if (!f) return set_error(GX_ERR_DATA, "gx_hepevt_read: cannot open %s", path);
  const bool physics = mode == GX_MODE_PHYSICS;
  const double unit = physics ? 1000.0 : 1.0; // GeV -> MeV; the reference keeps the GeV numbers
  int k = 0, nev = 0, bad = 0, rc = GX_OK;
  std::vector<HepEntry> ent;
  for (int e = 0; e < max_events; ++e) {
    int nhep;
    if (std::fscanf(f, "%d", &nhep) != 1) break; // end of file
    if (nhep < 0 || nhep > (1 << 24)) {
      rc = set_error(GX_ERR_DATA, "gx_hepevt_read: event %d: bad entry count %d", e, nhep);
      break;
    }
    ent.resize(nhep);
    bool ok = true;
    for (int i = 0; i < nhep && ok; ++i) {
      HepEntry &h = ent[i];
      ok = std::fscanf(f, "%d %d %d %d %lf %lf %lf %lf", &h.ist, &h.id, &h.jda1, &h.jda2, &h.p[0], &h.p[1], &h.p[2],
                       &h.p[3]) == 8;
    }
    if (!ok) {
      rc = set_error(GX_ERR_DATA, "gx_hepevt_read: event %d is truncated", e);
      break;
    }
    // daughters of an entry with daughters are marked; the primaries are the
    // marked entries without daughters (proxy/src/ProxyHepEvtGenerator.cpp:82-96)
    for (int i = 0; i < nhep; ++i) {
      if (ent[i].jda1 <= 0) continue;
      for (int j = ent[i].jda1 - 1; j <= ent[i].jda2 - 1; ++j) {
        if (j < 0 || j >= nhep) { // outside the event (the reference reads out of bounds)
          ++bad;
          continue;
        }
        if (ent[j].ist > 0) ent[j].ist = -1;
      }
    }
    for (int i = 0; i < nhep; ++i) {
      const HepEntry &h = ent[i];
      if (!(h.ist == -1 && h.jda1 == 0)) continue;
      if (k >= cap) {
        ++k; // counted, not stored
        continue;
      }
      const double pm = std::sqrt(h.p[0] * h.p[0] + h.p[1] * h.p[1] + h.p[2] * h.p[2]);
      const double pp = pm * unit;
      // the reference squares the mass (quirk); physics mode uses it as given
      const double mass = physics ? h.p[3] * unit : h.p[3] * h.p[3];
      h_event[k] = e;
      h_pdg[k] = h.id;
      h_E[k] = pp * pp / (std::sqrt(pp * pp + mass * mass) + mass);
      for (int c = 0; c < 3; ++c) h_dir[3 * k + c] = pm > 0 ? h.p[c] / pm : h.p[c];
      ++k;
    }
    ++nev;
  }
  std::fclose(f);
  *n_out = k;
  if (nev_out) *nev_out = nev;
  if (bad_out) *bad_out = bad;
  if (rc) return rc;
  if (k > cap) return set_error(GX_ERR_OVERFLOW, "gx_hepevt_read: %d particles, capacity %d", k, cap);
  return GX_OK;
}

int gx_hepevt_load(const char *path, int mode, int max_events, const double vertex[3], int cap, int *d_type,
                   double *d_E, double *d_pos, double *d_dir, int *d_event, int *n_prim, int *n_events,
                   int *n_skipped, gx_stream_t stream)
{
  if (!path || !n_prim || cap < 0 || (cap > 0 && (!d_type || !d_E || !d_pos || !d_dir || !d_event)))
    return set_error(GX_ERR_ARG, "gx_hepevt_load: bad arguments");
  // first pass: count the particles, then read them
  int n = 0, nev = 0, bad = 0;
  int rc = gx_hepevt_read(path, mode, max_events, 0, nullptr, nullptr, nullptr, nullptr, &n, &nev, &bad);
  if (rc != GX_OK && rc != GX_ERR_OVERFLOW) return rc;
  std::vector<int> ev(n > 0 ? n : 1), pdg(n > 0 ? n : 1);
  std::vector<double> E(n > 0 ? n : 1), dir(3 * (size_t)(n > 0 ? n : 1));
  if (n > 0 && (rc = gx_hepevt_read(path, mode, max_events, n, ev.data(), pdg.data(), E.data(), dir.data(), &n, &nev,
                                    &bad)) != GX_OK)
    return rc;
  std::vector<int> t_type, t_event;
  std::vector<double> t_E, t_pos, t_dir;
  int skipped = 0;
  for (int i = 0; i < n; ++i) {
    const int ty = pdg_to_type(pdg[i]);
    if (ty < 0) { // not transported by the EM path
      ++skipped;
      continue;
    }
    t_type.push_back(ty);
    t_event.push_back(ev[i]);
    t_E.push_back(E[i]);
    for (int c = 0; c < 3; ++c) {
      t_pos.push_back(vertex ? vertex[c] : 0.0);
      t_dir.push_back(dir[3 * i + c]);
    }
  }
  const int m = (int)t_type.size();
  *n_prim = m;
  if (n_events) *n_events = nev;
  if (n_skipped) *n_skipped = skipped;
  if (m > cap) return set_error(GX_ERR_OVERFLOW, "gx_hepevt_load: %d primaries, capacity %d", m, cap);
  if (m == 0) return GX_OK;
  cudaStream_t s = stream_of(stream);
  cudaError_t e;
  if ((e = cudaMemcpyAsync(d_type, t_type.data(), m * sizeof(int), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(d_event, t_event.data(), m * sizeof(int), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(d_E, t_E.data(), m * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(d_pos, t_pos.data(), 3 * m * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(d_dir, t_dir.data(), 3 * m * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_error(e, "gx_hepevt_load: copy to the device");
  // the host vectors go out of scope on return: wait for the copies
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "gx_hepevt_load: synchronise");
  return GX_OK;
}

} // extern "C"
