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
    r.s[c] = (double)v1[c];
    r.s[3 + c] = (double)v2[c];
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
