// gx_kernels.cu -- batch kernels behind the per-function entry points of the
// C ABI (RNG, tables, models, process step limits, helix).  These run the
// reference's functions one thread per track in FP64, for parity with the
// reference and for callers that drive their own step loop.
#include "gx_internal.cuh"

#include <cmath>
#include <cstring>
#include <mutex>

namespace gx {

constexpr int kBlock = 256;
static inline int grid_for(long long n) { return (int)((n + kBlock - 1) / kBlock); }

// ----------------------------------------------------------------- RNG
__device__ __forceinline__ uint32_t mulmod_add(uint64_t a, uint64_t s, uint64_t acc, uint64_t m)
{
  return (uint32_t)(((a * s) % m + acc) % m);
}

__device__ __forceinline__ void matvec3(const uint64_t *A, uint32_t v[3], uint64_t m)
{
  uint32_t r[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) acc = mulmod_add(A[3 * i + k], v[k], acc, m);
    r[i] = (uint32_t)acc;
  }
  v[0] = r[0];
  v[1] = r[1];
  v[2] = r[2];
}

// jump[c][b] = A_c^(2^(76+b)), b = 0..63
__global__ void k_rng_substreams(const uint64_t *__restrict__ jump, uint32_t s0, uint32_t s1, uint32_t s2,
                                 uint32_t s3, uint32_t s4, uint32_t s5, long long first, int n,
                                 uint32_t *__restrict__ out)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long k = (unsigned long long)(first + i);
  uint32_t v1[3] = {s0, s1, s2}, v2[3] = {s3, s4, s5};
  for (int b = 0; k != 0 && b < 64; ++b, k >>= 1) {
    if (k & 1ULL) {
      matvec3(jump + 9 * b, v1, 4294967087ULL);
      matvec3(jump + 9 * (64 + b), v2, 4294944443ULL);
    }
  }
  out[0LL * n + i] = v1[0];
  out[1LL * n + i] = v1[1];
  out[2LL * n + i] = v1[2];
  out[3LL * n + i] = v2[0];
  out[4LL * n + i] = v2[1];
  out[5LL * n + i] = v2[2];
}

struct Mat2 {
  uint64_t a[2][9];
};

__global__ void k_rng_matvec(Mat2 M, uint32_t *__restrict__ st, int n)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t v1[3] = {st[i], st[n + i], st[2LL * n + i]};
  uint32_t v2[3] = {st[3LL * n + i], st[4LL * n + i], st[5LL * n + i]};
  matvec3(M.a[0], v1, 4294967087ULL);
  matvec3(M.a[1], v2, 4294944443ULL);
  st[i] = v1[0];
  st[n + i] = v1[1];
  st[2LL * n + i] = v1[2];
  st[3LL * n + i] = v2[0];
  st[4LL * n + i] = v2[1];
  st[5LL * n + i] = v2[2];
}

__global__ void k_rng_uniform(uint32_t *__restrict__ st, int n, int k, double *__restrict__ out)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Mrg r;
  r.load(st, n, i);
  for (int j = 0; j < k; ++j) out[(long long)j * n + i] = r.u01();
  r.store(st, n, i);
}

static std::mutex g_jump_mu;
static uint64_t *g_jump_dev[64] = {nullptr};

// The skip-ahead table of the substream jumps: h[c][b] = A_c^(2^(76 + b))
// mod m_c for the two components c of MRG32k3a, b = 0..63 (A^(2^76) is one
// substream, MRG32k3a::AdvanceState(76, 0)).  The one host recipe of every
// copy of the table on a device.
void build_jump_host(uint64_t h[2][64][9])
{
  const uint64_t m[2] = {4294967087ULL, 4294944443ULL};
  for (int c = 0; c < 2; ++c) {
    uint64_t P[9];
    jump_matrix(c, 76, 0, P); // A^(2^76)
    for (int b = 0; b < 64; ++b) {
      std::memcpy(h[c][b], P, sizeof(P));
      mat_mul(P, P, P, m[c]);
    }
  }
}

int get_jump_table(uint64_t **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return set_error(GX_ERR_ARG, "device index %d", dev);
  std::lock_guard<std::mutex> lk(g_jump_mu);
  if (!g_jump_dev[dev]) {
    uint64_t h[2][64][9];
    build_jump_host(h);
    uint64_t *d = nullptr;
    e = cudaMalloc((void **)&d, sizeof(h));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc jump table");
    e = cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemcpy jump table");
    g_jump_dev[dev] = d;
  }
  *out = g_jump_dev[dev];
  return GX_OK;
}

int launch_substreams(const double seed[6], long long first, int n, uint32_t *d_states, cudaStream_t s)
{
  uint64_t *jt;
  int rc = get_jump_table(&jt);
  if (rc) return rc;
  if (n > 0)
    k_rng_substreams<<<grid_for(n), kBlock, 0, s>>>(jt, (uint32_t)seed[0], (uint32_t)seed[1], (uint32_t)seed[2],
                                                   (uint32_t)seed[3], (uint32_t)seed[4], (uint32_t)seed[5], first,
                                                   n, d_states);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GX_OK : cuda_error(e, "k_rng_substreams");
}

// --------------------------------------------------------------- tables
__global__ void k_table_value(const Data *__restrict__ d, int table, int mat, const double *__restrict__ E,
                              double *__restrict__ out, int n, int inv)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const VecDesc &v = d->vec[table][mat];
  out[i] = inv ? vec_invrange_ref(*d, v, E[i]) : vec_value_ref(*d, v, E[i]);
}

__global__ void k_sb_value(const Data *__restrict__ d, int which, const double *__restrict__ x,
                           const double *__restrict__ y, double *__restrict__ out, int n)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = sb_value<double>(d->sb[which], x[i], y[i]);
}

// ---------------------------------------------------------------- models
struct InterArgs {
  int model, n;
  ModelParams p;
  uint32_t *rng;
  const double *E, *dir;
  double *E_out, *dir_out, *edep, *sec_E, *sec_dir;
  int *status, *nsec, *sec_type;
  int *err;
};

__global__ void k_interact(const Data *__restrict__ d, InterArgs a)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  Mrg r;
  r.load(a.rng, a.n, i);
  Inter<double> io;
  io.E = a.E[i];
  io.dir[0] = a.dir[3 * i];
  io.dir[1] = a.dir[3 * i + 1];
  io.dir[2] = a.dir[3 * i + 2];
  io.edep = 0;
  io.status = 0;
  io.nsec = 0;
  int err = 0;
  switch (a.model) {
  case GX_KLEIN_NISHINA: kn_sample(r, a.p, io, &err); break;
  case GX_SAUTER_GAVRILA: sg_sample(r, *d, a.p, io, &err); break;
  case GX_BETHE_HEITLER: bh_sample(r, a.p, io, &err); break;
  case GX_SELTZER_BERGER: sb_sample(r, a.p, io, &err); break;
  case GX_MOLLER: mb_sample(r, a.p, io, &err); break;
  case GX_BHABHA: bhabha_sample(r, a.p, io, &err); break;
  case GX_ANNIHILATION: annih_sample(r, io, &err); break;
  default: break;
  }
  r.store(a.rng, a.n, i);
  a.E_out[i] = io.E;
  for (int k = 0; k < 3; ++k) a.dir_out[3 * i + k] = io.dir[k];
  a.edep[i] = io.edep;
  a.status[i] = io.status;
  a.nsec[i] = io.nsec;
  for (int s = 0; s < 2; ++s) {
    bool has = s < io.nsec;
    a.sec_type[2 * i + s] = has ? io.sec_type[s] : -1;
    a.sec_E[2 * i + s] = has ? io.sec_E[s] : 0.0;
    for (int k = 0; k < 3; ++k) a.sec_dir[6 * i + 3 * s + k] = has ? io.sec_dir[s][k] : 0.0;
  }
  if (err) atomicOr(a.err, err);
}

__global__ void k_field_value(const Data *__restrict__ d, int n, const double *__restrict__ pos,
                              double *__restrict__ B)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]}, b[3];
  field_map_value(d->fmap, p, b);
  B[3 * i] = b[0];
  B[3 * i + 1] = b[1];
  B[3 * i + 2] = b[2];
}

__global__ void k_xs(int model, double Z, double c, const double *__restrict__ E, double *__restrict__ out, int n)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = (model == GX_KLEIN_NISHINA) ? kn_xs_per_atom(Z, E[i]) : mb_xs_per_atom(Z, E[i], c, 10.0 * eV);
}

// ------------------------------------------------------------- processes
// ProxyEmProcess<T>::PostStepGPIL, ProxyEmProcess.hpp:122-151
__global__ void k_post_step_gpil(const Data *__restrict__ d, int table, int mat, int n, uint32_t *__restrict__ rng,
                                 const double *__restrict__ E, const double *__restrict__ pstep,
                                 double *__restrict__ nil, double *__restrict__ saved, double *__restrict__ step)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double lambda = vec_value_ref(*d, d->vec[table][mat], E[i]);
  double nl = nil[i];
  if (nl <= 0.0) {
    Mrg r;
    r.load(rng, n, i);
    nl = -::log(r.u01());
    r.store(rng, n, i);
  } else {
    nl -= pstep[i] / saved[i];
  }
  nil[i] = nl;
  step[i] = nl / lambda;
  saved[i] = 1.0 / lambda;
}

__global__ void k_along_gpil(const Data *__restrict__ d, int mode, int charge, const int *__restrict__ mat,
                             const double *__restrict__ E, double *__restrict__ out, int n)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = ioni_along_gpil_ref(*d, mode, charge, mat[i], E[i]);
}

__global__ void k_along_doit(const Data *__restrict__ d, int mode, int charge, const int *__restrict__ mat,
                             const double *__restrict__ step, double *__restrict__ E, double *__restrict__ edep,
                             int n)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double e = E[i], ed = edep[i];
  ioni_along_doit_ref(*d, mode, charge, mat[i], step[i], e, ed);
  E[i] = e;
  edep[i] = ed;
}

// ----------------------------------------------------------------- helix
struct HelixArgs {
  double B[3], kB2C;
  int n;
  const double *px, *py, *pz, *dx, *dy, *dz, *q, *p, *s;
  double *npx, *npy, *npz, *ndx, *ndy, *ndz;
};

__global__ void k_helix(HelixArgs a)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  double pos[3] = {a.px[i], a.py[i], a.pz[i]}, dir[3] = {a.dx[i], a.dy[i], a.dz[i]}, np[3], nd[3];
  helix_dostep(a.kB2C, a.B, pos, dir, a.q[i], a.p[i], a.s[i], np, nd);
  a.npx[i] = np[0];
  a.npy[i] = np[1];
  a.npz[i] = np[2];
  a.ndx[i] = nd[0];
  a.ndy[i] = nd[1];
  a.ndz[i] = nd[2];
}

static int check_launch(const char *what)
{
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GX_OK : cuda_error(e, what);
}

} // namespace gx

using namespace gx;

#define GX_CTX(c)                                                                                                    \
  if (!(c)) return set_error(GX_ERR_ARG, "%s: null context", __func__);                                            \
  Ctx *C = reinterpret_cast<Ctx *>(c)

// The elementary functions of the FP64 parity variant (gx_math.h), or CUDA's
// own (lib = 1), one thread per argument.
__global__ void k_math(int fn, int lib, int n, const double *__restrict__ x, const double *__restrict__ y,
                       double *__restrict__ out)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = x[i], b = y ? y[i] : 0.0;
  double r;
  switch (fn) {
  case 0: r = lib ? ::log(a) : gxm_log(a); break;
  case 1: r = lib ? ::exp(a) : gxm_exp(a); break;
  case 2: r = lib ? ::pow(a, b) : gxm_pow(a, b); break;
  case 3: r = lib ? ::sin(a) : gxm_sin(a); break;
  case 4: r = lib ? ::cos(a) : gxm_cos(a); break;
  case 5: r = lib ? ::expm1(a) : gxm_expm1(a); break;
  default: r = lib ? ::log1p(a) : gxm_log1p(a); break;
  }
  out[i] = r;
}

extern "C" {

int gx_rng_substreams(const double seed[6], long long first, int n, uint32_t *d_states, gx_stream_t s)
{
  if (!seed || (n > 0 && !d_states) || n < 0 || first < 0) return set_error(GX_ERR_ARG, "gx_rng_substreams: bad args");
  for (int k = 0; k < 6; ++k)
    if (!(seed[k] >= 0.0 && seed[k] < (k < 3 ? kM1 : kM2)) || seed[k] != std::floor(seed[k]))
      return set_error(GX_ERR_ARG, "gx_rng_substreams: seed word %d out of range", k);
  return launch_substreams(seed, first, n, d_states, stream_of(s));
}

int gx_rng_advance(uint32_t *d_states, int n, long long e, long long c, gx_stream_t s)
{
  if (n < 0 || (n > 0 && !d_states)) return set_error(GX_ERR_ARG, "gx_rng_advance: bad args");
  if (e > 4096 || e < -4096) return set_error(GX_ERR_ARG, "gx_rng_advance: |e| > 4096");
  Mat2 M;
  jump_matrix(0, e, c, M.a[0]);
  jump_matrix(1, e, c, M.a[1]);
  if (n > 0) k_rng_matvec<<<grid_for(n), kBlock, 0, stream_of(s)>>>(M, d_states, n);
  return check_launch("k_rng_matvec");
}

int gx_rng_uniform(uint32_t *d_states, int n, int k, double *d_out, gx_stream_t s)
{
  if (n < 0 || k < 0 || (n > 0 && (!d_states || !d_out))) return set_error(GX_ERR_ARG, "gx_rng_uniform: bad args");
  if (n > 0 && k > 0) k_rng_uniform<<<grid_for(n), kBlock, 0, stream_of(s)>>>(d_states, n, k, d_out);
  return check_launch("k_rng_uniform");
}

int gx_rng_stream_id(const long long *h_ids, int n, uint32_t *d_states, gx_stream_t s)
{
  if (n < 0 || (n > 0 && (!h_ids || !d_states))) return set_error(GX_ERR_ARG, "gx_rng_stream_id: bad args");
  std::vector<uint32_t> h(6 * (size_t)n);
  const uint64_t m[2] = {4294967087ULL, 4294944443ULL};
  for (int i = 0; i < n; ++i) {
    if (h_ids[i] < 0 || h_ids[i] > 32) return set_error(GX_ERR_ARG, "gx_rng_stream_id: id outside 0..32");
    for (int c = 0; c < 2; ++c) {
      uint64_t v[3] = {12345, 12345, 12345}, J[9];
      jump_matrix(c, 127 * h_ids[i], 0, J);
      mat_vec(J, v, m[c]);
      for (int k = 0; k < 3; ++k) h[(size_t)(3 * c + k) * n + i] = (uint32_t)v[k];
    }
  }
  cudaError_t e = cudaMemcpyAsync(d_states, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_of(s));
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_of(s));
  return e == cudaSuccess ? GX_OK : cuda_error(e, "gx_rng_stream_id copy");
}

int gx_table_value(gx_ctx *ctx, int table, int mat, const double *d_E, double *d_out, int n, gx_stream_t s)
{
  GX_CTX(ctx);
  if (table < 0 || table >= kNTables || mat < 0 || mat >= kNMat || n < 0) return set_error(GX_ERR_ARG, "gx_table_value: bad args");
  if (n > 0) k_table_value<<<grid_for(n), kBlock, 0, stream_of(s)>>>(C->dev, table, mat, d_E, d_out, n, 0);
  return check_launch("k_table_value");
}

int gx_table_invrange(gx_ctx *ctx, int table, int mat, const double *d_r, double *d_out, int n, gx_stream_t s)
{
  GX_CTX(ctx);
  if (table < 0 || table >= kNTables || mat < 0 || mat >= kNMat || n < 0) return set_error(GX_ERR_ARG, "gx_table_invrange: bad args");
  if (n > 0) k_table_value<<<grid_for(n), kBlock, 0, stream_of(s)>>>(C->dev, table, mat, d_r, d_out, n, 1);
  return check_launch("k_table_value");
}

int gx_sb_value(gx_ctx *ctx, int which, const double *d_x, const double *d_y, double *d_out, int n, gx_stream_t s)
{
  GX_CTX(ctx);
  if (which < 0 || which > 2 || n < 0) return set_error(GX_ERR_ARG, "gx_sb_value: bad args");
  if (n > 0) k_sb_value<<<grid_for(n), kBlock, 0, stream_of(s)>>>(C->dev, which, d_x, d_y, d_out, n);
  return check_launch("k_sb_value");
}

int gx_interact(gx_ctx *ctx, int model, const gx_model_params *p, int n, uint32_t *d_rng, const double *d_E,
                const double *d_dir, double *d_E_out, double *d_dir_out, double *d_edep, int *d_status,
                int *d_nsec, int *d_sec_type, double *d_sec_E, double *d_sec_dir, gx_stream_t s)
{
  GX_CTX(ctx);
  if (!p || model < GX_KLEIN_NISHINA || model > GX_ANNIHILATION || n < 0) return set_error(GX_ERR_ARG, "gx_interact: bad args");
  if (p->sb_table < 0 || p->sb_table > 2 || p->Z < 1 || p->Z > 99) return set_error(GX_ERR_ARG, "gx_interact: bad params");
  if (n == 0) return GX_OK;
  InterArgs a;
  a.model = model;
  a.n = n;
  a.p.mode = p->mode;
  a.p.Z = p->Z;
  a.p.cut = p->cut;
  a.p.density_factor = p->density_factor;
  a.p.sb = C->host.sb + p->sb_table;
  a.rng = d_rng;
  a.E = d_E;
  a.dir = d_dir;
  a.E_out = d_E_out;
  a.dir_out = d_dir_out;
  a.edep = d_edep;
  a.status = d_status;
  a.nsec = d_nsec;
  a.sec_type = d_sec_type;
  a.sec_E = d_sec_E;
  a.sec_dir = d_sec_dir;
  int *derr = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&derr, sizeof(int), stream_of(s));
  if (e != cudaSuccess) return cuda_error(e, "gx_interact scratch");
  cudaMemsetAsync(derr, 0, sizeof(int), stream_of(s));
  a.err = derr;
  k_interact<<<grid_for(n), kBlock, 0, stream_of(s)>>>(C->dev, a);
  int rc = check_launch("k_interact");
  int herr = 0;
  cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, stream_of(s));
  cudaFreeAsync(derr, stream_of(s));
  e = cudaStreamSynchronize(stream_of(s));
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_error(e, "gx_interact");
  if (herr) return set_error(GX_ERR_ITERCAP, "gx_interact: a rejection loop hit its iteration cap");
  return GX_OK;
}

int gx_field_value(gx_ctx *ctx, int n, const double *d_pos, double *d_B, gx_stream_t s)
{
  if (!ctx || n < 0 || (n > 0 && (!d_pos || !d_B))) return set_error(GX_ERR_ARG, "gx_field_value: bad arguments");
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->host.fmap) return set_error(GX_ERR_ARG, "gx_field_value: no field map loaded (gx_ctx_load_field_map)");
  if (n == 0) return GX_OK;
  k_field_value<<<grid_for(n), kBlock, 0, stream_of(s)>>>(c->dev, n, d_pos, d_B);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GX_OK : cuda_error(e, "k_field_value");
}

int gx_xs_per_atom(int model, double Z, const double *d_E, double *d_out, int n, gx_stream_t s)
{
  if ((model != GX_KLEIN_NISHINA && model != GX_MOLLER) || n < 0) return set_error(GX_ERR_ARG, "gx_xs_per_atom: bad args");
  // twopi mc2 rcl2 along the CLHEP definition chain
  const double eplus = 1., e_SI = 1.602176487e-19, coulomb = eplus / e_SI, second = 1.e+9, meter = 1000.;
  const double ampere = coulomb / second, volt = 1.e-6 * (1. / eplus), weber = volt * second, henry = weber / ampere;
  const double mu0 = 4 * kPi * 1.e-7 * henry / meter, c_light = 2.99792458e+8 * meter / second;
  const double epsilon0 = 1. / (c_light * c_light * mu0), elm = eplus * eplus / (4 * kPi * epsilon0);
  const double rcl = elm / kEMass, c = kTwoPi * kEMass * rcl * rcl;
  if (n > 0) k_xs<<<grid_for(n), kBlock, 0, stream_of(s)>>>(model, Z, c, d_E, d_out, n);
  return check_launch("k_xs");
}

int gx_post_step_gpil(gx_ctx *ctx, int process, int mat, int n, uint32_t *d_rng, const double *d_E,
                      const double *d_pstep_prev, double *d_nil, double *d_saved, double *d_step, gx_stream_t s)
{
  GX_CTX(ctx);
  static const int kTable[5] = {GX_Lambda_compt, GX_Lambda_conv, GX_LambdaPrim_phot, GX_Lambda_eBrem_em,
                                GX_Lambda_eIoni_em};
  if (process < 0 || process > 4 || mat < 0 || mat >= kNMat || n < 0) return set_error(GX_ERR_ARG, "gx_post_step_gpil: bad args");
  if (n > 0)
    k_post_step_gpil<<<grid_for(n), kBlock, 0, stream_of(s)>>>(C->dev, kTable[process], mat, n, d_rng, d_E,
                                                               d_pstep_prev, d_nil, d_saved, d_step);
  return check_launch("k_post_step_gpil");
}

int gx_ioni_along_gpil(gx_ctx *ctx, int mode, int charge, const int *d_mat, const double *d_E, double *d_out, int n,
                       gx_stream_t s)
{
  GX_CTX(ctx);
  if (n < 0) return set_error(GX_ERR_ARG, "gx_ioni_along_gpil: bad args");
  if (n > 0) k_along_gpil<<<grid_for(n), kBlock, 0, stream_of(s)>>>(C->dev, mode, charge, d_mat, d_E, d_out, n);
  return check_launch("k_along_gpil");
}

int gx_ioni_along_doit(gx_ctx *ctx, int mode, int charge, const int *d_mat, const double *d_step, double *d_E,
                       double *d_edep, int n, gx_stream_t s)
{
  GX_CTX(ctx);
  if (n < 0) return set_error(GX_ERR_ARG, "gx_ioni_along_doit: bad args");
  if (n > 0)
    k_along_doit<<<grid_for(n), kBlock, 0, stream_of(s)>>>(C->dev, mode, charge, d_mat, d_step, d_E, d_edep, n);
  return check_launch("k_along_doit");
}

int gx_helix_dostep(const double B[3], double kB2C, int n, const double *d_posx, const double *d_posy,
                    const double *d_posz, const double *d_dirx, const double *d_diry, const double *d_dirz,
                    const double *d_charge, const double *d_momentum, const double *d_step, double *d_newposx,
                    double *d_newposy, double *d_newposz, double *d_newdirx, double *d_newdiry, double *d_newdirz,
                    gx_stream_t s)
{
  if (!B || n < 0) return set_error(GX_ERR_ARG, "gx_helix_dostep: bad args");
  HelixArgs a = {{B[0], B[1], B[2]}, kB2C, n, d_posx, d_posy, d_posz, d_dirx, d_diry, d_dirz, d_charge, d_momentum,
                 d_step, d_newposx, d_newposy, d_newposz, d_newdirx, d_newdiry, d_newdirz};
  if (n > 0) k_helix<<<grid_for(n), kBlock, 0, stream_of(s)>>>(a);
  return check_launch("k_helix");
}

int gx_math_eval(int fn, int lib, int n, const double *d_x, const double *d_y, double *d_out, gx_stream_t s)
{
  if (fn < 0 || fn > 6 || lib < 0 || lib > 1 || n < 0 || (n > 0 && (!d_x || !d_out)) || (fn == 2 && n > 0 && !d_y))
    return set_error(GX_ERR_ARG, "gx_math_eval: bad args");
  if (n > 0) k_math<<<grid_for(n), kBlock, 0, stream_of(s)>>>(fn, lib, n, d_x, d_y, d_out);
  return check_launch("k_math");
}

} // extern "C"
