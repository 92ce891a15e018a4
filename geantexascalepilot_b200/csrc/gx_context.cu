// gx_context.cu -- host side of the C ABI: error reporting, physics-data
// loading and relocation to the device, MRG32k3a jump matrices.
#include "gx_internal.cuh"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace gx {

static thread_local char g_err[512] = "";

int set_error(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_error(cudaError_t e, const char *what)
{
  return set_error(GX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// ------------------------------------------------------------ table parsing
// Geant4 ASCII physics-vector format as read by ProxyPhysicsVector::Retrieve
// (source/Geant/proxy/src/ProxyPhysicsVector.cu:89-128): per vector a type,
// "emin emax n", the node count, then (energy, value) pairs.
struct HostVec {
  std::vector<double> x, y, d2;
};

// Second derivatives of the cubic spline with not-a-knot end conditions, in
// the recurrence of ProxyPhysicsVector::FillSecondDerivatives
// (ProxyPhysicsVector.cu:308-386) so that the node curvatures are the
// reference's own; fewer than 5 nodes use its simplified form (:211-238).
static void spline_d2(HostVec &v)
{
  const std::vector<double> &x = v.x, &y = v.y;
  int N = (int)x.size();
  std::vector<double> &d = v.d2;
  d.assign(N, 0.0);
  int n = N - 1;
  if (N < 5) {
    if (N < 3) return;
    for (int i = 1; i < n; ++i)
      d[i] = 3.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])) /
             (x[i + 1] - x[i - 1]);
    d[n] = d[n - 1];
    d[0] = d[1];
    return;
  }
  std::vector<double> u(n, 0.0);
  u[1] = ((y[2] - y[1]) / (x[2] - x[1]) - (y[1] - y[0]) / (x[1] - x[0]));
  u[1] = 6.0 * u[1] * (x[2] - x[1]) / ((x[2] - x[0]) * (x[2] - x[0]));
  d[1] = (2.0 * x[1] - x[0] - x[2]) / (2.0 * x[2] - x[0] - x[1]);
  for (int i = 2; i < n - 1; ++i) {
    double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
    double p = sig * d[i - 1] + 2.0;
    d[i] = (sig - 1.0) / p;
    u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
    u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1])) - sig * u[i - 1] / p;
  }
  double sig = (x[n - 1] - x[n - 2]) / (x[n] - x[n - 2]);
  double p = sig * d[n - 3] + 2.0;
  u[n - 1] = (y[n] - y[n - 1]) / (x[n] - x[n - 1]) - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
  u[n - 1] = 6.0 * sig * u[n - 1] / (x[n] - x[n - 2]) - (2.0 * sig - 1.0) * u[n - 2] / p;
  p = (1.0 + sig) + (2.0 * sig - 1.0) * d[n - 2];
  d[n - 1] = u[n - 1] / p;
  for (int k = n - 2; k > 1; --k) d[k] *= (d[k + 1] - u[k] * (x[k + 1] - x[k - 1]) / (x[k + 1] - x[k]));
  d[n] = (d[n - 1] - (1.0 - sig) * d[n - 2]) / sig;
  sig = 1.0 - ((x[2] - x[1]) / (x[2] - x[0]));
  d[1] *= (d[2] - u[1] / (1.0 - sig));
  d[0] = (d[1] - sig * d[2]) / (1.0 - sig);
}

static const char *kTableFile[kNTables] = {
    "DEDX.eBrem.e-.asc", "DEDX.eBrem.e+.asc", "DEDX.eIoni.e-.asc", "DEDX.eIoni.e+.asc",
    "InverseRange.eIoni.e-.asc", "InverseRange.eIoni.e+.asc", "Ionisation.eIoni.e-.asc",
    "Ionisation.eIoni.e+.asc", "Lambda.compt.gamma.asc", "Lambda.conv.gamma.asc",
    "Lambda.eBrem.e-.asc", "Lambda.eBrem.e+.asc", "Lambda.eIoni.e-.asc", "Lambda.eIoni.e+.asc",
    "LambdaMod1.msc.e-.asc", "LambdaMod1.msc.e+.asc", "LambdaPrim.compt.gamma.asc",
    "LambdaPrim.phot.gamma.asc", "Range.eIoni.e-.asc", "Range.eIoni.e+.asc"};

static bool read_table(const std::string &fn, HostVec out[kNMat])
{
  FILE *f = fopen(fn.c_str(), "r");
  if (!f) return false;
  int nv = 0;
  bool ok = fscanf(f, "%d", &nv) == 1 && nv == kNMat;
  for (int m = 0; ok && m < kNMat; ++m) {
    int type, n, siz;
    double emin, emax;
    ok = fscanf(f, "%d %lf %lf %d %d", &type, &emin, &emax, &n, &siz) == 5 && siz >= 2;
    if (!ok) break;
    out[m].x.resize(siz);
    out[m].y.resize(siz);
    for (int i = 0; ok && i < siz; ++i) ok = fscanf(f, "%lf %lf", &out[m].x[i], &out[m].y[i]) == 2;
    if (ok) spline_d2(out[m]);
  }
  fclose(f);
  return ok;
}

static bool read_sb(const std::string &dir, int Z, SBTable &t)
{
  std::string fn = dir + "/brem_SB/br" + std::to_string(Z);
  FILE *f = fopen(fn.c_str(), "r");
  if (!f) return false;
  int k, nx, ny;
  bool ok = fscanf(f, "%d %d %d", &k, &nx, &ny) == 3 && nx == 32 && ny == 57;
  for (int i = 0; ok && i < 32; ++i) ok = fscanf(f, "%lf", &t.x[i]) == 1;
  for (int j = 0; ok && j < 57; ++j) ok = fscanf(f, "%lf", &t.y[j]) == 1;
  for (int j = 0; ok && j < 57; ++j)
    for (int i = 0; ok && i < 32; ++i) ok = fscanf(f, "%lf", &t.v[j][i]) == 1;
  fclose(f);
  return ok;
}

// cut.dat as read by ProxyDataManager::RetrieveCutsTable (ProxyDataManager.cu:83-122)
static bool read_cuts(const std::string &dir, Data &d)
{
  FILE *f = fopen((dir + "/table/cut.dat").c_str(), "r");
  if (!f) return false;
  char ver[64];
  int nmat;
  bool ok = fscanf(f, "%63s %d", ver, &nmat) == 2 && nmat == kNMat;
  for (int i = 0; ok && i < 12; ++i) {
    double len, en;
    ok = fscanf(f, "%lf %lf", &len, &en) == 2;
    d.cut_raw[i] = en;
    d.cut_energy[i / kNMat][i % kNMat] = en * 1.0e-3;
    d.cut_length[i / kNMat][i % kNMat] = len;
  }
  fclose(f);
  return ok;
}

static bool read_sandia(const std::string &dir, Data &d, std::vector<double> &binding, std::vector<double> &sandia)
{
  FILE *f = fopen((dir + "/sandia.dat").c_str(), "r");
  if (!f) return false;
  char line[512];
  long pos = 0;
  do {
    pos = ftell(f);
    if (!fgets(line, sizeof(line), f)) {
      fclose(f);
      return false;
    }
  } while (line[0] == '#');
  fseek(f, pos, SEEK_SET);
  int n;
  bool ok = fscanf(f, " SHELLS %d", &n) == 1 && n == 101;
  for (int i = 0; ok && i < 101; ++i) ok = fscanf(f, "%d", &d.nshell[i]) == 1;
  for (int i = 0; ok && i < 101; ++i) ok = fscanf(f, "%d", &d.ishell[i]) == 1;
  ok = ok && fscanf(f, " BINDING %d", &n) == 1 && n == 1540;
  binding.resize(1540);
  for (int i = 0; ok && i < 1540; ++i) ok = fscanf(f, "%lf", &binding[i]) == 1;
  ok = ok && fscanf(f, " INTERVALS %d", &n) == 1 && n == 101;
  for (int i = 0; ok && i < 101; ++i) ok = fscanf(f, "%d", &d.nint[i]) == 1;
  ok = ok && fscanf(f, " SANDIA %d", &n) == 1 && n == 981;
  sandia.resize(981 * 5);
  for (int i = 0; ok && i < 981 * 5; ++i) ok = fscanf(f, "%lf", &sandia[i]) == 1;
  fclose(f);
  d.cumint[0] = 1;
  for (int z = 1; z < 101; ++z) d.cumint[z] = d.cumint[z - 1] + d.nint[z - 1];
  return ok;
}

// Derived electromagnetic constants, evaluated along the CLHEP definition
// chain (ProxySystemOfUnits.hpp / ProxyPhysicalConstants.hpp).
static void em_constants(double *rcl, double *compton_len, double *alpha)
{
  const double pi = kPi, eplus = 1., e_SI = 1.602176487e-19;
  const double coulomb = eplus / e_SI, second = 1.e+9, meter = 1000.;
  const double ampere = coulomb / second, megavolt = 1. / eplus, volt = 1.e-6 * megavolt;
  const double weber = volt * second, henry = weber / ampere;
  const double mu0 = 4 * pi * 1.e-7 * henry / meter;
  const double c_light = 2.99792458e+8 * meter / second;
  const double epsilon0 = 1. / (c_light * c_light * mu0);
  const double elm_coupling = eplus * eplus / (4 * pi * epsilon0);
  const double joule = eV / e_SI;
  const double h_Planck = 6.62606896e-34 * joule * second;
  const double hbarc = h_Planck / (2 * pi) * c_light;
  *rcl = elm_coupling / kEMass;
  *compton_len = hbarc / kEMass;
  *alpha = elm_coupling / hbarc;
}

// Tsai's radiation-length factor of an element (ProxyElementUtils.cu:40-61,
// its Coulomb correction :24-37), mm^2.
static double lrad_tsai_factor(double Z, double alpha, double rcl)
{
  static const double lrad_light[] = {5.31, 4.79, 4.74, 4.71};
  static const double lprad_light[] = {6.144, 5.621, 5.805, 5.924};
  const double logZ3 = std::log(Z) / 3.;
  double lrad, lprad;
  const int iz = (int)(Z + 0.5) - 1;
  if (iz <= 3) {
    lrad = lrad_light[iz];
    lprad = lprad_light[iz];
  } else {
    lrad = std::log(184.15) - logZ3;
    lprad = std::log(1194.) - 2 * logZ3;
  }
  const double az1 = alpha * Z, az2 = az1 * az1, az4 = az2 * az2;
  const double fc = (0.0083 * az4 + 0.20206 + 1. / (1. + az2)) * az2 - (0.0020 * az4 + 0.0369) * az4;
  return 4 * alpha * rcl * rcl * Z * (Z * (lrad - fc) + lprad);
}

static void material(Data &d, int m, double Z, double A, double density, double I, double rcl, double lc,
                     double alpha)
{
  const double avogadro = 6.02214179e+23;
  double n_atoms = avogadro * density / A * 1.e-3; // 1/mm3
  d.mat_Z[m] = Z;
  d.mat_A[m] = A;
  d.mat_I[m] = I;
  d.mat_density[m] = density;
  d.mat_nel[m] = Z * n_atoms;
  d.mat_dfactor[m] = d.mat_nel[m] * (4.0 * kPi * rcl * lc * lc); // n_el x the Migdal constant
  // radiation length (ProxyMaterial::ComputeDerivedQuantities, ProxyMaterial.cu:133-150)
  const double radinv = n_atoms * lrad_tsai_factor(Z, alpha, rcl);
  // the Urban model's Z-dependent constants: the theta0 correction and the
  // coefficients of the tail parameter (published with the model)
  const double z16 = std::exp(std::log(Z) / 6.0), z13 = z16 * z16;
  const double facz = 0.990395 + z16 * (-0.168386 + z16 * 0.093286);
  double *c = d.mat_msc[m];
  c[0] = radinv <= 0.0 ? 1.7976931348623157e308 : 1. / radinv;
  c[1] = facz * (1.0 - 8.7780e-2 / Z);
  c[2] = facz * (4.0780e-2 + 1.7315e-4 * Z);
  c[3] = 2.3785 - z13 * (4.1981e-1 - z13 * 6.3100e-2);
  c[4] = 4.7526e-1 + z13 * (1.7694 - z13 * 3.3885e-1);
  c[5] = 2.3683e-1 - z13 * (1.8111 - z13 * 3.2774e-1);
  c[6] = 1.7888e-2 + z13 * (1.9659e-2 - z13 * 2.6664e-3);
}

// Per node of a vector: the cubic of its bin as a polynomial in
// u = (E - x_i) / delta, {x_i, 1 / delta, c0, c1, c2, c3}, in FP64 and FP32.
static void append_coeffs(const HostVec &v, std::vector<double> &C64, std::vector<float> &C32)
{
  const int n = (int)v.x.size();
  for (int i = 0; i < n; ++i) {
    double x1 = v.x[i], x2 = (i + 1 < n) ? v.x[i + 1] : x1 + 1.0;
    double y1 = v.y[i], y2 = (i + 1 < n) ? v.y[i + 1] : y1;
    double a1 = v.d2[i], a2 = (i + 1 < n) ? v.d2[i + 1] : a1;
    double dl = x2 - x1, h = dl * dl / 6.0;
    double c[6] = {x1, 1.0 / dl, y1, (y2 - y1) - h * (2.0 * a1 + a2), 3.0 * h * a1, h * (a2 - a1)};
    for (int k = 0; k < 6; ++k) {
      C64.push_back(c[k]);
      C32.push_back((float)c[k]);
    }
  }
}

// New node values for vector (table, mat): second derivatives and per-bin
// coefficients recomputed on the host, all four node arrays updated on the
// device in place (the node energies stay).
int refit_vector(Ctx *ctx, int table, int mat, const double *ynew)
{
  const Data &d = ctx->host;
  const VecDesc &vd = d.vec[table][mat];
  const int n = vd.n;
  HostVec v;
  v.x.resize(n);
  v.y.assign(ynew, ynew + n);
  cudaError_t e = cudaMemcpy(v.x.data(), d.x + vd.off, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_error(e, "refit: node energies");
  spline_d2(v);
  std::vector<double> C64;
  std::vector<float> C32;
  append_coeffs(v, C64, C32);
  if ((e = cudaMemcpy(const_cast<double *>(d.y) + vd.off, v.y.data(), n * sizeof(double), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(const_cast<double *>(d.d2) + vd.off, v.d2.data(), n * sizeof(double), cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(const_cast<double *>(d.c64) + 6 * vd.off, C64.data(), C64.size() * sizeof(double),
                      cudaMemcpyHostToDevice)) ||
      (e = cudaMemcpy(const_cast<float *>(d.c32) + 6 * vd.off, C32.data(), C32.size() * sizeof(float),
                      cudaMemcpyHostToDevice)))
    return cuda_error(e, "refit: upload");
  return GX_OK;
}

// The same with new node abscissae as well (same count): the vector's
// descriptor follows and the context's device copy is updated.
int refit_vector_xy(Ctx *ctx, int table, int mat, const double *xnew, const double *ynew)
{
  Data &d = ctx->host;
  VecDesc &vd = d.vec[table][mat];
  const int n = vd.n;
  cudaError_t e = cudaMemcpy(const_cast<double *>(d.x) + vd.off, xnew, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_error(e, "refit: node abscissae");
  vd.emin = xnew[0];
  vd.emax = xnew[n - 1];
  vd.dbin = std::log(xnew[1] / vd.emin);
  vd.base = std::log(vd.emin) / vd.dbin;
  vd.invdbin = 1.0 / vd.dbin;
  vd.eminf = (float)vd.emin;
  vd.emaxf = (float)vd.emax;
  vd.invdbinf = (float)vd.invdbin;
  vd.basef = (float)vd.base;
  if ((e = cudaMemcpy(ctx->dev, &d, sizeof(Data), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_error(e, "refit: context upload");
  return refit_vector(ctx, table, mat, ynew);
}

template <class T> static int upload(const std::vector<T> &h, T **d)
{
  cudaError_t e = cudaMalloc((void **)d, sizeof(T) * (h.empty() ? 1 : h.size()));
  if (e != cudaSuccess) return cuda_error(e, "cudaMalloc tables");
  e = cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_error(e, "cudaMemcpy tables");
  return GX_OK;
}

int load_data(const char *datadir, Ctx *ctx)
{
  std::string dir(datadir);
  Data &d = ctx->host;
  std::memset(&d, 0, sizeof(d));
  std::vector<double> X, Y, D2, C64;
  std::vector<float> C32;
  for (int t = 0; t < kNTables; ++t) {
    HostVec v[kNMat];
    if (!read_table(dir + "/table/" + kTableFile[t], v))
      return set_error(GX_ERR_DATA, "cannot read table %s/table/%s", datadir, kTableFile[t]);
    for (int m = 0; m < kNMat; ++m) {
      VecDesc &vd = d.vec[t][m];
      int n = (int)v[m].x.size();
      vd.n = n;
      vd.off = (int)X.size();
      vd.emin = v[m].x[0];
      vd.emax = v[m].x[n - 1];
      vd.dbin = std::log(v[m].x[1] / vd.emin);
      vd.base = std::log(vd.emin) / vd.dbin;
      vd.invdbin = 1.0 / vd.dbin;
      vd.eminf = (float)vd.emin;
      vd.emaxf = (float)vd.emax;
      vd.invdbinf = (float)vd.invdbin;
      vd.basef = (float)vd.base;
      for (int i = 0; i < n; ++i) {
        X.push_back(v[m].x[i]);
        Y.push_back(v[m].y[i]);
        D2.push_back(v[m].d2[i]);
      }
      append_coeffs(v[m], C64, C32);
    }
  }
  if (!read_cuts(dir, d)) return set_error(GX_ERR_DATA, "cannot read %s/table/cut.dat", datadir);
  std::vector<SBTable> sb(3);
  if (!read_sb(dir, 11, sb[0]) || !read_sb(dir, 18, sb[1]) || !read_sb(dir, 82, sb[2]))
    return set_error(GX_ERR_DATA, "cannot read Seltzer-Berger tables in %s/brem_SB", datadir);
  std::vector<double> binding, sandia;
  if (!read_sandia(dir, d, binding, sandia)) return set_error(GX_ERR_DATA, "cannot read %s/sandia.dat", datadir);
  double rcl, lc, alpha;
  em_constants(&rcl, &lc, &alpha);
  d.pi_rcl2 = kPi * rcl * rcl;
  d.alpha = alpha;
  // mean excitation energies: ICRU Report 37 (the NIST values of these materials)
  material(d, 0, 1.0, 1.01, 1.e-25, 21.8e-6, rcl, lc, alpha); // Galactic
  material(d, 1, 82.0, 207.2, 11.35, 823.0e-6, rcl, lc, alpha); // G4_Pb
  material(d, 2, 18.0, 39.95, 1.396, 188.0e-6, rcl, lc, alpha); // G4_lAr
  double *px, *py, *pd2, *pc64, *pbind, *psandia;
  float *pc32;
  SBTable *psb;
  int rc;
  if ((rc = upload(X, &px)) || (rc = upload(Y, &py)) || (rc = upload(D2, &pd2)) || (rc = upload(C64, &pc64)) ||
      (rc = upload(C32, &pc32)) || (rc = upload(sb, &psb)) || (rc = upload(binding, &pbind)) ||
      (rc = upload(sandia, &psandia)))
    return rc;
  d.x = px;
  d.y = py;
  d.d2 = pd2;
  d.c64 = pc64;
  d.c32 = pc32;
  d.sb = psb;
  d.binding = pbind;
  d.sandia = psandia;
  ctx->owned = {px, py, pd2, pc64, pc32, psb, pbind, psandia};
  cudaError_t e = cudaMalloc((void **)&ctx->dev, sizeof(Data));
  if (e != cudaSuccess) return cuda_error(e, "cudaMalloc data");
  ctx->owned.push_back(ctx->dev);
  e = cudaMemcpy(ctx->dev, &d, sizeof(Data), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_error(e, "cudaMemcpy data");
  return GX_OK;
}

// ------------------------------------------------- MRG32k3a jump matrices
// Exact mod-m 3x3 matrix arithmetic in 64/128-bit integers (host side of the
// device skip-ahead).  A1, A2 are the two component recurrences.
static const uint64_t kMod[2] = {4294967087ULL, 4294944443ULL};
static const int64_t kA[2][3][3] = {{{0, 1, 0}, {0, 0, 1}, {-810728, 1403580, 0}},
                                    {{0, 1, 0}, {0, 0, 1}, {-1370589, 0, 527612}}};
// inverses of A1, A2 (MRG.hpp:82-90)
static const int64_t kAinv[2][3][3] = {{{184888585, 0, 1945170933}, {1, 0, 0}, {0, 1, 0}},
                                       {{0, 360363334, 4225571728LL}, {1, 0, 0}, {0, 1, 0}}};

void mat_mul(const uint64_t A[9], const uint64_t B[9], uint64_t C[9], uint64_t m)
{
  uint64_t T[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      unsigned __int128 s = 0;
      for (int k = 0; k < 3; ++k) s += (unsigned __int128)A[3 * i + k] * B[3 * k + j];
      T[3 * i + j] = (uint64_t)(s % m);
    }
  std::memcpy(C, T, sizeof(T));
}

static void base_matrix(int comp, bool inverse, uint64_t M[9])
{
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      int64_t a = inverse ? kAinv[comp][i][j] : kA[comp][i][j];
      int64_t m = (int64_t)kMod[comp];
      M[3 * i + j] = (uint64_t)(((a % m) + m) % m);
    }
}

// Transition matrix of AdvanceState(e, c) (MRG32k3a.cpp:167-205):
// n = 2^e + c (e > 0), -2^-e + c (e < 0), c (e = 0).
void jump_matrix(int comp, long long e, long long c, uint64_t out[9])
{
  uint64_t m = kMod[comp];
  uint64_t B[9], C[9], W[9];
  uint64_t I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::memcpy(C, I, sizeof(I));
  base_matrix(comp, c < 0, W);
  for (long long n = (c < 0) ? -c : c; n > 0; n >>= 1) {
    if (n & 1) mat_mul(W, C, C, m);
    mat_mul(W, W, W, m);
  }
  if (e != 0) {
    base_matrix(comp, e < 0, B);
    for (long long i = 0, k = (e < 0) ? -e : e; i < k; ++i) mat_mul(B, B, B, m);
    mat_mul(B, C, C, m);
  }
  std::memcpy(out, C, sizeof(C));
}

void mat_vec(const uint64_t A[9], uint64_t v[3], uint64_t m)
{
  uint64_t r[3];
  for (int i = 0; i < 3; ++i) {
    unsigned __int128 s = 0;
    for (int k = 0; k < 3; ++k) s += (unsigned __int128)A[3 * i + k] * v[k];
    r[i] = (uint64_t)(s % m);
  }
  std::memcpy(v, r, sizeof(r));
}

} // namespace gx

using namespace gx;

extern "C" {

const char *gx_last_error_string(void) { return g_err; }
int gx_version(void) { return 100; }

int gx_ctx_create(const char *datadir, int device, gx_ctx **out)
{
  if (!datadir || !out) return set_error(GX_ERR_ARG, "gx_ctx_create: null argument");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return set_error(GX_ERR_NODEVICE, "gx_ctx_create: no CUDA device");
  if (device < 0 || device >= ndev) return set_error(GX_ERR_ARG, "gx_ctx_create: bad device %d", device);
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  Ctx *c = new Ctx();
  c->device = device;
  int rc = load_data(datadir, c);
  if (rc != GX_OK) {
    for (void *p : c->owned) cudaFree(p);
    delete c;
    return rc;
  }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  *out = reinterpret_cast<gx_ctx *>(c);
  return GX_OK;
}

int gx_ctx_load_field_map(gx_ctx *ctx, const char *path)
{
  if (!ctx || !path) return set_error(GX_ERR_ARG, "gx_ctx_load_field_map: null argument");
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  FILE *f = std::fopen(path, "r");
  if (!f) return set_error(GX_ERR_DATA, "gx_ctx_load_field_map: cannot open %s", path);
  // ScalarCMSmagField::ReadVectorData (ScalarCMSmagField.h:162-199): one
  // lattice point per line, r outer and z inner, values read as float and
  // stored times 1 / (dr dz) in float
  const float kAInverse = (float)(1.0 / (50.0f * 200.0f));
  std::vector<float4> h((size_t)kFmapNr * kFmapNz);
  int ind = 0;
  char line[512];
  while (std::fgets(line, sizeof(line), f)) {
    float r, phi, z, bz, br, bphi;
    if (std::sscanf(line, "R(mm)= %f phi(deg)= %f Z(mm)= %f Bz(tesla)= %f Br(tesla)= %f Bphi(tesla)= %f", &r, &phi,
                    &z, &bz, &br, &bphi) != 6)
      continue;
    const int ir = ind / kFmapNz, iz = ind % kFmapNz;
    if (ind >= kFmapNr * kFmapNz || std::fabs(r - 50.0f * ir) > 1e-3f || std::fabs(z - (-16000.0f + 200.0f * iz)) > 1e-3f) {
      std::fclose(f);
      return set_error(GX_ERR_DATA, "gx_ctx_load_field_map: %s: point %d is not on the 181 x 161 (r, z) lattice", path,
                       ind);
    }
    h[ind] = make_float4(br * kAInverse, bphi * kAInverse, bz * kAInverse, 0.0f);
    ++ind;
  }
  std::fclose(f);
  if (ind != kFmapNr * kFmapNz)
    return set_error(GX_ERR_DATA, "gx_ctx_load_field_map: %s: %d lattice points, expected %d", path, ind,
                     kFmapNr * kFmapNz);
  cudaError_t e = cudaSetDevice(c->device);
  float4 *d = const_cast<float4 *>(c->host.fmap);
  if (e == cudaSuccess && !d) {
    e = cudaMalloc((void **)&d, h.size() * sizeof(float4));
    if (e == cudaSuccess) c->owned.push_back(d);
  }
  if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), h.size() * sizeof(float4), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_error(e, "gx_ctx_load_field_map: upload");
  c->host.fmap = d;
  e = cudaMemcpy(c->dev, &c->host, sizeof(Data), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? GX_OK : cuda_error(e, "gx_ctx_load_field_map: context upload");
}

int gx_ctx_destroy(gx_ctx *ctx)
{
  if (!ctx) return GX_OK;
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  release_engine(c);
  parity::release_engine(c);
  for (void *p : c->owned) cudaFree(p);
  if (c->host_buf) cudaFree(c->host_buf);
  if (c->host_stream) cudaStreamDestroy(c->host_stream);
  delete c;
  return GX_OK;
}

int gx_cut_value(gx_ctx *ctx, int index, int ipart, double *out)
{
  if (!ctx || !out) return set_error(GX_ERR_ARG, "gx_cut_value: null argument");
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  int k = 4 * ipart + index;
  *out = (k >= 0 && k < 12) ? c->host.cut_raw[k] : 0.0;
  return GX_OK;
}

} // extern "C"
