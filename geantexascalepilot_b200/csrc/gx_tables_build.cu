// gx_tables_build.cu -- macroscopic cross-section tables built on the device
// from the models' cross sections, in place of the Geant4-dumped ASCII tables.
//
// The reference builds nothing (its macroscopic cross section is
// ProxyEmModel::MacroscopicCrossSection, proxy/ProxyEmModel.hpp:57-76, the sum
// over elements of n_atoms x CrossSectionPerAtom, evaluated per call); its
// tables come from Geant4.  Here one thread per node energy evaluates:
//   Lambda.compt / LambdaPrim.compt   n_atoms sigma_KN(Z, E) (x E for Prim):
//     ProxyKleinNishina::CrossSectionPerAtom (ProxyKleinNishina.hpp:62-93)
//   Lambda.eIoni.e-   n_atoms sigma_Moller(Z, T, cut_e-): ProxyMollerScattering::
//     CrossSectionPerAtom (ProxyMollerScattering.hpp:61-89) with the
//     material's production cut instead of the reference's fixed 10 eV
//   Lambda.eIoni.e+   n_el sigma_Bhabha(T, cut_e-): the integral from the cut
//     to T of the differential cross section the Bhabha sampler draws from
//     (B(x) = 1/(beta^2 x^2) - b1/x + b2 - b3 x + b4 x^2, x = energy fraction)
//   Lambda.eBrem.e-   n_atoms sigma_SB(Z, T, cut_gamma): the Seltzer-Berger
//     tables chi(k/T, T) = (beta^2/Z^2) k dsigma/dk integrated in ln k from the
//     cut to T with the dielectric suppression k^2 / (k^2 + k_p^2),
//     k_p^2 = (Migdal constant x n_el) E_total^2; 16 x 8-point Gauss-Legendre.
//   Lambda.conv       n_atoms sigma_BH(Z, E): the Bethe-Heitler differential
//     cross section the pair sampler draws from (bh_sample: the screening
//     functions ScreenFunction1/2 of ProxyBetheHeitler.hpp:184-210, the
//     Coulomb correction above 50 MeV) integrated over the electron's energy
//     fraction, with Tsai's Z (Z + xi(Z)) for pair production in the field of
//     the atomic electrons (the reference has no CrossSectionPerAtom for it);
//   LambdaPrim.phot   E x the Sandia photo-absorption parameterisation (the
//     photo-electric cross section the transport already uses below 200 keV;
//     the reference has none).
//   DEDX.eIoni.e-/e+  the restricted collision stopping power of the
//     Berger-Seltzer formula (ICRU Report 37; energy transfers below the e-
//     production cut), with the density effect of Sternheimer and Peierls
//     (Phys. Rev. B 3 (1971) 3681) from the mean excitation energy and the
//     plasma energy; above 10 keV (below it the formula does not hold)
//   DEDX.eBrem.e-     the restricted radiative loss: k dsigma/dk of the
//     Seltzer-Berger tables (with the dielectric suppression) integrated from
//     0 to the gamma cut, up to 1 GeV
//   Lambda.eBrem.e+, DEDX.eBrem.e+  the same integrals with the positron's
//     Coulomb factor exp(2 pi alpha Z (1/beta1 - 1/beta2)) on the electron
//     tables (beta1, beta2: the positron's speed before and after emitting k),
//     the approximation of the positron-to-electron bremsstrahlung ratio that
//     the Geant4 Physics Reference Manual gives for the Seltzer-Berger model
//   Range / InverseRange.eIoni.e-/e+  the range integral of 1 / (dE/dx) over
//     the context's ionisation plus brems loss (rebuilt where built), from
//     2 E0 / (dE/dx)(E0) at the lowest node (dE/dx proportional to beta
//     there), 8-point Gauss-Legendre in ln E per node interval; the inverse
//     range is the same pairs swapped (host side, in gx_ctx_rebuild_tables).
// gx_ctx_rebuild_tables puts these values on the shipped tables' node
// energies (materials Pb and LAr; brems up to 1 GeV and pairs up to 100 GeV,
// where Geant4's tables switch to its relativistic models) and refits the
// splines; the shipped values remain where no model here applies.  Against
// the shipped Geant4 tables: Compton, ionisation to 2e-4 (the materials'
// atomic masses), brems 0.5%, pairs within 6% from 50 MeV to 10 TeV (up to
// +16% in lead at 10-30 MeV, where the Born approximation overestimates; the
// shipped values are kept below 4 MeV, near threshold), photo-electric within
// 6% in lead and 14-19% low in argon (the Sandia parameterisation against
// the photo-electric model of the Geant4 build), collision stopping power
// within 2.5% (lead: the density-effect parameters) and 1e-3 (argon),
// radiative loss 0.2%, positron brems: the shipped e+/e- ratio to 1e-4
// (cross sections) and 1e-3 (radiative loss; 1% in lead at 20-60 keV, where
// the factor leaves 10-20% of the electrons' loss), ranges within 4% (lead,
// whose shipped range integrates a loss table 2% below its own DEDX table)
// and 2e-3 (argon).
#include "gx_internal.cuh"

#include <cmath>
#include <vector>

namespace gx {

namespace {

// 8-point Gauss-Legendre on [0, 1]: nodes and weights
__constant__ double kGLx[8] = {0.019855071751231856, 0.10166676129318664, 0.2372337950418355,
                               0.40828267875217510,  0.59171732124782490, 0.7627662049581645,
                               0.89833323870681340,  0.98014492824876810};
__constant__ double kGLw[8] = {0.050614268145188130, 0.11119051722668724, 0.15685332293894363,
                               0.18134189168918100,  0.18134189168918100, 0.15685332293894363,
                               0.11119051722668724,  0.050614268145188130};

__device__ double bhabha_xs_per_electron(double kin, double cut, double twopi_mc2_rcl2)
{
  if (!(cut < kin)) return 0.0;
  const double energy = kin + kEMass, gam = energy / kEMass, beta2 = 1.0 - 1.0 / (gam * gam);
  const double y = 1.0 / (1.0 + gam), y2 = y * y, y12 = 1.0 - 2.0 * y;
  const double b1 = 2.0 - y2, b2 = y12 * (3.0 + y2), y122 = y12 * y12, b4 = y122 * y12, b3 = b4 + y122;
  const double x0 = cut / kin;
  const double I = (1.0 / x0 - 1.0) / beta2 - b1 * ::log(1.0 / x0) + b2 * (1.0 - x0) -
                   b3 * (1.0 - x0 * x0) / 2.0 + b4 * (1.0 - x0 * x0 * x0) / 3.0;
  return twopi_mc2_rcl2 / kin * I;
}

// Positron factor exp(2 pi alpha Z (1/beta1 - 1/beta2)) for emitting k at
// kinetic energy kin (pos_coef = 2 pi alpha Z; 0 for electrons: factor 1).
__device__ double positron_factor(double pos_coef, double kin, double k)
{
  if (pos_coef == 0.0) return 1.0;
  const double t2 = kin - k;
  if (!(t2 > 0.0)) return 0.0;
  const double ib1 = (kin + kEMass) / ::sqrt(kin * (kin + 2.0 * kEMass));
  const double ib2 = (t2 + kEMass) / ::sqrt(t2 * (t2 + 2.0 * kEMass));
  return ::exp(pos_coef * (ib1 - ib2));
}

__device__ double sb_xs_per_atom(const SBTable &t, double Z, double kin, double cut, double density_factor,
                                 double pos_coef)
{
  if (!(cut < kin)) return 0.0;
  const double E = kin + kEMass, beta2 = kin * (kin + 2.0 * kEMass) / (E * E), kp2 = density_factor * E * E;
  const double v0 = ::log(cut), dv = (::log(kin) - v0) / 16.0, lnT = ::log(kin);
  double s = 0.0;
  for (int l = 0; l < 16; ++l)
    for (int i = 0; i < 8; ++i) {
      const double k = ::exp(v0 + (l + kGLx[i]) * dv);
      s += kGLw[i] * sb_value<double>(t, k / kin, lnT) / (1.0 + kp2 / (k * k)) * positron_factor(pos_coef, kin, k);
    }
  return Z * Z / beta2 * s * dv * 1.0e-25; // millibarn -> mm^2
}

// Bethe-Heitler pair production per atom, mm^2:
//   dsigma/deps = alpha r_e^2 Z (Z + xi) { [eps^2 + (1 - eps)^2] (S1(d) - F_Z) / 2
//                                       + 2/3 eps (1 - eps) (S2(d) - F_Z) / 2 },
//   d = 136 m / (Z^(1/3) E eps (1 - eps)), F_Z = 8/3 ln Z (+ 8 f_c above 50 MeV),
//   xi = ln(1440 Z^(-2/3)) / (ln(183 Z^(-1/3)) - f_c)  (Y. S. Tsai, Rev. Mod. Phys.
//   46 (1974) 815), the negative parts of S - F_Z dropped as the sampler's
//   majorant does; symmetric in eps, so twice the integral over [m/E, 1/2]
//   (8 x 8-point Gauss-Legendre).
__device__ double bh_xs_per_atom(double Z, double E, double alpha, double rcl2)
{
  const double eps0 = kEMass / E;
  if (!(eps0 < 0.5)) return 0.0;
  const double fc = coulomb_factor(Z), lnZ = ::log(Z), Z3 = ::pow(Z, 1.0 / 3.0);
  const double FZ = 8.0 * lnZ / 3.0 + (E > 50.0 ? 8.0 * fc : 0.0);
  const double xi = ::log(1440.0 / (Z3 * Z3)) / (::log(183.0 / Z3) - fc);
  const double h = (0.5 - eps0) / 8.0;
  double s = 0.0;
  for (int l = 0; l < 8; ++l)
    for (int i = 0; i < 8; ++i) {
      const double eps = eps0 + (l + kGLx[i]) * h, u = eps * (1.0 - eps);
      const double d = 136.0 * eps0 / (Z3 * u);
      const double f1 = fmax(screen1<double>(d) - FZ, 0.0), f2 = fmax(screen2<double>(d) - FZ, 0.0);
      s += kGLw[i] * ((eps * eps + (1.0 - eps) * (1.0 - eps)) * f1 + (2.0 / 3.0) * u * f2);
    }
  return alpha * rcl2 * Z * (Z + xi) * s * h; // 2 x (1/2) x the bracket
}

// Density-effect correction of Sternheimer and Peierls for a condensed
// material: C = 1 + 2 ln(I / hw_p), hw_p = 28.816 eV sqrt(rho Z / A); x0, x1
// by their rules for I below / above 100 eV; m = 3.
__device__ double density_effect(double x, double I, double Z, double A, double rho)
{
  const double hwp = 28.816e-6 * ::sqrt(rho * Z / A), C = 1.0 + 2.0 * ::log(I / hwp);
  double x0, x1;
  if (I < 100.0e-6) {
    x1 = 2.0;
    x0 = C < 3.681 ? 0.2 : 0.326 * C - 1.0;
  } else {
    x1 = 3.0;
    x0 = C < 5.215 ? 0.2 : 0.326 * C - 1.5;
  }
  const double a = (C - 4.606 * x0) / ((x1 - x0) * (x1 - x0) * (x1 - x0));
  if (x < x0) return 0.0;
  if (x < x1) return 4.606 * x - C + a * (x1 - x) * (x1 - x) * (x1 - x);
  return 4.606 * x - C;
}

// Restricted collision stopping power (MeV/mm) of an electron (positron = 0)
// or positron (1) of kinetic energy T, energy transfers below cut: the
// Berger-Seltzer formula, 2 pi r_e^2 m n_el / beta^2 [ln(2 (tau + 2) / (I/m)^2)
// + F(tau, Delta) - delta].
__device__ double bs_dedx(double T, double cut, double I, double Z, double A, double rho, double n_el,
                          double twopi_mc2_rcl2, int positron)
{
  const double tau = T / kEMass, gam = tau + 1.0, b2 = tau * (tau + 2.0) / (gam * gam);
  const double x = ::log10(::sqrt(tau * (tau + 2.0)));
  const double lnI = ::log(2.0 * (tau + 2.0) / ((I / kEMass) * (I / kEMass)));
  double F;
  if (!positron) {
    const double d = fmin(cut, 0.5 * T) / kEMass;
    F = -1.0 - b2 + ::log((tau - d) * d) + tau / (tau - d) +
        (0.5 * d * d + (2.0 * tau + 1.0) * ::log(1.0 - d / tau)) / (gam * gam);
  } else {
    const double d = fmin(cut, T) / kEMass, y = 1.0 / (1.0 + gam), d2 = d * d, d3 = d2 * d, d4 = d3 * d;
    F = ::log(tau * d) - (b2 / tau) * (tau + 2.0 * d - 1.5 * d2 * y - (d - d3 / 3.0) * y * y -
                                       (0.5 * d2 - tau * d3 / 3.0 + 0.25 * d4) * y * y * y);
  }
  return twopi_mc2_rcl2 * n_el / b2 * (lnI + F - density_effect(x, I, Z, A, rho));
}

// Restricted radiative loss per atom (MeV mm^2): the integral of k dsigma/dk
// from 0 to min(kc, T) with the Seltzer-Berger tables (dsigma/dk = Z^2
// chi(k/T, T) / (beta^2 k) millibarn) and the dielectric suppression.
__device__ double sb_dedx_per_atom(const SBTable &t, double Z, double kin, double kc, double density_factor,
                                   double pos_coef)
{
  const double E = kin + kEMass, beta2 = kin * (kin + 2.0 * kEMass) / (E * E), kp2 = density_factor * E * E;
  const double kmax = fmin(kc, kin), dk = kmax / 16.0, lnT = ::log(kin);
  double s = 0.0;
  for (int l = 0; l < 16; ++l)
    for (int i = 0; i < 8; ++i) {
      const double k = (l + kGLx[i]) * dk;
      s += kGLw[i] * sb_value<double>(t, k / kin, lnT) / (1.0 + kp2 / (k * k)) * positron_factor(pos_coef, kin, k);
    }
  return Z * Z / beta2 * s * dk * 1.0e-25;
}

__global__ void k_table_build(const Data *__restrict__ D, int table, int mat, const double *__restrict__ E,
                              double *__restrict__ out, int n)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Data &d = *D;
  const double e = E[i], Z = d.mat_Z[mat], n_el = d.mat_nel[mat], n_atoms = n_el / Z;
  const double twopi_mc2_rcl2 = 2.0 * kEMass * d.pi_rcl2, pos_coef = 2.0 * kPi * d.alpha * Z;
  const SBTable &sb = d.sb[mat == 1 ? 2 : 1];
  double v = 0.0;
  switch (table) {
  case GX_Lambda_compt: v = fmax(0.0, n_atoms * kn_xs_per_atom(Z, e)); break;
  case GX_LambdaPrim_compt: v = fmax(0.0, e * n_atoms * kn_xs_per_atom(Z, e)); break;
  case GX_Lambda_eIoni_em: v = n_atoms * mb_xs_per_atom(Z, e, twopi_mc2_rcl2, d.cut_energy[1][mat]); break;
  case GX_Lambda_eIoni_ep: v = n_el * bhabha_xs_per_electron(e, d.cut_energy[1][mat], twopi_mc2_rcl2); break;
  case GX_Lambda_eBrem_em:
  case GX_Lambda_eBrem_ep:
    v = n_atoms * sb_xs_per_atom(sb, Z, e, d.cut_energy[0][mat], d.mat_dfactor[mat],
                                 table == GX_Lambda_eBrem_ep ? pos_coef : 0.0);
    break;
  case GX_Lambda_conv: v = n_atoms * bh_xs_per_atom(Z, e, d.alpha, d.pi_rcl2 / kPi); break;
  case GX_DEDX_eIoni_em:
  case GX_DEDX_eIoni_ep:
    v = bs_dedx(e, d.cut_energy[1][mat], d.mat_I[mat], Z, d.mat_A[mat], d.mat_density[mat], n_el, twopi_mc2_rcl2,
                table == GX_DEDX_eIoni_ep);
    break;
  case GX_DEDX_eBrem_em:
  case GX_DEDX_eBrem_ep:
    v = n_atoms * sb_dedx_per_atom(sb, Z, e, d.cut_energy[0][mat], d.mat_dfactor[mat],
                                   table == GX_DEDX_eBrem_ep ? pos_coef : 0.0);
    break;
  case GX_LambdaPrim_phot: v = e * pe_xs_sandia(d, (int)Z, d.mat_density[mat], e); break;
  default: v = 0.0;
  }
  out[i] = v;
}

bool buildable(int table, int mat)
{
  const bool t = table == GX_Lambda_compt || table == GX_LambdaPrim_compt || table == GX_Lambda_eIoni_em ||
                 table == GX_Lambda_eIoni_ep || table == GX_Lambda_eBrem_em || table == GX_Lambda_conv ||
                 table == GX_LambdaPrim_phot || table == GX_DEDX_eIoni_em || table == GX_DEDX_eIoni_ep ||
                 table == GX_DEDX_eBrem_em || table == GX_Lambda_eBrem_ep || table == GX_DEDX_eBrem_ep;
  return t && (mat == 1 || mat == 2); // the SB data cover lead and argon
}

// Values of the context's tables (the reference's spline) at n energies.
__global__ void k_table_eval(const Data *__restrict__ D, int table, int mat, const double *__restrict__ E,
                             double *__restrict__ out, int n)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = vec_value_ref(*D, D->vec[table][mat], E[i]);
}

// Range and inverse range of e- (ep = 0) or e+ (1) in material mat from the
// context's current loss tables (ionisation + brems), at the range table's
// node energies; refits both vectors.
int rebuild_range(Ctx *c, int mat, int ep)
{
  const int tr = ep ? GX_Range_ep : GX_Range_em, ti = ep ? GX_InverseRange_ep : GX_InverseRange_em;
  const int tion = ep ? GX_DEDX_eIoni_ep : GX_DEDX_eIoni_em, tbr = ep ? GX_DEDX_eBrem_ep : GX_DEDX_eBrem_em;
  const VecDesc &vd = c->host.vec[tr][mat];
  const int n = vd.n;
  std::vector<double> x(n);
  cudaError_t e = cudaMemcpy(x.data(), c->host.x + vd.off, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_error(e, "rebuild_range: nodes");
  // 8-point Gauss-Legendre in ln E on each node interval, plus the lowest node
  static const double gx[8] = {0.019855071751231856, 0.10166676129318664, 0.2372337950418355, 0.40828267875217510,
                               0.59171732124782490,  0.7627662049581645,  0.89833323870681340, 0.98014492824876810};
  static const double gw[8] = {0.050614268145188130, 0.11119051722668724, 0.15685332293894363, 0.18134189168918100,
                               0.18134189168918100,  0.15685332293894363, 0.11119051722668724, 0.050614268145188130};
  const int m = 1 + 8 * (n - 1);
  std::vector<double> E(m), D(m, 0.0);
  E[0] = x[0];
  for (int j = 1; j < n; ++j)
    for (int i = 0; i < 8; ++i) E[1 + 8 * (j - 1) + i] = std::exp(std::log(x[j - 1]) + gx[i] * std::log(x[j] / x[j - 1]));
  double *dE = nullptr, *dV = nullptr;
  if ((e = cudaMalloc((void **)&dE, 2 * m * sizeof(double))) != cudaSuccess) return cuda_error(e, "rebuild_range");
  dV = dE + m;
  cudaMemcpy(dE, E.data(), m * sizeof(double), cudaMemcpyHostToDevice);
  std::vector<double> V(m);
  for (int t : {tion, tbr}) {
    k_table_eval<<<(m + 127) / 128, 128>>>(c->dev, t, mat, dE, dV, m);
    if ((e = cudaMemcpy(V.data(), dV, m * sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess) break;
    for (int k = 0; k < m; ++k) D[k] += V[k];
  }
  cudaFree(dE);
  if (e != cudaSuccess) return cuda_error(e, "rebuild_range: loss tables");
  std::vector<double> r(n);
  r[0] = 2.0 * x[0] / D[0];
  for (int j = 1; j < n; ++j) {
    double s = 0.0;
    for (int i = 0; i < 8; ++i) {
      const int k = 1 + 8 * (j - 1) + i;
      s += gw[i] * E[k] / D[k];
    }
    r[j] = r[j - 1] + s * std::log(x[j] / x[j - 1]);
  }
  int rc = refit_vector(c, tr, mat, r.data());
  if (rc) return rc;
  return refit_vector_xy(c, ti, mat, r.data(), x.data());
}

} // namespace

} // namespace gx

using namespace gx;

extern "C" {

int gx_table_build(gx_ctx *ctx, int table, int mat, const double *d_E, double *d_out, int n, gx_stream_t s)
{
  if (!ctx || n < 0 || (n > 0 && (!d_E || !d_out))) return set_error(GX_ERR_ARG, "gx_table_build: bad arguments");
  if (!buildable(table, mat)) return set_error(GX_ERR_ARG, "gx_table_build: table %d, material %d not built", table, mat);
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (n == 0) return GX_OK;
  k_table_build<<<(n + 127) / 128, 128, 0, stream_of(s)>>>(c->dev, table, mat, d_E, d_out, n);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GX_OK : cuda_error(e, "k_table_build");
}

int gx_ctx_rebuild_tables(gx_ctx *ctx, double *max_rel_change)
{
  if (!ctx) return set_error(GX_ERR_ARG, "gx_ctx_rebuild_tables: null context");
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_error(e, "gx_ctx_rebuild_tables: cudaSetDevice");
  const int tables[] = {GX_Lambda_compt, GX_LambdaPrim_compt, GX_Lambda_eIoni_em, GX_Lambda_eIoni_ep,
                        GX_Lambda_eBrem_em, GX_Lambda_conv, GX_LambdaPrim_phot, GX_DEDX_eIoni_em,
                        GX_DEDX_eIoni_ep, GX_DEDX_eBrem_em, GX_Lambda_eBrem_ep, GX_DEDX_eBrem_ep};
  double *dv = nullptr;
  int nmax = 0;
  for (int t : tables)
    for (int m = 1; m <= 2; ++m) nmax = std::max(nmax, c->host.vec[t][m].n);
  if ((e = cudaMalloc((void **)&dv, nmax * sizeof(double))) != cudaSuccess)
    return cuda_error(e, "gx_ctx_rebuild_tables: scratch");
  double worst = 0.0;
  int rc = GX_OK;
  for (int t : tables)
    for (int m = 1; m <= 2 && rc == GX_OK; ++m) {
      const VecDesc &vd = c->host.vec[t][m];
      std::vector<double> x(vd.n), y(vd.n), old(vd.n);
      k_table_build<<<(vd.n + 127) / 128, 128>>>(c->dev, t, m, c->host.x + vd.off, dv, vd.n);
      if ((e = cudaMemcpy(y.data(), dv, vd.n * sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess ||
          (e = cudaMemcpy(x.data(), c->host.x + vd.off, vd.n * sizeof(double), cudaMemcpyDeviceToHost)) ||
          (e = cudaMemcpy(old.data(), c->host.y + vd.off, vd.n * sizeof(double), cudaMemcpyDeviceToHost))) {
        rc = cuda_error(e, "gx_ctx_rebuild_tables: download");
        break;
      }
      for (int i = 0; i < vd.n; ++i) {
        // brems: the Seltzer-Berger range only (Geant4 changes model at 1 GeV)
        if ((t == GX_Lambda_eBrem_em || t == GX_Lambda_eBrem_ep) && x[i] > 1.0e3) y[i] = old[i];
        // pairs: the Bethe-Heitler range (Geant4 changes to its relativistic,
        // LPM-suppressed model at 80 GeV)
        if (t == GX_Lambda_conv && (x[i] > 1.0e5 || x[i] < 4.0)) y[i] = old[i]; // and near threshold
        // stopping powers: the formulas hold above 10 keV; radiative loss in
        // the Seltzer-Berger range
        if ((t == GX_DEDX_eIoni_em || t == GX_DEDX_eIoni_ep) && x[i] < 0.01) y[i] = old[i];
        if ((t == GX_DEDX_eBrem_em || t == GX_DEDX_eBrem_ep) && x[i] > 1.0e3) y[i] = old[i];
        if (old[i] > 0.0 && y[i] > 0.0 && x[i] > 0.01) // above 10 keV (below it the shipped low-energy tails differ)
          worst = std::max(worst, std::fabs(y[i] / old[i] - 1.0));
      }
      rc = refit_vector(c, t, m, y.data());
    }
  cudaFree(dv);
  if (rc) return rc;
  // ranges from the rebuilt losses, and their inverses
  for (int m = 1; m <= 2 && rc == GX_OK; ++m)
    for (int ep = 0; ep <= 1 && rc == GX_OK; ++ep) rc = rebuild_range(c, m, ep);
  if (rc) return rc;
  if (max_rel_change) *max_rel_change = worst;
  return GX_OK;
}

} // extern "C"
