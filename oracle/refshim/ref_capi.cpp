// ref_capi.cpp -- ORACLE (test infrastructure only).
//
// extern "C" entry points that drive the reference's own hot-path code,
// compiled in place from the reference checkout through the headers in this
// directory (see ../build_ref.sh).  They are used to pin the plain-C oracle
// and to generate the committed golden vectors; nothing in the product links
// them.  The reference's data manager and Seltzer-Berger model read their data
// files relative to the working directory, so callers chdir to the
// reference's BasicCpuTransport directory before the first table or SB call.
#include "Geant/magneticfield/ConstFieldHelixStepper.hpp"
#include "Geant/proxy/ProxyBetheHeitler.hpp"
#include "Geant/proxy/ProxyBremsstrahlung.hpp"
#include "Geant/proxy/ProxyCompton.hpp"
#include "Geant/proxy/ProxyConversion.hpp"
#include "Geant/proxy/ProxyDataManager.cuh"
#include "Geant/proxy/ProxyIonization.hpp"
#include "Geant/proxy/ProxyKleinNishina.hpp"
#include "Geant/proxy/ProxyMollerScattering.hpp"
#include "Geant/proxy/ProxyPhotoElectric.hpp"
#include "Geant/proxy/ProxySauterGavrila.hpp"
#include "Geant/proxy/ProxySeltzerBerger.hpp"
#include "Geant/proxy/Proxy2DVector.hpp"
#include "Geant/random/MRG32k3a.hpp"
#include "Geant/proxy/ProxyEgammaGun.hpp"
#include "Geant/proxy/ProxyHepEvtGenerator.hpp"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <map>

namespace geantx {
thread_local std::vector<CapturedTrack> *gxrefCapture = nullptr;
thread_local long gxrefSeq = 0;
static thread_local MRG32k3a::State_t gState;
MRG32k3a::State_t *gxref_current_state() { return &gState; }
MRG32k3a &gxref_engine()
{
  static MRG32k3a engine;
  return engine;
}
} // namespace geantx

using namespace geantx;

namespace {
void load_state(const double *s) { std::memcpy(gState.fCg, s, 6 * sizeof(double)); }
void store_state(double *s) { std::memcpy(s, gState.fCg, 6 * sizeof(double)); }

// Advance-able access to the protected state of a reference MRG32k3a.
struct MrgAccess : public MRG32k3a {
  double *cg() { return this->GetState()->fCg; }
};
} // namespace

extern "C" {

// MRG32k3a: seed(6) -> Initialize() (SetNextStream) -> k Uniform() draws.
void gxref_mrg_draws(const double *seed, int k, double *out, double *state_out)
{
  double s[6];
  std::memcpy(s, seed, sizeof(s));
  MrgAccess r;
  r.SetSeed(s);
  r.Initialize();
  for (int i = 0; i < k; ++i) out[i] = r.Uniform();
  std::memcpy(state_out, r.cg(), sizeof(s));
}

// MRG32k3a::Initialize(long streamId) followed by k draws.
void gxref_mrg_stream_id(long id, int k, double *out)
{
  MrgAccess r;
  r.Initialize(id);
  for (int i = 0; i < k; ++i) out[i] = r.Uniform();
}

// MRG32k3a::AdvanceState(e, c) applied to a given state.
void gxref_mrg_advance(double *state, long e, long c)
{
  MrgAccess r;
  r.SetSeed(state);
  r.Initialize();
  r.AdvanceState(e, c);
  std::memcpy(state, r.cg(), 6 * sizeof(double));
}

// ---- tables (ProxyDataManager / ProxyPhysicsTable / ProxyPhysicsVector)
int gxref_tables_init() { return ProxyDataManager::Instance() ? 1 : 0; }
double gxref_table_value(int table, int mat, double e)
{
  return ProxyDataManager::Instance()->GetTable(table)->Value(mat, e);
}
double gxref_table_invrange(int table, int mat, double r)
{
  return ProxyDataManager::Instance()->GetTable(table)->GetPhysicsVector(mat)->InvRangeValue(r);
}
double gxref_cut_value(int index, int ipart) { return ProxyDataManager::Instance()->GetCutValue(index, ipart); }

// Proxy2DVector::Value on a Seltzer-Berger table read from data/brem_SB/br<Z>.
double gxref_sb2d_value(int Z, double x, double y)
{
  static std::map<int, Proxy2DVector *> cache;
  Proxy2DVector *v = cache[Z];
  if (!v) {
    v = new Proxy2DVector();
    char fn[256];
    std::snprintf(fn, sizeof(fn), "data/brem_SB/br%d", Z);
    std::ifstream in(fn);
    int k, nx, ny;
    in >> k >> nx >> ny;
    double val;
    for (size_t i = 0; i < data::numberOfXNodes; ++i) { in >> val; v->PutX(i, val); }
    for (size_t j = 0; j < data::numberOfYNodes; ++j) { in >> val; v->PutY(j, val); }
    for (size_t j = 0; j < data::numberOfYNodes; ++j)
      for (size_t i = 0; i < data::numberOfXNodes; ++i) { in >> val; v->PutValue(i, j, val); }
    cache[Z] = v;
  }
  return v->Value(x, y);
}

// ---- models: 0 KleinNishina, 1 SauterGavrila, 2 BetheHeitler, 3 SeltzerBerger, 4 Moller
void gxref_interact(int model, int n, double *states, const double *E, const double *dir, double *E_out,
                    double *dir_out, double *edep, int *status, int *nsec, int *sec_type, double *sec_E,
                    double *sec_dir)
{
  static ProxyKleinNishina *kn = new ProxyKleinNishina();
  static ProxySauterGavrila *sg = new ProxySauterGavrila();
  static ProxyBetheHeitler *bh = new ProxyBetheHeitler();
  static ProxyMollerScattering *mb = new ProxyMollerScattering();
  static ProxySeltzerBerger *sb = (model == 3) ? new ProxySeltzerBerger() : nullptr;
  if (model == 3 && !sb) sb = new ProxySeltzerBerger();
  static const int kSecType[5][2] = {{1, -1}, {1, -1}, {1, 2}, {0, -1}, {1, -1}};
  for (int i = 0; i < n; ++i) {
    load_state(&states[6 * i]);
    std::vector<CapturedTrack> cap;
    TrackState t;
    t.fCapture = false;
    t.fPhysicsState.fEkin = E[i];
    t.fDir = ThreeVector(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
    gxrefCapture = &cap;
    int ns = 0;
    switch (model) {
    case 0: ns = kn->SampleSecondaries(&t); break;
    case 1: ns = sg->SampleSecondaries(&t); break;
    case 2: ns = bh->SampleSecondaries(&t); break;
    case 3: ns = sb->SampleSecondaries(&t); break;
    case 4: ns = mb->SampleSecondaries(&t); break;
    default: break;
    }
    gxrefCapture = nullptr;
    std::sort(cap.begin(), cap.end(), [](const CapturedTrack &a, const CapturedTrack &b) { return a.seq < b.seq; });
    store_state(&states[6 * i]);
    E_out[i] = t.fPhysicsState.fEkin;
    dir_out[3 * i] = t.fDir.x();
    dir_out[3 * i + 1] = t.fDir.y();
    dir_out[3 * i + 2] = t.fDir.z();
    edep[i] = t.fPhysicsState.fEdep;
    status[i] = (t.fStatus == TrackStatus::Killed) ? 1 : 0;
    nsec[i] = ns;
    for (int s = 0; s < 2; ++s) {
      bool has = s < (int)cap.size();
      sec_type[2 * i + s] = has ? kSecType[model][s] : -1;
      sec_E[2 * i + s] = has ? cap[s].ekin : 0.0;
      for (int k = 0; k < 3; ++k) sec_dir[6 * i + 3 * s + k] = has ? cap[s].dir[k] : 0.0;
    }
  }
}

double gxref_kn_xs(double Z, double e)
{
  static ProxyKleinNishina *kn = new ProxyKleinNishina();
  return kn->CrossSectionPerAtom(Z, e);
}
double gxref_mb_xs(double Z, double e)
{
  static ProxyMollerScattering *mb = new ProxyMollerScattering();
  return mb->CrossSectionPerAtom(Z, e);
}
double gxref_sg_photo_energy(int Z, double e)
{
  static ProxySauterGavrila *sg = new ProxySauterGavrila();
  return sg->GetPhotoElectronEnergy(Z, e);
}
double gxref_coulomb(double Z)
{
  static ProxyBetheHeitler *bh = new ProxyBetheHeitler();
  return bh->ComputeCoulombFactor(Z);
}

// ---- processes: PostStepGPIL of 0 Compton, 1 Conversion, 2 PhotoElectric,
// 3 Bremsstrahlung, 4 Ionization on one TrackState carrying NIL / saved 1/lambda.
double gxref_post_step_gpil(int process, double *state, double e, double pstep_prev, double *nil,
                            double *saved, int mat)
{
  static ProxyCompton *pc = new ProxyCompton();
  static ProxyConversion *pv = new ProxyConversion();
  static ProxyPhotoElectric *pp = new ProxyPhotoElectric();
  static ProxyBremsstrahlung *pb = new ProxyBremsstrahlung();
  static ProxyIonization *pi = new ProxyIonization();
  static const int kIndex[5] = {kProxyCompton, kProxyConversion, kProxyPhotoElectric, kProxyBremsstrahlung,
                                kProxyIonization};
  load_state(state);
  TrackState t;
  t.fCapture = false;
  t.fPhysicsState.fEkin = e;
  t.fPhysicsState.fPstep = pstep_prev;
  t.fMaterialState.fMaterialId = mat;
  int k = kIndex[process];
  t.fPhysicsProcessState[k].fNumOfInteractLengthLeft = *nil;
  t.fPhysicsProcessState[k].fPhysicsInteractLength = *saved;
  double step = 0;
  switch (process) {
  case 0: step = pc->PostStepGPIL(&t); break;
  case 1: step = pv->PostStepGPIL(&t); break;
  case 2: step = pp->PostStepGPIL(&t); break;
  case 3: step = pb->PostStepGPIL(&t); break;
  case 4: step = pi->PostStepGPIL(&t); break;
  default: break;
  }
  *nil = t.fPhysicsProcessState[k].fNumOfInteractLengthLeft;
  *saved = t.fPhysicsProcessState[k].fPhysicsInteractLength;
  store_state(state);
  return step;
}

double gxref_ioni_along_gpil(int mat, double e)
{
  static ProxyIonization *pi = new ProxyIonization();
  TrackState t;
  t.fCapture = false;
  t.fPhysicsState.fEkin = e;
  t.fMaterialState.fMaterialId = mat;
  return pi->AlongStepGPIL(&t);
}

void gxref_ioni_along_doit(int mat, double step, double *e, double *edep)
{
  static ProxyIonization *pi = new ProxyIonization();
  TrackState t;
  t.fCapture = false;
  t.fPhysicsState.fEkin = *e;
  t.fPhysicsState.fPstep = step;
  t.fMaterialState.fMaterialId = mat;
  pi->AlongStepDoIt(&t);
  *e = t.fPhysicsState.fEkin;
  *edep = t.fPhysicsState.fEdep;
}

// ---- ConstFieldHelixStepper::DoStep (GeV, kilogauss, cm)
void gxref_helix(const double *B, int n, const double *pos, const double *dir, const double *charge,
                 const double *mom, const double *step, double *newpos, double *newdir)
{
  ConstFieldHelixStepper stepper(B[0], B[1], B[2]);
  for (int i = 0; i < n; ++i) {
    double x, y, z, dx, dy, dz;
    stepper.DoStep<double>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], dir[3 * i], dir[3 * i + 1], dir[3 * i + 2],
                           charge[i], mom[i], step[i], x, y, z, dx, dy, dz);
    newpos[3 * i] = x;
    newpos[3 * i + 1] = y;
    newpos[3 * i + 2] = z;
    newdir[3 * i] = dx;
    newdir[3 * i + 1] = dy;
    newdir[3 * i + 2] = dz;
  }
}

} // extern "C"


extern "C" {

// ProxyEgammaGun::GenerateOneEvent (proxy/src/ProxyEgammaGun.cpp:43-85), nevents
// events of nparticles, drawing from the stream state `state` (updated).  Per
// particle: PDG code, momentum, kinetic energy, direction.
int gxref_egamma_gun(double *state, int nevents, int nparticles, double gamma_fraction, double minp, double maxp,
                     double mineta, double maxeta, double minphi, double maxphi, int *pdg, double *p, double *ekin,
                     double *dir)
{
  load_state(state);
  // the one-argument constructor is ambiguous with the (nevents, nparticles = 1) one
  ProxyEgammaGun gun(nevents, nparticles);
  gun.SetGammaFraction(gamma_fraction);
  gun.SetMomentum(minp, maxp);
  gun.SetEta(mineta, maxeta);
  gun.SetPhi(minphi, maxphi);
  int k = 0;
  for (int e = 0; e < nevents; ++e) {
    ProxyEvent *ev = gun.GenerateOneEvent();
    ProxyVertex *v = (*ev->GetVertexVector())[0];
    for (int i = 0; i < v->GetNumberOfParticles(); ++i, ++k) {
      TrackState *t = v->GetParticle(i);
      t->fCapture = false;
      pdg[k] = t->fSchedulingState.fGVcode;
      p[k] = t->fPhysicsState.fMomentum;
      ekin[k] = t->fPhysicsState.fEkin;
      for (int j = 0; j < 3; ++j) dir[3 * k + j] = t->fDir.v[j];
    }
  }
  store_state(state);
  return k;
}

// ProxyEgammaGun::SetDirectionXYZ (ProxyEgammaGun.cpp:35-41): the direction of
// a particle generated with the eta and phi it sets (both ranges collapse to
// one value, so no draw changes it).
void gxref_egamma_direction(double x, double y, double z, double *dir)
{
  ProxyEgammaGun gun(1, 1);
  gun.SetDirectionXYZ(x, y, z);
  double st[6] = {12345., 12345., 12345., 12345., 12345., 12345.};
  load_state(st);
  ProxyEvent *ev = gun.GenerateOneEvent();
  TrackState *t = (*ev->GetVertexVector())[0]->GetParticle(0);
  t->fCapture = false;
  for (int j = 0; j < 3; ++j) dir[j] = t->fDir.v[j];
}

// ProxyHepEvtGenerator::GenerateOneEvent (proxy/src/ProxyHepEvtGenerator.cpp:48-132)
// for max_events events of `path`; per particle: event, PDG code, momentum,
// kinetic energy, direction.  Returns the number of particles (at most cap).
int gxref_hepevt(const char *path, int max_events, int cap, int *event, int *pdg, double *p, double *ekin, double *dir)
{
  // the path-only constructor leaves the event vector null, which the base
  // class destructor dereferences; the (nevents, path) one allocates it
  ProxyHepEvtGenerator gen(max_events, path);
  int k = 0;
  for (int e = 0; e < max_events; ++e) {
    ProxyEvent *ev = gen.GenerateOneEvent();
    ProxyVertex *v = (*ev->GetVertexVector())[0];
    for (int i = 0; i < v->GetNumberOfParticles() && k < cap; ++i, ++k) {
      TrackState *t = v->GetParticle(i);
      t->fCapture = false;
      event[k] = e;
      pdg[k] = t->fSchedulingState.fGVcode;
      p[k] = t->fPhysicsState.fMomentum;
      ekin[k] = t->fPhysicsState.fEkin;
      for (int j = 0; j < 3; ++j) dir[3 * k + j] = t->fDir.v[j];
    }
  }
  return k;
}

} // extern "C"
