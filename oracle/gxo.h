/*
 * gxo.h -- ORACLE (test infrastructure only).
 *
 * A plain-C, scalar CPU restatement of the reference's electromagnetic
 * particle-transport step path (Geant-RnD/GeantExascalePilot), against which
 * the CUDA product in geantexascalepilot_b200/ is tested: only the tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and never
 * as the thing measured or shipped.
 *
 * Each function cites the reference file:line it restates.  Parity of this
 * restatement is pinned against the reference's own code compiled in place
 * (oracle/refshim + oracle/build_ref.sh -> oracle/_ref/libgxref.so); the
 * generated golden vectors live in tests/golden/.
 *
 * Units: mm, MeV, ns (the reference's CLHEP units,
 * source/Geant/proxy/ProxySystemOfUnits.hpp); magnetic field in tesla.
 */
#ifndef GXO_H
#define GXO_H

#include <math.h>
#include <stdint.h>

/* The elementary functions of the per-step arithmetic (table lookups, models,
 * multiple scattering, helix).  Default build (liboracle.so): the C library's,
 * as the reference's std:: math -- this is the build pinned bit for bit
 * against the reference.  Parity build (liboracle_gxm.so, -DGXO_OWN_MATH):
 * the functions of gx_math.h, which the CUDA library's FP64 parity variant
 * compiles too, so that the two round alike and agree track by track; that
 * header is itself tested against the C library's functions to its stated
 * error bounds.  Set-up constants (materials, table grids, the multiple-
 * scattering material constants) stay on the C library in both builds, as in
 * the CUDA library's host code. */
#ifdef GXO_OWN_MATH
#include "gx_math.h"
#define gxo_log gxm_log
#define gxo_exp gxm_exp
#define gxo_pow gxm_pow
#define gxo_sin gxm_sin
#define gxo_cos gxm_cos
#define gxo_expm1 gxm_expm1
#define gxo_log1p gxm_log1p
#else
#define gxo_log log
#define gxo_exp exp
#define gxo_pow pow
#define gxo_sin sin
#define gxo_cos cos
#define gxo_expm1 expm1
#define gxo_log1p log1p
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- MRG32k3a */
/* source/Geant/random/MRG32k3a.hpp:45-49 -- state is six FP64 integers. */
typedef struct { double s[6]; } gxo_mrg_t;

double gxo_mrg_u01(gxo_mrg_t *r);                        /* MRG32k3a.cpp:124-163 */
uint32_t gxo_mrg_next_raw(gxo_mrg_t *r);                 /* numerator of the draw */
void gxo_mrg_advance(gxo_mrg_t *r, long e, long c);      /* MRG32k3a.cpp:171-178 */
void gxo_mrg_next_stream(double seed[6], gxo_mrg_t *r);  /* MRG32k3a.cpp:52-58 */
void gxo_mrg_next_substream(double bg[6], gxo_mrg_t *r); /* MRG32k3a.cpp:61-67 */
void gxo_mrg_init_stream_id(long id, gxo_mrg_t *r);      /* MRG32k3a.cpp:70-82 */
void gxo_mrg_seed_child(gxo_mrg_t *parent, gxo_mrg_t *child);

/* batch helpers for ctypes: states are n x 6 doubles, row-major */
void gxo_mrg_uniform_batch(int n, int k, double *states, double *out);
void gxo_mrg_substreams(const double seed[6], long first, int n, double *states);
void gxo_mrg_advance_batch(int n, double *states, long e, long c);

/* ------------------------------------------------------- physics vectors */
/* source/Geant/proxy/ProxyPhysicsVector.cuh / src/ProxyPhysicsVector.cu */
typedef struct {
  int n, type;
  double emin, emax, dbin, base;
  double *x, *y, *d2;
} gxo_pvec_t;

enum {
  GXO_DEDX_eBrem_em, GXO_DEDX_eBrem_ep, GXO_DEDX_eIoni_em, GXO_DEDX_eIoni_ep,
  GXO_InverseRange_em, GXO_InverseRange_ep, GXO_Ionisation_em, GXO_Ionisation_ep,
  GXO_Lambda_compt, GXO_Lambda_conv, GXO_Lambda_eBrem_em, GXO_Lambda_eBrem_ep,
  GXO_Lambda_eIoni_em, GXO_Lambda_eIoni_ep, GXO_LambdaMod1_msc_em, GXO_LambdaMod1_msc_ep,
  GXO_LambdaPrim_compt, GXO_LambdaPrim_phot, GXO_Range_em, GXO_Range_ep,
  GXO_NTABLES
};
#define GXO_NMAT 3

/* Seltzer-Berger 2-D table: source/Geant/proxy/Proxy2DVector.hpp:22-56 */
typedef struct { double x[32]; double y[57]; double v[57][32]; } gxo_sb_t;

typedef struct {
  gxo_pvec_t vec[GXO_NTABLES][GXO_NMAT];
  double cut_energy[4][GXO_NMAT]; /* [particle g,e-,e+,p][material], MeV */
  double cut_length[4][GXO_NMAT]; /* mm */
  double cut_raw[12];             /* file order, as the reference stores it */
  gxo_sb_t sb_slot10;             /* br11: the reference's fDataSB[10] */
  gxo_sb_t sb_ar, sb_pb;          /* br18, br82 */
  int nshell[101], ishell[101];
  double binding[1540];           /* eV */
  int nint[101], cumint[101];
  double sandia[981][5];
} gxo_data_t;

gxo_data_t *gxo_data_load(const char *datadir); /* NULL on failure */
void gxo_data_free(gxo_data_t *d);
double gxo_pvec_value(const gxo_pvec_t *v, double e);          /* PhysicsVector.cu:469-483 */
double gxo_pvec_invrange_value(const gxo_pvec_t *v, double r); /* PhysicsVector.cu:491-524 */
double gxo_table_value(const gxo_data_t *d, int table, int mat, double e);
double gxo_table_invrange(const gxo_data_t *d, int table, int mat, double r);
double gxo_sb_value(const gxo_sb_t *t, double x, double y);    /* Proxy2DVector.cpp:37-67 */
double gxo_get_cut_value(const gxo_data_t *d, int index, int ipart); /* ProxyDataManager.cuh:52-54 */
void gxo_table_value_batch(const gxo_data_t *d, int table, int mat, int n, const double *e, double *out);
void gxo_table_invrange_batch(const gxo_data_t *d, int table, int mat, int n, const double *r, double *out);

/* ------------------------------------------------------------ materials */
typedef struct {
  double Z, A, density;  /* g/mol, g/cm3 */
  double n_atoms;        /* 1/mm3 */
  double n_el;           /* electrons / mm3 */
  double density_factor; /* Migdal constant x electron density (MeV^-2 scale) */
  double radlen;         /* radiation length, mm (ProxyMaterial.cu:133-150) */
} gxo_material_t;
void gxo_material_make(double Z, double A, double density, gxo_material_t *m);

/* ------------------------------------------------------ interaction I/O */
/* The model entry points take the primary's kinetic energy and direction and
 * return the updated primary plus up to two secondaries, as the reference's
 * SampleSecondaries(TrackState*) does (source/Geant/proxy/ProxyEmModel.hpp:
 * 79-83).  status: 0 alive, 1 killed. */
typedef struct {
  double E, dir[3], edep;
  int status;
  int nsec;
  int sec_type[2];  /* 0 gamma, 1 e-, 2 e+ */
  double sec_E[2], sec_dir[2][3];
} gxo_inter_t;

enum { GXO_MODE_QUIRK = 0, GXO_MODE_PHYSICS = 1 };
typedef struct {
  int mode;
  int Z;                 /* element (quirk default 10) */
  double cut;            /* production cut, MeV (model specific) */
  double density_factor; /* SB dielectric suppression */
  const gxo_sb_t *sb;    /* SB table used */
  const gxo_data_t *data;
  int charge;            /* -1 e-, +1 e+ for Moller/Bhabha */
} gxo_model_params_t;

void gxo_rotate_to_lab(double *u, double *v, double *w, double u1, double u2, double u3);

int gxo_kn_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io);
int gxo_sg_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io);
int gxo_bh_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io);
int gxo_sb_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io);
int gxo_mb_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io);
int gxo_bhabha_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io);
int gxo_annih_sample(gxo_mrg_t *r, const gxo_model_params_t *p, gxo_inter_t *io);
double gxo_sg_photo_electron_energy(const gxo_data_t *d, int Z, double e, int mode);
double gxo_kn_xs_per_atom(double Z, double e);     /* ProxyKleinNishina.hpp:62-93 */
double gxo_mb_xs_per_atom(double Z, double e);     /* ProxyMollerScattering.hpp:61-89 */
double gxo_annih_xs_per_electron(double e);
double gxo_pe_xs_sandia(const gxo_data_t *d, int Z, double density, double e);
double gxo_coulomb_factor(double Zeff);            /* ProxyEmModel.hpp:114-128 */

/* models: 0 KN, 1 SG, 2 BH, 3 SB, 4 MB, 5 Bhabha, 6 annihilation */
void gxo_interact_batch(int model, const gxo_model_params_t *p, int n, double *states,
                        const double *E, const double *dir, double *E_out, double *dir_out,
                        double *edep, int *status, int *nsec, int *sec_type, double *sec_E,
                        double *sec_dir);

/* ------------------------------------------------------------ processes */
/* ProxyEmProcess<T>::PostStepGPIL, source/Geant/proxy/ProxyEmProcess.hpp:122-151 */
double gxo_post_step_gpil(gxo_mrg_t *r, double lambda_inv, double pstep_prev, double *nil,
                          double *inv_lambda_saved);
/* ProxyIonization::AlongStepGPIL / AlongStepDoIt, ProxyIonization.hpp:108-168 */
double gxo_ioni_along_gpil(const gxo_data_t *d, int mode, int charge, int mat, double e);
void gxo_ioni_along_doit(const gxo_data_t *d, int mode, int charge, int mat, double step,
                         double *e, double *edep);

/* --------------------------------------------------------------- helix */
/* ConstFieldHelixStepper::DoStep, source/Geant/magneticfield/ConstFieldHelixStepper.hpp:164-239 */
void gxo_helix_dostep(const double B[3], const double pos[3], const double dir[3], double charge,
                      double momentum, double step, double newpos[3], double newdir[3]);
/* the same step in mm / MeV / tesla for a field along z (kB2C = -0.299792458) */
void gxo_helix_dostep_mm(double Bz_tesla, const double pos[3], const double dir[3], double charge,
                         double momentum, double step, double newpos[3], double newdir[3]);
void gxo_helix_batch(const double B[3], int n, const double *pos, const double *dir,
                     const double *charge, const double *mom, const double *step, double *newpos,
                     double *newdir);

/* ---------------------------------------------------------- CSG geometry */
/* gxo_geom.c: a volume tree of placed solids, flattened into touchables
 * (transport config geometry = 2). */
enum { GXO_CSG_BOX = 0, GXO_CSG_TUBE = 1, GXO_CSG_SPHERE = 2, GXO_CSG_POLY = 3 };
#define GXO_CSG_TOL 1e-9 /* surface tolerance, mm */
typedef struct {
  int kind;             /* GXO_CSG_* */
  double a, b, c;       /* box: half lengths; tube: rmin, rmax, half length in z; sphere: rmin, rmax */
  double t[3], r[9];    /* global placement: x_global = R x_local + t (R row-major) */
  int rot;              /* 0: R is the identity */
  double lo[3], hi[3];  /* global bounding box, padded */
  int mat, parent, kid0, nkid, score, lv;
  int p0, np;           /* polyhedron: its planes in the plane table */
} gxo_csg_node_t;
typedef struct {
  int n, nscore;        /* touchables; scored ones (numbered depth-first) */
  gxo_csg_node_t *node; /* node 0 is the world */
  int *kids;
  double *planes;       /* polyhedra: unit outward normal and offset per plane */
} gxo_csg_t;
/* solids: kind and 3 parameters each (polyhedra: planes splanes[4 off[s] ..
 * 4 off[s+1]), normal and offset each); logical volumes: solid, material,
 * scored flag; placements: mother and daughter logical volume, translation (3)
 * and rotation (9, row-major; x_mother = R x_daughter + t).  NULL on error. */
gxo_csg_t *gxo_csg_build(int nsolid, const int *skind, const double *spar, const int *splane_off,
                         const double *splanes, int nlv, const int *lv_solid, const int *lv_mat, const int *lv_scored,
                         int npv, const int *pv_mother, const int *pv_lv, const double *pv_t, const double *pv_r,
                         int world);
void gxo_csg_free(gxo_csg_t *g);
int gxo_csg_contains(const gxo_csg_t *g, int v, const double *p, const double *d, double tol);
/* from touchable v (-1 or 0: the world) up until a touchable contains p, then down */
int gxo_csg_locate(const gxo_csg_t *g, int v, const double *p, const double *d, double tol);
/* distance to the next boundary from p in v (children closer than limit are
 * considered); *hit = the child entered, -1 when leaving v */
double gxo_csg_step(const gxo_csg_t *g, int v, const double *p, const double *d, double limit, int *hit);
double gxo_csg_safety(const gxo_csg_t *g, int v, const double *p);
/* the touchable entered at p after gxo_csg_step's crossing */
int gxo_csg_cross(const gxo_csg_t *g, int v, int hit, const double *p, const double *d);
/* batch front end for the tests: locate from the world, step (limit), safety,
 * touchable after the crossing (or the same one when the limit comes first) */
void gxo_csg_probe(const gxo_csg_t *g, int n, const double *pos, const double *dir, const double *limit, int *vol,
                   double *snext, int *next, double *safety);
int gxo_csg_node_count(const gxo_csg_t *g, int *nscore);
/* info: lv, parent, score, material, children; tr: t[3], R[9] */
void gxo_csg_node_info(const gxo_csg_t *g, int i, int *info, double *tr);

/* ------------------------------------------------------------ transport */
typedef struct {
  int geometry;            /* 0: single box of material box_mat; 1: layered calorimeter; 2: csg */
  int axis;                /* layering / box axis (0 x, 1 y, 2 z) */
  int nlayers;
  double t_abs, t_gap;     /* absorber (Pb) and gap (LAr) thickness, mm */
  double half_trans;       /* half transverse size, mm */
  double box_half[3];      /* geometry 0: half sizes; box centred at box_centre */
  double box_centre[3];
  int box_mat;
  double Bz;               /* tesla, along z */
  int charged_local;       /* 1: charged secondaries deposit locally (gamma-only transport) */
  int max_steps;           /* per-track safety cap */
  double seed[6];
  long first_substream;    /* substream index of primary 0 */
  int nthreads;
  int score_events;        /* number of event tallies (>=1) */
  int msc;                 /* 1: multiple scattering of e-/e+ (gxo_transport.c) */
  const float *field_map;  /* non-null: follow this field map (gxo_field_map_load) with RK4, Bz ignored */
  const gxo_csg_t *csg;    /* geometry 2: the volume tree; tallies are [score_events][csg->nscore] */
} gxo_config_t;

typedef struct {
  int type;         /* 0 gamma, 1 e-, 2 e+ */
  double E, pos[3], dir[3];
  int event;
} gxo_primary_t;

typedef struct {
  double *edep;          /* [score_events][nvol] FP64 */
  int nvol;
  double escaped;        /* kinetic energy leaving the world */
  long long steps;       /* track-steps (OneStep iterations) */
  long long substeps;    /* field propagation sub-steps */
  long long tracks;      /* tracks transported (primaries + secondaries) */
  long long secondaries[3];
  long long n_pair, n_annih;
  long long errors;
  int *primary_steps;    /* optional per-primary step count of the primary track */
} gxo_result_t;

int gxo_transport(const gxo_data_t *d, const gxo_config_t *cfg, int nprim,
                  const gxo_primary_t *prims, gxo_result_t *res);
/* flat-array front end for ctypes */
/* Tracks in flat arrays (pos, dir, nil: n x 3; rng: n x 6 state doubles;
 * event, primary, msc optional), status 0 alive. */
typedef struct {
  int n;
  int *type, *status, *event, *primary, *volume;
  double *pos, *dir, *ekin, *nil, *msc, *rng;
} gxo_tracks_t;
int gxo_step_tracks(const gxo_data_t *d, const gxo_config_t *cfg, gxo_tracks_t *t, gxo_tracks_t *sec,
                    double *edep, int nvol, double *escaped, long long *counters);
int gxo_transport_tracks(const gxo_data_t *d, const gxo_config_t *cfg, const gxo_tracks_t *t, double *edep, int nvol,
                         double *escaped, long long *counters);
int gxo_transport_flat(const gxo_data_t *d, const gxo_config_t *cfg, int nprim,
                       const int *type, const double *E, const double *pos, const double *dir,
                       const int *event, double *edep, int nvol, double *escaped,
                       long long *counters, int *primary_steps);

/* multiple scattering (gxo_transport.c), test front ends */
void gxo_msc_cos_batch(double Z, double X0, int n, double *states, double t, double lam0, double lam1, double e0,
                       double e1, double *out);
double gxo_msc_lambda1(const gxo_data_t *d, int type, int mat, double e);
double gxo_msc_true_to_geom(double t, double lam);
double gxo_msc_geom_to_true(double z, double lam, double tmax);

/* field map in the reference's CMS format (gxo_field.c): ScalarCMSmagField,
 * examples/magneticfield/simplifiedCMS/inc/Geant/ScalarCMSmagField.h:162-331.
 * load: 181 x 161 x 4 floats (Br, Bphi, Bz premultiplied by 1/(dr dz), pad),
 * NULL on error; value: tesla at pos (mm). */
float *gxo_field_map_load(const char *path);
void gxo_field_map_free(float *map);
void gxo_field_map_value(const float *map, const double pos[3], double B[3]);
void gxo_field_map_batch(const float *map, int n, const double *pos, double *B);

/* production-cut conversion (gxo_cuts.c): CutConverter, cuts/src/CutConverter*.cpp */
double gxo_cut_convert(int particle, int nelem, const double *Z, const double *n_atoms, double density, double cut,
                       int from_length);

/* ------------------------------------------------------ event generators */
/* gxo_events.c: ProxyEgammaGun (proxy/src/ProxyEgammaGun.cpp:35-85) and
 * ProxyHepEvtGenerator (proxy/src/ProxyHepEvtGenerator.cpp:48-132). */
int gxo_egamma_gun(gxo_mrg_t *r, int nevents, int nparticles, double gamma_fraction, double minp, double maxp,
                   double mineta, double maxeta, double minphi, double maxphi, int *pdg, double *p, double *ekin,
                   double *dir);
/* the library's beam-spot gun (gx_spot_gun), restated */
int gxo_spot_gun(const double seed[6], long stream, long first, int n, int ntypes, const int *types, double emin,
                 double emax, double cone_deg, int axis, const double centre[3], const double half[2], int *type,
                 double *E, double *pos, double *dir);
void gxo_egamma_dir(int physics, double x, double y, double z, double *eta, double *phi);
int gxo_hepevt_read(const char *path, int physics, int max_events, int cap, int *event, int *pdg, double *p,
                    double *ekin, double *dir, int *nev_read, int *bad);

#ifdef __cplusplus
}
#endif
#endif
