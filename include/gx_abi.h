/*
 * gx_abi.h -- C ABI of the B200-native EM particle-transport step path.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (GX_OK = 0, negative on error; gx_last_error_string() explains)
 * and never throws.  Pointers named d_* are device pointers; calls that take a
 * cudaStream_t are asynchronous on that stream.  The caller owns all buffers
 * it passes in (as the reference's ProxyDeviceManager does,
 * source/Geant/proxy/src/ProxyDeviceManager.cpp:100-204).
 *
 * Units: mm, MeV, ns (the reference's CLHEP units,
 * source/Geant/proxy/ProxySystemOfUnits.hpp); field in tesla.
 *
 * MRG32k3a states are six uint32 words per stream, stored as six planes of n
 * words (word k of stream i at index k * n + i).  The words are the six
 * integers the reference keeps as doubles (MRG32k3a.hpp:45-49).
 */
#ifndef GX_ABI_H
#define GX_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *gx_stream_t; /* a cudaStream_t */

enum {
  GX_OK = 0,
  GX_ERR_ARG = -1,      /* bad argument */
  GX_ERR_CUDA = -2,     /* a CUDA call failed */
  GX_ERR_DATA = -3,     /* physics data missing or malformed */
  GX_ERR_OVERFLOW = -4, /* a track store or stack ran out of room */
  GX_ERR_ITERCAP = -5,  /* an iteration cap was hit (tracks retired, see stats) */
  GX_ERR_NODEVICE = -6  /* no CUDA device */
};

/* physics-table ids, source/Geant/proxy/ProxyPhysicsTableIndex.hpp:23-45 */
enum {
  GX_DEDX_eBrem_em, GX_DEDX_eBrem_ep, GX_DEDX_eIoni_em, GX_DEDX_eIoni_ep,
  GX_InverseRange_em, GX_InverseRange_ep, GX_Ionisation_em, GX_Ionisation_ep,
  GX_Lambda_compt, GX_Lambda_conv, GX_Lambda_eBrem_em, GX_Lambda_eBrem_ep,
  GX_Lambda_eIoni_em, GX_Lambda_eIoni_ep, GX_LambdaMod1_msc_em, GX_LambdaMod1_msc_ep,
  GX_LambdaPrim_compt, GX_LambdaPrim_phot, GX_Range_em, GX_Range_ep,
  GX_NTABLES
};

/* interaction models (the reference's ProxyEmModel family, plus the two e+
 * models it lacks) */
enum { GX_KLEIN_NISHINA, GX_SAUTER_GAVRILA, GX_BETHE_HEITLER, GX_SELTZER_BERGER, GX_MOLLER,
       GX_BHABHA, GX_ANNIHILATION };
/* processes for gx_post_step_gpil, source/Geant/proxy/ProxyProcessIndex.cuh:23-41 */
enum { GX_PROC_COMPTON, GX_PROC_CONVERSION, GX_PROC_PHOTOELECTRIC, GX_PROC_BREMSSTRAHLUNG,
       GX_PROC_IONIZATION };
enum { GX_MODE_QUIRK = 0, GX_MODE_PHYSICS = 1 };

typedef struct gx_ctx gx_ctx;

/* ------------------------------------------------------------- context */
const char *gx_last_error_string(void);
int gx_version(void);
/* Loads the Geant4-format ASCII tables, cut table, Seltzer-Berger and shell
 * data from datadir and relocates them to the device.  Replaces
 * ProxyDataManager::ProxyDataManager + RetrievePhysicsData + RetrieveCutsTable
 * + RelocatePhysicsData (source/Geant/proxy/src/ProxyDataManager.cu:27-163). */
int gx_ctx_create(const char *datadir, int device, gx_ctx **out);
int gx_ctx_destroy(gx_ctx *ctx);

/* --------------------------------------------------------------- RNG */
/* Streams i = 0..n-1 start at substream (first + i) of the stream whose first
 * state is seed: seed * A^((first + i) 2^76), computed on the device by
 * skip-ahead.  Equivalent to (first + i) calls of MRG32k3a::AdvanceState(76, 0)
 * (source/Geant/random/src/MRG32k3a.cpp:167-178). */
int gx_rng_substreams(const double seed[6], long long first, int n, uint32_t *d_states, gx_stream_t s);
/* MRG32k3a::AdvanceState(e, c) applied to every stream (MRG32k3a.cpp:167-205). */
int gx_rng_advance(uint32_t *d_states, int n, long long e, long long c, gx_stream_t s);
/* k draws per stream, out[j * n + i]: RNG<MRG32k3a>::Uniform(State_t*)
 * (source/Geant/random/RNG.hpp:67-70, MRG32k3a.cpp:124-163). */
int gx_rng_uniform(uint32_t *d_states, int n, int k, double *d_out, gx_stream_t s);
/* MRG32k3a::Initialize(long streamId) (MRG32k3a.cpp:69-82), one state per id. */
int gx_rng_stream_id(const long long *h_ids, int n, uint32_t *d_states, gx_stream_t s);

/* ------------------------------------------------------------- tables */
/* ProxyPhysicsTable::Value(mat, E) (ProxyPhysicsTable.cu:121-125 ->
 * ProxyPhysicsVector::Value, ProxyPhysicsVector.cu:469-483), FP64. */
int gx_table_value(gx_ctx *ctx, int table, int mat, const double *d_E, double *d_out, int n, gx_stream_t s);
/* ProxyPhysicsVector::InvRangeValue (ProxyPhysicsVector.cu:491-524). */
int gx_table_invrange(gx_ctx *ctx, int table, int mat, const double *d_r, double *d_out, int n, gx_stream_t s);
/* Proxy2DVector::Value (Proxy2DVector.cpp:37-67) on Seltzer-Berger table
 * which: 0 = br11 (the reference's hard-coded slot 10), 1 = br18, 2 = br82. */
int gx_sb_value(gx_ctx *ctx, int which, const double *d_x, const double *d_y, double *d_out, int n,
                gx_stream_t s);
/* Loads a field map in the format of the reference's CMS map
 * (examples/magneticfield/simplifiedCMS/cmsmagfield2015.txt: lines
 * "R(mm)= r phi(deg)= p Z(mm)= z Bz(tesla)= . Br(tesla)= . Bphi(tesla)= .",
 * 181 x 161 (r, z) points, r outer, dr = 50 mm, dz = 200 mm, |z| <= 16 m) as
 * ScalarCMSmagField::ReadVectorData reads it (ScalarCMSmagField.h:162-199);
 * other lattices are rejected.  Used by transports with cfg.field_map = 1. */
int gx_ctx_load_field_map(gx_ctx *ctx, const char *path);
/* The map's field (tesla) at n points (mm, xyz interleaved):
 * ScalarCMSmagField::GetFieldValue (ScalarCMSmagField.h:207-331). */
int gx_field_value(gx_ctx *ctx, int n, const double *d_pos, double *d_B, gx_stream_t s);
/* ProxyDataManager::GetCutValue(index, ipart) (ProxyDataManager.cuh:52-54), host. */
int gx_cut_value(gx_ctx *ctx, int index, int ipart, double *out);
/* The production-cut converter of the reference, CutConverter::Convert
 * (source/Geant/cuts/src/CutConverter.cpp:107-128, with
 * CutConverterForGamma/Electron/Positron and Spline; 301 energies from 990 eV
 * to 10 GeV as MaterialCuts.cpp:88-93 sets it), on the host: particle 0 gamma,
 * 1 e-, 2 e+; a material of nelem elements Z with n_atoms per mm^3 and
 * density in g/cm^3; from_length 1: *out = energy (MeV) of a cut given as a
 * length (mm); 0: the length (mm) of a cut given as an energy (MeV). */
int gx_cut_convert(int particle, int nelem, const double *Z, const double *n_atoms, double density, double cut,
                   int from_length, double *out);
/* Replaces the context's cut table (read from cut.dat, the Geant4 dump) by one
 * computed with gx_cut_convert for a range cut of cut_mm in every material
 * (protons: 100 keV per mm, Geant4's rule; the reference has no proton
 * converter), and uploads it: the models' thresholds follow from then on. */
int gx_ctx_compute_cuts(gx_ctx *ctx, double cut_mm);

/* Macroscopic cross sections built on the device from the models' cross
 * sections instead of read from the Geant4 tables (the reference evaluates
 * ProxyEmModel::MacroscopicCrossSection, proxy/ProxyEmModel.hpp:57-76, and
 * ships the tables): d_out[i] for table id `table` of material mat (1 Pb,
 * 2 LAr) at energies d_E[i]: GX_Lambda_compt and GX_LambdaPrim_compt (Klein-
 * Nishina, ProxyKleinNishina.hpp:62-93), GX_Lambda_eIoni_em (Moller with the
 * material's e- cut, ProxyMollerScattering.hpp:61-89), GX_Lambda_eIoni_ep
 * (Bhabha, integrated from the cut), GX_Lambda_eBrem_em (Seltzer-Berger
 * tables integrated from the gamma cut, with dielectric suppression),
 * GX_Lambda_eBrem_ep (the same with the positron Coulomb factor
 * exp(2 pi alpha Z (1/beta1 - 1/beta2))), GX_Lambda_conv (Bethe-Heitler with
 * the sampler's screening functions and Tsai's xi(Z) for the atomic
 * electrons), GX_LambdaPrim_phot (E x the Sandia photo-absorption cross
 * section), GX_DEDX_eIoni_em/ep (Berger-Seltzer restricted collision stopping
 * power with the Sternheimer-Peierls density effect), GX_DEDX_eBrem_em/ep
 * (Seltzer-Berger radiative loss below the gamma cut). */
int gx_table_build(gx_ctx *ctx, int table, int mat, const double *d_E, double *d_out, int n, gx_stream_t s);
/* Replaces the node values of those tables with the built ones where their
 * models hold (brems up to 1 GeV, pairs from 4 MeV to 100 GeV, stopping powers
 * above 10 keV) and refits their splines, then rebuilds Range and
 * InverseRange (e-, e+) as the range integral of the rebuilt losses;
 * *max_rel_change (optional) receives the largest relative change of a table
 * value above 10 keV.  Synchronous. */
int gx_ctx_rebuild_tables(gx_ctx *ctx, double *max_rel_change);

/* ------------------------------------------------------------- models */
typedef struct {
  int mode;              /* GX_MODE_QUIRK: the reference's hard-coded values; GX_MODE_PHYSICS */
  int Z;                 /* element for physics mode */
  double cut;            /* production cut (MeV) for SB, Moller, Bhabha in physics mode */
  double density_factor; /* SB dielectric suppression factor */
  int sb_table;          /* 0 br11, 1 br18, 2 br82 */
} gx_model_params;

/* A batch of ProxyEmModel<T>::SampleSecondaries(TrackState*) calls
 * (source/Geant/proxy/ProxyEmModel.hpp:79-83; ProxyKleinNishina.hpp:96-166,
 * ProxySauterGavrila.hpp:67-130, ProxyBetheHeitler.hpp:64-182,
 * ProxySeltzerBerger.hpp:204-286, ProxyMollerScattering.hpp:92-159).
 * Track i has kinetic energy d_E[i], direction d_dir[3i..3i+2] and stream i
 * of d_rng; outputs: updated energy / direction / deposit / status (1 killed),
 * number of secondaries and up to two secondaries (type 0 gamma, 1 e-, 2 e+;
 * energies d_sec_E[2i+k], directions d_sec_dir[6i+3k..]).  The reference
 * builds its secondaries and drops them; these are returned. */
int gx_interact(gx_ctx *ctx, int model, const gx_model_params *p, int n, uint32_t *d_rng, const double *d_E,
                const double *d_dir, double *d_E_out, double *d_dir_out, double *d_edep, int *d_status,
                int *d_nsec, int *d_sec_type, double *d_sec_E, double *d_sec_dir, gx_stream_t s);
/* CrossSectionPerAtom(Z, E) of Klein-Nishina (ProxyKleinNishina.hpp:62-93) or
 * Moller (ProxyMollerScattering.hpp:61-89), mm^2. */
int gx_xs_per_atom(int model, double Z, const double *d_E, double *d_out, int n, gx_stream_t s);

/* ---------------------------------------------------------- processes */
/* ProxyEmProcess<T>::PostStepGPIL (ProxyEmProcess.hpp:122-151) for a batch:
 * reads lambda from the process's table at material mat (the reference
 * forces mat = 2 at :133), updates NIL d_nil and the saved 1/lambda d_saved,
 * returns the proposed step. */
int gx_post_step_gpil(gx_ctx *ctx, int process, int mat, int n, uint32_t *d_rng, const double *d_E,
                      const double *d_pstep_prev, double *d_nil, double *d_saved, double *d_step,
                      gx_stream_t s);
/* ProxyIonization::AlongStepGPIL (ProxyIonization.hpp:108-128). */
int gx_ioni_along_gpil(gx_ctx *ctx, int mode, int charge, const int *d_mat, const double *d_E, double *d_out,
                       int n, gx_stream_t s);
/* ProxyIonization::AlongStepDoIt (ProxyIonization.hpp:130-168): d_E updated, d_edep added to. */
int gx_ioni_along_doit(gx_ctx *ctx, int mode, int charge, const int *d_mat, const double *d_step, double *d_E,
                       double *d_edep, int n, gx_stream_t s);

/* ------------------------------------------------ elementary functions */
/* The elementary functions of the FP64 parity variant of the transport
 * (gx_math.h: log, exp, pow, sin, cos, expm1, log1p from published methods,
 * contraction-free, identical on the GPU and the CPU), or with lib = 1 CUDA's
 * own, at n device arguments: fn 0 log, 1 exp, 2 pow(x, y), 3 sin, 4 cos,
 * 5 expm1, 6 log1p.  No counterpart in the reference, whose std:: / VecCore
 * math these stand in for; for testing the parity build. */
int gx_math_eval(int fn, int lib, int n, const double *d_x, const double *d_y, double *d_out, gx_stream_t s);

/* -------------------------------------------------------------- helix */
/* ConstFieldHelixStepper::DoStepArr (ConstFieldHelixStepper.hpp:249-302):
 * SoA inputs and outputs; kB2C is the reference's -0.299792458e-3 for
 * GeV / kilogauss / cm, or -0.299792458 for MeV / tesla / mm. */
int gx_helix_dostep(const double B[3], double kB2C, int n, const double *d_posx, const double *d_posy,
                    const double *d_posz, const double *d_dirx, const double *d_diry, const double *d_dirz,
                    const double *d_charge, const double *d_momentum, const double *d_step, double *d_newposx,
                    double *d_newposy, double *d_newposz, double *d_newdirx, double *d_newdiry,
                    double *d_newdirz, gx_stream_t s);

/* ------------------------------------------------------- CSG geometry */
/* A volume tree for transport geometry 2, built with the calls a VecGeom
 * detector construction makes (the reference navigates VecGeom,
 * geometry/NavigationInterface.hpp:63-98, over a tree built in
 * proxy/test/BasicCpuTransport/ProxyDetectorConstruction.cpp:241-324):
 *   new UnplacedBox(hx, hy, hz)             -> gx_geom_box
 *   new UnplacedTube(rmin, rmax, dz, 0, 2pi) -> gx_geom_tube (a phi segment: gx_geom_tube_segment)
 *   new UnplacedSphere / UnplacedOrb (full)  -> gx_geom_sphere
 *   new UnplacedTrd(x1, x2, y1, y2, z) etc.  -> gx_geom_polyhedron (its planes)
 *   new LogicalVolume(name, solid) + SetMaterialPtr -> gx_geom_logical_volume
 *   lv->PlaceDaughter(name, daughter, new Transformation3D(...))
 *                                            -> gx_geom_place_daughter
 *   GeoManager::SetWorld + CloseGeometry     -> gx_geom_close
 * Lengths in mm; materials 0 Galactic, 1 Pb, 2 LAr (the context's tables).
 * A placement puts a daughter point x at R x + t in its mother (R row-major,
 * NULL: identity).  Closing unrolls the tree into touchables (one per placed
 * instance, depth-first, the world first); the touchables of logical volumes
 * created with scored != 0 get consecutive tally columns in that order
 * (*nscore of them: pass that as nvol to gx_transport_run).  Solid ids,
 * logical volume ids and placement ids count from 0 in creation order. */
typedef struct gx_geom gx_geom;
int gx_geom_create(gx_geom **out);
void gx_geom_destroy(gx_geom *g);
int gx_geom_box(gx_geom *g, double hx, double hy, double hz, int *solid);
int gx_geom_tube(gx_geom *g, double rmin, double rmax, double dz, int *solid);
/* new UnplacedTube(rmin, rmax, dz, sphi, dphi): the tube between the
 * half-planes at phi = sphi and sphi + dphi (radians, 0 < dphi; 2 pi or more
 * is the full tube) */
int gx_geom_tube_segment(gx_geom *g, double rmin, double rmax, double dz, double sphi, double dphi, int *solid);
int gx_geom_sphere(gx_geom *g, double rmin, double rmax, int *solid);
/* A convex polyhedron {x : n_k . x <= d_k, k < nplanes} (4 to 32 planes,
 * planes[4k .. 4k+3] = outward normal n_k, any length, and offset d_k, in the
 * same length scale): VecGeom's UnplacedTrd / UnplacedTrapezoid /
 * UnplacedParallelepiped and the like are such intersections.  Rejected when
 * the planes bound no finite volume. */
int gx_geom_polyhedron(gx_geom *g, int nplanes, const double *planes, int *solid);
int gx_geom_logical_volume(gx_geom *g, int solid, int material, int scored, int *lv);
int gx_geom_place_daughter(gx_geom *g, int mother, int daughter, const double translation[3],
                           const double rotation[9], int *pv);
int gx_geom_close(gx_geom *g, int world, int *ntouchables, int *nscore);
/* a touchable of a closed tree: its logical volume, parent touchable (-1 for
 * the world), tally column (-1: not scored) and global transform */
int gx_geom_touchable(const gx_geom *g, int i, int *lv, int *parent, int *score, double translation[3],
                      double rotation[9]);
/* upload a closed tree into the context (replacing the previous one) */
int gx_ctx_load_geometry(gx_ctx *ctx, const gx_geom *g);
/* Navigation probe, one thread per point (device arrays; pos and dir n x 3):
 * the touchable containing the point (-1 outside the world), the distance to
 * the next boundary along dir (children are considered up to limit; -1
 * outside), the touchable entered there (the same one when limit comes
 * first) and the isotropic safety. */
int gx_geom_probe(gx_ctx *ctx, int n, const double *d_pos, const double *d_dir, const double *d_limit, int *d_vol,
                  double *d_snext, int *d_next, double *d_safety, gx_stream_t s);

/* ---------------------------------------------------------- transport */
typedef struct {
  int geometry;            /* 0: one box of material box_mat; 1: layered calorimeter; 2: the context's
                              CSG tree (gx_ctx_load_geometry; axis, nlayers, t_abs, t_gap, half_trans
                              and box_* are ignored) */
  int axis;                /* layering (or box) axis: 0 x, 1 y, 2 z */
  int nlayers;
  double t_abs, t_gap;     /* absorber (Pb) and gap (LAr) thickness, mm */
  double half_trans;       /* calorimeter half transverse size, mm */
  double box_half[3], box_centre[3];
  int box_mat;             /* 1 Pb, 2 LAr */
  double Bz;               /* tesla, along z */
  int charged_local;       /* 1: e-/e+ secondaries deposit their kinetic energy locally */
  int max_steps;           /* per-track step cap (retired with an error count above it) */
  double seed[6];
  long long first_substream;
  int nevents;             /* tally rows */
  /* engine */
  int precision;           /* 0 FP64, 1 FP32-mixed */
  int engine;              /* 0 plain loop (one mixed queue, host-driven), 1 batched (per-type queues, graph) */
  int block_size;          /* threads per block (0: default); above 256 (up to 1024) only for the batched
                              engine with the uniform field, layered geometry and no multiple scattering */
  int blocks_per_sm;       /* resident blocks per SM for the grid (0: default, 5 for the FP32-mixed
                              batched engine, 4 otherwise) */
  long long capacity;      /* track slots per particle type (0: default) */
  long long refill_below;  /* inject / refill when fewer tracks than this are in flight (0: default) */
  int graph_iters;         /* iterations per CUDA-graph launch between host checks (0: default) */
  int profile;             /* 1: no graph; CUDA events around every step kernel (per-kernel times in stats) */
  double wave_energy;      /* energy (MeV) carried by live tracks before more primaries are injected,
                              at most (0: from capacity) */
  int steps_per_launch;    /* batched engine: steps of one track per transport launch, at most; a track
                              stays in registers between them (0: default 16; 1: one step per iteration) */
  int msc;                 /* 1: multiple scattering of e-/e+ (Urban-type: safety-based step limit, true /
                              geometric path conversion, angular deflection); 2: the same with lateral
                              displacement (within the safety); 0: off (the reference has none,
                              proxy/ProxyScattering.hpp:53-71) */
  int field_map;           /* 1: the context's field map (gx_ctx_load_field_map) with fourth-order
                              Runge-Kutta sub-steps, Bz ignored; 0: uniform Bz with the helix */
  int steps_per_launch_by_type[3]; /* batched engine: steps per transport launch for gamma, e-, e+
                              (0: from steps_per_launch; e+ a quarter of it, at least 1) */
  int interaction_interval; /* batched engine: the compaction interval -- tracks that reach an interaction wait
                              in their per-process buffers and the interaction kernels, which compact their
                              survivors and secondaries back into the stores, run every this many iterations
                              (0 or 1: every iteration).  Results do not depend on it. */
  int fp64_parity;         /* 1 (precision 0 only): the FP64 parity variant -- no contraction, the reference's
                              spline and ionisation forms, the general helix step and the elementary functions
                              of gx_math.h, the operations of the CPU oracle in its order, so that the two
                              agree track by track; 0: the library's FP64 kernels */
  int fetch_min_by_type[3]; /* batched engine: a warp of the transport kernel of gamma, e-, e+ takes new
                              records from its store only once at least this many of its 32 lanes are
                              idle (or all are): the record loads, NIL draws and cross sections of new
                              tracks then run for several lanes at once instead of one or two in every
                              pass (0: the defaults -- 12 for the photons of the FP32-mixed engine in
                              the layered geometry, 1 for the rest; 1 to 32).  Results do not depend
                              on it. */
} gx_transport_config;

typedef struct {
  long long steps, substeps, tracks;
  long long secondaries[3];
  long long n_pair, n_annih, errors;
  double escaped;
  long long iterations;
  long long peak_in_flight;
  double kernel_ms;        /* device time of the whole transport loop, CUDA events */
  /* per step kernel (gamma, e-, e+; the plain engine uses entry 0): */
  double step_ms[3];       /* summed device time (profile mode only) */
  long long step_launches[3];
  long long tracks_read[3];    /* track records read */
  long long tracks_written[3]; /* track records written (survivors and secondaries) */
  long long bytes_per_track;   /* size of one track record in the stores */
  /* the transport kernel of each type alone (batched engine; times in profile mode only): */
  double transport_ms[3];
  long long transport_read[3];    /* track records read */
  long long transport_written[3]; /* records written: survivors and interacting tracks */
  long long transport_queued[3];  /* of those, records written to the interaction buffers */
  long long transport_steps[3];   /* steps completed in the transport kernel */
} gx_transport_stats;

void gx_transport_config_default(gx_transport_config *cfg);
/* Transports nprim primaries (device arrays: type 0 gamma / 1 e- / 2 e+,
 * kinetic energy, position xyz, direction xyz, event index) to completion and
 * adds their energy deposits to d_edep[event * nvol + volume] (FP64).
 * Replaces the reference's DoStep / OneStep / InnerStep loop
 * (source/Geant/proxy/test/test_BasicCpuTransport.cpp:358-550) and its
 * device-side launch wrappers (source/Geant/kernel/KernelPhysicsProcess.cuh:22-36).
 * d_primary_steps (optional) receives the step count of each primary track. */
int gx_transport_run(gx_ctx *ctx, const gx_transport_config *cfg, int nprim, const int *d_type,
                     const double *d_E, const double *d_pos, const double *d_dir, const int *d_event,
                     double *d_edep, int nvol, int *d_primary_steps, gx_transport_stats *stats, gx_stream_t s);
/* The same from host buffers: copies the primaries in and the tallies out
 * inside the call (h_edep is overwritten).  The context keeps the stream and
 * the device staging buffer of these calls (grown when a call needs more), so
 * a call allocates nothing once the context has seen its size.  Synchronous. */
int gx_transport_run_host(gx_ctx *ctx, const gx_transport_config *cfg, int nprim, const int *h_type,
                          const double *h_E, const double *h_pos, const double *h_dir, const int *h_event,
                          double *h_edep, int nvol, int *h_primary_steps, gx_transport_stats *stats);

/* ------------------------------------------------- primary generation */
/* The e/gamma particle gun of the reference, ProxyEgammaGun
 * (source/Geant/proxy/ProxyEgammaGun.hpp:35-82, src/ProxyEgammaGun.cpp:43-85),
 * writing transport primaries straight into device arrays.  Particle
 * i = event x nparticles + j draws four uniforms from one MRG32k3a stream
 * (the stream whose state is seed, after first_draw draws), in the
 * reference's order: type (gamma below gamma_fraction, else e-), momentum
 * uniform in [min_p, max_p] (MeV), eta, phi uniform in their ranges; kinetic
 * energy p^2 / (sqrt(p^2 + m^2) + m), direction from eta and phi.  The
 * output equals the reference's sequential output for the same stream state
 * (the reference's ProxyRandom starts at the default seed, 12345 x 6).
 * Position = vertex (the reference leaves it at the origin); d_event[i] =
 * first_event + event; d_pdg (optional) gets 22 / 11.  Draws consumed:
 * 4 x nevents x nparticles. */
typedef struct {
  int nevents, nparticles;  /* particles per event */
  double gamma_fraction;    /* reference default 0.5 */
  double min_p, max_p;      /* MeV; reference default 1 GeV .. 1 TeV */
  double min_eta, max_eta;  /* reference default -3 .. 3 */
  double min_phi, max_phi;  /* reference default 0 .. 2 pi */
  double vertex[3];         /* mm */
  double seed[6];           /* MRG32k3a stream state */
  long long first_draw;     /* draws of that stream already used */
  int first_event;
} gx_egamma_gun_params;
int gx_egamma_gun(const gx_egamma_gun_params *p, int *d_type, double *d_E, double *d_pos, double *d_dir,
                  int *d_event, int *d_pdg, gx_stream_t s);
/* Beam-spot gun of the throughput workloads (C4: 2^16 e-/e+/gamma,
 * log-uniform 10 MeV - 100 GeV, 5 degree cone, 2 x 2 cm spot; C5's
 * directions): its own MRG32k3a stream, stream `stream` of the run seed
 * (streams 2^127 draws apart; C4 uses stream 1), separate from the transport
 * substreams of the same seed.  Primary i (counted from 0 over all calls;
 * first = index of the first one written) takes draws 5i .. 5i+4: u0 the
 * kinetic energy emin (emax / emin)^u0, u1 cos theta = 1 - u1 (1 - cos cone),
 * u2 phi = 2 pi u2 (direction about +axis; the transverse axes in cyclic
 * order), u3, u4 the start centre +- half[k] (2u - 1) in the two transverse
 * coordinates; type = types[i % ntypes] (0 gamma, 1 e-, 2 e+).  The device
 * version jumps each thread to its first draw; the host version draws in
 * sequence; both write the same primaries. */
typedef struct {
  double seed[6];           /* run seed (MRG32k3a state) */
  long long stream;         /* stream of the seed the gun draws from (>= 0) */
  long long first;          /* index of the first primary written */
  int ntypes, types[3];
  double emin, emax;        /* MeV, emin <= emax */
  double cone_deg;          /* half angle of the direction cone, degrees */
  int axis;                 /* beam axis 0 x, 1 y, 2 z */
  double centre[3];         /* spot centre, mm */
  double half[2];           /* spot half widths along the two transverse axes, mm */
} gx_spot_gun_params;
int gx_spot_gun(const gx_spot_gun_params *p, long long n, int *d_type, double *d_E, double *d_pos, double *d_dir,
                gx_stream_t s);
int gx_spot_gun_host(const gx_spot_gun_params *p, long long n, int *type, double *E, double *pos, double *dir);
/* Particle type of the transport (0 gamma, 1 e-, 2 e+) for a PDG code, -1 for
 * the particles the EM path does not transport. */
int gx_pdg_to_type(int pdg);
/* ProxyHepEvtGenerator::GenerateOneEvent (source/Geant/proxy/src/
 * ProxyHepEvtGenerator.cpp:48-132) for up to max_events events of a HEPEVT
 * ASCII file, on the host: per event NHEP, then NHEP lines "ISTHEP IDHEP
 * JDAHEP1 JDAHEP2 PX PY PZ M" (GeV).  The primaries are the daughters (of an
 * entry with daughters, status > 0) that have no daughters, in file order;
 * per primary: event index, PDG code, kinetic energy, unit direction.
 * GX_MODE_QUIRK reproduces the reference (mass squared, GeV numbers kept as
 * MeV); GX_MODE_PHYSICS uses the mass as given and converts GeV to MeV.
 * Daughter indices outside their event are skipped and counted in *bad (the
 * reference reads out of bounds there).  *n_out = primaries found; if that
 * exceeds cap, the first cap are stored and GX_ERR_OVERFLOW is returned.
 * A truncated event ends the read with GX_ERR_DATA. */
int gx_hepevt_read(const char *path, int mode, int max_events, int cap, int *h_event, int *h_pdg, double *h_E,
                   double *h_dir, int *n_out, int *nev_out, int *bad_out);
/* gx_hepevt_read, then the gamma / e- / e+ primaries into device arrays ready
 * for gx_transport_run (position = vertex, or the origin if null; other
 * particles are counted in *n_skipped).  Synchronises the stream. */
int gx_hepevt_load(const char *path, int mode, int max_events, const double vertex[3], int cap, int *d_type,
                   double *d_E, double *d_pos, double *d_dir, int *d_event, int *n_prim, int *n_events,
                   int *n_skipped, gx_stream_t s);

/* ------------------------------------------------- tracks in SoA form */
/* A batch of tracks: the hot fields of the reference's TrackState
 * (source/Geant/track/TrackState.hpp:30-232) as the arrays of a
 * TrackCollection (source/Geant/track/TrackCollection.hpp:23-42), one entry
 * per track in every array.  All arrays are device arrays of `capacity`
 * entries owned by the caller; entries 0 .. n-1 are tracks.  Units mm, MeV.
 * The fields, with the TrackState member each stands for:
 *   type          particle: 0 gamma, 1 e-, 2 e+ (fPhysicsState.fParticleType)
 *   status        GX_TRACK_* (fStatus)
 *   event         event index, a row of the tally (fHistoryState.fEvent)
 *   primary       index of the primary this track is, -1 for a secondary
 *                 (fHistoryState.fPrimaryIndx)
 *   volume        volume holding the track (layered calorimeter: 2 layer +
 *                 slab; box: 0; CSG tree: the touchable), -1 outside, < -1
 *                 "locate it" (fGeometryState.fPath)
 *   next_volume   volume after the step (fGeometryState.fNextpath)
 *   process       discrete process that limits the step, -1 none
 *                 (fPhysicsState.fProcess): gamma 0 Compton, 1 conversion,
 *                 2 photo-electric; e-/e+ 0 ionisation, 1 brems, e+
 *                 2 annihilation
 *   boundary      1 when the step ends on a boundary (fGeometryState.fBoundary)
 *   x, y, z       position (fPos)          dx, dy, dz  unit direction (fDir)
 *   ekin          kinetic energy (fPhysicsState.fEkin)
 *   nil0..2       number of interaction lengths left of each discrete process,
 *                 <= 0: draw a new one (fPhysicsProcessState[i].fNumOfInteractLengthLeft)
 *   lambda_inv0..2  its macroscopic cross section at the step start, 1/mm
 *                 (fPhysicsProcessState[i].fMacroscopicCrossSection)
 *   pstep         proposed physics step (fPhysicsState.fPstep)
 *   step          length of the last step taken (fStep)
 *   snext         distance to the next boundary along the direction, up to
 *                 pstep (fGeometryState.fSnext)
 *   safety        isotropic safety (fGeometryState.fSafety)
 *   msc_range     multiple scattering: range scale of the step limit in the
 *                 current volume, <= 0 unset (no TrackState member: the
 *                 reference has no multiple scattering)
 *   rng           MRG32k3a state, six planes of `capacity` words (the
 *                 reference keeps one generator per thread) */
enum { GX_TRACK_ALIVE = 0, GX_TRACK_KILLED = 1, GX_TRACK_INTERACT = 2, GX_TRACK_EXITED = 3 };
typedef struct {
  int n, capacity;
  int *type, *status, *event, *primary, *volume, *next_volume, *process, *boundary;
  double *x, *y, *z, *dx, *dy, *dz, *ekin;
  double *nil0, *nil1, *nil2, *lambda_inv0, *lambda_inv1, *lambda_inv2;
  double *pstep, *step, *snext, *safety, *msc_range;
  uint32_t *rng;
} gx_track_soa;

/* The four stages of one step of the reference's OneStep / InnerStep
 * (source/Geant/proxy/test/test_BasicCpuTransport.cpp:358-497), one thread per
 * track, for the tracks of `tracks` with status GX_TRACK_ALIVE (gx_post_step:
 * GX_TRACK_INTERACT), in FP64 (cfg->fp64_parity selects the parity variant).
 * cfg gives the geometry, field and physics options; multiple scattering
 * (cfg->msc) is not offered stage by stage (use gx_transport_tracks).
 *   gx_gpil        PostStepGPIL of every discrete process (NIL drawn when
 *                  <= 0; ProxyEmProcess.hpp:122-151), the ionisation range
 *                  limit (ProxyIonization.hpp:108-128), FindNextBoundary
 *                  (geometry/NavigationInterface.hpp:63-98): writes
 *                  lambda_inv*, nil*, pstep, process, snext, safety.
 *   gx_propagate   LinearPropagationHandler / FieldPropagationHandler::
 *                  Propagate (core/src/LinearPropagationHandler.cpp:12-56,
 *                  magneticfield/src/FieldPropagationHandler.cpp:87-360): moves
 *                  the track by pstep or to the first boundary; writes x..dz,
 *                  step, boundary, next_volume.
 *   gx_along_step  NIL update by step x lambda_inv, ProxyIonization::
 *                  AlongStepDoIt (ProxyIonization.hpp:130-168) scored into
 *                  d_edep[event * nvol + volume], then the outcome: status
 *                  KILLED (stopped, or left the world: EXITED, energy kept in
 *                  ekin), INTERACT (process set; a stopped e+ annihilates at
 *                  rest, process 2) or ALIVE (volume = next_volume).
 *   gx_post_step   PostStepDoIt (ProxyEmProcess.hpp:153-163): NIL of the
 *                  process reset and its model sampled; the track is updated in
 *                  place (KILLED when absorbed), its secondaries are written to
 *                  `secondaries` at entries 2i and 2i+1 (status ALIVE, fresh
 *                  NIL, streams seeded from the parent's; unused entries
 *                  KILLED with type -1), and deposits scored; secondaries->
 *                  capacity must be at least 2 tracks->n (secondaries->n is
 *                  set to 2 tracks->n).
 * Replace the reference's GPU launch wrappers (GPILGammaProcess,
 * StepGammaProcess and the electron ones, source/Geant/kernel/
 * KernelPhysicsProcess.cuh:22-36). */
int gx_gpil(gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *tracks, gx_stream_t s);
int gx_propagate(gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *tracks, gx_stream_t s);
int gx_along_step(gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *tracks, double *d_edep, int nvol,
                  gx_stream_t s);
int gx_post_step(gx_ctx *ctx, const gx_transport_config *cfg, gx_track_soa *tracks, gx_track_soa *secondaries,
                 double *d_edep, int nvol, gx_stream_t s);

/* The engine of gx_transport_run started from tracks instead of primaries:
 * the tracks of `in` (status ALIVE; entries with other status are skipped)
 * are injected as they are -- position, direction, energy, NIL, stream,
 * volume (< -1: located) -- and transported with their secondaries for at
 * most max_iterations iterations of the engine (0: to completion; one
 * iteration is one step of every track in flight with the plain engine,
 * up to steps_per_launch with the batched one), deposits added to d_edep.
 * Every track still alive then -- in flight, deferred, or not yet injected --
 * is written to `out` (out->n set; status ALIVE), so a caller can hand tracks
 * over and take them back: transporting `out` afterwards, here or in the
 * reference's host loop, continues each track exactly where it stopped (the
 * results do not depend on where the hand-over happens).  More tracks than
 * out->capacity: the first capacity are written and GX_ERR_OVERFLOW is
 * returned with out->n = the number alive.  Synchronous.  `in` and `out` must
 * not share arrays.  No counterpart in the reference (its TrackCollection is
 * host-side only). */
int gx_transport_tracks(gx_ctx *ctx, const gx_transport_config *cfg, const gx_track_soa *in, int max_iterations,
                        gx_track_soa *out, double *d_edep, int nvol, gx_transport_stats *stats, gx_stream_t s);

/* Launch-setting sweep of the batched engine.  No counterpart in the
 * reference (its kernels take nblocks / nthreads from the caller,
 * source/Geant/kernel/KernelPhysicsProcess.cuh:22-36).  Transports the given
 * primaries (the whole batch, or a representative subset of it) once per
 * candidate: block size {64, 128, 256, 512, 1024} (512 and 1024 with the
 * uniform field, layered geometry and no multiple scattering, at most 4096
 * threads per SM) x resident blocks per SM {1, 2, 4, 5, 6, 8}, then steps per track
 * and transport launch {1, 16, 64, 1024}, then iterations per CUDA-graph
 * launch {4, 8, 32, 64}, then the refill threshold {1/8, 1/4, 3/4 of the
 * capacity}, then the primary energy per injection wave {1/4, 1/2, 2 x the
 * default}, then the compaction interval (interaction_interval) {2, 4, 8},
 * then the photon kernel's fetch threshold (fetch_min_by_type[0]) {1, 8, 16,
 * 24} beside the default, each coordinate from the best so far.  Score: track-steps per millisecond of
 * device time, best of `repeats` runs (at least 1; the first run of a new
 * launch shape includes its graph capture).  Writes the winner into
 * cfg->block_size, blocks_per_sm, steps_per_launch, graph_iters,
 * refill_below, wave_energy, interaction_interval and fetch_min_by_type[0]; report (optional) lists
 * every trial.  cfg->engine must be 1; the precision and capacity are kept. */
#define GX_AUTOTUNE_MAX_TRIALS 64
typedef struct {
  int trials, best; /* number of trials listed; index of the winner */
  int block_size[GX_AUTOTUNE_MAX_TRIALS], blocks_per_sm[GX_AUTOTUNE_MAX_TRIALS];
  int steps_per_launch[GX_AUTOTUNE_MAX_TRIALS], graph_iters[GX_AUTOTUNE_MAX_TRIALS];
  long long refill_below[GX_AUTOTUNE_MAX_TRIALS];
  double wave_energy[GX_AUTOTUNE_MAX_TRIALS];
  int interaction_interval[GX_AUTOTUNE_MAX_TRIALS];
  double kernel_ms[GX_AUTOTUNE_MAX_TRIALS];    /* device time, best of the repeats (0: did not complete) */
  double steps_per_ms[GX_AUTOTUNE_MAX_TRIALS]; /* track-steps per device millisecond */
  int fetch_min_gamma[GX_AUTOTUNE_MAX_TRIALS];  /* fetch_min_by_type[0] of the trial */
} gx_autotune_report;
int gx_transport_autotune(gx_ctx *ctx, gx_transport_config *cfg, int nprim, const int *d_type, const double *d_E,
                          const double *d_pos, const double *d_dir, const int *d_event, int nvol, int repeats,
                          gx_autotune_report *report, gx_stream_t s);

/* Timeline tracing of the batched engine, in the library's tracing build
 * (geantexascalepilot_b200/build.py --timeline: lib/libgxb200_timeline.so);
 * the reference traces with timemory (its TIMEMORY_* markers), which has no
 * place in this build.  The step kernels of that build record, per iteration
 * and kernel, the GPU global timer (ns) at the start of their first block and
 * at the end of their last: h_out[((r * 16 + k) * 2) + {0, 1}] for row r =
 * (iteration + 1) mod 512 and kernel k (0 refill, 1 refill bookkeeping, 2-4
 * transport of gamma, e-, e+, 5 + 3 type + process interactions, 14 end of
 * iteration); a start of 2^64 - 1 means the kernel did not run.  reset clears
 * the record, read copies it out after a device synchronisation (n = 16384).
 * The product library returns GX_ERR_ARG from both. */
int gx_timeline_reset(gx_ctx *ctx);
int gx_timeline_read(gx_ctx *ctx, unsigned long long *h_out, long long n);

/* gx_transport_run without any device allocation.  No counterpart in the
 * reference.  For callers that must not allocate device memory while they
 * run: a host framework whose caching allocator already owns the device
 * memory, a process held to a fixed memory budget, or a time-critical loop
 * that cannot take the implicit device synchronisation of cudaMalloc /
 * cudaFree.  The plain FP64 loop runs on a static device array owned by the
 * library (about 6.3 MB, held on every device that loads the library until the
 * process exits): at most GX_NOALLOC_MAX_PRIMARIES primaries per call, at most
 * GX_NOALLOC_CAPACITY tracks in flight plus as many deferred; larger inputs
 * are rejected with GX_ERR_ARG and a message; more tracks than that in flight
 * and deferred at once end the call with GX_ERR_OVERFLOW (the tracks that did
 * not fit are scored where they were).  precision must be 0 (FP64); engine is
 * ignored; d_edep is added to as in gx_transport_run.  Every call shares the
 * array; calls that overlap on the GPU race on it.  The first call on a device
 * sets that device up (a symbol lookup and the skip-ahead table upload).  Each
 * call synchronises its stream after every iteration.  A cudaDeviceReset while the
 * library is loaded is not supported (the set-up is kept per process). */
#define GX_NOALLOC_CAPACITY 16384
#define GX_NOALLOC_MAX_PRIMARIES 4096
int gx_transport_run_noalloc(gx_ctx *ctx, const gx_transport_config *cfg, int nprim, const int *d_type,
                             const double *d_E, const double *d_pos, const double *d_dir, const int *d_event,
                             double *d_edep, int nvol, gx_transport_stats *stats, gx_stream_t s);

#ifdef __cplusplus
}
#endif
#endif
