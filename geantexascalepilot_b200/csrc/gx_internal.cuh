// gx_internal.cuh -- shared declarations of the C-ABI implementation files.
#pragma once

#include "../../include/gx_abi.h"
#include "gx_csg.cuh"
#include "gx_device.cuh"

#include <vector>

namespace gx {

struct Engine; // transport buffers, kept across calls (gx_transport.cu)
namespace parity {
struct Engine; // the same for the FP64 parity variant (gx_transport_parity.cu)
}

struct Ctx {
  int device = 0;
  int num_sms = 148;
  Data host;            // host copy (device pointers inside)
  Data *dev = nullptr;  // device copy
  std::vector<void *> owned;
  Engine *engine = nullptr;
  parity::Engine *parity_engine = nullptr;
  // the CSG volume tree (gx_ctx_load_geometry): touchables, children, tally column of each
  CsgNode *csg_node = nullptr;
  int *csg_kids = nullptr, *csg_score = nullptr, *csg_slab = nullptr, *csg_cand = nullptr;
  double *csg_planes = nullptr;
  int csg_n = 0, csg_nscore = 0;
  int csg_solids = 0; // the solid kinds in the tree (bit k: kind k)
  double *stage_scratch = nullptr; // escaped energy of the stage calls (gx_along_step)
  // gx_transport_run_host: its stream and device staging buffer, kept across calls
  cudaStream_t host_stream = nullptr;
  void *host_buf = nullptr;
  size_t host_buf_bytes = 0;
};

int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);
void jump_matrix(int comp, long long e, long long c, uint64_t out[9]);
void mat_mul(const uint64_t A[9], const uint64_t B[9], uint64_t C[9], uint64_t m);
void mat_vec(const uint64_t A[9], uint64_t v[3], uint64_t m);
void build_jump_host(uint64_t h[2][64][9]);
void release_engine(Ctx *c);
int launch_substreams(const double seed[6], long long first, int n, uint32_t *d_states, cudaStream_t s);
int get_jump_table(uint64_t **out);
int run_stage(int stage, Ctx *C, const gx_transport_config *cfg, gx_track_soa *t, gx_track_soa *sec, double *d_edep,
              int nvol, cudaStream_t s);
int run_tracks(Ctx *C, const gx_transport_config *cfg, const gx_track_soa *in, int max_iter, gx_track_soa *out,
               double *d_edep, int nvol, gx_transport_stats *stats, cudaStream_t s);
namespace parity {
int run_stage(int stage, Ctx *C, const gx_transport_config *cfg, gx_track_soa *t, gx_track_soa *sec, double *d_edep,
              int nvol, cudaStream_t s);
int run_tracks(Ctx *C, const gx_transport_config *cfg, const gx_track_soa *in, int max_iter, gx_track_soa *out,
               double *d_edep, int nvol, gx_transport_stats *stats, cudaStream_t s);
void release_engine(Ctx *c);
int run_transport(Ctx *C, const gx_transport_config *cfg, int nprim, const int *d_type, const double *d_E,
                  const double *d_pos, const double *d_dir, const int *d_event, double *d_edep, int nvol,
                  int *d_pstep, gx_transport_stats *stats, cudaStream_t s);
} // namespace parity
int refit_vector(Ctx *ctx, int table, int mat, const double *ynew);
int refit_vector_xy(Ctx *ctx, int table, int mat, const double *xnew, const double *ynew);

inline cudaStream_t stream_of(gx_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Launch defaults of the transport engines (the sweep of gx_transport_autotune
// found 128-thread blocks fastest for the batched engine on C3; the plain loop
// keeps 256).  The FP32-mixed step kernels of the uniform field, layered
// geometry and no multiple scattering are held to 96 registers, so five
// 128-thread blocks fit on an SM (20 warps); the others take up to 128 (four).
inline int default_block(int engine) { return engine == 1 ? 128 : 256; }
constexpr int kDefaultBlocksPerSM = 4;
inline int default_blocks_per_sm(const gx_transport_config &c)
{
  const bool plain = !c.field_map && c.geometry != 2 && !c.msc && !c.fp64_parity;
  return c.engine == 1 && c.precision == 1 && plain ? 5 : kDefaultBlocksPerSM;
}
// Steps of one track per transport-kernel launch in the batched engine, at
// most (a track is kept in registers while it neither interacts nor dies).
constexpr int kDefaultStepsPerLaunch = 16;
// Idle lanes of a warp before it takes new records in the transport kernel of
// type q (0 gamma, 1 e-, 2 e+).  Measured: the FP32-mixed photon kernels of the
// layered geometry gain 1.9% on C3, 2.7% on C4 and 0.9% with multiple
// scattering at 12 (8-16 within 0.5% of it); electrons gain nothing at 2-4 and
// lose above 8, positrons lose above 4; the FP64 kernels lose 2% and the CSG
// kernels 1-4% at 8-16.
inline int default_fetch_min(const gx_transport_config &c, int q)
{
  return (q == 0 && c.precision == 1 && c.geometry != 2 && !c.fp64_parity) ? 12 : 1;
}
// Live energy (injected primary energy not yet deposited or escaped) allowed
// before more primaries are injected, for stores of cap slots: showers started
// together in the Pb/LAr calorimeter peak at 0.052-0.062 tracks in flight per
// MeV (all types together; 10 MeV-100 GeV primaries, 4 T), so at 0.064 per MeV
// the population stays below `fill` x cap.  The batched engine keeps a store,
// an overflow stack and per-process interaction buffers of cap slots for each
// particle type, and uses fill 1.2 (C4 and C5 2.3-2.5% faster than at 0.8, in
// larger and fewer iterations; at 2.4 C5 overflowed an interaction buffer);
// the plain loop, one mixed store, 0.4.
constexpr double kWaveFillBatched = 1.2, kWaveFillPlain = 0.4;
inline double default_wave_energy(long long cap, double fill) { return fill * (double)cap / 0.064; }

} // namespace gx
