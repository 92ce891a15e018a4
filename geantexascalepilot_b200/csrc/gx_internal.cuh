// gx_internal.cuh -- shared declarations of the C-ABI implementation files.
#pragma once

#include "../../include/gx_abi.h"
#include "gx_device.cuh"

#include <vector>

namespace gx {

struct Engine; // transport buffers, kept across calls (gx_transport.cu)

struct Ctx {
  int device = 0;
  int num_sms = 148;
  Data host;            // host copy (device pointers inside)
  Data *dev = nullptr;  // device copy
  std::vector<void *> owned;
  Engine *engine = nullptr;
};

int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);
void jump_matrix(int comp, long long e, long long c, uint64_t out[9]);
void mat_mul(const uint64_t A[9], const uint64_t B[9], uint64_t C[9], uint64_t m);
void mat_vec(const uint64_t A[9], uint64_t v[3], uint64_t m);
void release_engine(Ctx *c);
int refit_vector(Ctx *ctx, int table, int mat, const double *ynew);

inline cudaStream_t stream_of(gx_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Launch defaults of the transport engines (the sweep of gx_transport_autotune
// found 128-thread blocks fastest for the batched engine on C3; the plain loop
// keeps 256).
inline int default_block(int engine) { return engine == 1 ? 128 : 256; }
constexpr int kDefaultBlocksPerSM = 4;
// Steps of one track per transport-kernel launch in the batched engine, at
// most (a track is kept in registers while it neither interacts nor dies).
constexpr int kDefaultStepsPerLaunch = 16;
// Primary energy per injection wave for stores of cap slots: a 10 GeV shower
// peaks near 800 tracks in flight, ~0.08 per MeV of primary energy; waves are
// sized so that their showers would peak at `fill` x cap if they all peaked
// together (they do not: waves overlap as showers age).  The batched engine
// uses fill 0.8 (fastest in the sweep on C3), the plain loop 0.4.
inline double default_wave_energy(long long cap, double fill) { return fill * (double)cap / 0.08; }

} // namespace gx
