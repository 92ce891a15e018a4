// gx_autotune.cu -- launch-setting sweep for the batched transport engine.
//
// The step kernels are register-heavy (110-130 registers per thread); block
// sizes of 64-256 threads run the kernels compiled for them, 512 and 1024
// threads (for the uniform field, layered geometry and no multiple
// scattering) the variants held to 64 registers per thread, which spill; the
// grid is a multiple of the SM count.  The sweep is coordinate descent: block
// size x resident blocks per SM first, then the steps a track may take per
// transport launch, then the number of iterations per CUDA-graph launch, then
// the refill threshold, then the primary energy per injection wave, then the
// compaction interval (how many iterations interacting tracks wait in their
// buffers before the interaction kernels compact them back into the stores),
// then the idle lanes a warp of the photon transport kernel waits for before
// it takes new records.
// Each candidate transports the caller's primaries completely; its score is
// track-steps per millisecond of device time, the best of `repeats` runs (the
// first run of a new launch shape also captures its graph).
#include "gx_internal.cuh"

#include <cstring>
#include <vector>

namespace {

struct Trial {
  int block, bpsm, steps, graph_iters;
  long long refill_below;
  double wave_energy;
  int interval;
  int fetch_g; // idle lanes before a warp of the photon kernel takes new records
};

} // namespace

extern "C" int gx_transport_autotune(gx_ctx *ctx, gx_transport_config *cfg, int nprim, const int *d_type,
                                     const double *d_E, const double *d_pos, const double *d_dir,
                                     const int *d_event, int nvol, int repeats, gx_autotune_report *rep,
                                     gx_stream_t stream)
{
  using namespace gx;
  if (!ctx || !cfg || nprim <= 0 || !d_type || !d_E || !d_pos || !d_dir || nvol <= 0 || cfg->nevents < 1)
    return set_error(GX_ERR_ARG, "gx_transport_autotune: bad arguments");
  if (cfg->engine != 1) return set_error(GX_ERR_ARG, "gx_transport_autotune: tunes the batched engine (engine 1)");
  if (repeats < 1) repeats = 2;
  Ctx *C = reinterpret_cast<Ctx *>(ctx);
  cudaError_t e = cudaSetDevice(C->device);
  if (e != cudaSuccess) return cuda_error(e, "gx_transport_autotune: cudaSetDevice");
  cudaStream_t s = stream_of(stream);
  const size_t nt = (size_t)cfg->nevents * nvol;
  double *edep = nullptr;
  if ((e = cudaMalloc((void **)&edep, nt * sizeof(double))) != cudaSuccess)
    return cuda_error(e, "gx_transport_autotune: tally scratch");

  gx_transport_config base = *cfg;
  base.profile = 0;
  const long long cap = base.capacity > 0 ? base.capacity : (1LL << 24);
  if (rep) std::memset(rep, 0, sizeof(*rep));
  int ntrials = 0, rc = GX_OK;
  double best_rate = -1.0;
  Trial best = {base.block_size > 0 ? base.block_size : default_block(1),
                base.blocks_per_sm > 0 ? base.blocks_per_sm : default_blocks_per_sm(base),
                base.steps_per_launch > 0 ? base.steps_per_launch : kDefaultStepsPerLaunch,
                base.graph_iters > 0 ? base.graph_iters : 16,
                base.refill_below > 0 ? base.refill_below : cap / 2, base.wave_energy,
                base.interaction_interval > 0 ? base.interaction_interval : 1,
                base.fetch_min_by_type[0] > 0 ? base.fetch_min_by_type[0] : default_fetch_min(base, 0)};

  auto measure = [&](const Trial &t) -> double {
    gx_transport_config c = base;
    c.block_size = t.block;
    c.blocks_per_sm = t.bpsm;
    c.steps_per_launch = t.steps;
    c.graph_iters = t.graph_iters;
    c.refill_below = t.refill_below;
    c.wave_energy = t.wave_energy;
    c.interaction_interval = t.interval;
    c.fetch_min_by_type[0] = t.fetch_g;
    double best_ms = 0.0, rate = 0.0;
    for (int r = 0; r < repeats; ++r) {
      cudaMemsetAsync(edep, 0, nt * sizeof(double), s);
      gx_transport_stats st;
      int k = gx_transport_run(ctx, &c, nprim, d_type, d_E, d_pos, d_dir, d_event, edep, nvol, nullptr, &st,
                               stream);
      if (k == GX_ERR_CUDA) {
        rc = k; // the device is in trouble: stop the sweep
        return -1.0;
      }
      if (k != GX_OK || st.kernel_ms <= 0.0) return 0.0; // e.g. overflow with this setting: not a candidate
      if (r == 0 || st.kernel_ms < best_ms) best_ms = st.kernel_ms;
      rate = (double)st.steps / best_ms;
    }
    if (rep && ntrials < GX_AUTOTUNE_MAX_TRIALS) {
      rep->block_size[ntrials] = t.block;
      rep->blocks_per_sm[ntrials] = t.bpsm;
      rep->steps_per_launch[ntrials] = t.steps;
      rep->graph_iters[ntrials] = t.graph_iters;
      rep->refill_below[ntrials] = t.refill_below;
      rep->wave_energy[ntrials] = t.wave_energy;
      rep->interaction_interval[ntrials] = t.interval;
      rep->fetch_min_gamma[ntrials] = t.fetch_g;
      rep->kernel_ms[ntrials] = best_ms;
      rep->steps_per_ms[ntrials] = rate;
    }
    ++ntrials;
    return rate;
  };
  auto consider = [&](const Trial &t) {
    if (rc) return;
    double r = measure(t);
    if (r > best_rate) {
      best_rate = r;
      best = t;
      if (rep) rep->best = ntrials - 1;
    }
  };

  // blocks above 256 threads only where their kernel variants exist
  const bool wide_ok = base.geometry != 2 && !base.msc && !base.field_map && !base.fp64_parity;
  const int blocks[] = {64, 128, 256, 512, 1024};
  const int bpsms[] = {1, 2, 4, 5, 6, 8};
  for (int b : blocks)
    for (int p : bpsms) {
      if (b > 256 && (!wide_ok || b * p > 4096)) continue;
      Trial t = best;
      t.block = b;
      t.bpsm = p;
      consider(t);
    }
  const Trial after_shape = best;
  for (int k : {1, 16, 64, 1024}) {
    Trial t = after_shape;
    t.steps = k;
    consider(t);
  }
  const Trial after_steps = best;
  for (int g : {4, 8, 32, 64}) {
    Trial t = after_steps;
    t.graph_iters = g;
    consider(t);
  }
  const Trial after_graph = best;
  for (long long r : {cap / 8, cap / 4, (3 * cap) / 4}) {
    Trial t = after_graph;
    t.refill_below = r;
    consider(t);
  }
  const Trial after_refill = best;
  // multiples of the engine's default widen or narrow the injection waves
  const double wave0 = default_wave_energy(cap, kWaveFillBatched);
  for (double m : {0.25, 0.5, 2.0}) {
    Trial t = after_refill;
    t.wave_energy = m * wave0;
    consider(t);
  }
  const Trial after_wave = best;
  for (int k : {2, 4, 8}) {
    Trial t = after_wave;
    t.interval = k;
    consider(t);
  }
  const Trial after_interval = best;
  for (int f : {1, 8, 16, 24}) {
    if (f == after_interval.fetch_g) continue;
    Trial t = after_interval;
    t.fetch_g = f;
    consider(t);
  }
  cudaFree(edep);
  if (rep) rep->trials = ntrials < GX_AUTOTUNE_MAX_TRIALS ? ntrials : GX_AUTOTUNE_MAX_TRIALS;
  if (rc) return rc;
  if (best_rate <= 0.0) return set_error(GX_ERR_OVERFLOW, "gx_transport_autotune: no setting completed the sample");
  cfg->block_size = best.block;
  cfg->blocks_per_sm = best.bpsm;
  cfg->steps_per_launch = best.steps;
  cfg->graph_iters = best.graph_iters;
  cfg->refill_below = best.refill_below;
  cfg->wave_energy = best.wave_energy;
  cfg->interaction_interval = best.interval;
  cfg->fetch_min_by_type[0] = best.fetch_g;
  return GX_OK;
}
