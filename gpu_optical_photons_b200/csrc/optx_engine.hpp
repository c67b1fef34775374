// optx_engine.hpp - internal interface between the C ABI (capi.cu) and the
// kernels (kernels.cu, compiled once per math mode into namespaces optx::fast,
// optx::exact and optx::approx). Not part of the public ABI (include/optx.h is).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "optx_device.cuh"

namespace optx {

// Tally binning as the kernels see it (transport.hpp:164-181 of the reference):
// tscale = float(time_bins) / time_max, computed on the host in float.
struct TallyDev {
  uint32_t time_bins;
  float tscale;
  uint32_t xy_bins;
  uint32_t len;  // 5 + time_bins + 1 + xy_bins^2 + 2
};

// Wavefront run description, resident in device memory (the host writes it
// before each run; kernels read it, so a captured graph stays valid).
struct WaveArgs {
  const DevParams* params;              // records: events, or gensteps (1 entry when not batched)
  const DevParams* phys;                // physics per event (= params unless gensteps)
  const unsigned long long* offsets;    // n_events + 1 relative photon offsets (batched)
  const uint32_t* ev_table;             // record of photon (k << ev_shift), k <= total >> ev_shift
  // n_events: records in `params` / `offsets` (events, or gensteps)
  uint32_t n_events;
  uint32_t threshold;                   // refill a warp when fewer lanes than this are alive (1..32)
  uint32_t cadence;                     // steps per photon per wave before a forced spill (0 = none)
  uint32_t qcap;                        // capacity of each state queue, photons
  unsigned long long total;             // photons in the run
  unsigned long long first_id;          // Philox id of relative photon 0
  unsigned long long wave_quota;        // fresh photons admitted per wave
  float4* qa;                           // state queues: tiles of 32 photons x 4 float4 (64 B each)
  float4* qb;
  unsigned long long* tally;            // tally mode: n_events x len u64
  TallyDev tc;
  DevRecords rec;                       // records mode
  const double* w_bin;                  // adjoint mode: time_bins + 1 weights
  double w_det;
  double inv_la, inv_la2, inv_ls, inv_ls2, inv_r, inv_tau, inv_tau2;
  uint32_t score_mask;                  // bit j: parameter j has a score term
  uint32_t moments_smem;                // 1: moments accumulate per block in shared memory first
  double* grad;                         // adjoint mode: 4 FP64 sums (accumulated)
  double* moments;                      // adjoint mode, optional: (time_bins + 1) x 5 FP64
                                        // per-bin (count, sum S_La, S_Ls, S_R, S_tau)
  unsigned long long graph_handle;      // cudaGraphConditionalHandle of the wave loop
  unsigned long long iter_cap;          // watchdog: max loop iterations per warp per wave
  uint32_t use_graph;                   // 1: the wave loop is a graph while node (set its condition)
  uint32_t wave_cap;                    // watchdog: max waves per run
  uint32_t chunk;                       // consecutive work items a warp claims per grab (>= 32)
  uint32_t n_tallies;                   // events = tally slices (= n_events unless gensteps)
  uint32_t ev_shift;                    // ev_table resolution: one entry per 2^ev_shift photons
  uint32_t tail_steps;                  // steps a photon makes in a wave before it may be spilled at its end
  const uint32_t* tally_of;             // record -> event (null: the record's own index)
  const float4* seg;                    // genstep records: 2 float4 each (end x,y,z,t0), (dt,-,-,-)
};

// Dynamic state of a wavefront run (device memory).
struct WaveCtrl {
  unsigned long long fresh_next;   // first fresh photon (relative index) of the current wave
  unsigned long long useful;       // lane-steps that advanced a photon
  unsigned long long issued;       // 32 x warp step iterations
  unsigned long long cursor;       // work items claimed (atomic; may run past the wave's items)
  unsigned int wave;               // current wave number
  unsigned int n_in;               // survivors carried into the current wave
  unsigned int fresh_count;        // fresh photons admitted in the current wave
  unsigned int n_out;              // survivors spilled (atomic)
  unsigned int blocks_done;        // blocks finished (atomic)
  unsigned int active;             // 0 once the run is complete
  unsigned int error;              // bit 0 queue overflow, bit 1 watchdog
  unsigned int spills;             // total photons spilled over the run
  unsigned int gs_error;           // device genstep upload: bit 0 an invalid genstep, bit 1 more
                                   // photons than the engine holds (kept until the next upload)
};

// kModeMoments: the adjoint replay that also fills the per-bin score moments
// (single configuration only; a kernel of its own keeps the gradient replay lean).
enum WaveMode : int { kModeTally = 0, kModeRecords = 1, kModeAdjoint = 2, kModeMoments = 3 };
// Wave kernel variants: one configuration (physics in the kernel argument); a
// batch of records with per-event physics; a batch whose events share their
// step physics (kernel argument), with per-record emission and per-event tallies.
enum WaveVariant : int { kSingle = 0, kBatch = 1, kBatchUniform = 2 };
constexpr uint32_t kEvShift = 7;  // coarsest event-table resolution: one entry per 128 photons
// Shared memory of one warp's pantry: 32 ready photons x 112 bytes (7 x 16 B;
// the 112-byte stride makes 8 lanes' 128-bit accesses hit 8 distinct bank groups).
constexpr uint32_t kPantryBytesPerWarp = 32u * 112u;
constexpr unsigned kErrQueue = 1u, kErrWatchdog = 2u;
// Batched tallies: each warp caches the counters of two events in shared memory
// (7 x u64 per event, padded to 8) and, when the tally has at most kSlotBins
// histogram bins, their time / hit-map bins too (u32).
constexpr uint32_t kSlotBins = 256u;
constexpr uint32_t kSlotCounterBytesPerWarp = 2u * 8u * 8u;
inline __host__ __device__ uint32_t slot_bin_bytes_per_warp(uint32_t n_bins) {
  return n_bins <= kSlotBins ? 2u * n_bins * 4u : 0u;
}
// Score moments: a block-private (time_bins + 1) x 5 FP64 table in shared memory,
// added to global memory once per block, when it takes at most this many bytes
// (818 time bins); larger tables accumulate with global atomics directly.
constexpr uint32_t kMomentSmemMaxBytes = 32u * 1024u;
inline __host__ __device__ uint32_t moment_smem_bytes(uint32_t time_bins) {
  const uint32_t b = (time_bins + 1u) * 5u * 8u;
  return b <= kMomentSmemMaxBytes ? b : 0u;
}

#define OPTX_DECLARE_LAUNCHERS(NS)                                                               \
  namespace NS {                                                                                 \
  cudaError_t launch_history_records(const DevParams& P, uint64_t first_id, uint64_t n,          \
                                     const DevRecords& out, int block, cudaStream_t st);         \
  cudaError_t launch_history_tally(const DevParams& P, const TallyDev& tc, uint64_t first_id,    \
                                   uint64_t n, unsigned long long* tally, int block, int grid,   \
                                   cudaStream_t st);                                             \
  int history_tally_blocks_per_sm(int block, size_t smem);                                       \
  /* Wavefront: prep (reset ctrl, zero tallies) and one wave. */                                 \
  cudaError_t launch_wave_prep(const WaveArgs* A_dev, WaveCtrl* ctrl, int grid, int block,       \
                               cudaStream_t st);                                                 \
  const void* wave_prep_fn();                                                                    \
  /* batch: kSingle, kBatch or kBatchUniform (see WaveVariant) */                               \
  const void* wave_kernel_fn(int mode, int batch, int minb);                                     \
  int wave_blocks_per_sm(int mode, int batch, int minb, int block, size_t smem);                 \
  cudaError_t wave_set_smem(int mode, int batch, int minb, size_t smem);                         \
  cudaError_t launch_wave(int mode, int batch, int minb, const DevParams& P,                     \
                          const WaveArgs* A_dev, WaveCtrl* ctrl, int grid, int block,            \
                          size_t smem, cudaStream_t st);                                         \
  cudaError_t launch_event_table(const unsigned long long* offsets, uint32_t n_events,           \
                                 uint32_t* table, unsigned long long total, uint32_t shift,      \
                                 cudaStream_t st);                                               \
  }

OPTX_DECLARE_LAUNCHERS(fast)
OPTX_DECLARE_LAUNCHERS(exact)
OPTX_DECLARE_LAUNCHERS(approx)

}  // namespace optx
