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
  unsigned long long total;             // the run covers relative photons [item_lo, total)
  unsigned long long item_lo;           // first relative photon of the run (0: the whole batch)
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
  uint32_t slot_cache;                  // batched tallies: 1 = warps may cache events in shared-memory
                                        // slots (every record's max_steps < kSlotMaxAdd)
  uint32_t keep_tally;                  // 1: the run adds to the tallies (no zeroing by the prep kernel)
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
// Dynamic shared memory above this needs the kernel's opt-in attribute: the
// default limit is 48 KB minus the kernel's static shared memory (at most 1 KB
// for the kernels here).
constexpr size_t kDynSmemOptIn = 47u * 1024u;
constexpr unsigned kErrQueue = 1u, kErrWatchdog = 2u;
// Batched tallies: each warp caches the counters of two events in shared memory
// (7 x u32 per event, padded to 8) and, when the tally has at most kSlotBins
// histogram bins, their time / hit-map bins too (u32). A warp flushes both its
// slots to the events' u64 slices once kSlotFlushPhotons photons have entered it
// since the last flush (checked at refills); events are cached only when every
// record's max_steps is below kSlotMaxAdd (WaveArgs::slot_cache), so a photon
// adds less than kSlotMaxAdd to a step sum. At most 64 more photons
// (32 lanes, 32 in the pantry) can finish before the next check, so a u32
// counter gains less than (kSlotFlushPhotons + 64) x kSlotMaxAdd < 2^32.
constexpr uint32_t kSlotBins = 256u;
constexpr uint32_t kSlotCounterBytesPerWarp = 2u * 8u * 4u;
constexpr uint32_t kSlotMaxAdd = 1u << 16;
constexpr uint32_t kSlotFlushPhotons = 1u << 14;
static_assert((static_cast<unsigned long long>(kSlotFlushPhotons) + 64u) * kSlotMaxAdd < (1ull << 32),
              "slot counters must not wrap between flushes");
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

// Per-interaction sorted run (sorted_kernel): between steps each photon waits in
// the state queue of its pending interaction; every iteration is one launch in
// which each warp takes 32 photons of one queue (or 32 fresh emissions), so the
// interaction code runs warp-uniform, and appends the survivors, moved to their
// next interaction, to the queues of the other parity.
enum SortQueue : uint32_t { kQScatter = 0, kQFresnel = 1, kQPainted = 2, kSortQueues = 3 };
// A queued photon: 5 x 16 B in tiles of 32 photons (px py pz t | dx dy dz path |
// window words 0-3 | words 4-7 | nb ns o+hit blk), plus its relative index.
constexpr uint32_t kSortVec4 = 5u;
constexpr int kSortThreads = 256;  // threads per block of sorted_kernel
constexpr uint32_t kSortBytesPerPhoton = kSortVec4 * 16u + 4u;

// Passed by value (kernel parameter: read through the constant bank).
struct SortArgs {
  float4* q[2][kSortQueues];            // [parity][queue] tiles
  uint32_t* qid[2][kSortQueues];        // relative photon index per slot
  uint32_t cap;                         // slots per queue = photons in flight (multiple of 32)
  uint32_t drain_below;                 // finish every photon in one launch once fewer are left
  unsigned long long n;                 // photons in the run
  unsigned long long first_id;          // Philox id of relative photon 0
  unsigned long long* tally;            // null: no tally (else ADDED to, flat layout)
  TallyDev tc;
  DevRecords rec;                       // rec.fate null: no records
  unsigned long long graph_handle;      // cudaGraphConditionalHandle of the iteration loop
  uint32_t iter_cap;                    // watchdog: max iterations per run
  uint32_t use_graph;                   // 1: iterations run as a graph while node (set its condition)
};

// A queue's append counter, alone in its 128-byte line: every warp of a launch
// adds to it, so the three queues' counters should not share an L2 sector.
struct alignas(128) SortCounter {
  unsigned int v;
  unsigned int pad[31];
};

struct SortCtrl {
  SortCounter count[2][kSortQueues];    // photons per queue [parity] (appends are atomic)
  unsigned int parity;                  // parity of this iteration's input queues
  unsigned int emit_count;              // fresh photons this iteration
  unsigned long long emit_base;         // relative index of the first of them
  unsigned int drain;                   // 1: this iteration runs every photon to its end
  unsigned int blocks_done;             // blocks finished (atomic)
  unsigned int iter;                    // iterations run
  unsigned int error;                   // kErrQueue, kErrWatchdog
  unsigned int active;                  // 0 once the run is complete (launches return at once)
  unsigned long long queued[kSortQueues];  // photons that went through each queue
  unsigned long long drained;           // photons finished by the drain launch
};
static_assert(sizeof(SortCtrl) <= 1024, "sorted control block");

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
  /* Per-interaction sorted run: prep (one thread) and one iteration. */                         \
  /* minb: 3 or 4 resident blocks per SM (the register budget) */                               \
  const void* sorted_prep_fn();                                                                  \
  const void* sorted_kernel_fn(int minb);                                                        \
  int sorted_blocks_per_sm(int minb, int block);                                                 \
  cudaError_t launch_sorted(int minb, const DevParams& P, const SortArgs& A, SortCtrl* ctrl,      \
                            int grid, int block, cudaStream_t st);                               \
  cudaError_t launch_sorted_prep(const SortArgs& A, SortCtrl* ctrl, cudaStream_t st);            \
  }

OPTX_DECLARE_LAUNCHERS(fast)
OPTX_DECLARE_LAUNCHERS(exact)
OPTX_DECLARE_LAUNCHERS(approx)

}  // namespace optx
