// kernels.cu - photon transport kernels for sm_100a.
//
// Compiled three times by the build: OPTX_NS=fast (CUDA libm, FMA contraction),
// OPTX_NS=exact (portable math, -fmad=false) and OPTX_NS=approx (the fast
// source with --use_fast_math). Kernels:
//
//  * history_records_kernel / history_tally_kernel: one thread per photon for
//    its whole history (a thread runs its photons one after another in one
//    loop, history_loop), the drop-in for the reference's transport_records_kernel
//    and transport_tally_kernel (src/gpu/gpu_backend.cu:47-100 of the reference).
//    The tally keeps fate counts and step sums in registers (no atomics) and the
//    time / hit-map histograms in block-private shared memory, flushed once per
//    block with 64-bit global atomics: integer sums, so the result does not depend
//    on the schedule (the property of gpu_backend.cu:68-100 and test_gpu.cpp:122-146).
//
//  * wave_kernel: the wavefront engine, the B200 form of the reference's
//    event_step_kernel (src/gpu/gpu_event.cu:125-170). A persistent grid of warps
//    keeps one photon per lane in registers. When fewer than `threshold` lanes of
//    a warp are alive, the idle lanes take photons from the warp's shared-memory
//    pantry, which all 32 lanes refill together (a fresh photon is emitted, or a
//    survivor of the previous wave is loaded from the state queue) from a chunk
//    of consecutive work items the warp claimed with one atomic. When the wave's
//    items are used up, or a photon has made `cadence` steps in this wave, the
//    warp spills its live photons: ballot + popc give each one a slot after a
//    single atomicAdd, and the state is written as 4 x 128-bit stores into an
//    AoSoA queue tile (32 photons x 64 B). The next wave (the next iteration of a
//    CUDA-graph while loop, or the next host launch) reads them back with 4 x
//    128-bit coalesced loads. The last block to finish a wave sets up the next one
//    (counters only; no block ever waits for another).
//    Variants: one configuration (physics in the kernel argument); a batch of
//    records (events or gensteps) whose photons read their event's physics record
//    per step; a batch whose events share their step physics (kernel argument).
//    Batched tallies go through two per-warp shared-memory event slots.
//    Records depend only on (seed, photon id), so they equal the history
//    kernel's bit for bit for any block size, threshold, cadence, chunk or wave size.
#include <cuda_runtime.h>

#include <algorithm>

#include "optx_device.cuh"
#include "optx_engine.hpp"

#ifndef OPTX_NS
#error "OPTX_NS must be defined (fast or exact)"
#endif

namespace optx {
namespace OPTX_NS {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ void store_record(const DevRecords& out, uint64_t i, const Photon& s,
                                             uint32_t fate) {
  out.fate[i] = static_cast<uint8_t>(fate);
  out.n_boundary[i] = s.nb;
  out.n_scatter[i] = s.ns;
  out.t[i] = s.t;
  out.x[i] = s.px;
  out.y[i] = s.py;
  out.z[i] = s.pz;
  out.path[i] = s.path;
}

// The histories of photons first_id + i for i = i0, i0 + stride, ... < n, one
// after another in this thread (transport.hpp:151-159 per photon), in one loop
// for all of them: a thread whose photon ended starts its next photon in the
// next iteration instead of waiting, at the end of a per-photon loop, for the
// longest history of its warp (measured: 1.7-2.2x on the single
// configurations). Each photon's arithmetic is that of its own history, so
// records and tallies do not depend on the grid. done(i, s, fate) is called
// once per photon.
template <class Done>
__device__ __forceinline__ void history_loop(const DevParams& P, uint64_t first_id, uint64_t n,
                                             uint64_t i, uint64_t stride, Done&& done) {
  Photon s;
  Rng r;
  ScoreAux aux{0u, 0.0f};
  // At most one photon for this thread (a launch that covers its photons in one
  // grid pass, e.g. one event of a batch): the plain per-photon loop, which is
  // tighter (measured: 4096 per-event launches 229 -> 182 ms; +1 % on 1e7-photon
  // launches, where threads run several photons through the single loop).
  if (i + stride >= n) {
    if (i < n) {
      const uint64_t id = first_id + i;
      r.init(id, P.key_lo, P.key_hi, 0u);
      start_photon<false>(P, s, r, id, aux);
      uint32_t fate = kMaxSteps;
      for (uint32_t st = 0; st < P.max_steps; ++st) {
        if (!step_photon<false>(P, s, r, id, fate, aux)) break;
      }
      done(i, s, fate);
    }
    return;
  }
  uint64_t cur = 0;
  uint32_t step = 0;
  bool alive = false;
  for (;;) {
    uint32_t fate = kMaxSteps;
    bool ended;
    if (!alive) {
      if (i >= n) break;
      cur = i;
      i += stride;
      const uint64_t id = first_id + cur;
      r.init(id, P.key_lo, P.key_hi, 0u);
      start_photon<false>(P, s, r, id, aux);
      step = 0;
      alive = true;
      ended = P.max_steps == 0u;
    } else {
      ended = !step_photon<false>(P, s, r, first_id + cur, fate, aux);
      if (!ended && ++step >= P.max_steps) ended = true;  // fate stays kMaxSteps
    }
    if (ended) {
      alive = false;
      done(cur, s, fate);
    }
  }
}

// Blocks of up to 1024 threads (the accepted block sizes): at most 64 registers.
__global__ void __launch_bounds__(1024, 1) history_records_kernel(const DevParams P, uint64_t first_id, uint64_t n,
                                       DevRecords out) {
  history_loop(P, first_id, n, static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x,
               static_cast<uint64_t>(gridDim.x) * blockDim.x,
               [&](uint64_t i, const Photon& s, uint32_t fate) { store_record(out, i, s, fate); });
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
  return v;
}

__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
  return v;
}

// Flat tally layout: [5 fates | time_bins + 1 | xy_bins^2 | sum nb | sum ns].
// Launch bounds: blocks of up to 1024 threads (the accepted block sizes), which
// caps the kernel at 64 registers: 4 resident blocks of 256, measured 6-8 %
// faster than the unbounded 75 registers (3 blocks) despite 12 B of spills.
__global__ void __launch_bounds__(1024, 1) history_tally_kernel(const DevParams P, const TallyDev tc, uint64_t first_id,
                                     uint64_t n, unsigned long long* __restrict__ gt) {
  extern __shared__ uint32_t s_hist[];  // [time_bins + 1 | xy_bins^2]
  const uint32_t n_bins = tc.len - 7u;
  for (uint32_t b = threadIdx.x; b < n_bins; b += blockDim.x) s_hist[b] = 0u;
  __syncthreads();

  uint32_t f0 = 0, f1 = 0, f2 = 0, f3 = 0, f4 = 0;
  unsigned long long snb = 0, sns = 0;
  history_loop(P, first_id, n, static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x,
               static_cast<uint64_t>(gridDim.x) * blockDim.x,
               [&](uint64_t, const Photon& s, uint32_t fate) {
                 f0 += fate == 0u;
                 f1 += fate == 1u;
                 f2 += fate == 2u;
                 f3 += fate == 3u;
                 f4 += fate == 4u;
                 snb += s.nb;
                 sns += s.ns;
                 if (fate == kDetected) {
                   atomicAdd(&s_hist[time_bin(s.t, tc.tscale, tc.time_bins)], 1u);
                   atomicAdd(&s_hist[tc.time_bins + 1u + xy_bin(s.px, s.py, P, tc.xy_bins)], 1u);
                 }
               });
  // Fates and sums: warp reductions, one global atomic per warp and counter.
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t r0 = __reduce_add_sync(kFull, f0), r1 = __reduce_add_sync(kFull, f1),
                 r2 = __reduce_add_sync(kFull, f2), r3 = __reduce_add_sync(kFull, f3),
                 r4 = __reduce_add_sync(kFull, f4);
  snb = warp_sum_u64(snb);
  sns = warp_sum_u64(sns);
  if (lane == 0) {
    if (r0) atomicAdd(&gt[0], static_cast<unsigned long long>(r0));
    if (r1) atomicAdd(&gt[1], static_cast<unsigned long long>(r1));
    if (r2) atomicAdd(&gt[2], static_cast<unsigned long long>(r2));
    if (r3) atomicAdd(&gt[3], static_cast<unsigned long long>(r3));
    if (r4) atomicAdd(&gt[4], static_cast<unsigned long long>(r4));
    if (snb) atomicAdd(&gt[tc.len - 2u], snb);
    if (sns) atomicAdd(&gt[tc.len - 1u], sns);
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < n_bins; b += blockDim.x) {
    if (s_hist[b] != 0u) atomicAdd(&gt[5u + b], static_cast<unsigned long long>(s_hist[b]));
  }
}

// ---------------------------------------------------------------------------
// Wavefront engine.

// Event (record) of relative photon g: the table gives the record holding photon
// (g >> shift) << shift; the scan moves past records that end before g (one or
// two steps when records hold at least 2^shift photons; the host picks the
// finest shift its table allocation allows).
__device__ __forceinline__ uint32_t find_event(const WaveArgs* __restrict__ A, unsigned long long g,
                                               uint32_t shift) {
  uint32_t e = __ldg(A->ev_table + (g >> shift));
  const unsigned long long* __restrict__ off = A->offsets;
  while (e + 1u < A->n_events && __ldg(off + e + 1u) <= g) ++e;
  return e;
}

// table[k] = the record that holds photon k << shift: the largest e with
// offsets[e] <= k << shift, which is never an empty record. Each record fills its
// own entries, k in [ceil(offsets[e] / 2^shift), ceil(offsets[e+1] / 2^shift)),
// one warp per record (an empty record has none): every entry is written once,
// with no search per entry. For the 4096-event batch's 519k entries: 7-9 us
// (CUDA events, warm), against 11-13 us for a thread per entry with a binary
// search over the offsets.
__global__ void event_table_kernel(const unsigned long long* __restrict__ offsets, uint32_t n_events,
                                   uint32_t* __restrict__ table, uint32_t shift) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const unsigned long long round_up = (1ull << shift) - 1ull;
  for (uint32_t e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < n_events; e += warps) {
    const unsigned long long k0 = (offsets[e] + round_up) >> shift;
    const unsigned long long k1 = (offsets[e + 1u] + round_up) >> shift;
    for (unsigned long long k = k0 + lane; k < k1; k += 32u) table[k] = e;
  }
}

__device__ __forceinline__ float4 make_uint4_as_float4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  return make_float4(__uint_as_float(a), __uint_as_float(b), __uint_as_float(c), __uint_as_float(d));
}

// Queue slot -> first float4 of the photon in its 32-photon tile.
__device__ __forceinline__ size_t qidx(uint32_t slot) {
  return static_cast<size_t>(slot >> 5) * 128u + (slot & 31u);
}

__global__ void wave_prep_kernel(const WaveArgs* __restrict__ A, WaveCtrl* __restrict__ ctrl) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned long long lo = A->item_lo < A->total ? A->item_lo : A->total;
    unsigned long long fresh = A->total - lo < A->wave_quota ? A->total - lo : A->wave_quota;
    if (A->cadence != 0u && fresh > A->qcap) fresh = A->qcap;
    ctrl->fresh_next = lo;
    ctrl->useful = 0ull;
    ctrl->issued = 0ull;
    ctrl->wave = 0u;
    ctrl->n_in = 0u;
    ctrl->fresh_count = static_cast<unsigned int>(fresh);
    ctrl->cursor = 0u;
    ctrl->n_out = 0u;
    ctrl->blocks_done = 0u;
    ctrl->active = fresh > 0ull ? 1u : 0u;
    ctrl->error = 0u;
    ctrl->spills = 0u;
  }
  if (blockIdx.x == 0 && threadIdx.x < 4u && A->grad != nullptr) A->grad[threadIdx.x] = 0.0;
  if (A->moments != nullptr) {
    const uint32_t nm = 5u * (A->tc.time_bins + 1u);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x)
      A->moments[i] = 0.0;
  }
  if (A->tally != nullptr && A->keep_tally == 0u) {
    const size_t total = static_cast<size_t>(A->n_tallies) * A->tc.len;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
      A->tally[i] = 0ull;
  }
}

// Physics of a lane's photon: the kernel argument (one configuration, or a batch
// whose events share their step physics: UNI) or its event's record in global
// memory, read field by field where the step uses it. Lanes hold event indices;
// records (events or gensteps) are read at emission only.
template <bool BATCH, bool UNI>
__device__ __forceinline__ const DevParams& params_of(const DevParams& P0,
                                                      const WaveArgs* __restrict__ A, uint32_t ev) {
  if (BATCH && !UNI) return A->phys[ev];
  return P0;
}

// MINB: the register budget, as the resident blocks per SM the allocation must
// allow: 2, 3 or 4 blocks of 256 threads (<= 128 / 80 / 64 registers), or 7
// blocks of 128 threads (<= 72 registers, 28 warps per SM); a tuning knob.
template <int MINB>
constexpr int wave_max_threads() { return MINB >= 5 ? 128 : 256; }

template <int MODE, bool BATCH, int MINB, bool UNI>
__global__ void __launch_bounds__(wave_max_threads<MINB>(), MINB) wave_kernel(const DevParams P0,
                                                      const WaveArgs* __restrict__ A,
                                                      WaveCtrl* __restrict__ ctrl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t nwarps = blockDim.x >> 5;
  // [pantries: nwarps x 32 x 112 B][block histograms (tally), bin weights (adjoint)
  //  or, batched tally, per-warp event slots: nwarps x 2 x 8 u32 counters, then
  //  nwarps x 2 x n_bins u32 bins when n_bins <= kSlotBins]
  constexpr bool kSlots = BATCH && MODE == kModeTally;
  constexpr bool kAdj = MODE == kModeAdjoint || MODE == kModeMoments;  // replay modes
  float4* pantry = reinterpret_cast<float4*>(smem_raw + warp * kPantryBytesPerWarp);
  unsigned char* extra = smem_raw + nwarps * kPantryBytesPerWarp;
  uint32_t* s_hist = reinterpret_cast<uint32_t*>(extra);
  double* s_w = reinterpret_cast<double*>(extra);
  double* s_mom = s_w + (A->tc.time_bins + 1u);  // adjoint, moments_smem: [time_bins + 1][5]
  uint32_t* s_evc = reinterpret_cast<uint32_t*>(extra) + warp * 16u;
  __shared__ double s_red[4][16];

  // Wave-constant values live in shared memory, not in each thread's registers.
  struct WaveShared {
    const float4* qin;
    float4* qout;
    unsigned long long fresh_next, first_id, iter_cap;
    uint32_t n_in, items, T, cadence, qcap, chunk, ev_shift, tail_steps, slot_cache;
    const uint32_t* tally_of;
    TallyDev tc;
  };
  __shared__ WaveShared ws;
  if (threadIdx.x == 0) {
    const uint32_t wave = ctrl->wave;
    ws.n_in = ctrl->n_in;
    ws.items = ws.n_in + ctrl->fresh_count;
    ws.fresh_next = ctrl->fresh_next;
    ws.qin = (wave & 1u) ? A->qb : A->qa;
    ws.qout = (wave & 1u) ? A->qa : A->qb;
    ws.T = A->threshold;
    ws.cadence = A->cadence;
    ws.qcap = A->qcap;
    ws.first_id = A->first_id;
    ws.iter_cap = A->iter_cap;
    ws.chunk = A->chunk < 32u ? 32u : A->chunk;
    ws.tally_of = A->tally_of;
    ws.ev_shift = A->ev_shift;
    ws.tail_steps = A->tail_steps < 1u ? 1u : A->tail_steps;
    ws.slot_cache = A->slot_cache;
    ws.tc = A->tc;
  }
  __syncthreads();
  const uint32_t& n_in = ws.n_in;
  const uint32_t& items = ws.items;
  const unsigned long long& fresh_next = ws.fresh_next;
  const uint32_t& T = ws.T;
  const uint32_t& cadence = ws.cadence;
  const uint32_t& qcap = ws.qcap;
  const unsigned long long& first_id = ws.first_id;
  const unsigned long long& iter_cap = ws.iter_cap;
  const uint32_t& wchunk = ws.chunk;
  const uint32_t& tail_steps = ws.tail_steps;
  // Event of a record (a genstep's event; a plain batch's records are its events).
  auto event_of = [&](uint32_t rec) -> uint32_t {
    const uint32_t* m = ws.tally_of;
    return m == nullptr ? rec : __ldg(m + rec);
  };
  const TallyDev& tc = ws.tc;
  const uint32_t n_bins = tc.len - 7u;
  const bool slot_bins = n_bins <= kSlotBins;
  uint32_t* s_sb = reinterpret_cast<uint32_t*>(extra + nwarps * kSlotCounterBytesPerWarp) +
                   warp * 2u * n_bins;  // this warp's [2][n_bins] (when slot_bins)

  if (MODE == kModeTally && !BATCH) {
    for (uint32_t b = threadIdx.x; b < n_bins; b += blockDim.x) s_hist[b] = 0u;
  }
  if (kSlots) {
    if (lane < 16u) s_evc[lane] = 0u;
    if (slot_bins) {
      for (uint32_t b = lane; b < 2u * n_bins; b += 32u) s_sb[b] = 0u;
    }
  }
  if (kAdj) {
    const double* wb = A->w_bin;
    for (uint32_t b = threadIdx.x; b <= tc.time_bins; b += blockDim.x) s_w[b] = wb ? wb[b] : 0.0;
    if (MODE == kModeMoments && A->moments_smem) {
      for (uint32_t i = threadIdx.x; i < 5u * (tc.time_bins + 1u); i += blockDim.x) s_mom[i] = 0.0;
    }
  }
  __syncthreads();

  Photon s{};
  Rng r{};
  ScoreAux aux{0u, 0.0f};
  uint32_t pidx = 0u, ev = 0u;
  bool alive = false;
  bool exhausted = false;  // warp-uniform: the wave's work items are all handed out
  uint32_t pc = 0u;        // warp-uniform: photons waiting in this warp's pantry
  uint32_t wsteps = 0u;
  // Warp-uniform bookkeeping: the work items [chunk_lo, chunk_hi) claimed by this
  // warp and not yet emitted; batched, the events cached in its two shared-memory
  // slots and the slot replaced next. Batched variants keep these in shared
  // memory (measured: fewer local-memory spills, -2.5 % per photon-step on the
  // batch), the single-configuration ones in registers.
  constexpr uint32_t kNoEvent = 0xffffffffu;
  // [warp][chunk_lo, chunk_hi, tag0, tag1, victim, photons since the last slot flush]
  __shared__ uint32_t s_book[8][8];
  uint32_t r_book[6] = {0u, 0u, kNoEvent, kNoEvent, 0u, 0u};
  uint32_t* book = BATCH ? s_book[warp] : r_book;
  if (BATCH && lane < 6u) s_book[warp][lane] = (lane == 2u || lane == 3u) ? kNoEvent : 0u;
  __syncwarp();
  uint32_t& chunk_lo = book[0];
  uint32_t& chunk_hi = book[1];
  uint32_t& tag0 = book[2];
  uint32_t& tag1 = book[3];
  uint32_t& victim = book[4];
  uint32_t& since = book[5];
  // Single configuration: per-lane tallies, flushed at the end of the wave.
  uint32_t f0 = 0, f1 = 0, f2 = 0, f3 = 0, f4 = 0, snb = 0, sns = 0;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0;
  uint32_t useful = 0u, iters = 0u;

  // Warp-collective: adds slot v's counters and bins to event `tag`'s tally
  // slice and clears the slot.
  auto flush_slot = [&](uint32_t v, uint32_t tag) {
    __syncwarp();
    if (tag != kNoEvent) {
      unsigned long long* G = A->tally + static_cast<size_t>(tag) * tc.len;
      if (lane < 7u) {  // 5 fates, then the nb and ns sums (the last two entries)
        const uint32_t c = s_evc[v * 8u + lane];
        if (c != 0u) {
          atomicAdd(&G[lane < 5u ? lane : tc.len - 7u + lane], static_cast<unsigned long long>(c));
          s_evc[v * 8u + lane] = 0u;
        }
      }
      if (slot_bins) {
        uint32_t* sb = s_sb + v * n_bins;
        for (uint32_t b = lane; b < n_bins; b += 32u) {
          const uint32_t c = sb[b];
          if (c != 0u) {
            atomicAdd(&G[5u + b], static_cast<unsigned long long>(c));
            sb[b] = 0u;
          }
        }
      }
    }
    __syncwarp();
  };

  // Bookkeeping of a finished photon.
  auto finish = [&](uint32_t fate, const DevParams& P) {
    if (MODE == kModeRecords) {
      store_record(A->rec, pidx, s, fate);
    } else if (MODE == kModeTally && BATCH) {
      // 32-bit shared-memory atomics into the event's slot when the warp caches
      // it (a 64-bit shared-memory add is not one atomic instruction: u64 slots
      // measured +10 % per photon-step on the batch), else 64-bit global atomics into the event's
      // slice. Events are cached only when every record's max_steps is below
      // kSlotMaxAdd (so is each photon's nb and ns), and the warp flushes its
      // slots every kSlotFlushPhotons photons (at a refill): no u32 counter wraps.
      const int slot = ev == tag0 ? 0 : (ev == tag1 ? 1 : -1);
      unsigned long long* G = A->tally + static_cast<size_t>(ev) * tc.len;
      if (slot >= 0) {
        uint32_t* C = s_evc + slot * 8;
        atomicAdd(&C[fate], 1u);
        if (s.nb) atomicAdd(&C[5], s.nb);
        if (s.ns) atomicAdd(&C[6], s.ns);
      } else {
        atomicAdd(&G[fate], 1ull);
        if (s.nb) atomicAdd(&G[tc.len - 2u], static_cast<unsigned long long>(s.nb));
        if (s.ns) atomicAdd(&G[tc.len - 1u], static_cast<unsigned long long>(s.ns));
      }
      if (fate == kDetected) {
        const uint32_t tb = time_bin(s.t, tc.tscale, tc.time_bins);
        const uint32_t xb = tc.time_bins + 1u + xy_bin(s.px, s.py, P, tc.xy_bins);
        if (slot >= 0 && slot_bins) {
          uint32_t* sb = s_sb + static_cast<uint32_t>(slot) * n_bins;
          atomicAdd(&sb[tb], 1u);
          atomicAdd(&sb[xb], 1u);
        } else {
          atomicAdd(&G[5u + tb], 1ull);
          atomicAdd(&G[5u + xb], 1ull);
        }
      }
    } else if (MODE == kModeTally) {
      f0 += fate == 0u;
      f1 += fate == 1u;
      f2 += fate == 2u;
      f3 += fate == 3u;
      f4 += fate == 4u;
      // Per-lane step sums stay far below 2^31 between flushes (a lane sees at
      // most wave_quota / lanes photons of max_steps steps); flush early if not.
      if (snb > 0x7fffffffu || sns > 0x7fffffffu) {
        atomicAdd(&A->tally[tc.len - 2u], static_cast<unsigned long long>(snb));
        atomicAdd(&A->tally[tc.len - 1u], static_cast<unsigned long long>(sns));
        snb = sns = 0u;
      }
      snb += s.nb;
      sns += s.ns;
      if (fate == kDetected) {
        atomicAdd(&s_hist[time_bin(s.t, tc.tscale, tc.time_bins)], 1u);
        atomicAdd(&s_hist[tc.time_bins + 1u + xy_bin(s.px, s.py, P, tc.xy_bins)], 1u);
      }
    } else {  // adjoint: score terms of detected photons (see WaveArgs)
      if (fate == kDetected) {
        const uint32_t tb = time_bin(s.t, tc.tscale, tc.time_bins);
        const double w = s_w[tb] + A->w_det;
        double* M = MODE == kModeMoments ? A->moments : nullptr;
        if (w != 0.0 || M != nullptr) {
          const double path = s.path;
          const uint32_t m = A->score_mask;
          const double s0 = (m & 1u) ? path * A->inv_la2 : 0.0;
          const double s1 = (m & 2u) ? path * A->inv_ls2 - static_cast<double>(s.ns) * A->inv_ls : 0.0;
          const double s2 = (m & 4u) ? static_cast<double>(aux.n_refl) * A->inv_r : 0.0;
          const double s3 = (m & 8u) ? static_cast<double>(aux.t_emit) * A->inv_tau2 - A->inv_tau : 0.0;
          g0 += w * s0;
          g1 += w * s1;
          g2 += w * s2;
          g3 += w * s3;
          if (M != nullptr) {  // per-bin (count, score sums): histogram and Jacobian in one pass
            double* mb = (MODE == kModeMoments && A->moments_smem ? s_mom : M) + 5u * tb;
            atomicAdd(mb, 1.0);
            if (s0 != 0.0) atomicAdd(mb + 1, s0);
            if (s1 != 0.0) atomicAdd(mb + 2, s1);
            if (s2 != 0.0) atomicAdd(mb + 3, s2);
            if (s3 != 0.0) atomicAdd(mb + 4, s3);
          }
        }
      }
    }
  };

  // Warp-collective: spill the lanes with `spill` set into the output queue.
  // Returns true for the lanes whose photon went to the queue; when the queue
  // is full the others keep their photon (the capacity only limits compaction).
  bool queue_full = false;  // warp-uniform
  auto spill_lanes = [&](bool spill) -> bool {
    const uint32_t smask = __ballot_sync(kFull, spill);
    if (smask == 0u) return false;
    uint32_t base = 0u;
    if (lane == 0u) base = atomicAdd(&ctrl->n_out, static_cast<unsigned>(__popc(smask)));
    base = __shfl_sync(kFull, base, 0);
    bool done = false;
    if (spill) {
      const uint32_t slot = base + static_cast<uint32_t>(__popc(smask & lt));
      if (slot < qcap) {
        float4* q = ws.qout + qidx(slot);
        q[0] = make_float4(s.px, s.py, s.pz, s.t);
        q[32] = make_float4(s.dx, s.dy, s.dz, s.path);
        q[64] = make_float4(__uint_as_float(s.nb), __uint_as_float(s.ns),
                            __uint_as_float(r.draws()), __uint_as_float(pidx));
        q[96] = make_float4(__uint_as_float(aux.n_refl), aux.t_emit, __uint_as_float(ev), 0.0f);
        done = true;
      }
    }
    if (__ballot_sync(kFull, spill && !done) != 0u) queue_full = true;
    return done;
  };

  for (;;) {
    if (static_cast<unsigned long long>(iters) > iter_cap) {
      if (lane == 0u) atomicOr(&ctrl->error, kErrWatchdog);
      break;
    }
    uint32_t amask = __ballot_sync(kFull, alive);
    uint32_t na = static_cast<uint32_t>(__popc(amask));
    if (na < T) {
      const uint32_t need = 32u - na;
      if (pc < need && !exhausted) {
        // Refill the pantry: all lanes emit (or load) one photon each together,
        // so emission code runs on full warps. Items come from the warp's claimed
        // chunk of consecutive items, then from a newly claimed chunk (one atomic
        // per `chunk` items keeps a warp on one event for many photons).
        const uint32_t room = 32u - pc;
        const uint32_t base1 = chunk_lo;
        const uint32_t got1 = min(room, chunk_hi - chunk_lo);
        chunk_lo += got1;
        uint32_t base2 = 0u, got = got1;
        if (got1 < room) {
          unsigned long long b = 0ull;
          if (lane == 0u) b = atomicAdd(&ctrl->cursor, static_cast<unsigned long long>(wchunk));
          b = __shfl_sync(kFull, b, 0);
          const unsigned long long hi = b + wchunk;
          chunk_lo = b < items ? static_cast<uint32_t>(b) : items;
          chunk_hi = hi < items ? static_cast<uint32_t>(hi) : items;
          const uint32_t got2 = min(room - got1, chunk_hi - chunk_lo);
          base2 = chunk_lo;
          chunk_lo += got2;
          got += got2;
        }
        // A fresh chunk holds >= 32 items unless the wave's items ran out.
        exhausted = got < room;
        uint32_t nev = 0u;
        if (lane < got) {
          const uint32_t item = lane < got1 ? base1 + lane : base2 + (lane - got1);
          Photon ns{};
          Rng nr{};
          ScoreAux na_aux{0u, 0.0f};
          uint32_t npidx;
          if (item < n_in) {
            // A survivor of the previous wave: 4 x 128-bit loads from its tile.
            const float4* q = ws.qin + qidx(item);
            const float4 a = q[0], b = q[32], c = q[64], d = q[96];
            ns.px = a.x; ns.py = a.y; ns.pz = a.z; ns.t = a.w;
            ns.dx = b.x; ns.dy = b.y; ns.dz = b.z; ns.path = b.w;
            ns.nb = __float_as_uint(c.x);
            ns.ns = __float_as_uint(c.y);
            npidx = __float_as_uint(c.w);
            if (kAdj) {
              na_aux.n_refl = __float_as_uint(d.x);
              na_aux.t_emit = d.y;
            }
            nev = __float_as_uint(d.z);
            const DevParams& P = params_of<BATCH, UNI>(P0, A, nev);
            nr.init(first_id + npidx, P.key_lo, P.key_hi, __float_as_uint(c.z));
          } else {
            const unsigned long long g = fresh_next + (item - n_in);
            npidx = static_cast<uint32_t>(g);
            if (BATCH) nev = find_event(A, g, ws.ev_shift);
            const DevParams& R = BATCH ? A->params[nev] : P0;  // the photon's record
            nr.init(first_id + g, R.key_lo, R.key_hi, 0u);
            const float4* sg = A->seg == nullptr ? nullptr : A->seg + 2u * nev;
            start_photon<kAdj>(R, ns, nr, first_id + g, na_aux, sg);
            if (BATCH) nev = event_of(nev);  // from here on the photon needs only its event
          }
          float4* e = pantry + (pc + lane) * 7u;
          e[0] = make_float4(ns.px, ns.py, ns.pz, ns.t);
          e[1] = make_float4(ns.dx, ns.dy, ns.dz, ns.path);
          e[2] = make_uint4_as_float4(ns.nb, ns.ns, npidx, nev);
          e[3] = make_uint4_as_float4(nr.w[0], nr.w[1], nr.w[2], nr.w[3]);
          e[4] = make_uint4_as_float4(nr.w[4], nr.w[5], nr.w[6], nr.w[7]);
          if (kAdj) {
            e[5] = make_float4(__uint_as_float(nr.o), __uint_as_float(nr.blk),
                               __uint_as_float(na_aux.n_refl), na_aux.t_emit);
          } else {
            reinterpret_cast<float2*>(e + 5)[0] =
                make_float2(__uint_as_float(nr.o), __uint_as_float(nr.blk));
          }
        }
        pc += got;
        if (kSlots) {
          // Slots to flush (bit v: slot v), through one flush site. (1) u32 slot
          // counters stay bounded: only photons that entered this warp through
          // its pantry finish here, so flushing both slots once kSlotFlushPhotons
          // photons have entered since the last flush keeps every counter below
          // (kSlotFlushPhotons + 64) x kSlotMaxAdd < 2^32. (2) The newest event
          // takes a slot: the slot of the oldest event of this refill is kept if
          // it has one, else the slots are replaced in turn.
          uint32_t fm = 0u, v = 2u, e_last = kNoEvent;
          since += got;
          if (since >= kSlotFlushPhotons) {
            fm = 3u;
            since = 0u;
          }
          if (got > 0u && ws.slot_cache) {
            const uint32_t e_first = __shfl_sync(kFull, nev, 0);
            e_last = __shfl_sync(kFull, nev, got - 1u);
            if (e_last != tag0 && e_last != tag1) {
              v = tag0 == e_first ? 1u : (tag1 == e_first ? 0u : victim);
              victim = v ^ 1u;
              fm |= 1u << v;
            }
          }
#pragma unroll 1
          for (uint32_t j = 0; j < 2u; ++j) {
            if (fm & (1u << j)) flush_slot(j, j == 0u ? tag0 : tag1);
          }
          if (v == 0u) tag0 = e_last;
          if (v == 1u) tag1 = e_last;
        }
        __syncwarp();
      }
      if (pc > 0u) {
        // Idle lanes take photons from the top of the pantry.
        const uint32_t take = min(need, pc);
        const uint32_t rank = static_cast<uint32_t>(__popc(~amask & lt));
        if (!alive && rank < take) {
          const float4* e = pantry + (pc - 1u - rank) * 7u;
          const float4 a = e[0], b = e[1], c = e[2], d = e[3], f = e[4];
          s.px = a.x; s.py = a.y; s.pz = a.z; s.t = a.w;
          s.dx = b.x; s.dy = b.y; s.dz = b.z; s.path = b.w;
          s.nb = __float_as_uint(c.x);
          s.ns = __float_as_uint(c.y);
          pidx = __float_as_uint(c.z);
          ev = __float_as_uint(c.w);
          r.w[0] = __float_as_uint(d.x); r.w[1] = __float_as_uint(d.y);
          r.w[2] = __float_as_uint(d.z); r.w[3] = __float_as_uint(d.w);
          r.w[4] = __float_as_uint(f.x); r.w[5] = __float_as_uint(f.y);
          r.w[6] = __float_as_uint(f.z); r.w[7] = __float_as_uint(f.w);
          if (kAdj) {
            const float4 h = e[5];
            r.o = __float_as_uint(h.x);
            r.blk = __float_as_uint(h.y);
            aux.n_refl = __float_as_uint(h.z);
            aux.t_emit = h.w;
          } else {
            const float2 h = reinterpret_cast<const float2*>(e + 5)[0];
            r.o = __float_as_uint(h.x);
            r.blk = __float_as_uint(h.y);
          }
          const DevParams& P = params_of<BATCH, UNI>(P0, A, ev);
          wsteps = 0u;
          alive = s.nb + s.ns < P.max_steps;
          if (!alive) finish(kMaxSteps, P);
        }
        pc -= take;
        __syncwarp();
        amask = __ballot_sync(kFull, alive);
        na = static_cast<uint32_t>(__popc(amask));
      }
      if (exhausted && pc == 0u) {
        if (na == 0u) break;
        // A photon moves on to the next wave (compaction into fuller warps) only
        // after `tail_steps` (>= 1) steps in this one: every item of a wave makes
        // progress, so the run ends, and long histories advance many steps per
        // wave instead of one step per wave once the waves are small.
        if (na < T && !queue_full) {
          if (spill_lanes(alive && wsteps >= tail_steps)) alive = false;
          if (__ballot_sync(kFull, alive) == 0u) break;
        }
      }
    }

    // One step for every live lane; the lanes whose photon ended reconverge
    // here to record it together (one pass of the tally code per warp step).
    // Batched variants also reconverge inside the step before the Philox
    // advance (measured: -6 % per photon-step on the batch; the
    // single-configuration kernels gain nothing from it and spill more).
    const uint32_t smask = BATCH ? __ballot_sync(kFull, alive) : 0u;
    uint32_t fate = kMaxSteps;
    bool ended = false;
    if (alive) {
      const DevParams& P = params_of<BATCH, UNI>(P0, A, ev);
      const bool still =
          step_photon<kAdj, BATCH && !UNI>(P, s, r, first_id + pidx, fate, aux, smask);
      ++wsteps;
      ended = !still || s.nb + s.ns >= P.max_steps;  // at max_steps fate stays kMaxSteps
    }
    __syncwarp();
    if (ended) {
      alive = false;
      finish(fate, params_of<BATCH, UNI>(P0, A, ev));
    }
    ++iters;
    useful += na;
    if (cadence != 0u && !queue_full) {  // forced compaction after `cadence` steps in this wave
      if (spill_lanes(alive && wsteps >= cadence)) alive = false;
    }
  }

  // ---- end of this block's share of the wave: flush --------------------------
  if (lane == 0u) {
    atomicAdd(&ctrl->useful, static_cast<unsigned long long>(useful));
    atomicAdd(&ctrl->issued, 32ull * iters);
  }
  if (MODE == kModeTally) {
    if (BATCH) {
      flush_slot(0u, tag0);
      flush_slot(1u, tag1);
    } else {
      const uint32_t r0 = __reduce_add_sync(kFull, f0), r1 = __reduce_add_sync(kFull, f1),
                     r2 = __reduce_add_sync(kFull, f2), r3 = __reduce_add_sync(kFull, f3),
                     r4 = __reduce_add_sync(kFull, f4);
      const unsigned long long wnb = warp_sum_u64(snb), wns = warp_sum_u64(sns);
      unsigned long long* gt = A->tally;
      if (lane == 0u) {
        if (r0) atomicAdd(&gt[0], static_cast<unsigned long long>(r0));
        if (r1) atomicAdd(&gt[1], static_cast<unsigned long long>(r1));
        if (r2) atomicAdd(&gt[2], static_cast<unsigned long long>(r2));
        if (r3) atomicAdd(&gt[3], static_cast<unsigned long long>(r3));
        if (r4) atomicAdd(&gt[4], static_cast<unsigned long long>(r4));
        if (wnb) atomicAdd(&gt[tc.len - 2u], wnb);
        if (wns) atomicAdd(&gt[tc.len - 1u], wns);
      }
      __syncthreads();
      for (uint32_t b = threadIdx.x; b < tc.len - 7u; b += blockDim.x) {
        if (s_hist[b] != 0u) atomicAdd(&gt[5u + b], static_cast<unsigned long long>(s_hist[b]));
      }
    }
  }
  if (kAdj) {
    g0 = warp_sum_f64(g0);
    g1 = warp_sum_f64(g1);
    g2 = warp_sum_f64(g2);
    g3 = warp_sum_f64(g3);
    if (lane == 0u) {
      s_red[0][warp] = g0;
      s_red[1][warp] = g1;
      s_red[2][warp] = g2;
      s_red[3][warp] = g3;
    }
    __syncthreads();
    if (threadIdx.x < 4u) {
      double acc = 0.0;
      for (uint32_t w = 0; w < nwarps; ++w) acc += s_red[threadIdx.x][w];
      if (acc != 0.0) atomicAdd(&A->grad[threadIdx.x], acc);
    }
    if (MODE == kModeMoments && A->moments_smem) {  // every lane's moments are in s_mom (barrier above)
      double* M = A->moments;
      for (uint32_t i = threadIdx.x; i < 5u * (tc.time_bins + 1u); i += blockDim.x) {
        if (s_mom[i] != 0.0) atomicAdd(M + i, s_mom[i]);
      }
    }
  }

  // ---- the last block to finish sets up the next wave --------------------------
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(&ctrl->blocks_done, 1u);
    if (done == gridDim.x - 1u) {
      __threadfence();
      volatile WaveCtrl* vc = ctrl;
      const unsigned n_out = vc->n_out < qcap ? vc->n_out : qcap;  // reservations past qcap were not written
      const unsigned long long next = vc->fresh_next + vc->fresh_count;
      const unsigned long long remaining = A->total - next;
      unsigned long long fresh = remaining < A->wave_quota ? remaining : A->wave_quota;
      if (A->cadence != 0u) {
        const unsigned long long room = qcap > n_out ? qcap - n_out : 0ull;
        if (fresh > room) fresh = room;
      }
      vc->fresh_next = next;
      vc->n_in = n_out;
      vc->fresh_count = static_cast<unsigned>(fresh);
      vc->n_out = 0u;
      vc->cursor = 0u;
      vc->blocks_done = 0u;
      vc->spills = vc->spills + n_out;
      vc->wave = vc->wave + 1u;
      if (vc->wave >= A->wave_cap && (n_out + fresh) > 0ull) vc->error = vc->error | kErrWatchdog;
      const bool more = (n_out + fresh) > 0ull && vc->error == 0u;
      vc->active = more ? 1u : 0u;
      __threadfence();
      if (!more && A->use_graph != 0u) cudaGraphSetConditional(A->graph_handle, 0u);
    }
  }
}

// ---------------------------------------------------------------------------
// Per-interaction sorted run: photons between steps wait in the state queue of
// their pending interaction (Rayleigh scatter, a polished face, a painted face);
// one launch per iteration. The launch's work items are the three input queues
// and the iteration's fresh emissions, each segment padded to a multiple of 32,
// so every warp takes 32 photons of one kind: step_act runs warp-uniform (the
// Philox advance once per warp step), then step_move takes each survivor to its
// next interaction and a warp-aggregated append (ballot + one atomic per queue)
// writes it, 5 x 128-bit stores, into that queue of the other parity. Absorption,
// black faces and the step limit end a photon at the move. The last block to
// finish sets up the next iteration: the output queues become the input, fresh
// photons fill the freed slots, and once nothing is left to emit and fewer than
// `drain_below` photons are in flight, one last launch runs every remaining photon
// to its end in place (the fused loop). Records depend only on (seed, photon id),
// so they equal the history kernel's bit for bit.

__device__ __forceinline__ float4 __uint_as_float4(uint4 v) {
  return make_float4(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z),
                     __uint_as_float(v.w));
}

// Offset, in float4, of word group g of queue slot `slot` (tiles of 32 photons).
__device__ __forceinline__ size_t sort_off(uint32_t slot, uint32_t g) {
  return ((static_cast<size_t>(slot >> 5) * kSortVec4 + g) << 5) + (slot & 31u);
}

__global__ void sorted_prep_kernel(const SortArgs A, SortCtrl* __restrict__ ctrl) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (uint32_t p = 0; p < 2u; ++p)
    for (uint32_t q = 0; q < kSortQueues; ++q) ctrl->count[p][q].v = 0u;
  const unsigned long long emit = A.n < A.cap ? A.n : A.cap;
  ctrl->parity = 0u;
  ctrl->emit_base = 0ull;
  ctrl->emit_count = static_cast<unsigned>(emit);
  ctrl->drain = (emit == A.n && emit < A.drain_below) ? 1u : 0u;
  ctrl->blocks_done = 0u;
  ctrl->iter = 0u;
  ctrl->error = 0u;
  ctrl->active = A.n > 0ull ? 1u : 0u;
  for (uint32_t q = 0; q < kSortQueues; ++q) ctrl->queued[q] = 0ull;
  ctrl->drained = 0ull;
}

template <int MINB>
__global__ void __launch_bounds__(kSortThreads, MINB)
    sorted_kernel(const DevParams P, const SortArgs A, SortCtrl* __restrict__ ctrl) {
  // Host-loop launches past the end of the run do nothing (the flag only changes
  // in the last block of a launch, after every block has read it).
  if (ctrl->active == 0u) return;
  __shared__ unsigned long long s_cnt[7];  // 5 fates, sum nb, sum ns
  if (threadIdx.x < 7u) s_cnt[threadIdx.x] = 0ull;
  __syncthreads();

  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t par = ctrl->parity, npar = par ^ 1u;
  const bool drain = ctrl->drain != 0u;
  const uint32_t c0 = ctrl->count[par][0].v, c1 = ctrl->count[par][1].v, c2 = ctrl->count[par][2].v;
  const uint32_t ce = ctrl->emit_count;
  const unsigned long long emit_base = ctrl->emit_base;
  const uint32_t e1 = (c0 + 31u) & ~31u, e2 = e1 + ((c1 + 31u) & ~31u),
                 e3 = e2 + ((c2 + 31u) & ~31u), e4 = e3 + ((ce + 31u) & ~31u);
  const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long* const tally = A.tally;
  const TallyDev tc = A.tc;

  const uint32_t stride = n_warps << 5;

  uint32_t f0 = 0, f1 = 0, f2 = 0, f3 = 0, f4 = 0, snb = 0, sns = 0;
  uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) << 5;
  for (; base < e4; base += stride) {
    // The warp's segment: queue 0, 1, 2, or 3 = fresh emissions (warp-uniform).
    const uint32_t seg = base < e1 ? 0u : (base < e2 ? 1u : (base < e3 ? 2u : 3u));
    const uint32_t start = seg == 0u ? 0u : (seg == 1u ? e1 : (seg == 2u ? e2 : e3));
    const uint32_t cnt = seg == 0u ? c0 : (seg == 1u ? c1 : (seg == 2u ? c2 : ce));
    const uint32_t idx = base - start + lane;
    const bool valid = idx < cnt;

    Photon s;
    Rng r;
    ScoreAux aux{0u, 0.0f};
    uint32_t rel = 0u, fate = kMaxSteps;
    int hit = 0;
    bool live = valid;
    if (valid) {
      if (seg < 3u) {
        // The warp reads one whole tile: 5 coalesced 512-byte loads, streamed
        // past L1 (each photon is read once per iteration).
        const uint4* q = reinterpret_cast<const uint4*>(A.q[par][seg]);
        const float4 v0 = __uint_as_float4(__ldcs(q + sort_off(idx, 0u)));
        const float4 v1 = __uint_as_float4(__ldcs(q + sort_off(idx, 1u)));
        const uint4 v2 = __ldcs(q + sort_off(idx, 2u)), v3 = __ldcs(q + sort_off(idx, 3u)),
                    v4 = __ldcs(q + sort_off(idx, 4u));
        rel = __ldcs(A.qid[par][seg] + idx);
        s.px = v0.x; s.py = v0.y; s.pz = v0.z; s.t = v0.w;
        s.dx = v1.x; s.dy = v1.y; s.dz = v1.z; s.path = v1.w;
        r.w[0] = v2.x; r.w[1] = v2.y; r.w[2] = v2.z; r.w[3] = v2.w;
        r.w[4] = v3.x; r.w[5] = v3.y; r.w[6] = v3.z; r.w[7] = v3.w;
        s.nb = v4.x; s.ns = v4.y;
        r.o = v4.z & 0xffu;
        hit = static_cast<int>(v4.z >> 8);
        r.blk = v4.w;
      } else {
        rel = static_cast<uint32_t>(emit_base + idx);
        r.init(A.first_id + rel, P.key_lo, P.key_hi, 0u);
        start_photon<false>(P, s, r, A.first_id + rel, aux);
      }
    }
    const uint64_t id = A.first_id + rel;
    if (seg < 3u) {
      const uint32_t m = __ballot_sync(kFull, valid);
      if (valid) live = step_act<false>(P, s, r, id, fate, aux, hit, m);
    }

    int next = -1;
    if (drain) {
      // Last launch: the rest of each history in place (transport.hpp:151-159).
      while (live) {
        if (s.nb + s.ns >= P.max_steps) { fate = kMaxSteps; live = false; break; }
        live = step_photon<false>(P, s, r, id, fate, aux);
      }
    } else if (live) {
      // Photons that have made max_steps steps end here (each live step counted
      // one boundary or one scatter).
      if (s.nb + s.ns >= P.max_steps) {
        fate = kMaxSteps;
        live = false;
      } else {
        hit = step_move(P, s, r);
        if (hit == kHitAbsorb) {  // bulk absorption (transport.hpp:98-101)
          fate = kAbsorbedBulk;
          live = false;
        } else if (hit == kHitScatter) {
          next = kQScatter;
        } else {
          const uint32_t model = face_model(P, hit);
          if (model == kBlack) {  // black face: absorbed, no draw (transport.hpp:129-132)
            ++s.nb;
            fate = kAbsorbedSurface;
            live = false;
          } else {
            next = model == kPolished ? kQFresnel : kQPainted;
          }
        }
      }
    }

    // Survivors: warp-aggregated appends to the queue of their next interaction.
    // Lanes 0-2 reserve the warp's slots in the three queues with one atomic
    // instruction (one round trip), then each survivor writes its state.
    const uint32_t m0 = __ballot_sync(kFull, next == static_cast<int>(kQScatter)),
                   m1 = __ballot_sync(kFull, next == static_cast<int>(kQFresnel)),
                   m2 = __ballot_sync(kFull, next == static_cast<int>(kQPainted));
    uint32_t base_q = 0u;
    if (lane < kSortQueues) {
      const uint32_t mq = lane == 0u ? m0 : (lane == 1u ? m1 : m2);
      if (mq != 0u) base_q = atomicAdd(&ctrl->count[npar][lane].v, static_cast<unsigned>(__popc(mq)));
    }
    const uint32_t b0 = __shfl_sync(kFull, base_q, 0), b1 = __shfl_sync(kFull, base_q, 1),
                   b2 = __shfl_sync(kFull, base_q, 2);
    if (next >= 0) {
      const uint32_t mq = next == 0 ? m0 : (next == 1 ? m1 : m2);
      const uint32_t slot = (next == 0 ? b0 : (next == 1 ? b1 : b2)) + __popc(mq & lt);
      if (slot < A.cap) {
        float4* q = A.q[npar][next];
        uint4* qu = reinterpret_cast<uint4*>(q);
        q[sort_off(slot, 0u)] = make_float4(s.px, s.py, s.pz, s.t);
        q[sort_off(slot, 1u)] = make_float4(s.dx, s.dy, s.dz, s.path);
        qu[sort_off(slot, 2u)] = make_uint4(r.w[0], r.w[1], r.w[2], r.w[3]);
        qu[sort_off(slot, 3u)] = make_uint4(r.w[4], r.w[5], r.w[6], r.w[7]);
        qu[sort_off(slot, 4u)] = make_uint4(s.nb, s.ns, r.o | (static_cast<uint32_t>(hit) << 8), r.blk);
        A.qid[npar][next][slot] = rel;
      } else {
        atomicOr(&ctrl->error, kErrQueue);
      }
    }

    // Finished photons: record and tally.
    if (valid && !live) {
      if (A.rec.fate != nullptr) store_record(A.rec, rel, s, fate);
      f0 += fate == 0u;
      f1 += fate == 1u;
      f2 += fate == 2u;
      f3 += fate == 3u;
      f4 += fate == 4u;
      snb += s.nb;
      sns += s.ns;
      if (fate == kDetected && tally != nullptr) {
        atomicAdd(tally + 5u + time_bin(s.t, tc.tscale, tc.time_bins), 1ull);
        atomicAdd(tally + 6u + tc.time_bins + xy_bin(s.px, s.py, P, tc.xy_bins), 1ull);
      }
    }
  }

  // Fates and step sums: warp reductions, shared atomics, one global atomic per
  // block and counter.
  const uint32_t r0 = __reduce_add_sync(kFull, f0), r1 = __reduce_add_sync(kFull, f1),
                 r2 = __reduce_add_sync(kFull, f2), r3 = __reduce_add_sync(kFull, f3),
                 r4 = __reduce_add_sync(kFull, f4);
  const unsigned long long rb = warp_sum_u64(snb), rs = warp_sum_u64(sns);
  if (lane == 0u && tally != nullptr) {
    if (r0) atomicAdd(&s_cnt[0], static_cast<unsigned long long>(r0));
    if (r1) atomicAdd(&s_cnt[1], static_cast<unsigned long long>(r1));
    if (r2) atomicAdd(&s_cnt[2], static_cast<unsigned long long>(r2));
    if (r3) atomicAdd(&s_cnt[3], static_cast<unsigned long long>(r3));
    if (r4) atomicAdd(&s_cnt[4], static_cast<unsigned long long>(r4));
    if (rb) atomicAdd(&s_cnt[5], rb);
    if (rs) atomicAdd(&s_cnt[6], rs);
  }
  __syncthreads();
  if (threadIdx.x < 7u && tally != nullptr && s_cnt[threadIdx.x] != 0ull) {
    const uint32_t at = threadIdx.x < 5u ? threadIdx.x : tc.len - 7u + threadIdx.x;
    atomicAdd(tally + at, s_cnt[threadIdx.x]);
  }

  // ---- the last block to finish sets up the next iteration ----------------------
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(&ctrl->blocks_done, 1u);
    if (done == gridDim.x - 1u) {
      __threadfence();
      volatile SortCtrl* vc = ctrl;
      unsigned long long live = 0ull;
      for (uint32_t q = 0; q < kSortQueues; ++q) {
        unsigned int k = vc->count[npar][q].v;
        if (k > A.cap) k = A.cap;  // appends past cap were not written (error set)
        vc->count[npar][q].v = k;
        vc->queued[q] = vc->queued[q] + k;
        vc->count[par][q].v = 0u;
        live += k;
      }
      if (vc->drain) vc->drained = vc->drained + (static_cast<unsigned long long>(c0) + c1 + c2 + ce);
      const unsigned long long next = vc->emit_base + vc->emit_count;
      const unsigned long long remaining = A.n - next;
      const unsigned long long room = A.cap > live ? A.cap - live : 0ull;
      const unsigned long long emit = remaining < room ? remaining : room;
      vc->emit_base = next;
      vc->emit_count = static_cast<unsigned>(emit);
      vc->parity = npar;
      vc->drain = (emit == remaining && live + emit < A.drain_below) ? 1u : 0u;
      vc->iter = vc->iter + 1u;
      vc->blocks_done = 0u;
      bool more = live + emit > 0ull && vc->error == 0u;
      if (more && vc->iter >= A.iter_cap) {
        vc->error = vc->error | kErrWatchdog;
        more = false;
      }
      vc->active = more ? 1u : 0u;
      __threadfence();
      if (!more && A.use_graph != 0u) cudaGraphSetConditional(A.graph_handle, 0u);
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers.

cudaError_t launch_history_records(const DevParams& P, uint64_t first_id, uint64_t n,
                                   const DevRecords& out, int block, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  // At most one wave of resident blocks: each thread runs several histories.
  int dev = 0, sms = 1, bps = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, history_records_kernel, block, 0) != cudaSuccess ||
      bps < 1)
    bps = 1;
  const uint64_t grid = std::min<uint64_t>((n + block - 1) / block, static_cast<uint64_t>(bps) * sms);
  history_records_kernel<<<static_cast<unsigned>(grid), block, 0, st>>>(P, first_id, n, out);
  return cudaGetLastError();
}

int history_tally_blocks_per_sm(int block, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, history_tally_kernel, block, smem) !=
      cudaSuccess)
    return 0;
  return b;
}

cudaError_t launch_history_tally(const DevParams& P, const TallyDev& tc, uint64_t first_id,
                                 uint64_t n, unsigned long long* tally, int block, int grid,
                                 cudaStream_t st) {
  const size_t smem = static_cast<size_t>(tc.len - 7u) * sizeof(uint32_t);
  if (smem > kDynSmemOptIn) {
    const cudaError_t e = cudaFuncSetAttribute(
        history_tally_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
  }
  history_tally_kernel<<<grid, block, smem, st>>>(P, tc, first_id, n, tally);
  return cudaGetLastError();
}

const void* wave_prep_fn() { return reinterpret_cast<const void*>(&wave_prep_kernel); }

cudaError_t launch_wave_prep(const WaveArgs* A_dev, WaveCtrl* ctrl, int grid, int block,
                             cudaStream_t st) {
  wave_prep_kernel<<<grid, block, 0, st>>>(A_dev, ctrl);
  return cudaGetLastError();
}

template <int MODE, bool BATCH, bool UNI>
static const void* kfn(int minb) {
  switch (minb) {
    case 3: return reinterpret_cast<const void*>(&wave_kernel<MODE, BATCH, 3, UNI>);
    case 4: return reinterpret_cast<const void*>(&wave_kernel<MODE, BATCH, 4, UNI>);
    case 7: return reinterpret_cast<const void*>(&wave_kernel<MODE, BATCH, 7, UNI>);
    default: return reinterpret_cast<const void*>(&wave_kernel<MODE, BATCH, 2, UNI>);
  }
}

template <int MODE>
static const void* kfn_variant(int batch, int minb) {
  switch (batch) {
    case kBatchUniform: return kfn<MODE, true, true>(minb);
    case kBatch: return kfn<MODE, true, false>(minb);
    default: return kfn<MODE, false, false>(minb);
  }
}

const void* wave_kernel_fn(int mode, int batch, int minb) {
  switch (mode) {
    case kModeTally: return kfn_variant<kModeTally>(batch, minb);
    case kModeRecords: return kfn_variant<kModeRecords>(batch, minb);
    case kModeMoments:  // single configuration only (the host checks)
      return batch == kSingle ? kfn<kModeMoments, false, false>(minb) : nullptr;
    default: return kfn_variant<kModeAdjoint>(batch, minb);
  }
}

int wave_blocks_per_sm(int mode, int batch, int minb, int block, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, wave_kernel_fn(mode, batch, minb), block,
                                                    smem) != cudaSuccess)
    return 0;
  return b;
}

cudaError_t wave_set_smem(int mode, int batch, int minb, size_t smem) {
  return cudaFuncSetAttribute(wave_kernel_fn(mode, batch, minb),
                              cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
}

cudaError_t launch_wave(int mode, int batch, int minb, const DevParams& P, const WaveArgs* A_dev,
                        WaveCtrl* ctrl, int grid, int block, size_t smem, cudaStream_t st) {
  void* args[] = {const_cast<DevParams*>(&P), &A_dev, &ctrl};
  return cudaLaunchKernel(wave_kernel_fn(mode, batch, minb), dim3(grid), dim3(block), args, smem, st);
}

const void* sorted_prep_fn() { return reinterpret_cast<const void*>(&sorted_prep_kernel); }
const void* sorted_kernel_fn(int minb) {
  return minb == 3 ? reinterpret_cast<const void*>(&sorted_kernel<3>)
                   : reinterpret_cast<const void*>(&sorted_kernel<4>);
}

cudaError_t launch_sorted(int minb, const DevParams& P, const SortArgs& A, SortCtrl* ctrl, int grid,
                          int block, cudaStream_t st) {
  void* args[] = {const_cast<DevParams*>(&P), const_cast<SortArgs*>(&A), &ctrl};
  return cudaLaunchKernel(sorted_kernel_fn(minb), dim3(grid), dim3(block), args, 0, st);
}

cudaError_t launch_sorted_prep(const SortArgs& A, SortCtrl* ctrl, cudaStream_t st) {
  sorted_prep_kernel<<<1, 32, 0, st>>>(A, ctrl);
  return cudaGetLastError();
}

int sorted_blocks_per_sm(int minb, int block) {
  const void* fn = sorted_kernel_fn(minb);
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, block, 0) != cudaSuccess) return 0;
  return b < minb ? b : minb;
}

cudaError_t launch_event_table(const unsigned long long* offsets, uint32_t n_events,
                               uint32_t* table, unsigned long long total, uint32_t shift,
                               cudaStream_t st) {
  (void)total;  // the records' offsets end at the total
  const unsigned blocks = static_cast<unsigned>(std::min<unsigned long long>((n_events + 7ull) / 8ull, 8192ull));
  if (blocks == 0u) return cudaSuccess;
  event_table_kernel<<<blocks, 256, 0, st>>>(offsets, n_events, table, shift);
  return cudaGetLastError();
}

}  // namespace OPTX_NS
}  // namespace optx
