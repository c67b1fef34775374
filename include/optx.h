/* optx.h - C ABI of the B200 optical-photon transport engine (liboptx.so).
 *
 * Drop-in boundary for the GPU path of the reference project
 * zmeskma/GPU_Optical_photons (file:line below are relative to that project).
 * Every entry point returns an int status (OPTX_OK = 0) and never throws;
 * optx_last_error() gives the message of the calling thread's last failure.
 * Plain pointers and sizes only: no C++ or torch types cross this boundary.
 *
 * Threading: calls from several host threads are serialised per device by the
 * library. Host-buffer calls are synchronous (like the reference); the
 * *_device calls are asynchronous on the given stream (NULL = legacy stream).
 */
#ifndef OPTX_H
#define OPTX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OPTX_ABI_VERSION 1

/* Status codes. */
#define OPTX_OK 0
#define OPTX_ERR_INVALID_ARGUMENT 1 /* reference: std::invalid_argument (gpu_event.cu:177-182) */
#define OPTX_ERR_RUNTIME 2          /* reference: std::runtime_error (gpu_backend.cu:171-185) */
#define OPTX_ERR_CUDA 3             /* reference: CUDA_CHECK -> runtime_error (cuda_util.cuh:17-24) */
#define OPTX_ERR_NO_DEVICE 4
#define OPTX_ERR_CAPACITY 5         /* a wavefront state queue overflowed */
#define OPTX_ERR_WATCHDOG 6         /* a device loop hit its iteration cap */

/* Math modes. FAST: CUDA logf/sincosf/cbrtf with FMA contraction (the
 * reference's default GPU build). EXACT: portable log/sincos/cbrt and no FMA
 * (the reference with OPTPHOT_PORTABLE_MATH and OPTPHOT_CUDA_FMAD=OFF); bit-
 * identical to the reference CPU build with OPTPHOT_PORTABLE_MATH. APPROX:
 * the fast kernels compiled with nvcc --use_fast_math (hardware log2 / sin /
 * cos / reciprocal / square root, denormals flushed); its per-photon agreement
 * with the reference CPU build meets the same >= 99.9% bar as FAST (tested). */
#define OPTX_MATH_FAST 0
#define OPTX_MATH_EXACT 1
#define OPTX_MATH_APPROX 2

/* optphot::SimParams, byte for byte (include/optphot/params.hpp:40-63). */
typedef struct optx_params {
  float hx, hy, hz;
  float n_scint, n_det, n_out, abs_length, scat_length;
  uint32_t surface; /* 0 polished, 1 black, 2 specular, 3 lambertian */
  float reflectivity;
  uint32_t source; /* 0 point, 1 uniform in the volume */
  float src_x, src_y, src_z, tau;
  uint32_t max_steps;
  uint64_t seed;
} optx_params;

/* Extension (no reference counterpart): surface model and reflectivity per
 * face 0..4 (0:-x 1:+x 2:-y 3:+y 4:-z); entry 5 (+z readout) is ignored. NULL
 * everywhere it is accepted means `surface` / `reflectivity` on all five faces
 * (params.hpp:60-66, transport.hpp:120-144). */
typedef struct optx_faces {
  uint32_t surface[6];
  float reflectivity[6];
} optx_faces;

/* optphot::TallyConfig (include/optphot/transport.hpp:164-168). */
typedef struct optx_tally_config {
  uint32_t time_bins;
  float time_max;
  uint32_t xy_bins;
} optx_tally_config;

/* Caller-owned structure-of-arrays records, n entries each
 * (optphot::PhotonRecords, include/optphot/backend.hpp:31-50). */
typedef struct optx_records {
  uint8_t* fate;
  uint32_t* n_boundary;
  uint32_t* n_scatter;
  float *t, *x, *y, *z, *path;
} optx_records;

/* optphot::RunTiming (backend.hpp:65-71), milliseconds. */
typedef struct optx_timing {
  double total_ms, kernel_ms, h2d_ms, d2h_ms, alloc_ms;
} optx_timing;

/* optphot::EventStats (backend.hpp:95-103) plus wavefront counters. */
typedef struct optx_event_stats {
  uint64_t launches;          /* waves run (wave-kernel launches) */
  uint64_t useful_lane_steps; /* photon steps done = sum of all photons' steps */
  uint64_t issued_lane_steps; /* 32 x warp step iterations */
  double kernels_ms;          /* device time of the transport */
  uint64_t spills;            /* photons written to the state queue */
} optx_event_stats;

/* Wavefront engine configuration. Zero fields take defaults. */
typedef struct optx_wave_config {
  int32_t block_size;    /* threads per block, multiple of 32, <= 256 (default 256) */
  int32_t blocks_per_sm; /* register budget as resident blocks per SM: 2, 3 or 4 blocks of 256
                            threads (<= 128 / 80 / 64 registers), or 7 blocks of 128 threads
                            (<= 72 registers; needs block_size 128); the persistent grid is that
                            x SMs (default 3) */
  uint32_t threshold;    /* refill a warp when fewer than this many lanes are alive, 1..32 (default 28) */
  uint32_t cadence;      /* steps per photon per wave before a forced spill, 0 = none (default 0) */
  uint64_t wave_quota;   /* fresh photons admitted per wave, 0 = all (default) */
  int32_t use_graph;     /* 1: waves run as a CUDA-graph while loop (default); -1: host loop */
  int32_t math;          /* OPTX_MATH_FAST / OPTX_MATH_EXACT / OPTX_MATH_APPROX */
  uint32_t chunk;        /* consecutive photons a warp claims per grab, 32..2^20 (default 256);
                            results do not depend on it */
  uint32_t max_gensteps; /* capacity for optx_engine_set_gensteps, 0 = none (default) */
  uint32_t tail_steps;   /* at the end of a wave a photon moves on to the next wave only after
                            this many steps in the wave (default 4096: in practice a warp keeps its
                            photons until they finish); results do not depend on it */
  uint32_t reserved;     /* must be 0 */
} optx_wave_config;

/* Extension (no reference counterpart; the reference lists generation on the GPU
 * from gensteps as future work, README.md section 9 item 7): a genstep, the
 * compact description of the photons one charged-particle step emits. Its
 * photons start uniformly on the segment (x0,y0,z0)-(x1,y1,z1), at a time
 * uniform in [t0, t1] plus the event's exponential decay time (tau), with
 * isotropic directions; they consume the same six emission draws as the
 * reference's sources (position fraction, time fraction, one unused word,
 * direction cos theta, azimuth, decay), then transport with the physics of
 * their event and add to that event's tally. */
typedef struct optx_genstep {
  float x0, y0, z0, t0;  /* segment start (mm), emission window start (ns) */
  float x1, y1, z1, t1;  /* segment end (mm), emission window end (ns), t1 >= t0 */
  uint32_t n_photons;    /* photons emitted along this step */
  uint32_t event;        /* index into the events array: physics and tally slice */
} optx_genstep;

/* ---- device ---------------------------------------------------------- */
int optx_abi_version(void);
/* reference: bool gpu_available() (backend.hpp:84) */
int optx_gpu_available(void);
/* reference: std::string gpu_device_name() (backend.hpp:85) */
int optx_gpu_device_name(char* buf, size_t len);
const char* optx_last_error(void);
/* Frees the library's cached device / pinned buffers and graphs. */
int optx_release_cache(void);

/* ---- history kernel, host buffers (the reference's GPU calls) ---------- */
/* reference: RunTiming run_gpu_records(const SimParams&, uint64_t n, PhotonRecords&,
 *   int block_size = 256, uint64_t first_id = 0, uint64_t chunk = 1 << 24)
 *   (backend.hpp:88-89; gpu_backend.cu:119-156). `out` holds n entries per array. */
int optx_run_records(const optx_params* p, const optx_faces* faces, uint64_t n,
                     const optx_records* out, int block_size, uint64_t first_id, uint64_t chunk,
                     int math, optx_timing* timing);
/* reference: RunTiming run_gpu_tally(const SimParams&, const TallyConfig&, uint64_t n,
 *   Tally&, int block_size = 256, uint64_t first_id = 0) (backend.hpp:90-91;
 *   gpu_backend.cu:158-212). tally_out: flat u64 array of
 *   5 + time_bins + 1 + xy_bins^2 + 2 entries = [fate counts | arrival-time histogram
 *   (last bin overflow) | hit map, row-major iy*xy_bins+ix | sum n_boundary | sum n_scatter];
 *   it is overwritten. */
int optx_run_tally(const optx_params* p, const optx_faces* faces, const optx_tally_config* c,
                   uint64_t n, uint64_t* tally_out, int block_size, uint64_t first_id, int math,
                   optx_timing* timing);
/* reference: RunTiming run_gpu_records_event(const SimParams&, uint64_t n, PhotonRecords&,
 *   uint32_t steps_per_launch, int block_size = 256, uint64_t first_id = 0,
 *   uint64_t chunk = 1 << 24, EventStats* = nullptr) (backend.hpp:110-115;
 *   gpu_event.cu:174-244). Runs the wavefront engine with cadence = steps_per_launch:
 *   each photon advances at most that many steps per wave. With steps_per_launch >=
 *   max_steps it runs one wave history style, as the reference's single launch: each
 *   warp holds photons 32w .. 32w + 31 until all have finished, so issued_lane_steps =
 *   sum over groups of 32 x the longest history. Records are bit-identical to
 *   optx_run_records for every steps_per_launch, block_size and chunk. */
int optx_run_records_event(const optx_params* p, const optx_faces* faces, uint64_t n,
                           const optx_records* out, uint32_t steps_per_launch, int block_size,
                           uint64_t first_id, uint64_t chunk, int math, optx_event_stats* stats,
                           optx_timing* timing);

/* ---- device-resident calls (caller device buffers, async on `stream`) --- */
/* Device buffers given to these calls and to optx_engine_run_records /
 * optx_sorted_run are written by kernels: the record arrays n_boundary,
 * n_scatter, t, x, y, z, path must be 4-byte aligned and tallies 8-byte
 * aligned, else OPTX_ERR_INVALID_ARGUMENT before any launch. */
/* History records kernel into device arrays of n entries. */
int optx_records_device(const optx_params* p, const optx_faces* faces, uint64_t n,
                        uint64_t first_id, const optx_records* dev_out, int block_size, int math,
                        void* stream);
/* History tally kernel; ADDS into dev_tally (flat layout as optx_run_tally). */
int optx_tally_device(const optx_params* p, const optx_faces* faces, const optx_tally_config* c,
                      uint64_t n, uint64_t first_id, uint64_t* dev_tally, int block_size, int math,
                      void* stream);

/* ---- per-interaction sorted kernels (extension) -------------------------
 * The design the reference's profiling notes name as the next step after the
 * fused event kernel (PROFILING.md:136-143, README.md:719-720): between steps
 * each photon waits in an HBM state queue for its pending interaction (Rayleigh
 * scatter, a polished face, a painted face), and each warp of an iteration's
 * launch takes 32 photons of one kind, so the interaction code runs without
 * divergence between kinds. One configuration per run; the records equal the
 * history kernel's (optx_records_device) bit for bit, and the tallies
 * optx_tally_device's. */
typedef struct optx_sorted optx_sorted;
typedef struct optx_sorted_counters {
  uint64_t iterations; /* launches of the last run (one per iteration) */
  uint64_t queued[3];  /* photons that went through the scatter, polished-face and
                          painted-face queues */
  uint64_t drained;    /* photons finished by the run's last, in-place launch */
  double kernel_ms;    /* device time of the last run */
} optx_sorted_counters;
/* Sorted-run configuration. Zero fields take defaults. */
typedef struct optx_sorted_config {
  uint32_t capacity;      /* photons in flight = slots per queue, rounded up to 32 (default 2^21);
                             the queues take 2 x 3 x 84 bytes per slot */
  uint32_t drain_below;   /* once nothing is left to emit and fewer photons than this are in
                             flight, one last launch runs each of them to its end (default: the
                             number of resident threads) */
  int32_t math;           /* OPTX_MATH_FAST / OPTX_MATH_EXACT / OPTX_MATH_APPROX */
  int32_t blocks_per_sm;  /* register budget: 4 (64 registers, default) or 3 (80) blocks of 256 */
  uint32_t host_loop;     /* 1: iterations launched from the host (one stream synchronisation per
                             8; optx_sorted_run is then synchronous) instead of a CUDA-graph
                             while loop, for profilers that do not see kernels inside
                             conditional graph nodes */
} optx_sorted_config;
int optx_sorted_create(const optx_sorted_config* cfg, optx_sorted** out);
int optx_sorted_destroy(optx_sorted* s);
/* n photons (ids first_id ..) of one configuration, async on `stream`: ADDS the
 * tally into dev_tally (flat layout as optx_run_tally; NULL = none) and writes
 * dev_records (n entries; NULL = none). n < 2^32. Run errors are reported by
 * the next optx_sorted_stats. A handle has one set of queues: a run given a
 * different stream than the previous run waits on the device for that run to
 * end (runs of one handle never overlap). */
int optx_sorted_run(optx_sorted* s, const optx_params* p, const optx_faces* faces,
                    const optx_tally_config* c, uint64_t n, uint64_t first_id,
                    uint64_t* dev_tally, const optx_records* dev_records, void* stream);
/* Counters of the last run; synchronises `stream`. OPTX_ERR_CAPACITY or
 * OPTX_ERR_WATCHDOG when the run failed. */
int optx_sorted_stats(optx_sorted* s, optx_sorted_counters* stats, void* stream);

/* ---- wavefront engine (extension: persistent, graph-captured, batched) -- */
typedef struct optx_engine optx_engine;
/* An engine for up to max_events events and max_photons photons per run. The
 * tally layout is per event as in optx_run_tally. */
int optx_engine_create(const optx_tally_config* c, uint32_t max_events, uint64_t max_photons,
                       const optx_wave_config* cfg, optx_engine** out);
int optx_engine_destroy(optx_engine* e);
/* Uploads a batch: events[i] (and faces[i] if faces != NULL) with counts[i] photons;
 * event i owns photon ids first_id + sum(counts[0..i-1]) + k, k < counts[i], so its
 * photons are those of the reference's run_cpu_* with first_id = that offset.
 * Asynchronous on `stream` (host arrays are copied before return). */
int optx_engine_set_events(optx_engine* e, const optx_params* events, const optx_faces* faces,
                           const uint64_t* counts, uint32_t n_events, uint64_t first_id,
                           void* stream);
/* Uploads a batch of gensteps (extension, see optx_genstep): n_events events
 * (physics; each event's source fields are ignored) and n_gensteps <= the
 * engine's max_gensteps gensteps in any order of events. The photons of genstep
 * g have the Philox ids first_id + (photons of gensteps 0..g-1) + 0, 1, ...; a
 * run expands them on the device and adds them to per-event tallies (n_events
 * slices). Blocks until the upload is done. */
int optx_engine_set_gensteps(optx_engine* e, const optx_params* events, const optx_faces* faces,
                             uint32_t n_events, const optx_genstep* gensteps, uint32_t n_gensteps,
                             uint64_t first_id, void* stream);
/* The same upload with the gensteps in device memory (extension), for a
 * producer that runs on the GPU: kernels on `stream` build the records, segment
 * table, event indices and photon offsets, and the next run takes its photon
 * total from the device, so neither the upload nor the run waits for the host
 * (the small per-event table in `events` is staged before the call returns).
 * dev_gensteps: device pointer, 4-byte aligned, n_gensteps <= min(max_gensteps,
 * 2^24). The gensteps are checked on the device as optx_engine_set_gensteps
 * checks them on the host; an invalid one, or more photons than the engine
 * holds, is reported as OPTX_ERR_INVALID_ARGUMENT by the next
 * optx_engine_get_tallies / optx_engine_stats (the run then tallies without
 * the invalid gensteps, or nothing when over capacity). Results equal those of
 * optx_engine_set_gensteps with the same gensteps. The photon total is known on
 * the device only: records arrays for optx_engine_run_records must hold the
 * engine's max_photons entries (those past the total are left untouched). */
int optx_engine_set_gensteps_device(optx_engine* e, const optx_params* events,
                                    const optx_faces* faces, uint32_t n_events,
                                    const optx_genstep* dev_gensteps, uint32_t n_gensteps,
                                    uint64_t first_id, void* stream);
/* Runs the uploaded batch; per-event tallies stay on the device (overwritten).
 * Asynchronous on `stream`. */
int optx_engine_run_tally(optx_engine* e, void* stream);
/* Checkpoint and resume of a batched run (the batch's counterpart of the
 * reference's restartable runs: first_id in backend.hpp:84-115 and a Philox
 * stream resumed from its draws, philox.hpp:117-134). Photon i of event j has
 * the relative index offset_j + i (offsets = prefix sums of the counts); a
 * photon's history depends only on (seed, first_id + relative index), so a batch
 * run as consecutive ranges [0, a), [a, b), ... gives the uninterrupted run's
 * tallies exactly. optx_engine_run_tally_range transports the relative photons
 * [lo, hi) in tally mode, async on `stream`; accumulate = 0 zeroes the per-event
 * tallies first (as optx_engine_run_tally does), 1 adds to them. A checkpoint is
 * (the batch, the next relative index, the tallies from
 * optx_engine_get_tallies); to resume — in this process or another — upload the
 * same batch with the same first_id, restore the tallies with
 * optx_engine_set_tallies, and continue with accumulate = 1. Not available after
 * optx_engine_set_gensteps_device (the photon total lives on the device). */
int optx_engine_run_tally_range(optx_engine* e, uint64_t lo, uint64_t hi, int accumulate,
                                void* stream);
/* Replaces the per-event tallies (n_events x tally length u64, host memory),
 * e.g. with a checkpoint's; synchronous on `stream`. */
int optx_engine_set_tallies(optx_engine* e, const uint64_t* host_tallies, void* stream);
/* Runs the uploaded batch writing records (device arrays indexed by photon
 * index relative to first_id, total entries = sum of counts). */
int optx_engine_run_records(optx_engine* e, const optx_records* dev_out, void* stream);
/* Path-replay adjoint (extension; the reference has no differentiation).
 * Replays the uploaded single-configuration batch from the photons' Philox
 * counters (no stored paths) and accumulates, in FP64, for every detected photon
 *   grad[j] += (w_bin[time_bin(t)] + w_det) * S_j
 * with the score S of its history with respect to theta = (abs_length,
 * scat_length, reflectivity, tau):
 *   S_La = path / La^2,  S_Ls = path / Ls^2 - n_scatter / Ls,
 *   S_R = (reflections at painted faces) / R,  S_tau = t_emit / tau^2 - 1 / tau
 * (terms of a disabled process are 0). R is the reflectivity of the painted
 * (specular and Lambertian) faces: with per-face surfaces (optx_faces) they must
 * all have the same reflectivity, else OPTX_ERR_INVALID_ARGUMENT; faces of other
 * models may carry any value. With w_bin = dLoss/dh (h = the run's
 * arrival-time histogram, time_bins + 1 entries) and w_det = dLoss/dD / n
 * (D = detected fraction), grad = dLoss/dtheta. dev_w_bin (time_bins + 1
 * doubles, 8-byte aligned, else OPTX_ERR_INVALID_ARGUMENT), dev_grad (4
 * doubles, overwritten): device pointers. Asynchronous on `stream`; a run that
 * ends on the watchdog or a full state queue is reported by the next
 * optx_engine_stats / optx_engine_get_tallies on the engine. */
int optx_engine_run_adjoint(optx_engine* e, const double* dev_w_bin, double w_det,
                            double* dev_grad, void* stream);
/* Per-bin score moments (extension, same replay as optx_engine_run_adjoint, on
 * an engine holding one configuration: one event, no gensteps):
 * for each arrival-time bin b (time_bins + 1 entries, the last = overflow)
 *   moments[5 b + 0] = detected photons in b  (the run's histogram h_b)
 *   moments[5 b + 1 + j] = sum over them of S_j
 * so that moments[5 b + 1 + j] estimates dE[h_b]/dtheta_j: the Jacobian of the
 * histogram, from which the Poisson Fisher information and Gauss-Newton steps
 * follow without one replay per bin. Counts are exact integers in FP64.
 * dev_moments: device pointer, (time_bins + 1) x 5 doubles, overwritten.
 * Asynchronous on `stream`; run errors are reported as for
 * optx_engine_run_adjoint. */
int optx_engine_run_score_moments(optx_engine* e, double* dev_moments, void* stream);
/* Device pointer of the per-event tallies (n_events x tally length u64). */
int optx_engine_tally_ptr(optx_engine* e, uint64_t** dev_ptr, uint64_t* len_per_event);
/* Copies the per-event tallies to host memory (synchronises `stream`). */
int optx_engine_get_tallies(optx_engine* e, uint64_t* host_out, void* stream);
/* Statistics of the last run (synchronises `stream`). */
int optx_engine_stats(optx_engine* e, optx_event_stats* stats, void* stream);
/* One-shot batched run with host buffers: H2D of the event table, one graph
 * launch, D2H of the per-event tallies (host_tallies: n_events x tally length),
 * with one wait for the run. On an error return host_tallies is unspecified. */
int optx_run_batch(optx_engine* e, const optx_params* events, const optx_faces* faces,
                   const uint64_t* counts, uint32_t n_events, uint64_t first_id,
                   uint64_t* host_tallies, optx_event_stats* stats, optx_timing* timing);

/* One-shot genstep run with host buffers (extension): set_gensteps, one graph
 * launch, D2H of the per-event tallies (host_tallies: n_events x tally length),
 * with one wait for the run. On an error return host_tallies is unspecified. */
int optx_run_gensteps(optx_engine* e, const optx_params* events, const optx_faces* faces,
                      uint32_t n_events, const optx_genstep* gensteps, uint32_t n_gensteps,
                      uint64_t first_id, uint64_t* host_tallies, optx_event_stats* stats,
                      optx_timing* timing);

/* ---- wavefront tally without device allocation -------------------------- */
/* No counterpart in the reference. For callers that cannot call cudaMalloc
 * (the device memory belongs to another runtime or framework allocator, or the
 * process may not grow its device footprint after start-up): the same result as
 * optx_run_tally (the wavefront engine on one configuration, host output), with
 * all device scratch in a static 2.6 MiB array of the library that every GPU
 * loading liboptx.so holds until the process exits. It calls no cudaMalloc,
 * cudaFree or other allocating routine. Limits: n < 2^32, and a tally length
 * (5 + time_bins + 1 + xy_bins^2 + 2) of at most (the device's opt-in shared
 * memory per block - the kernel's static shared memory - 28,672 B of photon
 * pantries) / 4 + 7 entries, capped at 65,536 by the array: 50,927 entries on
 * B200. Larger requests fail with OPTX_ERR_INVALID_ARGUMENT before any launch,
 * and the message gives the device's maximum. The first call on a device looks
 * up the array's device address (make that first call before any stream
 * capture; optx_release_cache makes the next call look it up again, e.g. after
 * a cudaDeviceReset). Every call
 * shares the one array: calls that overlap on the GPU (other streams or host
 * threads) race; the library serialises calls from one process. Synchronous on
 * `stream`; tally_out is a host array, overwritten. */
int optx_wavefront_tally_noalloc(const optx_params* p, const optx_faces* faces,
                                 const optx_tally_config* c, uint64_t n, uint64_t first_id,
                                 uint64_t* tally_out, int math, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPTX_H */
