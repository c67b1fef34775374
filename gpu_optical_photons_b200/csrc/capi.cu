// capi.cu - the extern "C" boundary of liboptx.so (declared in include/optx.h).
//
// Host side of the engine: argument checks with the reference's error
// behaviour (invalid_argument -> OPTX_ERR_INVALID_ARGUMENT, runtime_error ->
// OPTX_ERR_RUNTIME, CUDA_CHECK -> OPTX_ERR_CUDA; src/gpu/gpu_event.cu:177-182,
// src/gpu/gpu_backend.cu:171-185, src/gpu/cuda_util.cuh:17-24 of the reference),
// conversion of SimParams into the kernels' DevParams, cached device buffers,
// timing with CUDA events, and the wavefront engine object (state queues,
// control block, CUDA-graph while loop).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <thread>
#include <tuple>
#include <sys/mman.h>
#include <unistd.h>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/optx.h"
#include "optx_device.cuh"
#include "optx_engine.hpp"

using namespace optx;

namespace {

thread_local std::string g_err;
std::mutex g_mu;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// On failure the thread's last CUDA error is read back (cleared), so that a
// non-sticky error is not reported again by a later, unrelated launch.
#define OPTX_CUDA(call)                                                                   \
  do {                                                                                    \
    const cudaError_t err_ = (call);                                                      \
    if (err_ != cudaSuccess) {                                                            \
      (void)cudaGetLastError();                                                           \
      return fail(OPTX_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(err_) + \
                                     " at " __FILE__ ":" + std::to_string(__LINE__) +     \
                                     " (" #call ")");                                     \
    }                                                                                     \
  } while (0)

#define OPTX_TRY(call)            \
  do {                            \
    const int rc_ = (call);       \
    if (rc_ != OPTX_OK) return rc_; \
  } while (0)

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

constexpr float kSpeedOfLight = 299.792458f;  // mm/ns (hd.hpp:37 of the reference)

// Host-side fault injection for tests (unset in normal use). OPTX_TEST_FAULT=alloc
// makes the engine's device allocations fail as cudaMalloc does when the device
// is out of memory; OPTX_TEST_FAULT=watchdog caps every wavefront run at one wave
// and each warp at one loop iteration, so a run ends through the device-side
// watchdogs (the error word of the control block) instead of finishing.
bool test_fault(const char* what) {
  const char* v = std::getenv("OPTX_TEST_FAULT");
  return v != nullptr && std::strcmp(v, what) == 0;
}

int check_params(const optx_params* p, const optx_faces* f) {
  if (p == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "params must not be NULL");
  if (!(p->hx > 0.0f && p->hy > 0.0f && p->hz > 0.0f) || !std::isfinite(p->hx) ||
      !std::isfinite(p->hy) || !std::isfinite(p->hz))
    return fail(OPTX_ERR_INVALID_ARGUMENT, "box half-sizes must be positive and finite");
  if (!(p->n_scint > 0.0f && p->n_det > 0.0f && p->n_out > 0.0f))
    return fail(OPTX_ERR_INVALID_ARGUMENT, "refractive indices must be positive");
  if (!(p->abs_length > 0.0f) || !(p->scat_length > 0.0f))
    return fail(OPTX_ERR_INVALID_ARGUMENT, "abs_length and scat_length must be > 0 (inf disables)");
  if (p->surface > 3u) return fail(OPTX_ERR_INVALID_ARGUMENT, "surface must be 0..3");
  if (p->source > 1u) return fail(OPTX_ERR_INVALID_ARGUMENT, "source must be 0 (point) or 1 (volume)");
  if (!(p->tau >= 0.0f) || !std::isfinite(p->tau))
    return fail(OPTX_ERR_INVALID_ARGUMENT, "tau must be finite and >= 0");
  if (f != nullptr) {
    for (int i = 0; i < 5; ++i)
      if (f->surface[i] > 3u) return fail(OPTX_ERR_INVALID_ARGUMENT, "face surface must be 0..3");
  }
  return OPTX_OK;
}

// SimParams (+ optional per-face surfaces) -> the kernels' 112-byte record. The
// derived quantities use the reference's float expressions: inv_speed =
// n_scint / c (transport.hpp:74), eta = n1 / n2 and eta * eta (fresnel.hpp:32-33).
DevParams make_dev_params(const optx_params& p, const optx_faces* f) {
  DevParams d;
  std::memset(&d, 0, sizeof(d));
  d.hx = p.hx;
  d.hy = p.hy;
  d.hz = p.hz;
  volatile float ns = p.n_scint;  // keep the host division in float
  d.inv_speed = ns / kSpeedOfLight;
  d.n_scint = p.n_scint;
  d.n_det = p.n_det;
  d.n_out = p.n_out;
  d.abs_length = p.abs_length;
  d.scat_length = p.scat_length;
  d.tau = p.tau;
  d.src_x = p.src_x;
  d.src_y = p.src_y;
  d.src_z = p.src_z;
  uint32_t bits = 0;
  float refl[5];
  for (int i = 0; i < 5; ++i) {
    const uint32_t m = f ? f->surface[i] : p.surface;
    bits |= (m & 3u) << (2 * i);
    refl[i] = f ? f->reflectivity[i] : p.reflectivity;
  }
  d.surf_bits = bits;
  d.refl0 = refl[0];
  d.refl1 = refl[1];
  d.refl2 = refl[2];
  d.refl3 = refl[3];
  d.refl4 = refl[4];
  d.max_steps = p.max_steps;
  d.source = p.source;
  volatile float e1 = p.n_scint / p.n_det;
  volatile float e2 = p.n_scint / p.n_out;
  d.eta2_det = e1 * e1;
  d.eta2_out = e2 * e2;
  d.key_lo = static_cast<uint32_t>(p.seed);
  d.key_hi = static_cast<uint32_t>(p.seed >> 32);
  // Reciprocals for the hit-map binning (xy_bin): float divisions, correctly
  // rounded (2 hx is exact).
  volatile float two_hx = 2.0f * p.hx, two_hy = 2.0f * p.hy;
  d.inv2hx = 1.0f / two_hx;
  d.inv2hy = 1.0f / two_hy;
  return d;
}

int make_tally_dev(const optx_tally_config* c, TallyDev& t) {
  if (c == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "tally config must not be NULL");
  if (c->time_bins == 0u || c->xy_bins == 0u || !(c->time_max > 0.0f))
    return fail(OPTX_ERR_INVALID_ARGUMENT, "tally config needs time_bins, xy_bins >= 1, time_max > 0");
  const uint64_t len = 5ull + c->time_bins + 1ull + static_cast<uint64_t>(c->xy_bins) * c->xy_bins + 2ull;
  if (len > (1ull << 30)) return fail(OPTX_ERR_INVALID_ARGUMENT, "tally too large");
  t.time_bins = c->time_bins;
  volatile float tb = static_cast<float>(c->time_bins);
  t.tscale = tb / c->time_max;  // transport.hpp:171
  t.xy_bins = c->xy_bins;
  t.len = static_cast<uint32_t>(len);
  return OPTX_OK;
}

int check_block(int block) {
  if (block <= 0 || block % 32 != 0 || block > 1024)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "block_size must be a multiple of 32 <= 1024");
  return OPTX_OK;
}

int check_math(int math) {
  if (math != OPTX_MATH_FAST && math != OPTX_MATH_EXACT && math != OPTX_MATH_APPROX)
    return fail(OPTX_ERR_INVALID_ARGUMENT,
                "math must be OPTX_MATH_FAST, OPTX_MATH_EXACT or OPTX_MATH_APPROX");
  return OPTX_OK;
}

int ensure_device() {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(OPTX_ERR_NO_DEVICE, "no CUDA device available");
  }
  OPTX_CUDA(cudaFree(nullptr));  // context creation outside the timed region (cuda_util.cuh:63-65)
  return OPTX_OK;
}

// Forgets the looked-up device addresses of the allocation-free call's static
// scratch (defined with that call, at the end of this file).
void noalloc_forget_addresses();

int num_sms() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

// ---- math-mode dispatch -------------------------------------------------------
#define DISPATCH(math, fn, ...)                          \
  ((math) == OPTX_MATH_EXACT    ? exact::fn(__VA_ARGS__)  \
   : (math) == OPTX_MATH_APPROX ? approx::fn(__VA_ARGS__) \
                                : fast::fn(__VA_ARGS__))

// ---- cached device buffers (per process; the library serialises calls) ---------
// g_cache.rec belongs to optx_run_records_event, which holds g_event_mu for its
// whole call (its engine writes the buffer between its own g_mu sections).
// Lock order: g_event_mu, g_pipe_mu, an API engine's mu, g_mu.
std::mutex g_event_mu;
struct Cache {
  void* rec = nullptr;
  size_t rec_bytes = 0;
  unsigned long long* tally = nullptr;
  size_t tally_bytes = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};
Cache g_cache;

int cache_events() {
  if (g_cache.e0 == nullptr) {
    OPTX_CUDA(cudaEventCreate(&g_cache.e0));
    OPTX_CUDA(cudaEventCreate(&g_cache.e1));
  }
  return OPTX_OK;
}

int cache_records(size_t cap, DevRecords& d) {
  const size_t bytes = cap * (1 + 4 + 4 + 5 * 4) + 8 * 256;
  if (g_cache.rec_bytes < bytes) {
    if (g_cache.rec) cudaFree(g_cache.rec);
    g_cache.rec = nullptr;
    g_cache.rec_bytes = 0;
    OPTX_CUDA(cudaMalloc(&g_cache.rec, bytes));
    g_cache.rec_bytes = bytes;
  }
  auto* base = static_cast<unsigned char*>(g_cache.rec);
  size_t off = 0;
  auto take = [&](size_t b) {
    unsigned char* p = base + off;
    off += (b + 255) & ~size_t(255);
    return p;
  };
  d.fate = take(cap);
  d.n_boundary = reinterpret_cast<uint32_t*>(take(cap * 4));
  d.n_scatter = reinterpret_cast<uint32_t*>(take(cap * 4));
  d.t = reinterpret_cast<float*>(take(cap * 4));
  d.x = reinterpret_cast<float*>(take(cap * 4));
  d.y = reinterpret_cast<float*>(take(cap * 4));
  d.z = reinterpret_cast<float*>(take(cap * 4));
  d.path = reinterpret_cast<float*>(take(cap * 4));
  return OPTX_OK;
}

int cache_tally(size_t len) {
  if (g_cache.tally_bytes < len * 8) {
    if (g_cache.tally) cudaFree(g_cache.tally);
    g_cache.tally = nullptr;
    g_cache.tally_bytes = 0;
    OPTX_CUDA(cudaMalloc(&g_cache.tally, len * 8));
    g_cache.tally_bytes = len * 8;
  }
  return OPTX_OK;
}

int copy_records_d2h(const optx_records* out, uint64_t offset, const DevRecords& d, uint64_t m) {
  OPTX_CUDA(cudaMemcpy(out->fate + offset, d.fate, m, cudaMemcpyDeviceToHost));
  OPTX_CUDA(cudaMemcpy(out->n_boundary + offset, d.n_boundary, m * 4, cudaMemcpyDeviceToHost));
  OPTX_CUDA(cudaMemcpy(out->n_scatter + offset, d.n_scatter, m * 4, cudaMemcpyDeviceToHost));
  OPTX_CUDA(cudaMemcpy(out->t + offset, d.t, m * 4, cudaMemcpyDeviceToHost));
  OPTX_CUDA(cudaMemcpy(out->x + offset, d.x, m * 4, cudaMemcpyDeviceToHost));
  OPTX_CUDA(cudaMemcpy(out->y + offset, d.y, m * 4, cudaMemcpyDeviceToHost));
  OPTX_CUDA(cudaMemcpy(out->z + offset, d.z, m * 4, cudaMemcpyDeviceToHost));
  OPTX_CUDA(cudaMemcpy(out->path + offset, d.path, m * 4, cudaMemcpyDeviceToHost));
  return OPTX_OK;
}

int check_records(const optx_records* r) {
  if (r == nullptr || r->fate == nullptr || r->n_boundary == nullptr || r->n_scatter == nullptr ||
      r->t == nullptr || r->x == nullptr || r->y == nullptr || r->z == nullptr || r->path == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "records: every array must be non-NULL");
  return OPTX_OK;
}

// Device record arrays and tallies are written by kernels: n_boundary, n_scatter
// and the float fields with 4-byte stores, tallies with 64-bit atomics. A
// misaligned pointer would fault the GPU inside the kernel, so it is refused here.
int check_dev_records(const optx_records* r) {
  OPTX_TRY(check_records(r));
  const void* words[7] = {r->n_boundary, r->n_scatter, r->t, r->x, r->y, r->z, r->path};
  for (const void* w : words)
    if ((reinterpret_cast<uintptr_t>(w) & 3u) != 0u)
      return fail(OPTX_ERR_INVALID_ARGUMENT,
                  "device records: n_boundary, n_scatter, t, x, y, z and path must be 4-byte aligned");
  return OPTX_OK;
}

int check_dev_tally(const uint64_t* t) {
  if (t == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "dev_tally must not be NULL");
  if ((reinterpret_cast<uintptr_t>(t) & 7u) != 0u)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "dev_tally must be 8-byte aligned (64-bit atomics)");
  return OPTX_OK;
}

DevRecords to_dev(const optx_records* r) {
  return {r->fate, r->n_boundary, r->n_scatter, r->t, r->x, r->y, r->z, r->path};
}

// ---- gensteps from device memory ------------------------------------------------
// A producer on the GPU (a charged-particle step loop, say) hands its gensteps
// over in device memory: records, segments, event indices and the photon
// offsets are built by kernels, and the run takes its photon total from the
// device, so nothing waits for the host. Offsets come from a two-level scan of
// 4096-genstep tiles, hence at most 4096^2 gensteps per upload.
constexpr uint32_t kScanBlock = 1024;                     // threads per scan block
constexpr uint32_t kScanItems = 4;                        // gensteps per thread
constexpr uint32_t kScanTile = kScanBlock * kScanItems;   // gensteps per scan block
constexpr uint32_t kMaxDeviceGensteps = kScanTile * kScanTile;

// One thread per genstep: its parameter record (its event's physics, source =
// the segment from (x0, y0, z0)), segment entry, event index and photon count
// (the scan's input), with the checks of optx_engine_set_gensteps. An invalid
// genstep sets bit 0 of *error, adds no photons and points at event 0.
__global__ void genstep_records_kernel(const optx_genstep* __restrict__ gs, uint32_t n,
                                       const DevParams* __restrict__ phys, uint32_t n_events,
                                       DevParams* __restrict__ params, float4* __restrict__ seg,
                                       uint32_t* __restrict__ tally_of,
                                       unsigned long long* __restrict__ counts,
                                       unsigned int* __restrict__ error) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const optx_genstep s = gs[g];
  const float v[8] = {s.x0, s.y0, s.z0, s.t0, s.x1, s.y1, s.z1, s.t1};
  bool ok = s.event < n_events && s.t1 >= s.t0;
#pragma unroll
  for (int i = 0; i < 8; ++i) ok = ok && isfinite(v[i]);
  if (!ok) atomicOr(error, 1u);
  const uint32_t ev = ok ? s.event : 0u;
  DevParams d = phys[ev];
  d.source = kSourceSegment;
  d.src_x = s.x0;
  d.src_y = s.y0;
  d.src_z = s.z0;
  params[g] = d;
  seg[2ull * g] = make_float4(s.x1, s.y1, s.z1, s.t0);
  seg[2ull * g + 1] = make_float4(s.t1 - s.t0, 0.0f, 0.0f, 0.0f);
  tally_of[g] = ev;
  counts[g] = ok ? s.n_photons : 0ull;
}

// Exclusive scan of v[0, n) tile by tile (kScanTile entries per block), in
// place; each tile's sum goes to tile_sums[blockIdx.x].
__global__ void __launch_bounds__(kScanBlock) scan_tiles_kernel(unsigned long long* __restrict__ v,
                                                                uint32_t n,
                                                                unsigned long long* __restrict__ tile_sums) {
  __shared__ unsigned long long s[kScanBlock];
  const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
  unsigned long long x[kScanItems], t = 0ull;
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; ++k) {
    x[k] = base + k < n ? v[base + k] : 0ull;
    t += x[k];
  }
  s[threadIdx.x] = t;
  __syncthreads();
  for (uint32_t off = 1; off < kScanBlock; off <<= 1) {  // inclusive scan of the thread sums
    const unsigned long long y = threadIdx.x >= off ? s[threadIdx.x - off] : 0ull;
    __syncthreads();
    s[threadIdx.x] += y;
    __syncthreads();
  }
  unsigned long long run = s[threadIdx.x] - t;
#pragma unroll
  for (uint32_t k = 0; k < kScanItems; ++k) {
    if (base + k < n) v[base + k] = run;
    run += x[k];
  }
  if (threadIdx.x == kScanBlock - 1) tile_sums[blockIdx.x] = s[threadIdx.x];
}

// Adds each tile's prefix to its entries and writes the total to v[n]; a total
// above max_total sets bit 1 of *error and becomes 0 (the run then does nothing).
__global__ void scan_add_kernel(unsigned long long* __restrict__ v, uint32_t n,
                                const unsigned long long* __restrict__ tile_prefix,
                                const unsigned long long* __restrict__ grand, unsigned long long max_total,
                                unsigned int* __restrict__ error) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) v[i] += tile_prefix[i / kScanTile];
  if (i == 0) {
    const unsigned long long total = *grand;
    const bool over = total > max_total;
    if (over) atomicOr(error, 2u);
    v[n] = over ? 0ull : total;
  }
}

// Photon -> record table with the total read from the device (offsets[n_records]).
__global__ void event_table_dev_kernel(const unsigned long long* __restrict__ offsets, uint32_t n_records,
                                       uint32_t* __restrict__ table, uint32_t shift,
                                       unsigned long long entries) {
  const unsigned long long k = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= entries) return;
  const unsigned long long g = k << shift;
  if (g >= offsets[n_records]) return;
  uint32_t lo = 0, hi = n_records;
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (offsets[mid] <= g) lo = mid; else hi = mid;
  }
  table[k] = lo;
}

}  // namespace

// =============================================================================
// Wavefront engine object.
struct optx_engine {
  optx_wave_config cfg{};
  optx_tally_config tcfg{};
  TallyDev tdev{};
  uint32_t max_events = 0;   // tally slices
  uint32_t max_records = 0;  // parameter records (events, or gensteps)
  uint64_t max_photons = 0;
  uint64_t ev_entries = 0;   // capacity of the photon -> record table
  int n_sm = 0;
  uint32_t qcap = 0;
  // device memory
  WaveArgs* d_args = nullptr;
  WaveCtrl* d_ctrl = nullptr;
  DevParams* d_params = nullptr;
  unsigned long long* d_offsets = nullptr;
  uint32_t* d_evtable = nullptr;
  uint32_t* d_tally_of = nullptr;  // genstep -> event (gensteps only)
  DevParams* d_phys = nullptr;     // physics per event (gensteps only)
  float4* d_seg = nullptr;         // genstep segment ends and time windows
  unsigned long long* d_scan = nullptr;  // device genstep uploads: tile sums of the photon scan
  float4* d_qa = nullptr;
  float4* d_qb = nullptr;
  unsigned long long* d_tally = nullptr;
  double* d_grad = nullptr;
  // current batch: n_events records (events or gensteps) adding to n_tallies slices
  uint32_t n_events = 0;
  uint32_t n_tallies = 0;
  uint32_t ev_shift = kEvShift;
  bool gensteps = false;
  bool uniform = false;  // every event has the same step physics (see same_step_physics)
  uint64_t total = 0;              // photons of the batch (device gensteps: the capacity bound)
  // The next run covers relative photons [run_lo, run_hi) and adds to the
  // tallies when run_keep (optx_engine_run_tally_range); a plain run resets them.
  uint64_t run_lo = 0, run_hi = 0;
  bool run_range = false, run_keep = false;
  bool total_on_device = false;    // device gensteps: the run takes its total from d_offsets[n]
  uint64_t first_id = 0;
  DevParams P0{};
  std::vector<DevParams> h_params;
  std::vector<unsigned long long> h_offsets;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool timed = false;
  struct Graph {
    int mode;
    int batch;  // WaveVariant
    int grid, block;
    size_t smem;
    DevParams P0;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    cudaGraphConditionalHandle handle;
  };
  std::vector<Graph> graphs;
};

namespace {

size_t wave_smem(const optx_engine* e, int mode, int variant) {
  const bool batch = variant != kSingle;
  const size_t pantry = static_cast<size_t>(e->cfg.block_size / 32) * kPantryBytesPerWarp;
  if (mode == kModeTally && !batch) return pantry + static_cast<size_t>(e->tdev.len - 7u) * 4u;
  if (mode == kModeAdjoint || mode == kModeMoments)  // bin weights, then the block's moment table
    return pantry + static_cast<size_t>(e->tdev.time_bins + 1u) * 8u +
           (mode == kModeMoments ? moment_smem_bytes(e->tdev.time_bins) : 0u);
  if (mode == kModeTally && batch)  // per-warp event slots
    return pantry + static_cast<size_t>(e->cfg.block_size / 32) *
                        (kSlotCounterBytesPerWarp + slot_bin_bytes_per_warp(e->tdev.len - 7u));
  return pantry;
}

// Register-budget variant of the wave kernel: 2, 3 or 4 blocks of 256 threads
// per SM, or 7 blocks of 128 threads.
int engine_minb(const optx_engine* e) {
  const int b = e->cfg.blocks_per_sm > 0 ? e->cfg.blocks_per_sm : 3;
  if (b == 7) return 7;
  return std::max(2, std::min(4, b));
}

int engine_grid(optx_engine* e, int mode, int batch, int& grid) {
  const size_t smem = wave_smem(e, mode, batch);
  const int math = e->cfg.math;
  const int minb = engine_minb(e);
  int dev = 0, max_smem = 0;
  OPTX_CUDA(cudaGetDevice(&dev));
  OPTX_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  // The opt-in maximum covers the kernel's static shared memory too.
  cudaFuncAttributes fa{};
  OPTX_CUDA(cudaFuncGetAttributes(&fa, DISPATCH(math, wave_kernel_fn, mode, batch, minb)));
  if (smem + fa.sharedSizeBytes > static_cast<size_t>(max_smem))
    return fail(OPTX_ERR_RUNTIME, "wavefront kernel needs " + std::to_string(smem + fa.sharedSizeBytes) +
                                      " bytes of shared memory per block (" + std::to_string(max_smem) +
                                      " available); reduce xy_bins / time_bins");
  if (smem > kDynSmemOptIn) OPTX_CUDA(DISPATCH(math, wave_set_smem, mode, batch, minb, smem));
  int bps = DISPATCH(math, wave_blocks_per_sm, mode, batch, minb, e->cfg.block_size, smem);
  if (bps <= 0) return fail(OPTX_ERR_RUNTIME, "wavefront kernel cannot be resident with this block size / tally");
  if (e->cfg.blocks_per_sm == 7) bps = std::min(bps, 7);
  else if (e->cfg.blocks_per_sm > 0) bps = std::min(bps, e->cfg.blocks_per_sm * (256 / e->cfg.block_size));
  grid = bps * e->n_sm;
  return OPTX_OK;
}

// Writes the WaveArgs for a run (async on stream).
int engine_upload_args(optx_engine* e, int mode, int batch, int grid, cudaGraphConditionalHandle h,
                       const DevRecords* rec, const double* w_bin, double w_det,
                       const double* theta_inv, uint32_t score_mask, cudaStream_t st,
                       double* moments = nullptr) {
  WaveArgs a;
  std::memset(&a, 0, sizeof(a));
  a.params = e->d_params;
  a.phys = e->gensteps ? e->d_phys : e->d_params;
  a.offsets = e->d_offsets;
  a.ev_table = e->d_evtable;
  a.n_events = e->n_events;
  a.n_tallies = e->n_tallies;
  a.ev_shift = e->ev_shift;
  a.tally_of = e->gensteps ? e->d_tally_of : nullptr;
  a.seg = e->gensteps ? e->d_seg : nullptr;
  a.threshold = e->cfg.threshold;
  a.cadence = e->cfg.cadence;
  a.qcap = e->qcap;
  a.total = e->run_range ? e->run_hi : e->total;
  a.item_lo = e->run_range ? e->run_lo : 0ull;
  a.keep_tally = e->run_range && e->run_keep ? 1u : 0u;
  a.first_id = e->first_id;
  a.wave_quota = e->cfg.wave_quota ? e->cfg.wave_quota : (1ull << 31);
  if (a.wave_quota > (1ull << 30)) a.wave_quota = 1ull << 30;
  a.qa = e->d_qa;
  a.qb = e->d_qb;
  a.tally = (mode == kModeTally) ? e->d_tally : nullptr;
  a.tc = e->tdev;
  if (rec) a.rec = *rec;
  a.w_bin = w_bin;
  a.w_det = w_det;
  if (theta_inv) {
    a.inv_la = theta_inv[0];
    a.inv_la2 = theta_inv[1];
    a.inv_ls = theta_inv[2];
    a.inv_ls2 = theta_inv[3];
    a.inv_r = theta_inv[4];
    a.inv_tau = theta_inv[5];
    a.inv_tau2 = theta_inv[6];
  }
  a.score_mask = score_mask;
  a.grad = (mode == kModeAdjoint || mode == kModeMoments) ? e->d_grad : nullptr;
  a.moments = (mode == kModeMoments) ? moments : nullptr;
  a.moments_smem = (a.moments != nullptr && moment_smem_bytes(e->tdev.time_bins) != 0u) ? 1u : 0u;
  a.graph_handle = h;
  // Watchdog: no warp can iterate more than (photons + queue) x (max_steps + 2) times.
  uint32_t max_steps = 0;
  for (const DevParams& p : e->h_params) max_steps = std::max(max_steps, p.max_steps);
  a.iter_cap = (static_cast<unsigned long long>(e->total) + e->qcap + 64ull) *
                   (static_cast<unsigned long long>(max_steps) + 2ull) + 4096ull;
  // Every photon of a wave steps at least once, so a run needs at most about
  // (admission waves) + max_steps waves; the cap only stops a broken run.
  const unsigned long long per_wave = std::max<unsigned long long>(
      1ull, std::min<unsigned long long>(a.wave_quota, e->cfg.cadence ? e->qcap / 2 : a.wave_quota));
  const unsigned long long cap =
      4ull * (max_steps + 2ull) + 4ull * (e->total / per_wave) + 64ull;
  a.wave_cap = static_cast<uint32_t>(std::min<unsigned long long>(std::max(cap, 100000ull), 0xfffffff0ull));
  if (test_fault("watchdog")) {  // both watchdogs fire: one wave, one loop iteration per warp
    a.wave_cap = 1u;
    a.iter_cap = 1ull;
  }
  a.use_graph = (e->cfg.use_graph >= 0) ? 1u : 0u;
  a.chunk = e->cfg.chunk;
  a.tail_steps = e->cfg.tail_steps;
  a.slot_cache = max_steps < kSlotMaxAdd ? 1u : 0u;  // bounds the u32 slot sums
  (void)grid;
  (void)batch;
  OPTX_CUDA(cudaMemcpyAsync(e->d_args, &a, sizeof(a), cudaMemcpyHostToDevice, st));
  return OPTX_OK;
}

int engine_graph(optx_engine* e, int mode, int batch, int grid, optx_engine::Graph** out) {
  const size_t smem = wave_smem(e, mode, batch);
  const DevParams P0 = batch == kBatch ? DevParams{} : e->P0;
  for (auto& g : e->graphs) {
    if (g.mode == mode && g.batch == batch && g.grid == grid && g.block == e->cfg.block_size &&
        g.smem == smem && std::memcmp(&g.P0, &P0, sizeof(P0)) == 0) {
      *out = &g;
      return OPTX_OK;
    }
  }
  optx_engine::Graph g{};
  g.mode = mode;
  g.batch = batch;
  g.grid = grid;
  g.block = e->cfg.block_size;
  g.smem = smem;
  g.P0 = P0;
  const int math = e->cfg.math;
  OPTX_CUDA(cudaGraphCreate(&g.graph, 0));
  OPTX_CUDA(cudaGraphConditionalHandleCreate(&g.handle, g.graph, 1u, cudaGraphCondAssignDefault));

  // prep: reset the control block, zero the tallies
  cudaKernelNodeParams kp{};
  WaveArgs* a_ptr = e->d_args;
  WaveCtrl* c_ptr = e->d_ctrl;
  void* prep_args[] = {&a_ptr, &c_ptr};
  kp.func = const_cast<void*>(DISPATCH(math, wave_prep_fn));
  kp.gridDim = dim3(std::max(1, std::min(grid, 4 * e->n_sm)));
  kp.blockDim = dim3(256);
  kp.sharedMemBytes = 0;
  kp.kernelParams = prep_args;
  cudaGraphNode_t n_prep;
  OPTX_CUDA(cudaGraphAddKernelNode(&n_prep, g.graph, nullptr, 0, &kp));

  // while (active) { wave }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = g.handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t n_while;
  OPTX_CUDA(cudaGraphAddNode(&n_while, g.graph, &n_prep, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];

  DevParams p_copy = P0;
  void* wave_args[] = {&p_copy, &a_ptr, &c_ptr};
  cudaKernelNodeParams wp{};
  wp.func = const_cast<void*>(DISPATCH(math, wave_kernel_fn, mode, batch, engine_minb(e)));
  wp.gridDim = dim3(grid);
  wp.blockDim = dim3(e->cfg.block_size);
  wp.sharedMemBytes = static_cast<unsigned>(smem);
  wp.kernelParams = wave_args;
  cudaGraphNode_t n_wave;
  OPTX_CUDA(cudaGraphAddKernelNode(&n_wave, body, nullptr, 0, &wp));
  OPTX_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
  // Graphs of one configuration bake its parameters in; keep a few.
  constexpr size_t kMaxGraphs = 8;
  if (e->graphs.size() >= kMaxGraphs) {
    cudaGraphExecDestroy(e->graphs.front().exec);
    cudaGraphDestroy(e->graphs.front().graph);
    e->graphs.erase(e->graphs.begin());
  }
  e->graphs.push_back(g);
  *out = &e->graphs.back();
  return OPTX_OK;
}

// Device genstep uploads: the run's photon total is the scan's last entry,
// copied device to device behind the run arguments (no host synchronisation).
int engine_device_total(optx_engine* e, cudaStream_t st) {
  if (e->total_on_device)
    OPTX_CUDA(cudaMemcpyAsync(&e->d_args->total, e->d_offsets + e->n_events, sizeof(unsigned long long),
                              cudaMemcpyDeviceToDevice, st));
  return OPTX_OK;
}

// One complete run of the uploaded batch in `mode` (async on st).
int engine_run(optx_engine* e, int mode, const DevRecords* rec, const double* w_bin, double w_det,
               const double* theta_inv, uint32_t score_mask, cudaStream_t st,
               double* moments = nullptr) {
  if (e->n_events == 0) return fail(OPTX_ERR_INVALID_ARGUMENT, "no events uploaded");
  // Gensteps always run batched: each lane reads its genstep's record at emission.
  const int batch = (e->n_events > 1 || e->gensteps) ? (e->uniform ? kBatchUniform : kBatch) : kSingle;
  int grid = 0;
  OPTX_TRY(engine_grid(e, mode, batch, grid));
  const size_t smem = wave_smem(e, mode, batch);
  const int math = e->cfg.math;
  if (e->cfg.use_graph >= 0) {
    optx_engine::Graph* g = nullptr;
    OPTX_TRY(engine_graph(e, mode, batch, grid, &g));
    OPTX_TRY(engine_upload_args(e, mode, batch, grid, g->handle, rec, w_bin, w_det, theta_inv,
                                score_mask, st, moments));
    OPTX_TRY(engine_device_total(e, st));
    OPTX_CUDA(cudaEventRecord(e->ev0, st));
    OPTX_CUDA(cudaGraphLaunch(g->exec, st));
    OPTX_CUDA(cudaEventRecord(e->ev1, st));
  } else {
    OPTX_TRY(engine_upload_args(e, mode, batch, grid, 0ull, rec, w_bin, w_det, theta_inv,
                                score_mask, st, moments));
    OPTX_TRY(engine_device_total(e, st));
    OPTX_CUDA(cudaEventRecord(e->ev0, st));
    OPTX_CUDA(DISPATCH(math, launch_wave_prep, e->d_args, e->d_ctrl,
                       std::max(1, std::min(grid, 4 * e->n_sm)), 256, st));
    const DevParams P0 = batch == kBatch ? DevParams{} : e->P0;
    for (uint64_t w = 0;; ++w) {
      OPTX_CUDA(DISPATCH(math, launch_wave, mode, batch, engine_minb(e), P0, e->d_args, e->d_ctrl,
                         grid, e->cfg.block_size, smem, st));
      unsigned active = 0;
      OPTX_CUDA(cudaMemcpyAsync(&active, &e->d_ctrl->active, sizeof(active),
                                cudaMemcpyDeviceToHost, st));
      OPTX_CUDA(cudaStreamSynchronize(st));
      if (!active) break;  // the kernel stops the run itself at its wave cap
    }
    OPTX_CUDA(cudaEventRecord(e->ev1, st));
  }
  e->timed = true;
  return OPTX_OK;
}

// Status of a finished run from its control block's error word.
int run_error(unsigned error) {
  if (error & kErrQueue) return fail(OPTX_ERR_CAPACITY, "wavefront state queue overflow");
  if (error & kErrWatchdog) return fail(OPTX_ERR_WATCHDOG, "wavefront iteration cap reached");
  return OPTX_OK;
}

// The error a finished run left in its control block.
int ctrl_error(const WaveCtrl& c) {
  if (c.gs_error & 1u)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "a device genstep is invalid (event index out of range, "
                                           "non-finite coordinate or time, or t1 < t0)");
  if (c.gs_error & 2u)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "device gensteps exceed the engine's max_photons");
  return run_error(c.error);
}

int engine_check_ctrl(optx_engine* e, WaveCtrl& c, cudaStream_t st) {
  OPTX_CUDA(cudaMemcpyAsync(&c, e->d_ctrl, sizeof(c), cudaMemcpyDeviceToHost, st));
  OPTX_CUDA(cudaStreamSynchronize(st));
  return ctrl_error(c);
}

}  // namespace

// Records pipeline: chunk i's kernel runs on the compute stream while chunk
// i-1's records stream to the host on the copy stream, double-buffered on the
// device. Pinned caller arrays receive the DMA directly; pageable ones are
// filled from cached pinned staging buffers by a multi-threaded host copy that
// overlaps the next chunk's kernel (the reference copies synchronously into
// pageable vectors, gpu_backend.cu:119-156, cuda_util.cuh:98-111).
namespace {

struct RecPipe {
  uint64_t cap = 0;  // photons per buffer set
  void* dev[2] = {nullptr, nullptr};
  unsigned char* pin[2] = {nullptr, nullptr};
  cudaStream_t comp = nullptr, copy = nullptr;
  cudaEvent_t k0[2], k1[2], c1[2];
  unsigned* err = nullptr;  // pinned: the engine run's error word per buffer set
  bool events = false;
};
RecPipe g_pipe;

// Structure-of-arrays views of one buffer set of `cap` photons (256-B aligned arrays).
template <class Ptr>
void carve(unsigned char* base, uint64_t cap, Ptr& fate, Ptr (&w)[7]) {
  size_t off = 0;
  auto take = [&](size_t b) {
    unsigned char* q = base + off;
    off += (b + 255) & ~size_t(255);
    return q;
  };
  fate = take(cap);
  for (int i = 0; i < 7; ++i) w[i] = take(cap * 4);
}
size_t set_bytes(uint64_t cap) { return cap + 7 * ((cap * 4 + 255) & ~size_t(255)) + 256; }

int pipe_ensure(uint64_t cap) {
  if (!g_pipe.events) {
    OPTX_CUDA(cudaStreamCreateWithFlags(&g_pipe.comp, cudaStreamNonBlocking));
    OPTX_CUDA(cudaStreamCreateWithFlags(&g_pipe.copy, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
      OPTX_CUDA(cudaEventCreate(&g_pipe.k0[b]));
      OPTX_CUDA(cudaEventCreate(&g_pipe.k1[b]));
      OPTX_CUDA(cudaEventCreate(&g_pipe.c1[b]));
    }
    OPTX_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&g_pipe.err), 2 * sizeof(unsigned),
                            cudaHostAllocDefault));
    g_pipe.events = true;
  }
  if (g_pipe.cap >= cap) return OPTX_OK;
  for (int b = 0; b < 2; ++b) {
    if (g_pipe.dev[b]) cudaFree(g_pipe.dev[b]);
    if (g_pipe.pin[b]) cudaFreeHost(g_pipe.pin[b]);
    g_pipe.dev[b] = nullptr;
    g_pipe.pin[b] = nullptr;
  }
  g_pipe.cap = 0;
  for (int b = 0; b < 2; ++b) {
    OPTX_CUDA(cudaMalloc(&g_pipe.dev[b], set_bytes(cap)));
    OPTX_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&g_pipe.pin[b]), set_bytes(cap),
                            cudaHostAllocDefault));
  }
  g_pipe.cap = cap;
  return OPTX_OK;
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Host threads for copies into pageable memory (up to 8; more compete with the
// staging copies for host memory bandwidth).
unsigned copy_threads() { return std::max(1u, std::min(8u, std::thread::hardware_concurrency())); }

// memcpy of large blocks split over a few host threads.
void parallel_copy(const std::vector<std::tuple<void*, const void*, size_t>>& jobs) {
  size_t total = 0;
  for (auto& j : jobs) total += std::get<2>(j);
  const unsigned hw = copy_threads();
  if (total < (8u << 20) || hw == 1) {
    for (auto& j : jobs) std::memcpy(std::get<0>(j), std::get<1>(j), std::get<2>(j));
    return;
  }
  std::vector<std::thread> th;
  for (unsigned t = 0; t < hw; ++t) {
    th.emplace_back([&, t] {
      for (auto& j : jobs) {
        const size_t b = std::get<2>(j), lo = b * t / hw, hi = b * (t + 1) / hw;
        std::memcpy(static_cast<char*>(std::get<0>(j)) + lo, static_cast<const char*>(std::get<1>(j)) + lo,
                    hi - lo);
      }
    });
  }
  for (auto& x : th) x.join();
}

// Fraction of the pages of [p, p + len) resident in memory (1 when unknown).
double resident_fraction(void* p, size_t len, size_t page) {
  const uintptr_t lo = reinterpret_cast<uintptr_t>(p) & ~(uintptr_t(page) - 1);
  const uintptr_t hi = reinterpret_cast<uintptr_t>(p) + len;
  const size_t pages = (hi - lo + page - 1) / page;
  std::vector<unsigned char> v(pages);
  if (pages == 0 || mincore(reinterpret_cast<void*>(lo), hi - lo, v.data()) != 0) return 1.0;
  size_t r = 0;
  for (unsigned char c : v) r += c & 1u;
  return static_cast<double>(r) / static_cast<double>(pages);
}

// Writes one byte per page of pageable output arrays on host threads, so that
// the first-touch page faults of freshly allocated arrays happen while the GPU
// computes rather than during the copies (measured: 1e7 records into new numpy
// arrays 19.1 -> 15.3 ms). Skipped when most pages are already resident. The
// arrays are overwritten afterwards in full. Joined on destruction (every
// return path).
class PageToucher {
 public:
  PageToucher(const std::vector<std::pair<void*, size_t>>& ranges) {
    size_t total = 0;
    for (auto& r : ranges) total += r.second;
    const unsigned hw = copy_threads();
    if (total < (8u << 20) || hw == 1) return;
    const size_t page = static_cast<size_t>(std::max(4096L, sysconf(_SC_PAGESIZE)));
    size_t res = 0;
    for (auto& r : ranges)
      res += static_cast<size_t>(resident_fraction(r.first, r.second, page) * static_cast<double>(r.second));
    if (res * 2 >= total) return;
    for (unsigned t = 0; t < hw; ++t) {
      th_.emplace_back([ranges, t, hw, page] {
        for (auto& r : ranges) {
          volatile char* q = static_cast<volatile char*>(r.first);
          const size_t lo = r.second * t / hw, hi = r.second * (t + 1) / hw;
          for (size_t off = lo; off < hi; off += page) q[off] = 0;
        }
      });
    }
  }
  void join() {
    for (auto& x : th_) x.join();
    th_.clear();
  }
  ~PageToucher() { join(); }

 private:
  std::vector<std::thread> th_;
};

// ---- engines behind the reference-API host calls ------------------------------
// optx_run_tally and optx_run_records run the wavefront engine: the same
// per-photon arithmetic as the history kernels (bit-identical records, equal
// integer tallies) at 2-4x their speed on one configuration. One engine per
// (device, math mode, tally configuration, photon capacity) is created on first
// use; the most recent kApiMaxEngines are kept (until optx_release_cache). A call
// holds a reference to its engine, so an engine dropped from the cache lives until
// its last call ends; its mutex serialises a call's upload / run / read-back
// sequence. Lock order: g_event_mu, g_pipe_mu, then an engine's mu, then g_mu (taken inside
// the optx_engine_* calls).
struct ApiEngine {
  int device = -1;
  int math = 0;
  optx_tally_config tc{};
  uint64_t cap = 0;
  optx_engine* e = nullptr;
  std::mutex mu;
  ~ApiEngine() { optx_engine_destroy(e); }
};
// Guarded by g_mu, oldest first. Never destroyed: at process exit the CUDA
// runtime may already be gone, so cached engines are not freed then.
std::vector<std::shared_ptr<ApiEngine>>& g_api = *new std::vector<std::shared_ptr<ApiEngine>>();
constexpr size_t kApiMaxEngines = 8;
std::mutex g_pipe_mu;                           // the records pipeline (g_pipe)
constexpr uint64_t kApiMaxCap = 1ull << 27;     // photons per engine run

// Photon capacity of an engine serving runs of n photons: a power of two in
// [2^20, 2^27], so that a few engines serve all sizes.
uint64_t api_capacity(uint64_t n) {
  uint64_t c = 1ull << 20;
  while (c < n && c < kApiMaxCap) c <<= 1;
  return c;
}

// Finds or creates the engine. OPTX_ERR_RUNTIME means the wave kernel cannot be
// resident beside these histograms (the caller then runs the history kernel).
int api_engine(int math, const optx_tally_config& tc, uint64_t cap, std::shared_ptr<ApiEngine>& out) {
  int dev = 0;
  OPTX_CUDA(cudaGetDevice(&dev));
  auto match = [&](const ApiEngine& a) {
    return a.device == dev && a.math == math && a.cap >= cap && a.tc.time_bins == tc.time_bins &&
           a.tc.time_max == tc.time_max && a.tc.xy_bins == tc.xy_bins;
  };
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto& a : g_api)
      if (match(*a)) {
        out = a;
        return OPTX_OK;
      }
  }
  optx_wave_config cfg{};
  cfg.block_size = 128;   // the 72-register budget: 28 warps per SM, the fastest
  cfg.blocks_per_sm = 7;  // single-configuration variant on the reference setups
  cfg.threshold = 28;
  cfg.use_graph = 1;
  cfg.math = math;
  optx_engine* e = nullptr;
  OPTX_TRY(optx_engine_create(&tc, 1, cap, &cfg, &e));
  auto a = std::make_shared<ApiEngine>();
  a->device = dev;
  a->math = math;
  a->tc = tc;
  a->cap = cap;
  a->e = e;
  out = a;
  std::shared_ptr<ApiEngine> dropped;  // released after g_mu
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_api.size() >= kApiMaxEngines) {
    dropped = g_api.front();
    g_api.erase(g_api.begin());
  }
  g_api.push_back(std::move(a));
  return OPTX_OK;
}

}  // namespace

// =============================================================================
extern "C" {

int optx_abi_version(void) { return OPTX_ABI_VERSION; }

int optx_gpu_available(void) {
  int count = 0;
  const bool ok = cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
  if (!ok) cudaGetLastError();
  return ok ? 1 : 0;
}

int optx_gpu_device_name(char* buf, size_t len) {
  if (buf == nullptr || len == 0) return fail(OPTX_ERR_INVALID_ARGUMENT, "buffer must not be empty");
  int dev = 0;
  cudaDeviceProp prop{};
  std::string s = "none";
  if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
    s = std::string(prop.name) + " (sm_" + std::to_string(prop.major) + std::to_string(prop.minor) +
        ", " + std::to_string(prop.multiProcessorCount) + " SMs)";
  } else {
    cudaGetLastError();
  }
  std::snprintf(buf, len, "%s", s.c_str());
  return OPTX_OK;
}

const char* optx_last_error(void) { return g_err.c_str(); }

int optx_release_cache(void) {
  // No records call is in flight while g_event_mu (held to the end, so that
  // g_cache.rec is not in use when it is freed) and g_pipe_mu are held.
  std::lock_guard<std::mutex> elk(g_event_mu);
  std::vector<std::shared_ptr<ApiEngine>> engines;  // destroyed after g_mu, once unused
  {
    // Copies left queued by a records call that returned an error are drained first.
    std::lock_guard<std::mutex> plk(g_pipe_mu);
    if (g_pipe.events) {
      cudaStreamSynchronize(g_pipe.comp);
      cudaStreamSynchronize(g_pipe.copy);
    }
    for (int b = 0; b < 2; ++b) {
      if (g_pipe.dev[b]) cudaFree(g_pipe.dev[b]);
      if (g_pipe.pin[b]) cudaFreeHost(g_pipe.pin[b]);
      g_pipe.dev[b] = nullptr;
      g_pipe.pin[b] = nullptr;
    }
    g_pipe.cap = 0;
    cudaGetLastError();  // release reports nothing; a stale error must not reach the next call
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_cache.rec) cudaFree(g_cache.rec);
    if (g_cache.tally) cudaFree(g_cache.tally);
    if (g_cache.e0) cudaEventDestroy(g_cache.e0);
    if (g_cache.e1) cudaEventDestroy(g_cache.e1);
    g_cache = Cache{};
    engines.swap(g_api);
    // After a device reset the module is loaded again, possibly elsewhere: the
    // next allocation-free call looks the scratch address up afresh.
    noalloc_forget_addresses();
  }
  engines.clear();  // an engine still used by a call is destroyed when that call ends
  return OPTX_OK;
}

int optx_run_records(const optx_params* p, const optx_faces* faces, uint64_t n,
                                const optx_records* out, int block_size, uint64_t first_id,
                                uint64_t chunk, int math, optx_timing* timing) {
  std::lock_guard<std::mutex> lk(g_pipe_mu);
  OPTX_TRY(check_params(p, faces));
  OPTX_TRY(check_block(block_size));
  OPTX_TRY(check_math(math));
  if (n > 0) OPTX_TRY(check_records(out));
  OPTX_TRY(ensure_device());
  optx_timing tm{};
  const auto t0 = std::chrono::steady_clock::now();
  if (n == 0) {
    if (timing) *timing = tm;
    return OPTX_OK;
  }
  const DevParams P = make_dev_params(*p, faces);
  // `chunk` bounds the device memory as in the reference; the pipeline holds two
  // buffer sets of at most 2^22 photons each within it.
  const uint64_t cap = std::max<uint64_t>(
      1, std::min<uint64_t>({n, chunk ? chunk : (uint64_t{1} << 24), uint64_t{1} << 22}));
  const auto ta = std::chrono::steady_clock::now();
  OPTX_TRY(pipe_ensure(cap));
  // The wavefront engine writes each chunk's records (the history kernel when the
  // engine cannot be created, which a records run never needs in practice).
  std::shared_ptr<ApiEngine> ae;
  const optx_tally_config no_tally{1u, 1.0f, 1u};
  const int erc = api_engine(math, no_tally, api_capacity(cap), ae);
  if (erc != OPTX_OK && erc != OPTX_ERR_RUNTIME) return erc;
  std::unique_lock<std::mutex> elk;
  if (erc == OPTX_OK) elk = std::unique_lock<std::mutex>(ae->mu);
  tm.alloc_ms = ms_since(ta);
  void* outs[8] = {out->fate, out->n_boundary, out->n_scatter, out->t, out->x, out->y, out->z, out->path};
  bool direct = true;
  for (void* q : outs) direct = direct && is_pinned(q);
  const size_t elem[8] = {1, 4, 4, 4, 4, 4, 4, 4};
  auto views = [&](int b, bool host) {
    unsigned char* base = host ? g_pipe.pin[b] : static_cast<unsigned char*>(g_pipe.dev[b]);
    unsigned char* fate;
    unsigned char* w[7];
    carve(base, cap, fate, w);
    std::array<unsigned char*, 8> v{fate, w[0], w[1], w[2], w[3], w[4], w[5], w[6]};
    return v;
  };
  const uint64_t chunks = (n + cap - 1) / cap;
  float kms = 0.f, cms = 0.f;
  std::unique_ptr<PageToucher> touch;  // started once the first chunk is queued
  auto host_fill = [&](uint64_t i) {  // staging set (i % 2) -> caller arrays
    if (touch) touch->join();
    const uint64_t done = i * cap, m = std::min(cap, n - done);
    auto src = views(static_cast<int>(i % 2), true);
    std::vector<std::tuple<void*, const void*, size_t>> jobs;
    for (int k = 0; k < 8; ++k)
      jobs.emplace_back(static_cast<char*>(outs[k]) + done * elem[k], src[k], m * elem[k]);
    parallel_copy(jobs);
  };
  for (uint64_t i = 0; i < chunks; ++i) {
    const int b = static_cast<int>(i % 2);
    const uint64_t done = i * cap, m = std::min(cap, n - done);
    auto dv = views(b, false);
    // the device set b is free once the copy of chunk i - 2 has finished
    if (i >= 2) OPTX_CUDA(cudaStreamWaitEvent(g_pipe.comp, g_pipe.c1[b], 0));
    OPTX_CUDA(cudaEventRecord(g_pipe.k0[b], g_pipe.comp));
    const DevRecords d{dv[0], reinterpret_cast<uint32_t*>(dv[1]), reinterpret_cast<uint32_t*>(dv[2]),
                       reinterpret_cast<float*>(dv[3]), reinterpret_cast<float*>(dv[4]),
                       reinterpret_cast<float*>(dv[5]), reinterpret_cast<float*>(dv[6]),
                       reinterpret_cast<float*>(dv[7])};
    if (ae != nullptr) {
      const uint64_t cnt = m;
      const optx_records dr{d.fate, d.n_boundary, d.n_scatter, d.t, d.x, d.y, d.z, d.path};
      OPTX_TRY(optx_engine_set_events(ae->e, p, faces, &cnt, 1, first_id + done, g_pipe.comp));
      OPTX_TRY(optx_engine_run_records(ae->e, &dr, g_pipe.comp));
      OPTX_CUDA(cudaMemcpyAsync(&g_pipe.err[b], &ae->e->d_ctrl->error, sizeof(unsigned),
                                cudaMemcpyDeviceToHost, g_pipe.comp));
    } else {
      OPTX_CUDA(DISPATCH(math, launch_history_records, P, first_id + done, m, d, block_size, g_pipe.comp));
    }
    OPTX_CUDA(cudaEventRecord(g_pipe.k1[b], g_pipe.comp));
    OPTX_CUDA(cudaStreamWaitEvent(g_pipe.copy, g_pipe.k1[b], 0));
    auto hv = views(b, true);
    for (int k = 0; k < 8; ++k) {
      void* dst = direct ? static_cast<void*>(static_cast<char*>(outs[k]) + done * elem[k])
                         : static_cast<void*>(hv[k]);
      OPTX_CUDA(cudaMemcpyAsync(dst, dv[k], m * elem[k], cudaMemcpyDeviceToHost, g_pipe.copy));
    }
    OPTX_CUDA(cudaEventRecord(g_pipe.c1[b], g_pipe.copy));
    if (i == 0 && !direct) {
      std::vector<std::pair<void*, size_t>> ranges;
      for (int k = 0; k < 8; ++k) ranges.emplace_back(outs[k], n * elem[k]);
      touch.reset(new PageToucher(ranges));
    }
    if (i >= 1) {  // finish chunk i - 1 on the host while chunk i computes and copies
      const int pb = static_cast<int>((i - 1) % 2);
      OPTX_CUDA(cudaEventSynchronize(g_pipe.c1[pb]));
      float ms = 0.f;
      OPTX_CUDA(cudaEventElapsedTime(&ms, g_pipe.k0[pb], g_pipe.k1[pb]));
      kms += ms;
      OPTX_CUDA(cudaEventElapsedTime(&ms, g_pipe.k1[pb], g_pipe.c1[pb]));
      cms += ms;
      if (ae != nullptr) OPTX_TRY(run_error(g_pipe.err[pb]));
      if (!direct) host_fill(i - 1);
    }
  }
  const int lb = static_cast<int>((chunks - 1) % 2);
  OPTX_CUDA(cudaEventSynchronize(g_pipe.c1[lb]));
  float ms = 0.f;
  OPTX_CUDA(cudaEventElapsedTime(&ms, g_pipe.k0[lb], g_pipe.k1[lb]));
  kms += ms;
  OPTX_CUDA(cudaEventElapsedTime(&ms, g_pipe.k1[lb], g_pipe.c1[lb]));
  cms += ms;
  if (ae != nullptr) OPTX_TRY(run_error(g_pipe.err[lb]));
  if (!direct) host_fill(chunks - 1);
  tm.kernel_ms = kms;
  tm.d2h_ms = cms;  // kernel end to copy end per chunk (copies overlap later kernels)
  tm.total_ms = ms_since(t0);
  if (timing) *timing = tm;
  return OPTX_OK;
}

// History tally grid: one wave of resident blocks, each thread running its
// photons one after another in one loop (history_loop). Measured on B200 at 1e7
// photons: 1 wave takes 1-14 % less time than 4 waves with that loop.
constexpr uint64_t kHistoryGridWaves = 1;

int optx_run_tally(const optx_params* p, const optx_faces* faces, const optx_tally_config* c,
                   uint64_t n, uint64_t* tally_out, int block_size, uint64_t first_id, int math,
                   optx_timing* timing) {
  OPTX_TRY(check_params(p, faces));
  OPTX_TRY(check_block(block_size));
  OPTX_TRY(check_math(math));
  TallyDev td{};
  OPTX_TRY(make_tally_dev(c, td));
  if (tally_out == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "tally_out must not be NULL");
  OPTX_TRY(ensure_device());
  optx_timing tm{};
  const auto t0 = std::chrono::steady_clock::now();
  if (n > 0) {
    // The wavefront engine, in runs of at most its capacity, tallies summed on the host.
    std::shared_ptr<ApiEngine> ae;
    const int erc = api_engine(math, *c, api_capacity(n), ae);
    if (erc != OPTX_OK && erc != OPTX_ERR_RUNTIME) return erc;
    if (erc == OPTX_OK) {
      tm.alloc_ms = ms_since(t0);
      std::lock_guard<std::mutex> elk(ae->mu);
      std::vector<uint64_t> part(td.len);
      std::memset(tally_out, 0, td.len * 8ull);
      for (uint64_t done = 0; done < n;) {
        const uint64_t m = std::min(ae->cap, n - done);
        OPTX_TRY(optx_engine_set_events(ae->e, p, faces, &m, 1, first_id + done, nullptr));
        OPTX_TRY(optx_engine_run_tally(ae->e, nullptr));
        const auto tc = std::chrono::steady_clock::now();
        OPTX_TRY(optx_engine_get_tallies(ae->e, part.data(), nullptr));
        tm.d2h_ms += ms_since(tc);
        for (uint32_t k = 0; k < td.len; ++k) tally_out[k] += part[k];
        optx_event_stats s{};
        OPTX_TRY(optx_engine_stats(ae->e, &s, nullptr));
        tm.kernel_ms += s.kernels_ms;
        done += m;
      }
      tm.total_ms = ms_since(t0);
      if (timing) *timing = tm;
      return OPTX_OK;
    }
  }
  // The history kernel: n = 0, or the wave kernel's pantries do not fit beside
  // these histograms in shared memory.
  std::lock_guard<std::mutex> lk(g_mu);
  OPTX_TRY(cache_events());
  const DevParams P = make_dev_params(*p, faces);
  const size_t smem = static_cast<size_t>(td.len - 7u) * 4u;
  int dev = 0, max_smem = 0;
  OPTX_CUDA(cudaGetDevice(&dev));
  OPTX_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem > static_cast<size_t>(max_smem))
    return fail(OPTX_ERR_RUNTIME, "tally histograms need " + std::to_string(smem) +
                                      " bytes of shared memory; reduce xy_bins / time_bins");
  const int bps = DISPATCH(math, history_tally_blocks_per_sm, block_size, smem);
  const uint64_t needed = (n + block_size - 1) / block_size;
  const int grid = static_cast<int>(std::max<uint64_t>(
      1, std::min<uint64_t>(needed, kHistoryGridWaves * static_cast<uint64_t>(std::max(bps, 1)) *
                                        num_sms())));
  if (n / grid >= 0xffffffffull)
    return fail(OPTX_ERR_RUNTIME, "too many photons for one tally launch; split the run");
  const auto ta = std::chrono::steady_clock::now();
  OPTX_TRY(cache_tally(td.len));
  OPTX_CUDA(cudaMemset(g_cache.tally, 0, td.len * 8ull));
  tm.alloc_ms = ms_since(ta);
  OPTX_CUDA(cudaEventRecord(g_cache.e0, 0));
  if (n > 0) OPTX_CUDA(DISPATCH(math, launch_history_tally, P, td, first_id, n, g_cache.tally, block_size, grid, nullptr));
  OPTX_CUDA(cudaEventRecord(g_cache.e1, 0));
  OPTX_CUDA(cudaEventSynchronize(g_cache.e1));
  float ms = 0.f;
  OPTX_CUDA(cudaEventElapsedTime(&ms, g_cache.e0, g_cache.e1));
  tm.kernel_ms = ms;
  const auto tc = std::chrono::steady_clock::now();
  OPTX_CUDA(cudaMemcpy(tally_out, g_cache.tally, td.len * 8ull, cudaMemcpyDeviceToHost));
  tm.d2h_ms = ms_since(tc);
  tm.total_ms = ms_since(t0);
  if (timing) *timing = tm;
  return OPTX_OK;
}

int optx_records_device(const optx_params* p, const optx_faces* faces, uint64_t n,
                        uint64_t first_id, const optx_records* dev_out, int block_size, int math,
                        void* stream) {
  OPTX_TRY(check_params(p, faces));
  OPTX_TRY(check_block(block_size));
  OPTX_TRY(check_math(math));
  if (n > 0) OPTX_TRY(check_dev_records(dev_out));
  OPTX_TRY(ensure_device());
  const DevParams P = make_dev_params(*p, faces);
  const DevRecords d = to_dev(dev_out);
  // The grid is 32-bit: launch in pieces of at most 2^31 photons.
  for (uint64_t done = 0; done < n;) {
    const uint64_t m = std::min<uint64_t>(n - done, 1ull << 31);
    DevRecords dd = d;
    dd.fate += done;
    dd.n_boundary += done;
    dd.n_scatter += done;
    dd.t += done;
    dd.x += done;
    dd.y += done;
    dd.z += done;
    dd.path += done;
    OPTX_CUDA(DISPATCH(math, launch_history_records, P, first_id + done, m, dd, block_size,
                       static_cast<cudaStream_t>(stream)));
    done += m;
  }
  return OPTX_OK;
}

int optx_tally_device(const optx_params* p, const optx_faces* faces, const optx_tally_config* c,
                      uint64_t n, uint64_t first_id, uint64_t* dev_tally, int block_size, int math,
                      void* stream) {
  OPTX_TRY(check_params(p, faces));
  OPTX_TRY(check_block(block_size));
  OPTX_TRY(check_math(math));
  TallyDev td{};
  OPTX_TRY(make_tally_dev(c, td));
  OPTX_TRY(check_dev_tally(dev_tally));
  OPTX_TRY(ensure_device());
  const size_t smem = static_cast<size_t>(td.len - 7u) * 4u;
  int dev = 0, max_smem = 0;
  OPTX_CUDA(cudaGetDevice(&dev));
  OPTX_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem > static_cast<size_t>(max_smem))
    return fail(OPTX_ERR_RUNTIME, "tally histograms need " + std::to_string(smem) +
                                      " bytes of shared memory; reduce xy_bins / time_bins");
  if (n == 0) return OPTX_OK;
  const DevParams P = make_dev_params(*p, faces);
  const int bps = DISPATCH(math, history_tally_blocks_per_sm, block_size, smem);
  const uint64_t needed = (n + block_size - 1) / block_size;
  const int grid = static_cast<int>(std::max<uint64_t>(
      1, std::min<uint64_t>(needed, kHistoryGridWaves * static_cast<uint64_t>(std::max(bps, 1)) *
                                        num_sms())));
  if (n / grid >= 0xffffffffull)
    return fail(OPTX_ERR_RUNTIME, "too many photons for one tally launch; split the run");
  OPTX_CUDA(DISPATCH(math, launch_history_tally, P, td, first_id, n,
                     reinterpret_cast<unsigned long long*>(dev_tally), block_size, grid,
                     static_cast<cudaStream_t>(stream)));
  return OPTX_OK;
}

// ---- wavefront engine ---------------------------------------------------------

int optx_engine_create(const optx_tally_config* c, uint32_t max_events, uint64_t max_photons,
                       const optx_wave_config* cfg, optx_engine** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (out == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "out must not be NULL");
  *out = nullptr;
  if (max_events == 0) return fail(OPTX_ERR_INVALID_ARGUMENT, "max_events must be >= 1");
  if (max_photons == 0 || max_photons > 0xffffffffull)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "max_photons must be in [1, 2^32 - 1] per run");
  TallyDev td{};
  OPTX_TRY(make_tally_dev(c, td));
  optx_wave_config k{};
  if (cfg) k = *cfg;
  if (k.block_size == 0) k.block_size = 256;
  if (k.block_size <= 0 || k.block_size % 32 != 0 || k.block_size > 256)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "wavefront block_size must be a multiple of 32 <= 256");
  if (k.blocks_per_sm == 7 && k.block_size != 128)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "blocks_per_sm 7 (72-register budget) needs block_size 128");
  if (k.blocks_per_sm != 0 && k.blocks_per_sm != 7 && (k.blocks_per_sm < 2 || k.blocks_per_sm > 4))
    return fail(OPTX_ERR_INVALID_ARGUMENT, "blocks_per_sm must be 0 (default), 2, 3, 4 or 7");
  if (k.threshold == 0) k.threshold = 28;
  if (k.threshold > 32) return fail(OPTX_ERR_INVALID_ARGUMENT, "threshold must be 1..32");
  if (k.use_graph == 0) k.use_graph = 1;
  if (k.chunk == 0) k.chunk = 256;
  if (k.tail_steps == 0) k.tail_steps = 4096;
  if (k.reserved != 0) return fail(OPTX_ERR_INVALID_ARGUMENT, "reserved must be 0");
  if (k.chunk < 32 || k.chunk > (1u << 20))
    return fail(OPTX_ERR_INVALID_ARGUMENT, "chunk must be in [32, 2^20]");
  if (k.max_gensteps > (1u << 30)) return fail(OPTX_ERR_INVALID_ARGUMENT, "max_gensteps must be <= 2^30");
  OPTX_TRY(check_math(k.math));
  OPTX_TRY(ensure_device());
  auto* e = new optx_engine();
  e->cfg = k;
  e->tcfg = *c;
  e->tdev = td;
  e->max_events = max_events;
  e->max_records = std::max(max_events, k.max_gensteps);
  e->max_photons = max_photons;
  // One table entry per 128 photons at least; finer (down to one per photon)
  // when records are small and the table has room: 2 entries per record.
  e->ev_entries = (max_photons >> kEvShift) + 2ull + 2ull * e->max_records;
  e->n_sm = num_sms();
  auto cleanup = [&](int rc) {
    optx_engine_destroy(e);
    return rc;
  };
  int grid_max = 0;
  for (int mode = 0; mode < 3; ++mode) {
    for (int b = kSingle; b <= kBatchUniform; ++b) {
      int g = 0;
      const int rc = engine_grid(e, mode, b, g);
      if (rc != OPTX_OK && mode == kModeTally) return cleanup(rc);
      grid_max = std::max(grid_max, g);
    }
  }
  const uint64_t lanes = static_cast<uint64_t>(grid_max) * k.block_size;
  uint64_t qcap = lanes;
  if (k.cadence != 0) qcap = std::max<uint64_t>(lanes, std::min<uint64_t>(max_photons, 1ull << 23));
  qcap = (qcap + 31) & ~uint64_t(31);
  e->qcap = static_cast<uint32_t>(qcap);
  auto alloc = [&](void** p, size_t bytes) -> int {
    if (test_fault("alloc"))
      return fail(OPTX_ERR_CUDA, "cudaMalloc: out of memory (injected by OPTX_TEST_FAULT=alloc)");
    const cudaError_t err = cudaMalloc(p, bytes);
    if (err != cudaSuccess) {
      cudaGetLastError();
      return fail(OPTX_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(err));
    }
    return OPTX_OK;
  };
  int rc = OPTX_OK;
  if ((rc = alloc(reinterpret_cast<void**>(&e->d_args), sizeof(WaveArgs))) ||
      (rc = alloc(reinterpret_cast<void**>(&e->d_ctrl), sizeof(WaveCtrl))) ||
      (rc = alloc(reinterpret_cast<void**>(&e->d_params), sizeof(DevParams) * e->max_records)) ||
      (rc = alloc(reinterpret_cast<void**>(&e->d_offsets), 8ull * (e->max_records + 1ull))) ||
      (rc = alloc(reinterpret_cast<void**>(&e->d_evtable), 4ull * e->ev_entries)) ||
      (k.max_gensteps > 0 &&
       (rc = alloc(reinterpret_cast<void**>(&e->d_tally_of), 4ull * k.max_gensteps))) ||
      (k.max_gensteps > 0 &&
       (rc = alloc(reinterpret_cast<void**>(&e->d_seg), 32ull * k.max_gensteps))) ||
      (k.max_gensteps > 0 &&
       (rc = alloc(reinterpret_cast<void**>(&e->d_phys), sizeof(DevParams) * max_events))) ||
      (k.max_gensteps > 0 &&
       (rc = alloc(reinterpret_cast<void**>(&e->d_scan), 8ull * (kScanTile + 1ull)))) ||
      (rc = alloc(reinterpret_cast<void**>(&e->d_qa), qcap * 64ull)) ||
      (rc = alloc(reinterpret_cast<void**>(&e->d_qb), qcap * 64ull)) ||
      (rc = alloc(reinterpret_cast<void**>(&e->d_tally), 8ull * td.len * max_events)) ||
      (rc = alloc(reinterpret_cast<void**>(&e->d_grad), 8ull * 4)))
    return cleanup(rc);
  if (cudaMemset(e->d_ctrl, 0, sizeof(WaveCtrl)) != cudaSuccess) {  // no error, no run yet
    cudaGetLastError();
    return cleanup(fail(OPTX_ERR_CUDA, "cudaMemset of the control block failed"));
  }
  if (cudaEventCreate(&e->ev0) != cudaSuccess || cudaEventCreate(&e->ev1) != cudaSuccess)
    return cleanup(fail(OPTX_ERR_CUDA, "cudaEventCreate failed"));
  *out = e;
  return OPTX_OK;
}

int optx_engine_destroy(optx_engine* e) {
  if (e == nullptr) return OPTX_OK;
  for (auto& g : e->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  cudaFree(e->d_args);
  cudaFree(e->d_ctrl);
  cudaFree(e->d_params);
  cudaFree(e->d_offsets);
  cudaFree(e->d_evtable);
  cudaFree(e->d_tally_of);
  cudaFree(e->d_seg);
  cudaFree(e->d_phys);
  cudaFree(e->d_scan);
  cudaFree(e->d_qa);
  cudaFree(e->d_qb);
  cudaFree(e->d_tally);
  cudaFree(e->d_grad);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  delete e;
  return OPTX_OK;
}

}  // extern "C"

// True when two records have the same step physics (everything a step reads;
// the source fields and tau act at emission only), bit for bit.
static bool same_step_physics(DevParams a, DevParams b) {
  for (DevParams* d : {&a, &b}) {
    d->tau = 0.0f;
    d->src_x = d->src_y = d->src_z = 0.0f;
    d->source = 0u;
    d->pad2 = 0u;
  }
  return std::memcmp(&a, &b, sizeof(DevParams)) == 0;
}

// Uploads the record table and offsets of the current batch and builds the
// photon -> record table at the finest resolution the table holds.
static int engine_upload_records(optx_engine* e, cudaStream_t st) {
  const uint32_t n = e->n_events;
  e->total_on_device = false;
  OPTX_CUDA(cudaMemsetAsync(&e->d_ctrl->gs_error, 0, sizeof(unsigned), st));
  OPTX_CUDA(cudaMemcpyAsync(e->d_params, e->h_params.data(), sizeof(DevParams) * n,
                            cudaMemcpyHostToDevice, st));
  OPTX_CUDA(cudaMemcpyAsync(e->d_offsets, e->h_offsets.data(), 8ull * (n + 1ull),
                            cudaMemcpyHostToDevice, st));
  uint32_t shift = 0;
  while (shift < kEvShift && (e->total >> shift) + 2ull > e->ev_entries) ++shift;
  e->ev_shift = shift;
  if ((n > 1 || e->gensteps) && e->total > 0)
    OPTX_CUDA(DISPATCH(e->cfg.math, launch_event_table, e->d_offsets, n, e->d_evtable, e->total,
                       shift, st));
  return OPTX_OK;
}

static int fill_stats(optx_engine* e, const WaveCtrl& c, optx_event_stats* stats) {
  stats->launches = c.wave;
  stats->useful_lane_steps = c.useful;
  stats->issued_lane_steps = c.issued;
  stats->spills = c.spills;
  float ms = 0.f;
  if (e->timed) OPTX_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
  stats->kernels_ms = ms;
  return OPTX_OK;
}

// End of the one-shot host-buffer runs: one wait for the run. The tallies and
// the control block are copied back together (the tally copy first, so that a
// pageable host_out does not wait twice) and the statistics come from that copy;
// optx_engine_get_tallies followed by optx_engine_stats would wait three times.
static int read_back_one_shot(optx_engine* e, uint64_t* host_tallies, optx_event_stats* stats) {
  std::lock_guard<std::mutex> lk(g_mu);
  WaveCtrl c{};
  OPTX_CUDA(cudaMemcpyAsync(host_tallies, e->d_tally, 8ull * e->tdev.len * e->n_tallies,
                            cudaMemcpyDeviceToHost, nullptr));
  OPTX_CUDA(cudaMemcpyAsync(&c, e->d_ctrl, sizeof(c), cudaMemcpyDeviceToHost, nullptr));
  OPTX_CUDA(cudaStreamSynchronize(nullptr));
  OPTX_TRY(ctrl_error(c));
  return fill_stats(e, c, stats);
}

extern "C" {

int optx_engine_set_events(optx_engine* e, const optx_params* events, const optx_faces* faces,
                           const uint64_t* counts, uint32_t n_events, uint64_t first_id,
                           void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "engine must not be NULL");
  if (n_events == 0 || n_events > e->max_events)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "n_events must be in [1, max_events]");
  if (events == nullptr || counts == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "events and counts must not be NULL");
  // Built aside and committed only when every event is valid: a rejected batch
  // leaves the engine's current batch as it was.
  std::vector<DevParams> hp(n_events);
  std::vector<unsigned long long> ho(n_events + 1ull);
  uint64_t total = 0;
  for (uint32_t i = 0; i < n_events; ++i) {
    OPTX_TRY(check_params(&events[i], faces ? &faces[i] : nullptr));
    hp[i] = make_dev_params(events[i], faces ? &faces[i] : nullptr);
    ho[i] = total;
    total += counts[i];
    if (total > e->max_photons)
      return fail(OPTX_ERR_INVALID_ARGUMENT, "batch exceeds the engine's max_photons");
  }
  ho[n_events] = total;
  e->h_params.swap(hp);
  e->h_offsets.swap(ho);
  e->n_events = n_events;
  e->n_tallies = n_events;
  e->gensteps = false;
  e->uniform = true;
  for (uint32_t i = 1; i < n_events && e->uniform; ++i)
    e->uniform = same_step_physics(e->h_params[0], e->h_params[i]);
  e->total = total;
  e->first_id = first_id;
  e->P0 = e->h_params[0];
  return engine_upload_records(e, static_cast<cudaStream_t>(stream));
}

int optx_engine_set_gensteps(optx_engine* e, const optx_params* events, const optx_faces* faces,
                             uint32_t n_events, const optx_genstep* gensteps, uint32_t n_gensteps,
                             uint64_t first_id, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "engine must not be NULL");
  if (n_events == 0 || n_events > e->max_events)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "n_events must be in [1, max_events]");
  if (n_gensteps == 0 || n_gensteps > e->cfg.max_gensteps)
    return fail(OPTX_ERR_INVALID_ARGUMENT,
                "n_gensteps must be in [1, max_gensteps] (set max_gensteps in optx_wave_config)");
  if (events == nullptr || gensteps == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "events and gensteps must not be NULL");
  std::vector<DevParams> ev(n_events);
  for (uint32_t i = 0; i < n_events; ++i) {
    OPTX_TRY(check_params(&events[i], faces ? &faces[i] : nullptr));
    ev[i] = make_dev_params(events[i], faces ? &faces[i] : nullptr);
  }
  std::vector<DevParams> hp(n_gensteps);  // committed only when every genstep is valid
  std::vector<unsigned long long> ho(n_gensteps + 1ull);
  std::vector<float4> seg(2ull * n_gensteps);
  std::vector<uint32_t> tally_of(n_gensteps);
  uint64_t total = 0;
  for (uint32_t g = 0; g < n_gensteps; ++g) {
    const optx_genstep& gs = gensteps[g];
    if (gs.event >= n_events) return fail(OPTX_ERR_INVALID_ARGUMENT, "genstep event index out of range");
    const float v[8] = {gs.x0, gs.y0, gs.z0, gs.t0, gs.x1, gs.y1, gs.z1, gs.t1};
    for (float f : v)
      if (!std::isfinite(f)) return fail(OPTX_ERR_INVALID_ARGUMENT, "genstep coordinates and times must be finite");
    if (gs.t1 < gs.t0) return fail(OPTX_ERR_INVALID_ARGUMENT, "genstep t1 must be >= t0");
    DevParams d = ev[gs.event];
    d.source = kSourceSegment;
    d.src_x = gs.x0;
    d.src_y = gs.y0;
    d.src_z = gs.z0;
    hp[g] = d;
    seg[2ull * g] = make_float4(gs.x1, gs.y1, gs.z1, gs.t0);
    seg[2ull * g + 1] = make_float4(gs.t1 - gs.t0, 0.0f, 0.0f, 0.0f);
    tally_of[g] = gs.event;
    ho[g] = total;
    total += gs.n_photons;
    if (total > e->max_photons)
      return fail(OPTX_ERR_INVALID_ARGUMENT, "gensteps exceed the engine's max_photons");
  }
  ho[n_gensteps] = total;
  e->h_params.swap(hp);
  e->h_offsets.swap(ho);
  e->n_events = n_gensteps;
  e->n_tallies = n_events;
  e->gensteps = true;
  e->uniform = true;
  for (uint32_t i = 1; i < n_events && e->uniform; ++i) e->uniform = same_step_physics(ev[0], ev[i]);
  e->total = total;
  e->first_id = first_id;
  e->P0 = e->h_params[0];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  OPTX_CUDA(cudaMemcpyAsync(e->d_seg, seg.data(), sizeof(float4) * seg.size(), cudaMemcpyHostToDevice, st));
  OPTX_CUDA(cudaMemcpyAsync(e->d_tally_of, tally_of.data(), 4ull * n_gensteps, cudaMemcpyHostToDevice, st));
  OPTX_CUDA(cudaMemcpyAsync(e->d_phys, ev.data(), sizeof(DevParams) * n_events, cudaMemcpyHostToDevice, st));
  OPTX_TRY(engine_upload_records(e, st));
  // The host vectors must outlive the asynchronous copies.
  OPTX_CUDA(cudaStreamSynchronize(st));
  return OPTX_OK;
}

int optx_engine_set_gensteps_device(optx_engine* e, const optx_params* events,
                                    const optx_faces* faces, uint32_t n_events,
                                    const optx_genstep* dev_gensteps, uint32_t n_gensteps,
                                    uint64_t first_id, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "engine must not be NULL");
  if (n_events == 0 || n_events > e->max_events)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "n_events must be in [1, max_events]");
  if (n_gensteps == 0 || n_gensteps > e->cfg.max_gensteps || n_gensteps > kMaxDeviceGensteps)
    return fail(OPTX_ERR_INVALID_ARGUMENT,
                "n_gensteps must be in [1, min(max_gensteps, 2^24)] for device gensteps");
  if (events == nullptr || dev_gensteps == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "events and dev_gensteps must not be NULL");
  if ((reinterpret_cast<uintptr_t>(dev_gensteps) & 3u) != 0u)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "dev_gensteps must be 4-byte aligned");
  std::vector<DevParams> ev(n_events);
  for (uint32_t i = 0; i < n_events; ++i) {
    OPTX_TRY(check_params(&events[i], faces ? &faces[i] : nullptr));
    ev[i] = make_dev_params(events[i], faces ? &faces[i] : nullptr);
    ev[i].source = kSourceSegment;  // the records the device builds from them
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t n = n_gensteps;
  const uint32_t tiles = (n + kScanTile - 1u) / kScanTile;
  // ev is staged by the copy before it returns (pageable host memory).
  OPTX_CUDA(cudaMemcpyAsync(e->d_phys, ev.data(), sizeof(DevParams) * n_events, cudaMemcpyHostToDevice, st));
  OPTX_CUDA(cudaMemsetAsync(&e->d_ctrl->gs_error, 0, sizeof(unsigned), st));
  genstep_records_kernel<<<(n + 255u) / 256u, 256, 0, st>>>(
      dev_gensteps, n, e->d_phys, n_events, e->d_params, e->d_seg, e->d_tally_of, e->d_offsets,
      &e->d_ctrl->gs_error);
  OPTX_CUDA(cudaGetLastError());
  scan_tiles_kernel<<<tiles, kScanBlock, 0, st>>>(e->d_offsets, n, e->d_scan);
  OPTX_CUDA(cudaGetLastError());
  scan_tiles_kernel<<<1, kScanBlock, 0, st>>>(e->d_scan, tiles, e->d_scan + kScanTile);
  OPTX_CUDA(cudaGetLastError());
  scan_add_kernel<<<(n + 255u) / 256u, 256, 0, st>>>(e->d_offsets, n, e->d_scan, e->d_scan + kScanTile,
                                                     e->max_photons, &e->d_ctrl->gs_error);
  OPTX_CUDA(cudaGetLastError());
  // The photon -> record table at the resolution the capacity allows.
  uint32_t shift = 0;
  while (shift < kEvShift && (e->max_photons >> shift) + 2ull > e->ev_entries) ++shift;
  const unsigned long long entries = (e->max_photons >> shift) + 1ull;
  event_table_dev_kernel<<<static_cast<unsigned>((entries + 255ull) / 256ull), 256, 0, st>>>(
      e->d_offsets, n, e->d_evtable, shift, entries);
  OPTX_CUDA(cudaGetLastError());
  e->h_params.swap(ev);  // per-event physics on the host: caps and the adjoint's coefficients
  e->h_offsets.clear();
  e->n_events = n;
  e->n_tallies = n_events;
  e->gensteps = true;
  e->uniform = true;
  for (uint32_t i = 1; i < n_events && e->uniform; ++i)
    e->uniform = same_step_physics(e->h_params[0], e->h_params[i]);
  e->ev_shift = shift;
  e->total = e->max_photons;  // bound for the watchdog caps; the run reads the real total
  e->total_on_device = true;
  e->first_id = first_id;
  e->P0 = e->h_params[0];
  return OPTX_OK;
}

int optx_run_gensteps(optx_engine* e, const optx_params* events, const optx_faces* faces,
                      uint32_t n_events, const optx_genstep* gensteps, uint32_t n_gensteps,
                      uint64_t first_id, uint64_t* host_tallies, optx_event_stats* stats,
                      optx_timing* timing) {
  if (e == nullptr || host_tallies == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "engine and host_tallies must not be NULL");
  optx_timing tm{};
  const auto t0 = std::chrono::steady_clock::now();
  OPTX_TRY(optx_engine_set_gensteps(e, events, faces, n_events, gensteps, n_gensteps, first_id, nullptr));
  OPTX_TRY(optx_engine_run_tally(e, nullptr));
  optx_event_stats s{};
  OPTX_TRY(read_back_one_shot(e, host_tallies, &s));
  tm.total_ms = ms_since(t0);
  tm.kernel_ms = s.kernels_ms;
  if (stats) *stats = s;
  if (timing) *timing = tm;
  return OPTX_OK;
}

int optx_engine_run_tally(optx_engine* e, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "engine must not be NULL");
  return engine_run(e, kModeTally, nullptr, nullptr, 0.0, nullptr, 0u,
                    static_cast<cudaStream_t>(stream));
}

int optx_engine_run_tally_range(optx_engine* e, uint64_t lo, uint64_t hi, int accumulate,
                                void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "engine must not be NULL");
  if (e->n_events == 0) return fail(OPTX_ERR_INVALID_ARGUMENT, "no events uploaded");
  if (e->total_on_device)
    return fail(OPTX_ERR_INVALID_ARGUMENT,
                "photon ranges need a photon total known on the host (not device gensteps)");
  if (lo > hi || hi > e->total)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "photon range [" + std::to_string(lo) + ", " +
                                               std::to_string(hi) + ") is not inside [0, " +
                                               std::to_string(e->total) + "]");
  e->run_range = true;
  e->run_lo = lo;
  e->run_hi = hi;
  e->run_keep = accumulate != 0;
  const int rc = engine_run(e, kModeTally, nullptr, nullptr, 0.0, nullptr, 0u,
                            static_cast<cudaStream_t>(stream));
  e->run_range = false;  // the arguments are on the device: later runs cover the whole batch
  e->run_keep = false;
  return rc;
}

int optx_engine_set_tallies(optx_engine* e, const uint64_t* host_tallies, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr || host_tallies == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "engine and host_tallies must not be NULL");
  if (e->n_tallies == 0) return fail(OPTX_ERR_INVALID_ARGUMENT, "no events uploaded");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  OPTX_CUDA(cudaMemcpyAsync(e->d_tally, host_tallies, 8ull * e->tdev.len * e->n_tallies,
                            cudaMemcpyHostToDevice, st));
  OPTX_CUDA(cudaStreamSynchronize(st));
  return OPTX_OK;
}

int optx_engine_run_records(optx_engine* e, const optx_records* dev_out, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "engine must not be NULL");
  OPTX_TRY(check_dev_records(dev_out));
  const DevRecords d = to_dev(dev_out);
  return engine_run(e, kModeRecords, &d, nullptr, 0.0, nullptr, 0u,
                    static_cast<cudaStream_t>(stream));
}

namespace {

// Score coefficients of the uploaded single configuration, theta = (abs_length,
// scat_length, reflectivity, tau): inv = (1/La, 1/La^2, 1/Ls, 1/Ls^2, 1/R, 1/tau,
// 1/tau^2) and the mask of parameters whose process is on.
int adjoint_setup(optx_engine* e, double inv[7], uint32_t& mask) {
  if (e->n_tallies != 1)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "the adjoint runs on a single-configuration batch");
  const DevParams& P = e->h_params[0];
  // R is the reflectivity of the painted (specular / Lambertian) faces: the score
  // of a reflection there is 1 / R, so with per-face surfaces every painted face
  // must have that one reflectivity (faces of other models carry none).
  const float refl[5] = {P.refl0, P.refl1, P.refl2, P.refl3, P.refl4};
  bool painted = false;
  float Rf = 0.0f;
  for (int f = 0; f < 5; ++f) {
    const uint32_t m = (P.surf_bits >> (2 * f)) & 3u;
    if (m != kSpecular && m != kLambertian) continue;
    if (painted && refl[f] != Rf)
      return fail(OPTX_ERR_INVALID_ARGUMENT,
                  "the adjoint's reflectivity parameter is one value: the painted faces must share one "
                  "reflectivity");
    Rf = refl[f];
    painted = true;
  }
  const double la = P.abs_length, ls = P.scat_length, R = Rf, tau = P.tau;
  mask = 0;
  if (std::isfinite(la)) mask |= 1u;
  if (std::isfinite(ls)) mask |= 2u;
  if (painted && R > 0.0) mask |= 4u;
  if (tau > 0.0) mask |= 8u;
  inv[0] = 1.0 / la;
  inv[1] = 1.0 / (la * la);
  inv[2] = 1.0 / ls;
  inv[3] = 1.0 / (ls * ls);
  inv[4] = R > 0.0 ? 1.0 / R : 0.0;
  inv[5] = tau > 0.0 ? 1.0 / tau : 0.0;
  inv[6] = tau > 0.0 ? 1.0 / (tau * tau) : 0.0;
  return OPTX_OK;
}

}  // namespace

int optx_engine_run_adjoint(optx_engine* e, const double* dev_w_bin, double w_det,
                            double* dev_grad, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr || dev_w_bin == nullptr || dev_grad == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "engine, dev_w_bin and dev_grad must not be NULL");
  if ((reinterpret_cast<uintptr_t>(dev_w_bin) & 7u) != 0u)  // the kernel reads it as doubles
    return fail(OPTX_ERR_INVALID_ARGUMENT, "dev_w_bin must be 8-byte aligned");
  double inv[7];
  uint32_t mask = 0;
  OPTX_TRY(adjoint_setup(e, inv, mask));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  OPTX_TRY(engine_run(e, kModeAdjoint, nullptr, dev_w_bin, w_det, inv, mask, st));
  OPTX_CUDA(cudaMemcpyAsync(dev_grad, e->d_grad, 4 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return OPTX_OK;
}

int optx_engine_run_score_moments(optx_engine* e, double* dev_moments, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr || dev_moments == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "engine and dev_moments must not be NULL");
  if ((reinterpret_cast<uintptr_t>(dev_moments) & 7u) != 0u)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "dev_moments must be 8-byte aligned");
  if (e->n_events != 1 || e->gensteps)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "score moments run on one configuration (one event, no gensteps)");
  double inv[7];
  uint32_t mask = 0;
  OPTX_TRY(adjoint_setup(e, inv, mask));
  return engine_run(e, kModeMoments, nullptr, nullptr, 0.0, inv, mask,
                    static_cast<cudaStream_t>(stream), dev_moments);
}

int optx_engine_tally_ptr(optx_engine* e, uint64_t** dev_ptr, uint64_t* len_per_event) {
  if (e == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "engine must not be NULL");
  if (dev_ptr) *dev_ptr = reinterpret_cast<uint64_t*>(e->d_tally);
  if (len_per_event) *len_per_event = e->tdev.len;
  return OPTX_OK;
}

int optx_engine_get_tallies(optx_engine* e, uint64_t* host_out, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr || host_out == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "engine and host_out must not be NULL");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WaveCtrl c{};
  OPTX_TRY(engine_check_ctrl(e, c, st));
  OPTX_CUDA(cudaMemcpyAsync(host_out, e->d_tally, 8ull * e->tdev.len * e->n_tallies,
                            cudaMemcpyDeviceToHost, st));
  OPTX_CUDA(cudaStreamSynchronize(st));
  return OPTX_OK;
}

int optx_engine_stats(optx_engine* e, optx_event_stats* stats, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e == nullptr || stats == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "engine and stats must not be NULL");
  WaveCtrl c{};
  OPTX_TRY(engine_check_ctrl(e, c, static_cast<cudaStream_t>(stream)));
  return fill_stats(e, c, stats);
}

int optx_run_batch(optx_engine* e, const optx_params* events, const optx_faces* faces,
                   const uint64_t* counts, uint32_t n_events, uint64_t first_id,
                   uint64_t* host_tallies, optx_event_stats* stats, optx_timing* timing) {
  if (e == nullptr || host_tallies == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "engine and host_tallies must not be NULL");
  optx_timing tm{};
  const auto t0 = std::chrono::steady_clock::now();
  OPTX_TRY(optx_engine_set_events(e, events, faces, counts, n_events, first_id, nullptr));
  OPTX_TRY(optx_engine_run_tally(e, nullptr));
  optx_event_stats s{};
  OPTX_TRY(read_back_one_shot(e, host_tallies, &s));
  tm.total_ms = ms_since(t0);
  tm.kernel_ms = s.kernels_ms;
  if (stats) *stats = s;
  if (timing) *timing = tm;
  return OPTX_OK;
}

int optx_run_records_event(const optx_params* p, const optx_faces* faces, uint64_t n,
                           const optx_records* out, uint32_t steps_per_launch, int block_size,
                           uint64_t first_id, uint64_t chunk, int math, optx_event_stats* stats,
                           optx_timing* timing) {
  OPTX_TRY(check_params(p, faces));
  OPTX_TRY(check_block(block_size));
  if (steps_per_launch == 0)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "event-based backend: steps_per_launch must be >= 1");
  OPTX_TRY(check_math(math));
  if (n > 0) OPTX_TRY(check_records(out));
  OPTX_TRY(ensure_device());
  std::lock_guard<std::mutex> event_lk(g_event_mu);  // g_cache.rec is in use until the end
  const auto t0 = std::chrono::steady_clock::now();
  const uint64_t cap = std::max<uint64_t>(1, std::min<uint64_t>({n, chunk ? chunk : (uint64_t{1} << 24), uint64_t{1} << 31}));
  optx_tally_config tc{1u, 1.0f, 1u};
  optx_wave_config cfg{};
  cfg.block_size = std::min(block_size, 256);  // launch geometry only; records do not depend on it
  if (steps_per_launch >= p->max_steps) {
    // One launch, history style (gpu_event.cu with k >= max_steps): each warp
    // claims photons 32w .. 32w + 31 and runs until all have finished, so the
    // issued lane-steps are 32 x the longest history of each such group.
    cfg.threshold = 1;
    cfg.chunk = 32;
    cfg.cadence = 0;
  } else {
    cfg.threshold = 32;
    cfg.cadence = steps_per_launch;
  }
  cfg.use_graph = 1;
  cfg.math = math;
  optx_engine* e = nullptr;
  OPTX_TRY(optx_engine_create(&tc, 1, cap, &cfg, &e));
  optx_timing tm{};
  optx_event_stats st{};
  int rc = OPTX_OK;
  {
    std::unique_lock<std::mutex> lk(g_mu);
    DevRecords d{};
    rc = cache_records(cap, d);
    lk.unlock();
    for (uint64_t done = 0; rc == OPTX_OK && done < n; done += cap) {
      const uint64_t m = std::min(cap, n - done);
      const uint64_t cnt = m;
      if ((rc = optx_engine_set_events(e, p, faces, &cnt, 1, first_id + done, nullptr)) != OPTX_OK) break;
      const optx_records dr{d.fate, d.n_boundary, d.n_scatter, d.t, d.x, d.y, d.z, d.path};
      if ((rc = optx_engine_run_records(e, &dr, nullptr)) != OPTX_OK) break;
      optx_event_stats s{};
      if ((rc = optx_engine_stats(e, &s, nullptr)) != OPTX_OK) break;
      st.launches += s.launches;
      st.useful_lane_steps += s.useful_lane_steps;
      st.issued_lane_steps += s.issued_lane_steps;
      st.spills += s.spills;
      st.kernels_ms += s.kernels_ms;
      const auto tcp = std::chrono::steady_clock::now();
      lk.lock();
      rc = copy_records_d2h(out, done, d, m);
      lk.unlock();
      tm.d2h_ms += ms_since(tcp);
    }
  }
  optx_engine_destroy(e);
  if (rc != OPTX_OK) return rc;
  tm.kernel_ms = st.kernels_ms;
  tm.total_ms = ms_since(t0);
  if (stats) *stats = st;
  if (timing) *timing = tm;
  return OPTX_OK;
}

}  // extern "C"

// =============================================================================
// Per-interaction sorted run: state queues per pending interaction, one launch
// per iteration inside a CUDA-graph while loop (kernels.cu, sorted_kernel).
struct optx_sorted {
  std::mutex mu;
  int math = OPTX_MATH_FAST;
  int minb = 4;  // resident blocks per SM (register budget)
  uint32_t cap = 0, drain_below = 0;
  bool host_loop = false;
  int grid = 0;
  unsigned char* d_mem = nullptr;  // queues, ids and the control block in one allocation
  SortCtrl* d_ctrl = nullptr;
  float4* q[2][kSortQueues] = {};
  uint32_t* qid[2][kSortQueues] = {};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool ran = false;
  // The run's configuration and arguments are kernel parameters, so a graph
  // belongs to one (P, args) pair; repeated runs of the same work reuse it.
  struct Graph {
    DevParams P;
    SortArgs A;  // graph_handle zeroed in the key
    cudaGraph_t graph;
    cudaGraphExec_t exec;
  };
  std::vector<Graph> graphs;
};

namespace {

constexpr int kSortBlock = kSortThreads;
constexpr uint32_t kSortDefaultCap = 1u << 21;

int sorted_free(optx_sorted* s) {
  if (s->ran && s->ev1 != nullptr) cudaEventSynchronize(s->ev1);  // the last run no longer uses the queues
  for (auto& g : s->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  cudaFree(s->d_mem);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  delete s;
  return OPTX_OK;
}

// The run's graph: prep (control block), then while (photons left) { iteration }.
int sorted_graph(optx_sorted* s, const DevParams& P, const SortArgs& key, optx_sorted::Graph** out) {
  for (auto& g : s->graphs) {
    if (std::memcmp(&g.P, &P, sizeof(P)) == 0 && std::memcmp(&g.A, &key, sizeof(key)) == 0) {
      *out = &g;
      return OPTX_OK;
    }
  }
  optx_sorted::Graph g{};
  g.P = P;
  g.A = key;
  cudaGraphConditionalHandle handle;
  OPTX_CUDA(cudaGraphCreate(&g.graph, 0));
  OPTX_CUDA(cudaGraphConditionalHandleCreate(&handle, g.graph, 1u, cudaGraphCondAssignDefault));
  SortArgs a = key;
  a.graph_handle = handle;
  a.use_graph = 1u;
  SortCtrl* c_ptr = s->d_ctrl;
  void* prep_args[] = {&a, &c_ptr};
  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(DISPATCH(s->math, sorted_prep_fn));
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(32);
  kp.kernelParams = prep_args;
  cudaGraphNode_t n_prep;
  OPTX_CUDA(cudaGraphAddKernelNode(&n_prep, g.graph, nullptr, 0, &kp));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t n_while;
  OPTX_CUDA(cudaGraphAddNode(&n_while, g.graph, &n_prep, 1, &cp));
  DevParams p_copy = P;
  void* it_args[] = {&p_copy, &a, &c_ptr};
  cudaKernelNodeParams ip{};
  ip.func = const_cast<void*>(DISPATCH(s->math, sorted_kernel_fn, s->minb));
  ip.gridDim = dim3(s->grid);
  ip.blockDim = dim3(kSortBlock);
  ip.kernelParams = it_args;
  cudaGraphNode_t n_it;
  OPTX_CUDA(cudaGraphAddKernelNode(&n_it, cp.conditional.phGraph_out[0], nullptr, 0, &ip));
  OPTX_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
  constexpr size_t kMaxGraphs = 8;
  if (s->graphs.size() >= kMaxGraphs) {
    cudaGraphExecDestroy(s->graphs.front().exec);
    cudaGraphDestroy(s->graphs.front().graph);
    s->graphs.erase(s->graphs.begin());
  }
  s->graphs.push_back(g);
  *out = &s->graphs.back();
  return OPTX_OK;
}

}  // namespace

extern "C" {

int optx_sorted_create(const optx_sorted_config* cfg, optx_sorted** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (out == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "out must not be NULL");
  *out = nullptr;
  const optx_sorted_config k = cfg != nullptr ? *cfg : optx_sorted_config{};
  OPTX_TRY(check_math(k.math));
  if (k.host_loop != 0u && k.host_loop != 1u)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "host_loop must be 0 or 1");
  if (k.blocks_per_sm != 0 && k.blocks_per_sm != 3 && k.blocks_per_sm != 4)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "blocks_per_sm must be 0, 3 or 4");
  const uint64_t cap = k.capacity == 0u ? kSortDefaultCap : ((uint64_t(k.capacity) + 31u) & ~uint64_t(31));
  if (cap > (1ull << 28)) return fail(OPTX_ERR_INVALID_ARGUMENT, "capacity must be <= 2^28 photons");
  OPTX_TRY(ensure_device());
  const int minb = k.blocks_per_sm != 0 ? k.blocks_per_sm : 4;
  const int bps = DISPATCH(k.math, sorted_blocks_per_sm, minb, kSortBlock);
  if (bps <= 0) return fail(OPTX_ERR_RUNTIME, "sorted kernel cannot be resident");
  optx_sorted* s = new optx_sorted();
  s->math = k.math;
  s->minb = minb;
  s->host_loop = k.host_loop != 0u;
  s->cap = static_cast<uint32_t>(cap);
  s->grid = bps * num_sms();
  s->drain_below = k.drain_below != 0u ? k.drain_below : static_cast<uint32_t>(s->grid) * kSortBlock;
  const size_t q_bytes = cap * kSortVec4 * 16ull, id_bytes = cap * 4ull;
  const size_t ctrl_off = 2ull * kSortQueues * (q_bytes + id_bytes);
  const size_t total = ctrl_off + sizeof(SortCtrl);
  cudaError_t err = test_fault("alloc") ? cudaErrorMemoryAllocation
                                        : cudaMalloc(reinterpret_cast<void**>(&s->d_mem), total);
  if (err != cudaSuccess) {
    cudaGetLastError();
    sorted_free(s);
    return fail(OPTX_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(err));
  }
  size_t off = 0;
  for (int p = 0; p < 2; ++p)
    for (uint32_t q = 0; q < kSortQueues; ++q) {
      s->q[p][q] = reinterpret_cast<float4*>(s->d_mem + off);
      off += q_bytes;
      s->qid[p][q] = reinterpret_cast<uint32_t*>(s->d_mem + off);
      off += id_bytes;
    }
  // 128-byte aligned, as SortCounter wants: ctrl_off = 504 bytes x cap, cap a multiple of 32.
  s->d_ctrl = reinterpret_cast<SortCtrl*>(s->d_mem + ctrl_off);
  if (cudaMemset(s->d_ctrl, 0, sizeof(SortCtrl)) != cudaSuccess ||
      cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) {
    cudaGetLastError();
    sorted_free(s);
    return fail(OPTX_ERR_CUDA, "sorted run set-up failed");
  }
  *out = s;
  return OPTX_OK;
}

int optx_sorted_destroy(optx_sorted* s) {
  if (s == nullptr) return OPTX_OK;
  return sorted_free(s);
}

int optx_sorted_run(optx_sorted* s, const optx_params* p, const optx_faces* faces,
                    const optx_tally_config* c, uint64_t n, uint64_t first_id, uint64_t* dev_tally,
                    const optx_records* dev_records, void* stream) {
  if (s == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "sorted run must not be NULL");
  OPTX_TRY(check_params(p, faces));
  if (dev_tally == nullptr && dev_records == nullptr)
    return fail(OPTX_ERR_INVALID_ARGUMENT, "give dev_tally, dev_records or both");
  TallyDev td{};
  if (dev_tally != nullptr) OPTX_TRY(make_tally_dev(c, td));
  if (dev_tally != nullptr) OPTX_TRY(check_dev_tally(dev_tally));
  if (dev_records != nullptr) OPTX_TRY(check_dev_records(dev_records));
  if (n >= (1ull << 32)) return fail(OPTX_ERR_INVALID_ARGUMENT, "at most 2^32 - 1 photons per run");
  std::lock_guard<std::mutex> lk(s->mu);
  if (n == 0) return OPTX_OK;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const DevParams P = make_dev_params(*p, faces);
  SortArgs a{};  // value-initialised: padding is zero, so the graph key compares bytes
  for (int q = 0; q < 2; ++q)
    for (uint32_t k = 0; k < kSortQueues; ++k) {
      a.q[q][k] = s->q[q][k];
      a.qid[q][k] = s->qid[q][k];
    }
  a.cap = s->cap;
  a.drain_below = s->drain_below;
  a.n = n;
  a.first_id = first_id;
  a.tally = reinterpret_cast<unsigned long long*>(dev_tally);
  a.tc = td;
  if (dev_records != nullptr) a.rec = to_dev(dev_records);
  // Each photon needs at most max_steps + 1 iterations in flight, and the
  // queues admit `cap` photons at a time.
  const unsigned long long bound =
      (n / s->cap + 2ull) * (static_cast<unsigned long long>(P.max_steps) + 2ull) + 64ull;
  a.iter_cap = test_fault("watchdog") ? 1u : static_cast<uint32_t>(std::min(bound, 0xfffffff0ull));
  // One set of queues and one control block per handle: a run on another stream
  // waits on the device for the previous run to end.
  if (s->ran) OPTX_CUDA(cudaStreamWaitEvent(st, s->ev1, 0));
  OPTX_CUDA(cudaEventRecord(s->ev0, st));
  s->ran = true;
  if (!s->host_loop) {
    optx_sorted::Graph* g = nullptr;
    OPTX_TRY(sorted_graph(s, P, a, &g));
    OPTX_CUDA(cudaGraphLaunch(g->exec, st));
  } else {
    OPTX_CUDA(DISPATCH(s->math, launch_sorted_prep, a, s->d_ctrl, st));
    for (;;) {  // the kernel's own watchdog ends a run that does not finish
      for (int k = 0; k < 8; ++k)
        OPTX_CUDA(DISPATCH(s->math, launch_sorted, s->minb, P, a, s->d_ctrl, s->grid, kSortBlock, st));
      unsigned active = 0;
      OPTX_CUDA(cudaMemcpyAsync(&active, &s->d_ctrl->active, sizeof(active), cudaMemcpyDeviceToHost, st));
      OPTX_CUDA(cudaStreamSynchronize(st));
      if (!active) break;
    }
  }
  OPTX_CUDA(cudaEventRecord(s->ev1, st));
  return OPTX_OK;
}

int optx_sorted_stats(optx_sorted* s, optx_sorted_counters* out, void* stream) {
  if (s == nullptr || out == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = optx_sorted_counters{};
  if (!s->ran) return OPTX_OK;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  SortCtrl c{};
  OPTX_CUDA(cudaMemcpyAsync(&c, s->d_ctrl, sizeof(c), cudaMemcpyDeviceToHost, st));
  OPTX_CUDA(cudaStreamSynchronize(st));
  OPTX_CUDA(cudaEventSynchronize(s->ev1));
  float ms = 0.0f;
  OPTX_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
  out->iterations = c.iter;
  for (uint32_t q = 0; q < kSortQueues; ++q) out->queued[q] = c.queued[q];
  out->drained = c.drained;
  out->kernel_ms = ms;
  if (c.error & kErrQueue) return fail(OPTX_ERR_CAPACITY, "sorted run: state queue overflow");
  if (c.error & kErrWatchdog) return fail(OPTX_ERR_WATCHDOG, "sorted run: iteration cap reached");
  return OPTX_OK;
}

}  // extern "C"

// =============================================================================
// Wavefront tally without device allocation.
//
// For callers that cannot call cudaMalloc: code running where another runtime
// or framework owns the device memory (a caching allocator that must see every
// allocation, a memory-capped process, a plugin that may not grow its footprint
// after start-up). All of the run's device scratch lives in the file-scope
// array below, which the library holds on every GPU that loads it, until exit.
namespace {

constexpr uint32_t kNoAllocQueuePhotons = 16384;  // per state queue (64 B per photon)
constexpr uint32_t kNoAllocMaxTally = 65536;      // max tally length (u64 entries)
constexpr size_t kNoAllocArgsOff = 0;
constexpr size_t kNoAllocCtrlOff = 1024;
constexpr size_t kNoAllocTallyOff = 2048;
constexpr size_t kNoAllocQaOff = kNoAllocTallyOff + 8ull * kNoAllocMaxTally;
constexpr size_t kNoAllocQbOff = kNoAllocQaOff + 64ull * kNoAllocQueuePhotons;
constexpr size_t kNoAllocScratchBytes = kNoAllocQbOff + 64ull * kNoAllocQueuePhotons;  // 2.6 MiB
static_assert(sizeof(WaveArgs) <= kNoAllocCtrlOff && sizeof(WaveCtrl) <= kNoAllocTallyOff - kNoAllocCtrlOff,
              "no-alloc scratch layout");

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};  // device address of the array, per device

}  // namespace

namespace {
void noalloc_forget_addresses() {  // called with g_mu held, like the allocation-free call
  for (void*& p : g_noalloc_ptr) p = nullptr;
}
}  // namespace

extern "C" int optx_wavefront_tally_noalloc(const optx_params* p, const optx_faces* faces,
                                            const optx_tally_config* c, uint64_t n,
                                            uint64_t first_id, uint64_t* tally_out, int math,
                                            void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  OPTX_TRY(check_params(p, faces));
  OPTX_TRY(check_math(math));
  TallyDev td{};
  OPTX_TRY(make_tally_dev(c, td));
  if (n > 0xffffffffull)
    return fail(OPTX_ERR_INVALID_ARGUMENT,
                "optx_wavefront_tally_noalloc: at most 2^32 - 1 photons per call");
  if (tally_out == nullptr) return fail(OPTX_ERR_INVALID_ARGUMENT, "tally_out must not be NULL");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(OPTX_ERR_NO_DEVICE, "no CUDA device available");
  }
  int dev = 0;
  OPTX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(OPTX_ERR_RUNTIME, "device ordinal out of range");
  constexpr int kBlock = 256, kMinB = 4;
  // The histograms sit in shared memory beside the 8 warps' pantries, so the
  // longest tally is what the opt-in shared memory per block leaves (B200:
  // 232,448 B), capped by the static tally accumulator.
  int max_optin = 0;
  OPTX_CUDA(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  OPTX_CUDA(cudaFuncGetAttributes(&fa, DISPATCH(math, wave_kernel_fn, kModeTally, kSingle, kMinB)));
  const long long pantries = static_cast<long long>(kBlock / 32) * kPantryBytesPerWarp;
  const long long room = static_cast<long long>(max_optin) - static_cast<long long>(fa.sharedSizeBytes) - pantries;
  const uint64_t max_len = std::min<uint64_t>(kNoAllocMaxTally, room > 0 ? static_cast<uint64_t>(room / 4) + 7u : 0u);
  if (td.len > max_len)
    return fail(OPTX_ERR_INVALID_ARGUMENT,
                "optx_wavefront_tally_noalloc: tally length " + std::to_string(td.len) +
                    " exceeds the maximum of " + std::to_string(max_len) +
                    " entries on this device (5 + time_bins + 1 + xy_bins^2 + 2; the histograms "
                    "share the opt-in shared memory per block with the pantries)");
  // First call on this device: the host-side name of the array is not a device
  // address, so look the address up once (with this device current).
  if (g_noalloc_ptr[dev] == nullptr) {
    void* ptr = nullptr;
    OPTX_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    g_noalloc_ptr[dev] = ptr;
  }
  unsigned char* base = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  auto* d_args = reinterpret_cast<WaveArgs*>(base + kNoAllocArgsOff);
  auto* d_ctrl = reinterpret_cast<WaveCtrl*>(base + kNoAllocCtrlOff);
  auto* d_tally = reinterpret_cast<unsigned long long*>(base + kNoAllocTallyOff);
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  const DevParams P = make_dev_params(*p, faces);
  const size_t smem = static_cast<size_t>(kBlock / 32) * kPantryBytesPerWarp +
                      static_cast<size_t>(td.len - 7u) * 4u;
  if (smem > kDynSmemOptIn) OPTX_CUDA(DISPATCH(math, wave_set_smem, kModeTally, kSingle, kMinB, smem));
  const int bps = DISPATCH(math, wave_blocks_per_sm, kModeTally, kSingle, kMinB, kBlock, smem);
  if (bps <= 0)
    return fail(OPTX_ERR_RUNTIME, "tally histograms need too much shared memory; reduce xy_bins / time_bins");
  const int grid = std::min(bps, kMinB) * num_sms();

  WaveArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n_events = 1;
  a.n_tallies = 1;
  a.ev_shift = kEvShift;
  a.threshold = 28;
  a.cadence = 0;
  a.qcap = kNoAllocQueuePhotons;
  a.total = n;
  a.first_id = first_id;
  a.wave_quota = 1ull << 30;
  a.qa = reinterpret_cast<float4*>(base + kNoAllocQaOff);
  a.qb = reinterpret_cast<float4*>(base + kNoAllocQbOff);
  a.tally = d_tally;
  a.tc = td;
  a.use_graph = 0u;
  a.chunk = 256u;
  a.tail_steps = 4096u;
  a.iter_cap = (static_cast<unsigned long long>(n) + a.qcap + 64ull) * (P.max_steps + 2ull) + 4096ull;
  a.wave_cap = static_cast<uint32_t>(std::min<unsigned long long>(
      std::max<unsigned long long>(4ull * (P.max_steps + 2ull) + 64ull, 100000ull), 0xfffffff0ull));
  OPTX_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(a), cudaMemcpyHostToDevice, st));
  // The prep kernel clears what must start at zero: the control block and the
  // tally accumulator (the array keeps the previous call's contents).
  OPTX_CUDA(DISPATCH(math, launch_wave_prep, d_args, d_ctrl, std::min(grid, 4 * num_sms()), 256, st));
  for (;;) {
    OPTX_CUDA(DISPATCH(math, launch_wave, kModeTally, kSingle, kMinB, P, d_args, d_ctrl, grid, kBlock,
                       smem, st));
    unsigned active = 0;
    OPTX_CUDA(cudaMemcpyAsync(&active, &d_ctrl->active, sizeof(active), cudaMemcpyDeviceToHost, st));
    OPTX_CUDA(cudaStreamSynchronize(st));
    if (!active) break;  // the kernel ends the run itself at its wave cap
  }
  unsigned error = 0;
  OPTX_CUDA(cudaMemcpyAsync(&error, &d_ctrl->error, sizeof(error), cudaMemcpyDeviceToHost, st));
  OPTX_CUDA(cudaMemcpyAsync(tally_out, d_tally, 8ull * td.len, cudaMemcpyDeviceToHost, st));
  OPTX_CUDA(cudaStreamSynchronize(st));
  if (error & kErrWatchdog) return fail(OPTX_ERR_WATCHDOG, "wavefront iteration cap reached");
  return OPTX_OK;
}
