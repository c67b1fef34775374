// ref_gpu_capi.cpp - a C ABI over the reference project's own GPU backend.
//
// TEST INFRASTRUCTURE ONLY. oracle/relink.py compiles it with the reference's
// src/gpu/gpu_backend.cu and src/gpu/gpu_event.cu (nvcc, sm_100a, the
// reference's default or portable build options) and src/cpu/cpu_backend.cpp,
// read in place from the reference checkout, into oracle/_ref/libref_gpu*.so.
// Used to compare this repository's kernels with the reference kernels on the
// same B200 (parity and speed); never part of the product.
//
// Wraps (reference paths): include/optphot/backend.hpp:84-115 gpu_available,
// run_gpu_records, run_gpu_tally, run_gpu_records_event.
#include <cstring>
#include <exception>

#include "optphot/backend.hpp"

using namespace optphot;

namespace {

void copy_out(const PhotonRecords& r, uint64_t n, uint8_t* fate, uint32_t* nb, uint32_t* ns, float* t,
              float* x, float* y, float* z, float* path) {
  std::memcpy(fate, r.fate.data(), n);
  std::memcpy(nb, r.n_boundary.data(), n * 4);
  std::memcpy(ns, r.n_scatter.data(), n * 4);
  std::memcpy(t, r.t.data(), n * 4);
  std::memcpy(x, r.x.data(), n * 4);
  std::memcpy(y, r.y.data(), n * 4);
  std::memcpy(z, r.z.data(), n * 4);
  std::memcpy(path, r.path.data(), n * 4);
}

}  // namespace

extern "C" {

int refgpu_available() { return gpu_available() ? 1 : 0; }

int refgpu_portable_math() {
#if defined(OPTPHOT_PORTABLE_MATH)
  return 1;
#else
  return 0;
#endif
}

// timing[5] = total, kernel, h2d, d2h, alloc (ms). Returns 0, or 1 on an exception.
int refgpu_records(const void* params, uint64_t n, int block_size, uint64_t first_id, uint64_t chunk,
                   uint8_t* fate, uint32_t* nb, uint32_t* ns, float* t, float* x, float* y, float* z,
                   float* path, double* timing) {
  try {
    SimParams p;
    std::memcpy(&p, params, sizeof(p));
    PhotonRecords rec;
    const RunTiming tm = run_gpu_records(p, n, rec, block_size, first_id, chunk);
    copy_out(rec, n, fate, nb, ns, t, x, y, z, path);
    const double v[5] = {tm.total_ms, tm.kernel_ms, tm.h2d_ms, tm.d2h_ms, tm.alloc_ms};
    if (timing) std::memcpy(timing, v, sizeof(v));
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}

// Flat tally [5 fates | time_bins + 1 | xy_bins^2 | sum nb | sum ns].
int refgpu_tally(const void* params, uint32_t time_bins, float time_max, uint32_t xy_bins, uint64_t n,
                 int block_size, uint64_t first_id, uint64_t* out, double* timing) {
  try {
    SimParams p;
    std::memcpy(&p, params, sizeof(p));
    TallyConfig c;
    c.time_bins = time_bins;
    c.time_max = time_max;
    c.xy_bins = xy_bins;
    Tally tally;
    const RunTiming tm = run_gpu_tally(p, c, n, tally, block_size, first_id);
    uint64_t k = 0;
    for (int f = 0; f < kNumFates; ++f) out[k++] = tally.fate_counts[f];
    for (uint64_t v : tally.time_hist) out[k++] = v;
    for (uint64_t v : tally.xy_hist) out[k++] = v;
    out[k++] = tally.boundary_sum;
    out[k++] = tally.scatter_sum;
    const double v[5] = {tm.total_ms, tm.kernel_ms, tm.h2d_ms, tm.d2h_ms, tm.alloc_ms};
    if (timing) std::memcpy(timing, v, sizeof(v));
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}

// stats[4] = launches, useful lane-steps, issued lane-steps, kernels_ms (as double).
int refgpu_records_event(const void* params, uint64_t n, uint32_t k, int block_size, uint64_t first_id,
                         uint64_t chunk, uint8_t* fate, uint32_t* nb, uint32_t* ns, float* t, float* x,
                         float* y, float* z, float* path, double* stats, double* timing) {
  try {
    SimParams p;
    std::memcpy(&p, params, sizeof(p));
    PhotonRecords rec;
    EventStats es;
    const RunTiming tm = run_gpu_records_event(p, n, rec, k, block_size, first_id, chunk, &es);
    copy_out(rec, n, fate, nb, ns, t, x, y, z, path);
    if (stats) {
      stats[0] = static_cast<double>(es.launches);
      stats[1] = static_cast<double>(es.useful_lane_steps);
      stats[2] = static_cast<double>(es.issued_lane_steps);
      stats[3] = es.kernels_ms;
    }
    const double v[5] = {tm.total_ms, tm.kernel_ms, tm.h2d_ms, tm.d2h_ms, tm.alloc_ms};
    if (timing) std::memcpy(timing, v, sizeof(v));
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}

}  // extern "C"
