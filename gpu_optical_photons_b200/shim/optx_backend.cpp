// optx_backend.cpp - the reference project's GPU backend functions, implemented
// on the optx C ABI.
//
// zmeskma/GPU_Optical_photons declares its GPU entry points in
// include/optphot/backend.hpp:84-115 and implements them in
// src/gpu/gpu_backend.cu and src/gpu/gpu_event.cu. This file defines the same
// symbols (same namespace, names, signatures and default arguments, which the
// header supplies) by forwarding to liboptx.so, so the reference's apps
// (apps/optphot_main.cpp, optphot_bench.cpp, optphot_compare.cpp,
// optphot_event_bench.cpp) and its GPU tests (tests/test_gpu.cpp) link against
// it in place of the two .cu files without a source change.
//
// Build: compile with the reference's include directory and this repository's
// include/ on the include path, define OPTPHOT_HAVE_CUDA for the callers (as
// the reference's CMake does for its GPU library), and link liboptx.so.
//
// Math mode: the reference's GPU build follows its CMake options. With
// OPTPHOT_PORTABLE_MATH and OPTPHOT_NO_FMAD defined (the reference's
// bit-reproducible configuration) this file asks for OPTX_MATH_EXACT, which is
// bit-identical to the reference CPU build with OPTPHOT_PORTABLE_MATH; otherwise
// OPTX_MATH_FAST (CUDA libm and FMA contraction, the reference's default GPU
// build). Defining OPTX_SHIM_MATH (0 fast, 1 exact, 2 approx) overrides both.
//
// Errors: a non-zero optx status becomes the exception the reference throws:
// std::invalid_argument for OPTX_ERR_INVALID_ARGUMENT (gpu_event.cu:177-182),
// std::runtime_error otherwise (cuda_util.cuh:17-24, gpu_backend.cu:171-185).
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "optphot/backend.hpp"
#include "optx.h"

#ifndef OPTX_SHIM_MATH
#if defined(OPTPHOT_PORTABLE_MATH) && defined(OPTPHOT_NO_FMAD)
#define OPTX_SHIM_MATH OPTX_MATH_EXACT
#else
#define OPTX_SHIM_MATH OPTX_MATH_FAST
#endif
#endif

namespace optphot {

namespace {

// optx_params is declared byte for byte as SimParams (params.hpp:40-63).
static_assert(sizeof(SimParams) == sizeof(optx_params), "SimParams and optx_params differ in size");
static_assert(offsetof(SimParams, seed) == offsetof(optx_params, seed), "SimParams layout");
static_assert(offsetof(SimParams, max_steps) == offsetof(optx_params, max_steps), "SimParams layout");
static_assert(sizeof(TallyConfig) == sizeof(optx_tally_config), "TallyConfig layout");

void check(int rc) {
  if (rc == OPTX_OK) return;
  if (rc == OPTX_ERR_INVALID_ARGUMENT) throw std::invalid_argument(optx_last_error());
  throw std::runtime_error(optx_last_error());
}

const optx_params* as_optx(const SimParams& p) { return reinterpret_cast<const optx_params*>(&p); }

optx_records view(PhotonRecords& r) {
  return optx_records{r.fate.data(), r.n_boundary.data(), r.n_scatter.data(), r.t.data(),
                      r.x.data(),    r.y.data(),          r.z.data(),         r.path.data()};
}

RunTiming timing_of(const optx_timing& t) {
  RunTiming r;
  r.total_ms = t.total_ms;
  r.kernel_ms = t.kernel_ms;
  r.h2d_ms = t.h2d_ms;
  r.d2h_ms = t.d2h_ms;
  r.alloc_ms = t.alloc_ms;
  return r;
}

}  // namespace

bool gpu_available() { return optx_gpu_available() != 0; }

std::string gpu_device_name() {
  char buf[256] = {0};
  check(optx_gpu_device_name(buf, sizeof(buf)));
  return std::string(buf);
}

RunTiming run_gpu_records(const SimParams& p, uint64_t n, PhotonRecords& out, int block_size,
                          uint64_t first_id, uint64_t chunk) {
  out.resize(static_cast<std::size_t>(n));  // the callee sizes the caller's vectors
  const optx_records r = view(out);
  optx_timing t{};
  check(optx_run_records(as_optx(p), nullptr, n, &r, block_size, first_id, chunk, OPTX_SHIM_MATH, &t));
  return timing_of(t);
}

RunTiming run_gpu_tally(const SimParams& p, const TallyConfig& c, uint64_t n, Tally& out,
                        int block_size, uint64_t first_id) {
  out.reset(c);
  const optx_tally_config tc{c.time_bins, c.time_max, c.xy_bins};
  const std::size_t xy = static_cast<std::size_t>(c.xy_bins) * c.xy_bins;
  // Flat layout: [fates | time_bins + 1 | xy_bins^2 | sum nb | sum ns].
  std::vector<uint64_t> flat(kNumFates + (c.time_bins + 1u) + xy + 2u);
  optx_timing t{};
  check(optx_run_tally(as_optx(p), nullptr, &tc, n, flat.data(), block_size, first_id,
                       OPTX_SHIM_MATH, &t));
  std::size_t k = 0;
  for (auto& f : out.fate_counts) f = flat[k++];
  for (auto& v : out.time_hist) v = flat[k++];
  for (auto& v : out.xy_hist) v = flat[k++];
  out.boundary_sum = flat[k++];
  out.scatter_sum = flat[k++];
  return timing_of(t);
}

RunTiming run_gpu_records_event(const SimParams& p, uint64_t n, PhotonRecords& out,
                                uint32_t steps_per_launch, int block_size, uint64_t first_id,
                                uint64_t chunk, EventStats* stats) {
  out.resize(static_cast<std::size_t>(n));
  const optx_records r = view(out);
  optx_event_stats s{};
  optx_timing t{};
  check(optx_run_records_event(as_optx(p), nullptr, n, &r, steps_per_launch, block_size, first_id,
                               chunk, OPTX_SHIM_MATH, &s, &t));
  if (stats != nullptr) {
    stats->launches = s.launches;
    stats->useful_lane_steps = s.useful_lane_steps;
    stats->issued_lane_steps = s.issued_lane_steps;
    stats->kernels_ms = s.kernels_ms;
  }
  return timing_of(t);
}

}  // namespace optphot
