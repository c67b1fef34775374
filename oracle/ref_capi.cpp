// ref_capi.cpp - a C ABI over the reference project's own CPU backend.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile together with the
// reference's src/cpu/cpu_backend.cpp and its include/ tree, read in place
// from the reference checkout (nothing of it is copied into this repository).
// The resulting oracle/_ref/libref_cpu*.so files are used to pin the oracle
// restatement (optx_oracle.cpp) and as the timed CPU baseline.
//
// Wraps (reference paths): include/optphot/backend.hpp:76-79 run_cpu_records /
// run_cpu_tally, include/optphot/philox.hpp:64-76 philox4x32_10.
#include <cstring>

#include "optphot/backend.hpp"
#include "optphot/philox.hpp"

using namespace optphot;

static_assert(sizeof(SimParams) == 72, "SimParams layout");

extern "C" {

int ref_portable_math() {
#if defined(OPTPHOT_PORTABLE_MATH)
  return 1;
#else
  return 0;
#endif
}

int ref_max_threads() { return cpu_max_threads(); }

void ref_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  const U32x4 r = philox4x32_10(U32x4{ctr[0], ctr[1], ctr[2], ctr[3]}, U32x2{key[0], key[1]});
  out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

double ref_records(const void* params, uint64_t n, uint64_t first_id, int threads, uint8_t* fate,
                   uint32_t* nb, uint32_t* ns, float* t, float* x, float* y, float* z, float* path) {
  SimParams p;
  std::memcpy(&p, params, sizeof(p));
  PhotonRecords rec;
  const RunTiming tm = run_cpu_records(p, n, rec, threads, first_id);
  std::memcpy(fate, rec.fate.data(), n);
  std::memcpy(nb, rec.n_boundary.data(), n * 4);
  std::memcpy(ns, rec.n_scatter.data(), n * 4);
  std::memcpy(t, rec.t.data(), n * 4);
  std::memcpy(x, rec.x.data(), n * 4);
  std::memcpy(y, rec.y.data(), n * 4);
  std::memcpy(z, rec.z.data(), n * 4);
  std::memcpy(path, rec.path.data(), n * 4);
  return tm.kernel_ms;
}

// Tally in the flat layout [5 fates | time_bins+1 | xy_bins^2 | sum nb | sum ns].
double ref_tally(const void* params, uint32_t time_bins, float time_max, uint32_t xy_bins,
                 uint64_t n, uint64_t first_id, int threads, uint64_t* out) {
  SimParams p;
  std::memcpy(&p, params, sizeof(p));
  TallyConfig c;
  c.time_bins = time_bins;
  c.time_max = time_max;
  c.xy_bins = xy_bins;
  Tally tally;
  const RunTiming tm = run_cpu_tally(p, c, n, tally, threads, first_id);
  uint64_t k = 0;
  for (int f = 0; f < kNumFates; ++f) out[k++] = tally.fate_counts[f];
  for (uint64_t v : tally.time_hist) out[k++] = v;
  for (uint64_t v : tally.xy_hist) out[k++] = v;
  out[k++] = tally.boundary_sum;
  out[k++] = tally.scatter_sum;
  return tm.kernel_ms;
}

}  // extern "C"
