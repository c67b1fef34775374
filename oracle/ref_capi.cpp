// ref_capi.cpp - a C ABI over the reference project's own CPU backend.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile together with the
// reference's src/cpu/cpu_backend.cpp and its include/ tree, read in place
// from the reference checkout (nothing of it is copied into this repository).
// The resulting oracle/_ref/libref_cpu*.so files are used to pin the oracle
// restatement (optx_oracle.cpp) and as the timed CPU baseline.
//
// Wraps (reference paths): include/optphot/backend.hpp:76-79 run_cpu_records /
// run_cpu_tally, include/optphot/philox.hpp:64-76 philox4x32_10, and (to pin the
// package's output files and comparison harness) src/core/io.cpp write_records /
// write_tally, src/core/config.cpp params_to_json, src/core/compare.cpp.
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

// ---- output formats and comparison (src/core/io.cpp, config.cpp, compare.cpp) ----

#include <string>

#include "optphot/compare.hpp"
#include "optphot/config.hpp"

namespace {

PhotonRecords make_records(uint64_t n, const uint8_t* fate, const uint32_t* nb, const uint32_t* ns,
                           const float* t, const float* x, const float* y, const float* z,
                           const float* path) {
  PhotonRecords r;
  r.resize(n);
  std::memcpy(r.fate.data(), fate, n);
  std::memcpy(r.n_boundary.data(), nb, n * 4);
  std::memcpy(r.n_scatter.data(), ns, n * 4);
  std::memcpy(r.t.data(), t, n * 4);
  std::memcpy(r.x.data(), x, n * 4);
  std::memcpy(r.y.data(), y, n * 4);
  std::memcpy(r.z.data(), z, n * 4);
  std::memcpy(r.path.data(), path, n * 4);
  return r;
}

int copy_out(const std::string& s, char* out, size_t len) {
  if (s.size() + 1 > len) return -1;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return static_cast<int>(s.size());
}

}  // namespace

extern "C" {

// params_to_json(p, o) (config.cpp:230-253) into `out`; returns its length or -1.
int ref_params_to_json(const void* params, const char* backend, const char* mode, uint64_t n_photons,
                       int threads, int block_size, uint32_t time_bins, float time_max,
                       uint32_t xy_bins, char* out, size_t len) {
  SimParams p;
  std::memcpy(&p, params, sizeof(p));
  RunOptions o;
  o.backend = backend;
  o.mode = mode;
  o.n_photons = n_photons;
  o.threads = threads;
  o.block_size = block_size;
  o.tally.time_bins = time_bins;
  o.tally.time_max = time_max;
  o.tally.xy_bins = xy_bins;
  return copy_out(params_to_json(p, o), out, len);
}

// write_records(dir, records, meta) (io.cpp:48-60).
int ref_write_records(const char* dir, uint64_t n, const uint8_t* fate, const uint32_t* nb,
                      const uint32_t* ns, const float* t, const float* x, const float* y,
                      const float* z, const float* path, const char* meta) {
  try {
    write_records(dir, make_records(n, fate, nb, ns, t, x, y, z, path), meta);
  } catch (...) {
    return 1;
  }
  return 0;
}

// write_tally(dir, tally, meta) (io.cpp:62-72); tally in the flat layout.
int ref_write_tally(const char* dir, uint32_t time_bins, uint32_t xy_bins, const uint64_t* flat,
                    const char* meta) {
  TallyConfig c;
  c.time_bins = time_bins;
  c.xy_bins = xy_bins;
  Tally t;
  t.reset(c);
  uint64_t k = 0;
  for (auto& f : t.fate_counts) f = flat[k++];
  for (auto& v : t.time_hist) v = flat[k++];
  for (auto& v : t.xy_hist) v = flat[k++];
  t.boundary_sum = flat[k++];
  t.scatter_sum = flat[k++];
  try {
    write_tally(dir, t, meta);
  } catch (...) {
    return 1;
  }
  return 0;
}

// to_json(compare_histories(a, b)) and to_json(compare_distributions(a, b, p, ...))
// (compare.cpp:39-120) into out_hist / out_dist; returns 0, or -1 if a buffer is short.
int ref_compare_json(uint64_t na, const uint8_t* fa, const uint32_t* nba, const uint32_t* nsa,
                     const float* ta, const float* xa, const float* ya, const float* za,
                     const float* pa, uint64_t nb_, const uint8_t* fb, const uint32_t* nbb,
                     const uint32_t* nsb, const float* tb, const float* xb, const float* yb,
                     const float* zb, const float* pb, const void* params, int time_bins,
                     float t_max, int xy_bins, char* out_hist, char* out_dist, size_t len) {
  SimParams p;
  std::memcpy(&p, params, sizeof(p));
  const PhotonRecords a = make_records(na, fa, nba, nsa, ta, xa, ya, za, pa);
  const PhotonRecords b = make_records(nb_, fb, nbb, nsb, tb, xb, yb, zb, pb);
  std::string h = "null";
  if (na == nb_) h = to_json(compare_histories(a, b));
  const std::string d = to_json(compare_distributions(a, b, p, time_bins, t_max, xy_bins));
  if (copy_out(h, out_hist, len) < 0 || copy_out(d, out_dist, len) < 0) return -1;
  return 0;
}

}  // extern "C"
