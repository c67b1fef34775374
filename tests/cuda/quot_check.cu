// Checks the hit-map quotient of the kernels (quot_rn in
// gpu_optical_photons_b200/csrc/optx_device.cuh: a / b from the rounded
// reciprocal y = 1 / b, the product and two FMA corrections) against the IEEE
// division __fdiv_rn: for every float a in [b 2^-100, b] of each listed
// divisor, and for random (a, b) pairs. Prints one line per case and exits
// non-zero on a mismatch. Built and run by tests/test_gpu_quotient.py.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_runtime.h>

#include "optx_device.cuh"

namespace {

__global__ void every_a(float b, float y, uint32_t lo_bits, uint32_t hi_bits, unsigned long long* bad) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = lo_bits + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= hi_bits;
       i += stride) {
    const float a = __uint_as_float(static_cast<uint32_t>(i));
    if (__float_as_uint(__fdiv_rn(a, b)) != __float_as_uint(optx::quot_rn(a, b, y))) atomicAdd(bad, 1ull);
  }
}

__global__ void random_a(const float* bs, const float* ys, uint32_t nb, uint32_t per_b, unsigned long long* bad) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t total = static_cast<uint64_t>(nb) * per_b;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
    const uint32_t j = static_cast<uint32_t>(i / per_b);
    uint32_t h = static_cast<uint32_t>(i * 2654435761ull) ^ (static_cast<uint32_t>(i >> 17) * 40503u);
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    const float a = bs[j] * (((h >> 8) + 1u) * (1.0f / 16777216.0f));  // (0, b]
    if (__float_as_uint(__fdiv_rn(a, bs[j])) != __float_as_uint(optx::quot_rn(a, bs[j], ys[j])))
      atomicAdd(bad, 1ull);
  }
}

}  // namespace

int main() {
  unsigned long long* bad = nullptr;
  if (cudaMalloc(&bad, sizeof(unsigned long long)) != cudaSuccess) return 2;
  int rc = 0;
  const float divisors[] = {50.0f, 20.0f, 10.0f, 1.9999999f, 1.0000001f, 123.456f};
  for (const float b : divisors) {
    volatile float one = 1.0f;
    const float y = one / b;  // the host's correctly rounded reciprocal, as make_dev_params computes it
    const float lo_f = b * 0x1p-100f;
    uint32_t lo = 0, hi = 0;
    std::memcpy(&lo, &lo_f, 4);
    std::memcpy(&hi, &b, 4);
    cudaMemset(bad, 0, sizeof(unsigned long long));
    every_a<<<148 * 16, 256>>>(b, y, lo, hi, bad);
    unsigned long long n = 0;
    cudaMemcpy(&n, bad, sizeof(n), cudaMemcpyDeviceToHost);
    std::printf("b = %.9g: %u values of a, %llu mismatches\n", b, hi - lo + 1u, n);
    rc |= n != 0ull;
  }
  std::mt19937 g(7);
  std::uniform_real_distribution<float> e(-8.0f, 12.0f);
  const uint32_t nb = 1024, per_b = 1u << 18;
  std::vector<float> bs(nb), ys(nb);
  for (uint32_t j = 0; j < nb; ++j) {
    bs[j] = std::exp2(e(g));
    volatile float one = 1.0f;
    ys[j] = one / bs[j];
  }
  float *dbs = nullptr, *dys = nullptr;
  cudaMalloc(&dbs, nb * sizeof(float));
  cudaMalloc(&dys, nb * sizeof(float));
  cudaMemcpy(dbs, bs.data(), nb * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(dys, ys.data(), nb * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(bad, 0, sizeof(unsigned long long));
  random_a<<<148 * 16, 256>>>(dbs, dys, nb, per_b, bad);
  unsigned long long n = 0;
  cudaMemcpy(&n, bad, sizeof(n), cudaMemcpyDeviceToHost);
  std::printf("random: %u divisors x %u values of a, %llu mismatches\n", nb, per_b, n);
  rc |= n != 0ull;
  const cudaError_t err = cudaDeviceSynchronize();
  std::printf("cuda: %s\n", cudaGetErrorString(err));
  cudaFree(dbs);
  cudaFree(dys);
  cudaFree(bad);
  return rc | (err != cudaSuccess ? 2 : 0);
}
