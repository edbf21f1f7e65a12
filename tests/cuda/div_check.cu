// Test-only kernels: clv::div_by against the IEEE division on the device.
#include <cstdint>
#include "../../clvisc_b200/csrc/clv_device.cuh"

__device__ __forceinline__ bool same_f(float x, float y) {
  return __float_as_uint(x) == __float_as_uint(y) || (x != x && y != y);
}
__device__ __forceinline__ bool same_d(double x, double y) {
  return __double_as_longlong(x) == __double_as_longlong(y) || (x != x && y != y);
}

// every float bit pattern as the dividend
__global__ void check_all_f32(float b, unsigned long long* bad, unsigned int* first) {
  const float y = 1.0f / b;
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < (1ull << 32);
       t += (unsigned long long)gridDim.x * blockDim.x) {
    float a = __uint_as_float((unsigned int)t);
    float q = clv::div_by<float>(a, b, y);
    float r = a / b;
    if (!same_f(q, r)) {
      unsigned long long k = atomicAdd(bad, 1ull);
      if (k < 4) first[k] = (unsigned int)t;
    }
  }
}

// n pseudo-random double bit patterns (splitmix64) as dividends
__global__ void check_rand_f64(double b, unsigned long long n, unsigned long long seed, unsigned long long* bad,
                               unsigned long long* first) {
  const double y = 1.0 / b;
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long z = seed + t * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    // half the samples spread over all exponents, half near the values the kernels see
    if (t & 1) z = (z & 0x800FFFFFFFFFFFFFull) | ((unsigned long long)(1023 - 40 + (int)((z >> 52) % 80)) << 52);
    double a = __longlong_as_double((long long)z);
    double q = clv::div_by<double>(a, b, y);
    double r = a / b;
    if (!same_d(q, r)) {
      unsigned long long k = atomicAdd(bad, 1ull);
      if (k < 4) first[k] = z;
    }
  }
}

extern "C" int run_f32(float b, unsigned long long* bad_out, unsigned int* first_out) {
  unsigned long long* bad;
  unsigned int* first;
  cudaMalloc(&bad, sizeof(unsigned long long));
  cudaMalloc(&first, 4 * sizeof(unsigned int));
  cudaMemset(bad, 0, sizeof(unsigned long long));
  cudaMemset(first, 0, 4 * sizeof(unsigned int));
  check_all_f32<<<148 * 16, 256>>>(b, bad, first);
  cudaMemcpy(bad_out, bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaMemcpy(first_out, first, 4 * sizeof(unsigned int), cudaMemcpyDeviceToHost);
  cudaFree(bad);
  cudaFree(first);
  return (int)cudaGetLastError();
}

extern "C" int run_f64(double b, unsigned long long n, unsigned long long seed, unsigned long long* bad_out,
                       unsigned long long* first_out) {
  unsigned long long *bad, *first;
  cudaMalloc(&bad, sizeof(unsigned long long));
  cudaMalloc(&first, 4 * sizeof(unsigned long long));
  cudaMemset(bad, 0, sizeof(unsigned long long));
  cudaMemset(first, 0, 4 * sizeof(unsigned long long));
  check_rand_f64<<<148 * 16, 256>>>(b, n, seed, bad, first);
  cudaMemcpy(bad_out, bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaMemcpy(first_out, first, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaFree(bad);
  cudaFree(first);
  return (int)cudaGetLastError();
}
