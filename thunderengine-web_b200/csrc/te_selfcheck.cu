// Exhaustive self-check of rr_pow_fast (te_math.cuh): for an exponent p, every binary32
// bit pattern in [lo, hi) is raised to p by both routes, and the patterns whose results
// differ (as bits) are counted.  A diagnostic of the library's own arithmetic: the
// kernels call rr_pow_fast only with exponents this check has passed on all 2^31
// non-negative patterns (tests/test_gpu_parity.py).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/thunderstep.h"
#include "te_math.cuh"

namespace te {

__global__ void k_check_pow(float p, uint32_t lo, uint32_t hi, unsigned long long* bad, uint32_t* first) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)lo + blockIdx.x * blockDim.x + threadIdx.x; b < hi; b += step) {
    const float x = __uint_as_float((uint32_t)b);
    const uint32_t r1 = __float_as_uint(rr_pow_fast(x, p)), r2 = __float_as_uint(rr_pow_cr(x, p));
    if (r1 != r2) {
      atomicAdd(bad, 1ull);
      atomicMin(first, (uint32_t)b);
    }
  }
}

}  // namespace te

extern "C" int te_check_pow(float p, uint32_t lo, uint32_t hi, uint64_t* mismatches, uint32_t* first_bad) {
  if (!mismatches || !first_bad || hi < lo) return TE_EINVAL;
  unsigned long long* bad = nullptr;
  uint32_t* first = nullptr;
  cudaError_t e = cudaMalloc(&bad, sizeof(unsigned long long) + sizeof(uint32_t));
  if (e != cudaSuccess) return TE_ECUDA;
  first = reinterpret_cast<uint32_t*>(bad + 1);
  const uint32_t init_first = 0xffffffffu;
  e = cudaMemset(bad, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemcpy(first, &init_first, sizeof(uint32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    te::k_check_pow<<<148 * 8, 256>>>(p, lo, hi, bad, first);
    e = cudaGetLastError();
  }
  unsigned long long n = 0;
  uint32_t f = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&n, bad, sizeof(n), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&f, first, sizeof(f), cudaMemcpyDeviceToHost);
  cudaFree(bad);
  if (e != cudaSuccess) return TE_ECUDA;
  *mismatches = n;
  *first_bad = f;
  return TE_OK;
}
