// selftest.cu -- on-device self-check of arithmetic the kernels rely on.
//
// adc_selftest_div_const compares div3/div6/div12 (adc_internal.cuh), which
// replace full divisions by those constants in the FP64 element kernels,
// with IEEE division bit for bit over random finite inputs of every
// exponent in the normal range, over inputs built next to multiples of the
// divisor (quotients with a zero, one-third and two-thirds fractional ulp),
// over signed zeros and infinities, and over a NaN.
#include "adc_internal.cuh"

namespace adc {

__device__ __forceinline__ unsigned long long splitmix(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_selftest_div(long long n, unsigned long long seed, unsigned long long *bad) {
  unsigned long long local = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const unsigned long long h = splitmix(seed + (unsigned long long)k);
    double x;
    if ((k & 3) != 3) {
      // random significand and sign, exponent in [-1000, 1000]
      const unsigned long long ex = 1023 - 1000 + (h >> 52) % 2001;
      x = __longlong_as_double((long long)((h & 0x800FFFFFFFFFFFFFull) | (ex << 52)));
    } else {
      // 3*m + d for a random integer m < 2^51 and d in {-1, 0, 1}, scaled
      const long long m = (long long)((h >> 13) & ((1ull << 51) - 1));
      const long long d = (long long)(h % 3) - 1;
      x = ldexp((double)(3 * m + d), (int)((h >> 8) % 400) - 200);
      if (h & 1) x = -x;
    }
    if (k == 0) x = 0.0;
    if (k == 1) x = -0.0;
    if (k == 2) x = __longlong_as_double(0x7FF0000000000000ll);    // +inf
    if (k == 3) x = __longlong_as_double((long long)0xFFF0000000000000ull);  // -inf
    if (k == 4) x = __longlong_as_double(0x7FF8000000000000ll);    // NaN
    const double q3 = x / 3.0, q6 = x / 6.0, q12 = x / 12.0;
    if (isnan(x)) {   // a NaN must stay a NaN (payload bits are not compared)
      local += !isnan(div3(x)) + !isnan(div6(x)) + !isnan(div12(x));
      continue;
    }
    if (__double_as_longlong(div3(x)) != __double_as_longlong(q3)) ++local;
    if (__double_as_longlong(div6(x)) != __double_as_longlong(q6)) ++local;
    if (__double_as_longlong(div12(x)) != __double_as_longlong(q12)) ++local;
  }
  if (local) atomicAdd(bad, local);
}

}  // namespace adc

using namespace adc;

extern "C" int adc_selftest_div_const(long long n, unsigned long long seed, long long *mismatches) {
  if (n < 0 || !mismatches) { set_error("adc_selftest_div_const: bad arguments"); return ADC_ERR_ARG; }
  unsigned long long *d = nullptr;
  ADC_CUDA(cudaMalloc((void **)&d, sizeof(unsigned long long)));
  ADC_CUDA(cudaMemset(d, 0, sizeof(unsigned long long)));
  k_selftest_div<<<4 * 148, 256>>>(n, seed, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "adc_selftest_div_const");
  *mismatches = (long long)h;
  return ADC_OK;
}
