// tri_selftest.cu -- tri_selftest_division: checks on the device that the
// exact quotients from a correctly rounded reciprocal equal the IEEE quotient
// bit for bit: div_by_rcp over operands shaped like the step's (dt*d/dx,
// h*dx/2/dt: magnitudes 1e-14 .. 1e7 over divisors 1e-3 .. 1e3) and
// div_shared over every finite dividend magnitude (subnormals included,
// zeros of both signs) and divisors of either sign from 1e-30 to 1e30.
#include <cuda_runtime.h>

#include "tri_common.cuh"
#include "tri_internal.h"

using namespace tri;

namespace {

__device__ __forceinline__ unsigned long long mix(unsigned long long x) {
  // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ double unit(unsigned long long r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

__global__ void k_div_check(long long n, unsigned long long seed, unsigned long long* bad) {
  unsigned long long local = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long r1 = mix(seed ^ (2 * i)), r2 = mix(seed ^ (2 * i + 1));
    const double ea = -14.0 + 21.0 * unit(r1);  // |a| in 1e-14 .. 1e7
    const double eb = -3.0 + 6.0 * unit(r2);    // b in 1e-3 .. 1e3
    double a = exp10(ea) * ((r1 & 1) ? -1.0 : 1.0);
    const double b = exp10(eb);
    if ((r2 & 0xFF) == 0) a = 0.0;
    const double y = 1.0 / b;
    const double q = div_by_rcp(a, b, y);
    const double ref = a / b;
    if (__double_as_longlong(q) != __double_as_longlong(ref)) local++;
    // div_shared over any finite dividend (subnormal to 1e300) and divisors
    // 1e-30 .. 1e30
    const unsigned long long r3 = mix(seed ^ (0x5DEECE66Dull + 2 * i)), r4 = mix(r3);
    double a2 = exp10(-320.0 + 620.0 * unit(r3)) * ((r3 & 1) ? -1.0 : 1.0);
    if ((r4 & 0x3F) == 0) a2 = (r4 & 0x40) ? -0.0 : 0.0;
    const double b2 = exp10(-30.0 + 60.0 * unit(r4)) * ((r4 & 0x80) ? -1.0 : 1.0);
    const double q2 = div_shared(a2, b2, 1.0 / b2);
    if (__double_as_longlong(q2) != __double_as_longlong(a2 / b2)) local++;
  }
  if (local) atomicAdd(bad, local);
}

}  // namespace

extern "C" int tri_selftest_division(int64_t n, uint64_t seed, int64_t* mismatches) {
  TRI_CHECK_ARG(mismatches && n >= 0, "bad argument");
  unsigned long long* dbad = nullptr;
  TRI_CUDA_TRY(cudaMalloc(&dbad, sizeof(unsigned long long)));
  cudaMemset(dbad, 0, sizeof(unsigned long long));
  k_div_check<<<148 * 8, 256>>>(n, seed, dbad);
  cudaError_t e = cudaGetLastError();
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, dbad, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(dbad);
  if (e != cudaSuccess) return set_error(TRI_E_CUDA, "division self-test: %s", cudaGetErrorString(e));
  *mismatches = (int64_t)h;
  return TRI_OK;
}
