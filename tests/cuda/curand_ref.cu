// Test-only: cuRAND's Philox4_32_10 device generator, to pin the tracer's own
// Philox against NVIDIA's.  Output i is the first curand4() of a state
// initialised with (seed, subsequence = sub0 + i, offset = 4 * k).
#include <curand_kernel.h>
#include <stdint.h>

__global__ void curand_philox_kernel(unsigned long long seed, unsigned long long sub0, unsigned long long k, int n,
                                     uint4* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  curandStatePhilox4_32_10_t st;
  curand_init(seed, sub0 + i, 4ull * k, &st);
  out[i] = curand4(&st);
}

extern "C" int curand_ref_philox(unsigned long long seed, unsigned long long sub0, unsigned long long k, int n,
                                 void* d_out) {
  curand_philox_kernel<<<(n + 127) / 128, 128>>>(seed, sub0, k, n, (uint4*)d_out);
  if (cudaGetLastError() != cudaSuccess) return 1;
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}
