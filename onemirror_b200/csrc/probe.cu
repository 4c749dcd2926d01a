// probe.cu — measurement and test hooks: an FP32 FMA issue-rate probe (the
// roofline denominator for the FP32-bound tracer) and a Philox block dump.
#include <algorithm>

#include "internal.hpp"

using namespace qm;

namespace qm {

constexpr int kChains = 8;

// kChains independent FMA chains per thread; the result is written so the
// compiler keeps every FMA.
__global__ void __launch_bounds__(256) fma_probe_kernel(float* sink, int iters, float a, float b) {
  float acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = (float)(threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = fmaf(acc[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c];
  if (s == 1.2345f) sink[blockIdx.x] = s;  // never true for the probe's inputs; keeps the chains live
}

__global__ void recip_kernel(const double* x, int64_t n, double* rcp, double* rsq) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (rcp) rcp[i] = rcp_nr(x[i]);
  if (rsq) rsq[i] = rsqrt_nr(x[i]);
}

__global__ void philox_kernel(uint4 c0, uint2 key, int64_t n, uint4* out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint4 c = c0;
  c.x += (uint32_t)i;
  out[i] = philox4x32_10(c, key);
}

}  // namespace qm

extern "C" {

qmcrt_status qmcrt_fp32_peak_probe(float* d_sink, int32_t iters, double* flops, void* stream) {
  if (!d_sink || !flops || iters <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad probe arguments");
  int dev = 0, sms = 0;
  QM_CUDA(cudaGetDevice(&dev));
  QM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int blocks = sms * 8;
  fma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(d_sink, iters, 0.999999f, 1e-7f);
  QM_CUDA(cudaGetLastError());
  *flops = 2.0 * kChains * (double)iters * 256.0 * blocks;
  return QMCRT_OK;
}

qmcrt_status qmcrt_fp64_recip_probe(const double* d_x, int64_t n, double* d_rcp, double* d_rsqrt, void* stream) {
  if (!d_x || n <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad probe arguments");
  recip_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_x, n, d_rcp, d_rsqrt);
  QM_CUDA(cudaGetLastError());
  return QMCRT_OK;
}

qmcrt_status qmcrt_philox_blocks(const uint32_t ctr0[4], const uint32_t key[2], int64_t n, uint32_t* d_out,
                                 void* stream) {
  if (!ctr0 || !key || !d_out || n <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad philox arguments");
  philox_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      make_uint4(ctr0[0], ctr0[1], ctr0[2], ctr0[3]), make_uint2(key[0], key[1]), n, (uint4*)d_out);
  QM_CUDA(cudaGetLastError());
  return QMCRT_OK;
}

}  // extern "C"
