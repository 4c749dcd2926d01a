// smooth.cu — trimmed-mean smoothing of flux maps (ImageSmoother::image_smooth,
// image_smooth.cu:10-115).
//
// Each CTA stages its 32x8 output tile plus a halo of `radius` into shared
// memory with coalesced loads, then each thread forms its clipped window.
// Exact order statistics for radii 1-3 sort the window in registers with a
// sorting network (smooth_sorted_kernel); larger radii insertion-sort into a
// per-thread array.
// Two definitions:
//  - QMCRT_TRIM_SORTED: exact order statistics.  On integer counts the kept
//    sum is an exact 64-bit integer and the mean is one IEEE division, so the
//    result is bit-exact against any correct implementation.
//  - QMCRT_TRIM_HEAPS: the reference's streaming max-heap / min-heap pair with
//    its else-if chain (heap.cuh:9-212), replayed in float in the same
//    row-major order with the same operation order, bit-exact against a float
//    replica of the reference kernel.
#include <algorithm>
#include <type_traits>

#include "internal.hpp"

using namespace qm;

namespace qm {

constexpr int kTileX = 32, kTileY = 8, kMaxRadius = 7;
constexpr int kMaxWin = (2 * kMaxRadius + 1) * (2 * kMaxRadius + 1);

template <typename T>
__device__ __forceinline__ float as_float(T v) {
  return (float)v;
}

// Heap with elements[1..num-1] and comparison `larger` (max) or `smaller` (min).
template <bool MAX>
struct RefHeap {
  float* e;
  int num, max;
  __device__ bool cmp(float a, float b) const { return MAX ? (a > b) : (a < b); }
  __device__ void insert(float v) {
    if (num == max) return;
    int i = num++;
    for (; i != 1 && cmp(v, e[i / 2]); i /= 2) e[i] = e[i / 2];
    e[i] = v;
  }
  __device__ void delete_and_insert(float v) {
    if (num == 1) return;
    int i = 1, c;
    for (; 2 * i < num;) {
      c = (2 * i + 1 >= num || cmp(e[2 * i], e[2 * i + 1])) ? 2 * i : 2 * i + 1;
      if (cmp(e[c], v)) {
        e[i] = e[c];
        i = c;
      } else {
        break;
      }
    }
    e[i] = v;
  }
  __device__ float sum() const {
    float s = 0.0f;
    for (int i = 1; i < num; ++i) s = __fadd_rn(s, e[i]);
    return s;
  }
};

// Exact order statistics for a small radius R, all in registers: the
// (2R+1)^2 window values (positions outside the map hold the type's largest
// value, so they sort after every real one) go through Batcher's odd-even
// merge sort network, fully unrolled so every index is a compile-time
// constant; the kept sum then runs over the sorted positions [k, cnt - k) in
// ascending order, the order the general path's insertion sort gives.
template <typename T>
__device__ __forceinline__ void cmp_swap(T& a, T& b) {
  const T lo = a < b ? a : b, hi = a < b ? b : a;
  a = lo;
  b = hi;
}

// The comparators of Batcher's odd-even merge sort for N keys, listed at
// compile time.
struct SortNet {
  int n;
  short a[640], b[640];
};

template <int N>
constexpr SortNet batcher_net() {
  SortNet net{};
  int c = 0;
  for (int p = 1; p < N; p <<= 1)
    for (int k = p; k >= 1; k >>= 1)
      for (int j = k % p; j + k < N; j += 2 * k)
        for (int i = 0; i < k; ++i)
          if (i + j + k < N && (i + j) / (2 * p) == (i + j + k) / (2 * p)) {
            net.a[c] = (short)(i + j);
            net.b[c] = (short)(i + j + k);
            ++c;
          }
  net.n = c;
  return net;
}

template <int N, typename T>
__device__ __forceinline__ void batcher_sort(T (&v)[N]) {
  constexpr SortNet net = batcher_net<N>();
  static_assert(net.n <= 640, "sorting network larger than its table");
#pragma unroll
  for (int c = 0; c < net.n; ++c) cmp_swap(v[net.a[c]], v[net.b[c]]);
}

template <typename T>
__device__ __forceinline__ T sort_pad() {
  if constexpr (std::is_integral<T>::value) return (T)0xFFFFFFFFu;
  else return __int_as_float(0x7f800000);  // +inf
}

template <typename T, int R>
__global__ void __launch_bounds__(kTileX* kTileY) smooth_sorted_kernel(const T* __restrict__ in,
                                                                       float* __restrict__ out, int w, int h,
                                                                       float ratio) {
  pdl_wait();
  pdl_trigger();
  constexpr int W = 2 * R + 1, N = W * W, TW = kTileX + 2 * R, TH = kTileY + 2 * R;
  __shared__ T tile[TW * TH];
  const int x0 = blockIdx.x * kTileX - R, y0 = blockIdx.y * kTileY - R;
  const int tid = threadIdx.y * kTileX + threadIdx.x;
  for (int i = tid; i < TW * TH; i += kTileX * kTileY) {
    const int yy = y0 + i / TW, xx = x0 + i % TW;
    tile[i] = (xx >= 0 && xx < w && yy >= 0 && yy < h) ? in[(int64_t)yy * w + xx] : sort_pad<T>();
  }
  __syncthreads();
  const int x = blockIdx.x * kTileX + threadIdx.x, y = blockIdx.y * kTileY + threadIdx.y;
  if (x >= w || y >= h) return;
  const int lx = max(x - R, 0), ly = max(y - R, 0), rx = min(x + R, w - 1), ry = min(y + R, h - 1);
  const int cnt = (rx - lx + 1) * (ry - ly + 1);
  const int k = (int)((float)cnt * ratio);  // image_smooth.cu:34
  T v[N];
#pragma unroll
  for (int dy = 0; dy < W; ++dy)
#pragma unroll
    for (int dx = 0; dx < W; ++dx) v[dy * W + dx] = tile[(threadIdx.y + dy) * TW + threadIdx.x + dx];
  batcher_sort<N>(v);
  const int lo = k, hi = cnt - k;
  if constexpr (std::is_integral<T>::value) {  // integer counts: exact sum
    unsigned long long s = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) s += (i >= lo && i < hi) ? (unsigned long long)v[i] : 0ull;
    out[(int64_t)y * w + x] = __fdiv_rn(__ull2float_rn(s), (float)(cnt - 2 * k));
  } else {
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i)
      if (i >= lo && i < hi) s = __fadd_rn(s, as_float(v[i]));
    out[(int64_t)y * w + x] = __fdiv_rn(s, (float)(cnt - 2 * k));
  }
}

template <typename T, int METHOD>
__global__ void __launch_bounds__(kTileX* kTileY) smooth_kernel(const T* __restrict__ in, float* __restrict__ out,
                                                                int w, int h, int r, float ratio) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);
  const int tw = kTileX + 2 * r, th = kTileY + 2 * r;
  const int x0 = blockIdx.x * kTileX - r, y0 = blockIdx.y * kTileY - r;
  const int tid = threadIdx.y * kTileX + threadIdx.x;
  for (int i = tid; i < tw * th; i += kTileX * kTileY) {
    int yy = y0 + i / tw, xx = x0 + i % tw;
    tile[i] = (xx >= 0 && xx < w && yy >= 0 && yy < h) ? in[(int64_t)yy * w + xx] : T(0);
  }
  __syncthreads();
  const int x = blockIdx.x * kTileX + threadIdx.x, y = blockIdx.y * kTileY + threadIdx.y;
  if (x >= w || y >= h) return;
  const int lx = max(x - r, 0), ly = max(y - r, 0), rx = min(x + r, w - 1), ry = min(y + r, h - 1);
  const int cnt = (rx - lx + 1) * (ry - ly + 1);
  const int k = (int)((float)cnt * ratio);  // image_smooth.cu:34
  if (METHOD == QMCRT_TRIM_HEAPS) {
    float buf[2 * (kMaxWin / 2 + 2)];
    RefHeap<true> mx{buf, 1, k + 1};
    RefHeap<false> mn{buf + kMaxWin / 2 + 2, 1, k + 1};
    float value = 0.0f;
    for (int rr = ly; rr <= ry; ++rr)
      for (int cc = lx; cc <= rx; ++cc) {
        float cur = as_float(tile[(rr - y0) * tw + (cc - x0)]);
        value = __fadd_rn(value, cur);
        if (mx.num != mx.max) {
          mx.insert(cur);
          mn.insert(cur);
        } else if (mx.num > 1 && cur < mx.e[1]) {
          mx.delete_and_insert(cur);
        } else if (mn.num > 1 && cur > mn.e[1]) {
          mn.delete_and_insert(cur);
        }
      }
    float num = __fsub_rn(__fsub_rn(value, mx.sum()), mn.sum());
    out[(int64_t)y * w + x] = __fdiv_rn(num, (float)(cnt - 2 * k));
    return;
  }
  T v[kMaxWin];
  int m = 0;
  for (int rr = ly; rr <= ry; ++rr)
    for (int cc = lx; cc <= rx; ++cc) {
      T cur = tile[(rr - y0) * tw + (cc - x0)];
      int j = m++;
      while (j > 0 && v[j - 1] > cur) {
        v[j] = v[j - 1];
        --j;
      }
      v[j] = cur;
    }
  if constexpr (std::is_integral<T>::value) {  // integer counts: exact sum
    unsigned long long s = 0;
    for (int i = k; i < cnt - k; ++i) s += (unsigned long long)v[i];
    out[(int64_t)y * w + x] = __fdiv_rn(__ull2float_rn(s), (float)(cnt - 2 * k));
  } else {
    float s = 0.0f;
    for (int i = k; i < cnt - k; ++i) s = __fadd_rn(s, as_float(v[i]));
    out[(int64_t)y * w + x] = __fdiv_rn(s, (float)(cnt - 2 * k));
  }
}

template <typename T>
static qmcrt_status smooth(const T* d_in, float* d_out, int w, int h, int r, float ratio, int method,
                           cudaStream_t st) {
  if (!d_in || !d_out) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL map");
  if (w <= 0 || h <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "map size must be positive");
  if (r < 0 || r > kMaxRadius) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "radius must be in [0, 7]");
  if (!(ratio >= 0.f && ratio < 0.5f)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "ratio must be in [0, 0.5)");
  const char* a0 = (const char*)d_in;
  const char* a1 = a0 + (size_t)w * h * sizeof(T);
  const char* b0 = (const char*)d_out;
  const char* b1 = b0 + (size_t)w * h * sizeof(float);
  if (a0 < b1 && b0 < a1) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "input and output maps overlap");
  dim3 block(kTileX, kTileY), grid((w + kTileX - 1) / kTileX, (h + kTileY - 1) / kTileY);
  size_t smem = (size_t)(kTileX + 2 * r) * (kTileY + 2 * r) * sizeof(T);
  // launched with programmatic stream serialization: each kernel waits for
  // the stream's previous kernel in pdl_wait() before touching memory
  cudaError_t ce;
  if (method == QMCRT_TRIM_SORTED && r == 1) ce = launch_pdl(true, smooth_sorted_kernel<T, 1>, grid, block, 0, st, d_in, d_out, w, h, ratio);
  else if (method == QMCRT_TRIM_SORTED && r == 2) ce = launch_pdl(true, smooth_sorted_kernel<T, 2>, grid, block, 0, st, d_in, d_out, w, h, ratio);
  else if (method == QMCRT_TRIM_SORTED && r == 3) ce = launch_pdl(true, smooth_sorted_kernel<T, 3>, grid, block, 0, st, d_in, d_out, w, h, ratio);
  else if (method == QMCRT_TRIM_SORTED) ce = launch_pdl(true, smooth_kernel<T, QMCRT_TRIM_SORTED>, grid, block, smem, st, d_in, d_out, w, h, r, ratio);
  else if (method == QMCRT_TRIM_HEAPS) ce = launch_pdl(true, smooth_kernel<T, QMCRT_TRIM_HEAPS>, grid, block, smem, st, d_in, d_out, w, h, r, ratio);
  else return set_error(QMCRT_ERR_INVALID_ARGUMENT, "unknown trimmed-mean method");
  QM_CUDA(ce);
  return QMCRT_OK;
}

}  // namespace qm

extern "C" {

qmcrt_status qmcrt_smooth_trimmed_u32(const uint32_t* d_in, float* d_out, int32_t width, int32_t height,
                                      int32_t radius, float ratio, int32_t method, void* stream) {
  return smooth<uint32_t>(d_in, d_out, width, height, radius, ratio, method, (cudaStream_t)stream);
}

qmcrt_status qmcrt_smooth_trimmed_f32(const float* d_in, float* d_out, int32_t width, int32_t height,
                                      int32_t radius, float ratio, int32_t method, void* stream) {
  return smooth<float>(d_in, d_out, width, height, radius, ratio, method, (cudaStream_t)stream);
}

}  // extern "C"
