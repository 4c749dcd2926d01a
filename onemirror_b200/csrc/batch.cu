// batch.cu — many (field, sun) items in one persistent launch.
//
// The reference traces one heliostat per launch and synchronises after each
// (ray_tracing.cu:23-27), once per sun position (main.cpp:56-114).  Here a
// whole day over several fields is one pass: per item the aiming and grid
// kernels, then ONE persistent trace kernel whose CTAs pull fixed-size ray
// chunks from a global counter (load balance across items of uneven size and
// no per-item tail), then one flux-scaling kernel over all items.  The pass is
// stream-ordered and host-free, so it is captured once into a CUDA graph and
// replayed.  An autotuner picks the chunk size, the resident CTAs per SM and
// the side of a CTA-private shared-memory flux tile.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <type_traits>
#include <vector>

#include "internal.hpp"
#include "trace.cuh"

using namespace qm;

namespace qm {
void fill_trace_args(qmcrt_scene* s, const SunGeom& geo, const qmcrt_sun* sun, uint32_t quirks, TraceArgs* a);

constexpr int kBatchThreads = 256;

// Deposit through a CTA-private tile of T x T pixels anchored at (r0, c0);
// pixels outside the tile go straight to the global maps.
template <int T>
struct TileDeposit {
  uint32_t* s_cnt;
  float* s_en;
  int r0, c0, res_x;
  uint32_t* counts;
  float* energy;
  __device__ __forceinline__ void operator()(int pix, float e) const {
    int r = pix / res_x - r0, c = pix - (pix / res_x) * res_x - c0;
    if (T > 0 && (unsigned)r < (unsigned)T && (unsigned)c < (unsigned)T) {
      atomicAdd(s_cnt + r * T + c, 1u);
      atomicAdd(s_en + r * T + c, e);
    } else {
      red_add(counts + pix, 1u);
      red_add(energy + pix, e);
    }
  }
};

// Anchor of a chunk's tile: the pixel hit by the unperturbed reflection of
// the sun axis from the chunk's first point (tile centred there), or no tile.
__device__ bool chunk_anchor(const TraceArgs& a, uint32_t ray, int T, int* r0, int* c0) {
  const uint32_t g = a.rpp_shift >= 0 ? ray >> a.rpp_shift : ray / (uint32_t)a.rpp;
  const int h = __ldg(a.point_helio + g);
  const double* F = a.frame + kFrameStride * h;
  frame64 fr;
  fr.u = mk(__ldg(F + 0), __ldg(F + 1), __ldg(F + 2));
  fr.n = mk(__ldg(F + 3), __ldg(F + 4), __ldg(F + 5));
  fr.v = mk(__ldg(F + 6), __ldg(F + 7), __ldg(F + 8));
  const float2 xz = __ldg(a.point_xz + g);
  d3 o = mk(__ldg(F + 9), __ldg(F + 10), __ldg(F + 11)) + (double)xz.x * fr.u + (double)xz.y * fr.v;
  d3 s = mk(a.sdir[0], a.sdir[1], a.sdir[2]);
  d3 rd = s - (2.0 * dot(s, fr.n)) * fr.n;
  int pix = -1;
  if (!receiver_hit(a, o, rd, pix) || pix < 0) return false;
  *r0 = pix / a.res_x - T / 2;
  *c0 = pix % a.res_x - T / 2;
  return true;
}

// The Philox round keys of a batch's seed (every item shares it), passed as
// a launch parameter so that the rounds read them from the constant bank
// rather than from the shared-memory copy of the item's arguments.
struct PhiloxKeys {
  uint2 rk[10];
};

// LEAN: every item has a flat receiver and takes the plain tracer's lean
// build (power-of-two rays per point, point masks, no attenuation, no
// quirks).
template <int T, bool LEAN = false>
__global__ void __launch_bounds__(kBatchThreads, 4)
    batch_trace_kernel(const TraceArgs* __restrict__ items, const unsigned long long* __restrict__ chunk_begin,
                       int n_items, uint32_t chunk_rays, unsigned long long total_chunks,
                       unsigned long long* counter, const __grid_constant__ PhiloxKeys keys) {
  __shared__ TraceArgs s_a;
  __shared__ float4 s_tab[kBuieRecords];
  __shared__ unsigned long long s_c;
  __shared__ int s_item, s_anchor[3];
  // the flux tile (T > 0) in dynamic shared memory: T^2 counts, then T^2 energies
  extern __shared__ uint32_t s_cnt[];
  float* s_en = reinterpret_cast<float*>(s_cnt + T * T);
  int cur = -1;
  const float* loaded = nullptr;
  float fy0 = 0.f, fy1 = 0.f;
  RayCounters cnt;
  if constexpr (T > 0)
    for (int i = threadIdx.x; i < T * T; i += blockDim.x) {
      s_cnt[i] = 0;
      s_en[i] = 0.f;
    }
  for (;;) {
    if (threadIdx.x == 0) {
      unsigned long long c = atomicAdd(counter, 1ull);
      int it = -1;
      if (c < total_chunks) {  // largest item whose first chunk is <= c
        int lo = 0, hi = n_items - 1;
        while (lo < hi) {
          int mid = (lo + hi + 1) >> 1;
          if (__ldg(chunk_begin + mid) <= c) lo = mid;
          else hi = mid - 1;
        }
        it = lo;
      }
      s_c = c;
      s_item = it;
    }
    __syncthreads();
    const unsigned long long c = s_c;
    const int it = s_item;
    if (c >= total_chunks) break;
    if (it != cur) {
      const int* src = reinterpret_cast<const int*>(items + it);
      int* dst = reinterpret_cast<int*>(&s_a);
      for (int i = threadIdx.x; i < (int)(sizeof(TraceArgs) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
      __syncthreads();
      if (s_a.buie != loaded) {
        load_buie(s_a.buie, s_tab);
        loaded = s_a.buie;
      }
      fy0 = from_ordered(__ldg(s_a.field_yr));
      fy1 = from_ordered(__ldg(s_a.field_yr + 1));
      cur = it;
      __syncthreads();
    }
    const unsigned long long r0 = (c - __ldg(chunk_begin + it)) * (unsigned long long)chunk_rays;
    const unsigned long long r1 = min(r0 + chunk_rays, (unsigned long long)s_a.rays);
    if constexpr (T > 0) {
      if (threadIdx.x == 0) {
        int ar = 0, ac = 0;
        s_anchor[2] = chunk_anchor(s_a, (uint32_t)r0, T, &ar, &ac) ? 1 : 0;
        s_anchor[0] = ar;
        s_anchor[1] = ac;
      }
      __syncthreads();
      const TileDeposit<T> dep{s_cnt, s_en, s_anchor[2] ? s_anchor[0] : -(1 << 30), s_anchor[1], s_a.res_x,
                               s_a.counts, s_a.energy};
      for (unsigned long long r = r0 + threadIdx.x; r < r1; r += blockDim.x)
        trace_ray<false, false, false, 3, std::decay_t<decltype(dep)>, LEAN ? QMCRT_RECEIVER_FLAT : -1, LEAN>(
            s_a, s_tab, (uint32_t)r, fy0, fy1, cnt, dep, keys.rk);
      __syncthreads();
      if (s_anchor[2]) {  // flush the tile's non-zero pixels, then clear it
        for (int i = threadIdx.x; i < T * T; i += blockDim.x) {
          uint32_t k = s_cnt[i];
          if (k) {
            int pr = s_anchor[0] + i / T, pc = s_anchor[1] + i % T;
            int pix = pr * s_a.res_x + pc;
            red_add(s_a.counts + pix, k);
            red_add(s_a.energy + pix, s_en[i]);
            s_cnt[i] = 0;
            s_en[i] = 0.f;
          }
        }
      }
    } else {
      const GlobalDeposit dep{s_a.counts, s_a.energy};
      for (unsigned long long r = r0 + threadIdx.x; r < r1; r += blockDim.x)
        trace_ray<false, false, false, 3, std::decay_t<decltype(dep)>, LEAN ? QMCRT_RECEIVER_FLAT : -1, LEAN>(
            s_a, s_tab, (uint32_t)r, fy0, fy1, cnt, dep, keys.rk);
    }
    __syncthreads();  // everyone is done with s_c / s_a / the tile before the next chunk
  }
}

struct BatchFinalize {
  const uint32_t* counts;
  const float* energy;
  float* flux;
  float scale;
  int64_t res;
  double* intercepted;  // sum of energy
};

__global__ void batch_finalize_kernel(const BatchFinalize* __restrict__ f) {
  const BatchFinalize a = f[blockIdx.y];
  double acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.res; i += (int64_t)gridDim.x * blockDim.x) {
    float e = a.energy[i];
    acc += e;
    a.flux[i] = e * a.scale;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc != 0) atomicAdd(a.intercepted, acc);
}

template <class T>
static qmcrt_status balloc(T** p, size_t count) {
  *p = nullptr;
  QM_CUDA(cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T)));
  return QMCRT_OK;
}

}  // namespace qm

struct qmcrt_batch {
  bool lean = false;  // every item takes the lean build of the tracer (batch_trace_kernel's LEAN)
  struct Item {
    qmcrt_scene* scene = nullptr;
    qmcrt_sun sun{};
    double sdir[3];
    qm::SunGeom geo;
    uint32_t* d_counts = nullptr;
    float* d_energy = nullptr;
    float* d_flux = nullptr;
    uint4* d_mask = nullptr;  // per-point candidate masks (and sigma, weight) for this item's sun
    double4* d_origin = nullptr;  // the points in world coordinates for this item's sun
    const float* weight = nullptr;  // [n] mirror area per point of the item's scene
    const float2* pts = nullptr;
    const int32_t* pts_helio = nullptr;
    int64_t points = 0;
    int64_t res = 0;
    float scale = 0.f;
  };
  std::vector<Item> items;
  // the scenes' sample points and weights, copied so later traces of a scene
  // with other point parameters cannot move them under the batch
  std::vector<float2*> pts;
  std::vector<int32_t*> pts_helio;
  std::vector<float*> weights;
  qmcrt_trace_params params{};
  std::map<float, qm::BuieTable> tables;
  std::map<float, float*> d_tables;
  qm::TraceArgs* d_args = nullptr;
  unsigned long long* d_chunk_begin = nullptr;
  unsigned long long* d_counter = nullptr;
  double* d_intercepted = nullptr;  // [items]
  qm::BatchFinalize* d_fin = nullptr;
  std::vector<unsigned long long> chunk_begin;  // host copy [items+1]
  qmcrt_batch_tuning tuning{65536, 4, 0, 0.f};
  int sms = 148;
  qm::PhiloxKeys keys{};  // round keys of params.seed
  cudaStream_t cap_stream = nullptr;
  // the items' geometry is rebuilt on kGeomStreams side streams forked from
  // the pass's stream and joined before the trace (parallel graph branches)
  static constexpr int kGeomStreams = 8;
  cudaStream_t side[kGeomStreams] = {};
  cudaEvent_t fork = nullptr, join[kGeomStreams] = {};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace qm {

static qmcrt_status upload_chunks(qmcrt_batch* b, cudaStream_t st) {
  b->chunk_begin.assign(b->items.size() + 1, 0);
  uint64_t per = ((uint64_t)b->params.rays + b->tuning.chunk_rays - 1) / b->tuning.chunk_rays;
  for (size_t i = 0; i < b->items.size(); ++i) b->chunk_begin[i + 1] = b->chunk_begin[i] + per;
  QM_CUDA(cudaMemcpyAsync(b->d_chunk_begin, b->chunk_begin.data(), b->chunk_begin.size() * sizeof(unsigned long long),
                          cudaMemcpyHostToDevice, st));
  QM_CUDA(cudaStreamSynchronize(st));  // the host vector may change before a later upload
  return QMCRT_OK;
}

// Dynamic shared memory of the batched kernel's T x T tile: T^2 counts and
// T^2 energies, beside the staged Buie table.
template <int T>
constexpr int batch_tile_bytes() {
  return T * T * (int)(sizeof(uint32_t) + sizeof(float));
}

// Allow the tiles' dynamic shared memory (static + dynamic above 48 KB);
// done once per batch, outside any graph capture.
static cudaError_t batch_allow_tiles() {
  cudaError_t ce = cudaFuncSetAttribute(batch_trace_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        batch_tile_bytes<32>());
  if (ce == cudaSuccess)
    ce = cudaFuncSetAttribute(batch_trace_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              batch_tile_bytes<48>());
  if (ce == cudaSuccess)
    ce = cudaFuncSetAttribute(batch_trace_kernel<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              batch_tile_bytes<32>());
  if (ce == cudaSuccess)
    ce = cudaFuncSetAttribute(batch_trace_kernel<48, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              batch_tile_bytes<48>());
  return ce;
}

// One launch of the batched kernel with a T x T tile (T = 0: none).
template <int T>
static cudaError_t launch_batch(qmcrt_batch* b, int ctas, int items, unsigned long long total, cudaStream_t st) {
  if (b->lean)
    batch_trace_kernel<T, true><<<ctas, kBatchThreads, batch_tile_bytes<T>(), st>>>(
        b->d_args, b->d_chunk_begin, items, b->tuning.chunk_rays, total, b->d_counter, b->keys);
  else
    batch_trace_kernel<T><<<ctas, kBatchThreads, batch_tile_bytes<T>(), st>>>(
        b->d_args, b->d_chunk_begin, items, b->tuning.chunk_rays, total, b->d_counter, b->keys);
  return cudaGetLastError();
}

// The trace pass alone over the first n items (all items when n < 0).
static qmcrt_status enqueue_trace(qmcrt_batch* b, int n, cudaStream_t st) {
  int items = n < 0 ? (int)b->items.size() : std::min<int>(n, (int)b->items.size());
  unsigned long long total = b->chunk_begin[items];
  QM_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), st));
  int ctas = std::max(1, std::min(4, b->tuning.ctas_per_sm)) * b->sms;
  ctas = (int)std::min<unsigned long long>((unsigned long long)ctas, std::max<unsigned long long>(total, 1));
  switch (b->tuning.tile) {
    case 32:
      QM_CUDA(launch_batch<32>(b, ctas, items, total, st));
      break;
    case 48:
      QM_CUDA(launch_batch<48>(b, ctas, items, total, st));
      break;
    default:
      QM_CUDA(launch_batch<0>(b, ctas, items, total, st));
  }
  return QMCRT_OK;
}

static qmcrt_status enqueue_pass(qmcrt_batch* b, cudaStream_t st) {
  qmcrt_status e;
  // every item's geometry depends only on its own sun and scene: the small
  // kernels of different items run side by side
  constexpr int K = qmcrt_batch::kGeomStreams;
  QM_CUDA(cudaEventRecord(b->fork, st));
  for (int j = 0; j < K; ++j) QM_CUDA(cudaStreamWaitEvent(b->side[j], b->fork, 0));
  for (size_t i = 0; i < b->items.size(); ++i) {
    auto& it = b->items[i];
    cudaStream_t s = b->side[i % K];
    // the items' rays test occluder candidates: their grids are built only
    // where a list overflows, or for every ray when the sunshape is too wide
    // for the candidate cones
    if ((e = launch_sun_geom(it.scene, it.geo, it.sdir, 0, s, false, !b->tables.at(it.sun.csr).within_alpha))) return e;
    if ((e = launch_point_masks(it.scene, it.geo, it.sdir, it.pts, it.pts_helio, it.weight, it.points, it.d_mask, it.d_origin, s)))
      return e;
    QM_CUDA(cudaMemsetAsync(it.d_counts, 0, it.res * sizeof(uint32_t), s));
    QM_CUDA(cudaMemsetAsync(it.d_energy, 0, it.res * sizeof(float), s));
  }
  for (int j = 0; j < K; ++j) {
    QM_CUDA(cudaEventRecord(b->join[j], b->side[j]));
    QM_CUDA(cudaStreamWaitEvent(st, b->join[j], 0));
  }
  QM_CUDA(cudaMemsetAsync(b->d_intercepted, 0, b->items.size() * sizeof(double), st));
  if ((e = enqueue_trace(b, -1, st))) return e;
  int64_t maxres = 0;
  for (auto& it : b->items) maxres = std::max(maxres, it.res);
  dim3 grid((unsigned)std::min<int64_t>((maxres + 255) / 256, 64), (unsigned)b->items.size());
  batch_finalize_kernel<<<grid, 256, 0, st>>>(b->d_fin);
  QM_CUDA(cudaGetLastError());
  return QMCRT_OK;
}

static void drop_graph(qmcrt_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

}  // namespace qm

extern "C" {

qmcrt_status qmcrt_batch_create(qmcrt_scene* const* scenes, int32_t n_scenes, const qmcrt_batch_item* items,
                                int32_t n_items, const qmcrt_trace_params* params, qmcrt_batch** out) {
  if (!out || !scenes || !items || !params || n_scenes <= 0 || n_items <= 0)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL or empty batch arguments");
  *out = nullptr;
  if (params->quirks & (QMCRT_QUIRK_SKIP_ORIGIN_CELL | QMCRT_QUIRK_AABB_RADIUS | QMCRT_QUIRK_SELF_HIT |
                        QMCRT_QUIRK_PIXEL_EDGE))
    return set_error(QMCRT_ERR_NOT_SUPPORTED, "batches trace in corrected mode only");
  if (params->attenuation != QMCRT_ATTEN_NONE && params->attenuation != QMCRT_ATTEN_POLY_EXP)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "unknown attenuation mode");
  if (params->ray_end != 0) return set_error(QMCRT_ERR_NOT_SUPPORTED, "batch items trace every ray");
  if (params->point_mode != QMCRT_POINTS_POISSON || params->rays_per_point <= 0 || params->rays == 0 ||
      params->rays > 0xFFFFFFFFull)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "batches need Poisson points and 0 < rays < 2^32");
  {
    const cudaError_t ce = batch_allow_tiles();
    if (ce != cudaSuccess) return cuda_error(ce, "batch tile shared memory");
  }
  qmcrt_batch* b = new qmcrt_batch();
  b->params = *params;
  qmcrt_status e = QMCRT_OK;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t st = nullptr;
  std::vector<TraceArgs> args(n_items);
  std::vector<BatchFinalize> fin(n_items);
  b->pts.assign(n_scenes, nullptr);
  b->pts_helio.assign(n_scenes, nullptr);
  b->weights.assign(n_scenes, nullptr);
  for (int s = 0; s < n_scenes; ++s) {
    if (!scenes[s]) { e = set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL scene"); goto fail; }
    if ((e = ensure_points(scenes[s], params, st))) goto fail;
    int64_t np = scenes[s]->points;
    if ((e = balloc(&b->pts[s], np)) || (e = balloc(&b->pts_helio[s], np)) || (e = balloc(&b->weights[s], scenes[s]->n)))
      goto fail;
    cudaError_t ce = cudaMemcpy(b->pts[s], scenes[s]->d_point_xz, np * sizeof(float2), cudaMemcpyDeviceToDevice);
    if (ce == cudaSuccess)
      ce = cudaMemcpy(b->pts_helio[s], scenes[s]->d_point_helio, np * sizeof(int32_t), cudaMemcpyDeviceToDevice);
    if (ce == cudaSuccess)
      ce = cudaMemcpy(b->weights[s], scenes[s]->d_helio_weight, scenes[s]->n * sizeof(float), cudaMemcpyDeviceToDevice);
    if (ce != cudaSuccess) { e = cuda_error(ce, "batch point copy"); goto fail; }
  }
  if ((e = balloc(&b->d_intercepted, n_items))) goto fail;
  b->items.resize(n_items);
  for (int i = 0; i < n_items; ++i) {
    auto& it = b->items[i];
    if (items[i].scene < 0 || items[i].scene >= n_scenes) { e = set_error(QMCRT_ERR_INVALID_ARGUMENT, "item scene index out of range"); goto fail; }
    it.scene = scenes[items[i].scene];
    it.sun = items[i].sun;
    double l = std::sqrt((double)it.sun.dir[0] * it.sun.dir[0] + (double)it.sun.dir[1] * it.sun.dir[1] +
                         (double)it.sun.dir[2] * it.sun.dir[2]);
    if (!(l > 0) || !(it.sun.csr > 0.f && it.sun.csr < 1.f)) { e = set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad item sun"); goto fail; }
    for (int k = 0; k < 3; ++k) it.sdir[k] = it.sun.dir[k] / l;
    if ((e = alloc_sun_geom(it.scene, &it.geo))) goto fail;
    it.res = (int64_t)it.scene->rg.res_x * it.scene->rg.res_y;
    if ((e = balloc(&it.d_counts, it.res)) || (e = balloc(&it.d_energy, it.res)) || (e = balloc(&it.d_flux, it.res))) goto fail;
    float csr = it.sun.csr;
    if (!b->tables.count(csr)) {
      if (!buie_bucket_table(csr, &b->tables[csr])) {
        e = set_error(QMCRT_ERR_INTERNAL, "Buie table: a bucket holds two interval boundaries");
        goto fail;
      }
      float* d = nullptr;
      if ((e = balloc(&d, b->tables[csr].host.size()))) goto fail;
      b->d_tables[csr] = d;
      cudaError_t ce = cudaMemcpy(d, b->tables[csr].host.data(), b->tables[csr].host.size() * sizeof(float),
                                  cudaMemcpyHostToDevice);
      if (ce != cudaSuccess) { e = cuda_error(ce, "batch table upload"); goto fail; }
    }
    TraceArgs& a = args[i];
    std::memset(&a, 0, sizeof(a));
    fill_trace_args(it.scene, it.geo, &it.sun, 0, &a);
    const BuieTable& t = b->tables[csr];
    a.buie = b->d_tables[csr];
    if (!t.within_alpha) { a.cand = nullptr; a.cand_n = nullptr; }  // the item's rays walk the grid
    a.b_total = t.params[3];
    a.b_core = t.params[2];
    a.b_B = t.params[4];
    a.b_C = t.params[5];
    a.b_inv = 1 / (t.params[1] + 1);
    a.b_inv_bucket = t.inv_bucket;
    a.rays = (uint32_t)params->rays;
    a.atten = params->attenuation;
    a.rpp = params->rays_per_point;
    a.rpp_shift = (a.rpp & (a.rpp - 1)) ? -1 : __builtin_ctz((unsigned)a.rpp);
    philox_round_keys(make_uint2((uint32_t)params->seed, (uint32_t)(params->seed >> 32)), a.rk);
    std::memcpy(b->keys.rk, a.rk, sizeof(b->keys.rk));
    a.item = (uint32_t)i;
    a.point_xz = b->pts[items[i].scene];
    a.point_helio = b->pts_helio[items[i].scene];
    it.pts = a.point_xz;
    it.pts_helio = a.point_helio;
    it.weight = b->weights[items[i].scene];
    it.points = scenes[items[i].scene]->points;
    if ((e = balloc(&it.d_mask, it.points)) || (e = balloc(&it.d_origin, it.points))) goto fail;
    // all bits set until a pass builds the masks, sigmas and weights for the
    // item's sun (every pass builds them before it traces)
    if (cudaMemset(it.d_mask, 0xFF, it.points * sizeof(uint4)) != cudaSuccess) {
      e = set_error(QMCRT_ERR_CUDA, "batch mask initialisation");
      goto fail;
    }
    a.point_mask = it.d_mask;
    a.point_origin = it.d_origin;
    a.weight = b->weights[items[i].scene];
    a.counts = it.d_counts;
    a.energy = it.d_energy;
    it.scale = (float)((double)it.sun.dni * params->reflectivity / ((double)params->rays_per_point * it.scene->rg.pixel_area));
    fin[i] = BatchFinalize{it.d_counts, it.d_energy, it.d_flux, it.scale, it.res, b->d_intercepted + i};
  }
  if ((e = balloc(&b->d_args, n_items)) || (e = balloc(&b->d_fin, n_items)) ||
      (e = balloc(&b->d_chunk_begin, n_items + 1)) || (e = balloc(&b->d_counter, 1)))
    goto fail;
  {
    cudaError_t ce = cudaMemcpy(b->d_args, args.data(), n_items * sizeof(TraceArgs), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(b->d_fin, fin.data(), n_items * sizeof(BatchFinalize), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    for (int j = 0; j < qmcrt_batch::kGeomStreams && ce == cudaSuccess; ++j) {
      ce = cudaStreamCreateWithFlags(&b->side[j], cudaStreamNonBlocking);
      if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&b->join[j], cudaEventDisableTiming);
    }
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (ce != cudaSuccess) { e = cuda_error(ce, "batch upload"); goto fail; }
  }
  // the lean build when every item allows it: flat receivers, power-of-two
  // rays per point, no attenuation (items carry no quirks; every item has
  // point masks)
  b->lean = (params->rays_per_point & (params->rays_per_point - 1)) == 0 &&
            params->attenuation == QMCRT_ATTEN_NONE;
  for (auto& it : b->items) b->lean = b->lean && it.scene->rg.type == QMCRT_RECEIVER_FLAT;
  if ((e = upload_chunks(b, nullptr))) goto fail;
  *out = b;
  return QMCRT_OK;
fail:
  qmcrt_batch_destroy(b);
  return e;
}

qmcrt_status qmcrt_batch_destroy(qmcrt_batch* b) {
  if (!b) return QMCRT_OK;
  drop_graph(b);
  for (auto& it : b->items) {
    free_sun_geom(&it.geo);
    cudaFree(it.d_mask);
    cudaFree(it.d_origin);
    cudaFree(it.d_counts);
    cudaFree(it.d_energy);
    cudaFree(it.d_flux);
  }
  for (auto& kv : b->d_tables) cudaFree(kv.second);
  for (auto* p : b->pts) cudaFree(p);
  for (auto* p : b->pts_helio) cudaFree(p);
  for (auto* p : b->weights) cudaFree(p);
  cudaFree(b->d_args);
  cudaFree(b->d_fin);
  cudaFree(b->d_chunk_begin);
  cudaFree(b->d_counter);
  cudaFree(b->d_intercepted);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  for (int j = 0; j < qmcrt_batch::kGeomStreams; ++j) {
    if (b->side[j]) cudaStreamDestroy(b->side[j]);
    if (b->join[j]) cudaEventDestroy(b->join[j]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
  return QMCRT_OK;
}

qmcrt_status qmcrt_batch_set_tuning(qmcrt_batch* b, const qmcrt_batch_tuning* t) {
  if (!b || !t) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (t->chunk_rays < 256 || t->chunk_rays % 256 || t->ctas_per_sm < 1 || t->ctas_per_sm > 4 ||
      (t->tile != 0 && t->tile != 32 && t->tile != 48))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "tuning out of range");
  b->tuning = *t;
  drop_graph(b);
  return upload_chunks(b, nullptr);
}

qmcrt_status qmcrt_batch_autotune(qmcrt_batch* b, qmcrt_batch_tuning* chosen, void* stream) {
  if (!b) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL batch");
  cudaStream_t st = (cudaStream_t)stream;
  qmcrt_status e;
  // geometry of the items the tuner runs on
  int n = std::min<int>((int)b->items.size(), 12);
  for (int i = 0; i < n; ++i) {
    auto& it = b->items[i];
    if ((e = launch_sun_geom(it.scene, it.geo, it.sdir, 0, st, false, !b->tables.at(it.sun.csr).within_alpha))) return e;
    if ((e = launch_point_masks(it.scene, it.geo, it.sdir, it.pts, it.pts_helio, it.weight, it.points, it.d_mask, it.d_origin, st)))
      return e;
  }
  cudaEvent_t e0, e1;
  QM_CUDA(cudaEventCreate(&e0));
  QM_CUDA(cudaEventCreate(&e1));
  qmcrt_batch_tuning best{0, 0, 0, 1e30f};
  const int chunks[] = {16384, 65536, 262144};
  const int ctas[] = {3, 4};
  const int tiles[] = {0, 32, 48};
  for (int ch : chunks)
    for (int ct : ctas)
      for (int ti : tiles) {
        qmcrt_batch_tuning t{ch, ct, ti, 0.f};
        b->tuning = t;
        if ((e = upload_chunks(b, st))) return e;
        float ms = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
          QM_CUDA(cudaEventRecord(e0, st));
          if ((e = enqueue_trace(b, n, st))) return e;
          QM_CUDA(cudaEventRecord(e1, st));
          QM_CUDA(cudaEventSynchronize(e1));
          float m = 0;
          QM_CUDA(cudaEventElapsedTime(&m, e0, e1));
          if (rep) ms = m;  // the first run warms the caches
        }
        if (ms < best.ms) {
          best = t;
          best.ms = ms;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tuning = best;
  drop_graph(b);
  if ((e = upload_chunks(b, st))) return e;
  if (chosen) *chosen = best;
  return QMCRT_OK;
}

qmcrt_status qmcrt_batch_run(qmcrt_batch* b, void* stream) {
  if (!b) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL batch");
  return enqueue_pass(b, (cudaStream_t)stream);
}

qmcrt_status qmcrt_batch_capture(qmcrt_batch* b) {
  if (!b) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL batch");
  drop_graph(b);
  QM_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
  qmcrt_status e = enqueue_pass(b, b->cap_stream);
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(b->cap_stream, &g);
  if (e) {
    if (g) cudaGraphDestroy(g);
    return e;
  }
  if (ce != cudaSuccess) return cuda_error(ce, "cudaStreamEndCapture");
  b->graph = g;
  QM_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
  return QMCRT_OK;
}

qmcrt_status qmcrt_batch_launch(qmcrt_batch* b, void* stream) {
  if (!b || !b->exec) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "no captured graph (call qmcrt_batch_capture)");
  QM_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return QMCRT_OK;
}

qmcrt_status qmcrt_batch_maps(qmcrt_batch* b, int32_t item, uint32_t** d_counts, float** d_flux) {
  if (!b || item < 0 || item >= (int)b->items.size()) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad item");
  if (d_counts) *d_counts = b->items[item].d_counts;
  if (d_flux) *d_flux = b->items[item].d_flux;
  return QMCRT_OK;
}

qmcrt_status qmcrt_batch_read(qmcrt_batch* b, int32_t item, uint32_t* h_counts, float* h_flux,
                              qmcrt_trace_stats* stats, void* stream) {
  if (!b || item < 0 || item >= (int)b->items.size()) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad item");
  cudaStream_t st = (cudaStream_t)stream;
  auto& it = b->items[item];
  if (h_counts) QM_CUDA(cudaMemcpyAsync(h_counts, it.d_counts, it.res * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (h_flux) QM_CUDA(cudaMemcpyAsync(h_flux, it.d_flux, it.res * sizeof(float), cudaMemcpyDeviceToHost, st));
  double tp = 0, ie = 0;
  QM_CUDA(cudaMemcpyAsync(&tp, it.geo.power, sizeof(double), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaMemcpyAsync(&ie, b->d_intercepted + item, sizeof(double), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaStreamSynchronize(st));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->rays = b->params.rays;
    stats->total_power = tp * it.sun.dni * b->params.reflectivity;
    stats->intercepted_power = ie * it.sun.dni * b->params.reflectivity / b->params.rays_per_point;
    stats->intercept_ratio = stats->total_power > 0 ? stats->intercepted_power / stats->total_power : 0.0;
  }
  return QMCRT_OK;
}

}  // extern "C"
