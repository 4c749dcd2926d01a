// trace.cu — the tracing kernel and its C-ABI entry points.
//
// One thread per ray, rays numbered point-major so a warp's 32 rays leave
// the same micro-heliostat point in nearly the same direction (coherent DDA
// paths).  Per ray (map_tracing, rectgrid_raytracing.cu:155-196):
//   1. sun sample from the Buie inverse CDF held in shared memory, Philox
//      keyed by (seed, ray id) -> world direction through the sun frame;
//   2. shadow test: 3D-DDA toward the sun over the uniform grid;
//   3. slope-error normal (Gaussian theta, uniform phi), reflection;
//   4. block test: 3D-DDA toward the reflected direction;
//   5. receiver hit -> pixel -> count and energy deposit.
// Precision: sampling and both traversals (the loops) run in FP32; the
// per-ray frame products, reflection and receiver intersection run in FP64
// so pixel indices agree with the FP64 oracle except where a hit lies within
// ~1e-6 m of a pixel edge.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

#include "internal.hpp"
#include "trace.cuh"

using namespace qm;

namespace qm {

qmcrt_status ensure_points(qmcrt_scene* s, const qmcrt_trace_params* p, cudaStream_t st);
qmcrt_status upload_field(qmcrt_scene* s, const qmcrt_field* f, cudaStream_t st);

// ------------------------------------------------------------ finalize
struct FinalizeArgs {
  int64_t res;
  const uint32_t* counts;
  const float* energy;
  uint32_t* out_counts;
  float* out_energy;
  float* out_flux;
  float scale;
  int accumulate;
  unsigned long long* stats;
};

__global__ void finalize_kernel(FinalizeArgs a) {
  pdl_wait();
  pdl_trigger();
  double acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.res; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t c = a.counts[i];
    float e = a.energy[i];
    acc += e;
    if (a.out_counts) a.out_counts[i] = (a.accumulate ? a.out_counts[i] : 0u) + c;
    if (a.out_energy) a.out_energy[i] = (a.accumulate ? a.out_energy[i] : 0.f) + e;
    if (a.out_flux) a.out_flux[i] = (a.accumulate ? a.out_flux[i] : 0.f) + e * a.scale;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc != 0) atomicAdd((double*)&a.stats[9], acc);
}

// Clears a trace's count and energy maps and its statistics words (0-7 and
// the intercepted-energy sum in 9; word 8, the field's total power, belongs
// to the per-sun geometry): one launch in place of four memsets, so that it
// joins the chain of kernels launched with programmatic dependent launch.
__global__ void zero_maps_kernel(uint32_t* counts, float* energy, int64_t res, unsigned long long* stats) {
  pdl_wait();
  pdl_trigger();
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, step = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = i0; i < res; i += step) {
    counts[i] = 0u;
    energy[i] = 0.f;
  }
  if (i0 < 10 && i0 != 8) stats[i0] = 0ull;
}

// SM count of the current device, cached per device (the process may drive
// several GPUs; the attribute query is cheap but not free per launch).
static std::atomic<int> g_sm_count[64];
static int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  int v = g_sm_count[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    int q = 0;
    if (cudaDeviceGetAttribute(&q, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || q <= 0) q = 148;
    g_sm_count[dev].store(q, std::memory_order_relaxed);
    v = q;
  }
  return v;
}

template <bool TABLES, bool RECORDS, bool STATS, int CULL, int MINB = 1, int RT = -1, bool LEAN = false>
static cudaError_t launch_trace(const TraceArgs& a, cudaStream_t st) {
  auto k = trace_kernel<TABLES, RECORDS, STATS, CULL, MINB, RT, LEAN>;
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTraceThreads, 0);
  if (e != cudaSuccess) return e;
  int64_t blocks = (int64_t)std::max(per_sm, 1) * sm_count();
  int64_t need = ((int64_t)a.rays - a.ray0 + kTraceThreads - 1) / kTraceThreads;
  blocks = std::max<int64_t>(1, std::min(blocks, need));
  return launch_pdl(true, k, dim3((unsigned)blocks), dim3(kTraceThreads), 0, st, a);
}

template <bool TABLES, bool RECORDS>
static cudaError_t dispatch2(const TraceArgs& a, bool stats, int cull, cudaStream_t st) {
  if (cull == 3 && !TABLES)
    return stats ? launch_trace<false, RECORDS, true, 3>(a, st) : launch_trace<false, RECORDS, false, 3>(a, st);
  if (stats) {
    if (cull == 2) return launch_trace<TABLES, RECORDS, true, 2>(a, st);
    return cull ? launch_trace<TABLES, RECORDS, true, 1>(a, st) : launch_trace<TABLES, RECORDS, true, 0>(a, st);
  }
  if (cull == 2) return launch_trace<TABLES, RECORDS, false, 2>(a, st);
  return cull ? launch_trace<TABLES, RECORDS, false, 1>(a, st) : launch_trace<TABLES, RECORDS, false, 0>(a, st);
}

static cudaError_t dispatch(const TraceArgs& a, bool tables, bool records, bool stats, int cull, int variant,
                            cudaStream_t st) {
  // the production path (no records, no statistics) is compiled for 4 resident
  // CTAs per SM (64 registers); variant 3 keeps the unconstrained build
  // (the candidate path, one build per receiver type, and a lean one of each
  // for the common case: power-of-two rays per point, point masks, no
  // attenuation, no pixel-edge quirk)
  if (variant != 3 && !tables && !records && !stats && cull == 3) {
    const bool lean = a.rpp_shift >= 0 && a.point_mask && a.atten == QMCRT_ATTEN_NONE &&
                      !(a.quirks & QMCRT_QUIRK_PIXEL_EDGE);
    if (a.rtype == QMCRT_RECEIVER_CYLINDER)
      return lean ? launch_trace<false, false, false, 3, 4, QMCRT_RECEIVER_CYLINDER, true>(a, st)
                  : launch_trace<false, false, false, 3, 4, QMCRT_RECEIVER_CYLINDER>(a, st);
    return lean ? launch_trace<false, false, false, 3, 4, QMCRT_RECEIVER_FLAT, true>(a, st)
                : launch_trace<false, false, false, 3, 4, QMCRT_RECEIVER_FLAT>(a, st);
  }
  if (variant != 3 && !tables && !records && !stats && cull == 2) return launch_trace<false, false, false, 2, 4>(a, st);
  if (variant != 3 && !tables && !records && !stats && cull) return launch_trace<false, false, false, 1, 4>(a, st);
  if (tables) return records ? dispatch2<true, true>(a, stats, cull, st) : dispatch2<true, false>(a, stats, cull, st);
  return records ? dispatch2<false, true>(a, stats, cull, st) : dispatch2<false, false>(a, stats, cull, st);
}

// Buie table in the layout the kernels stage into shared memory: for each
// uniform bucket of [0, core) (index (int)(uu * inv_bucket), one float
// multiply: the same rounding here), the 16-byte record {angle, cdf, slope,
// next interval's cdf} of the interval holding the bucket's smallest value,
// plus one record past the last bucket.  The kernel takes record b, or
// record b + 1 once uu reaches the record's next cdf; that is the interval
// max_less_index finds as long as no bucket holds two interval boundaries,
// which this checks (the core table does not depend on csr; its narrowest
// interval, the last, is 0.88 buckets wide).  Returns false if a bucket
// holds two.
bool buie_bucket_table(float csr, BuieTable* t) {
  std::vector<float> raw(1025 + 1025 + 1024);
  float* cx = raw.data();
  float* cy = cx + 1025;
  buie_build(csr, cx, cy, cy + 1025, t->params);
  const float* sl = cy + 1025;
  const float inv_bucket = (float)kBuieBuckets / t->params[2];
  auto bucket_of = [inv_bucket](float x) {
    volatile float p = x * inv_bucket;  // rounded to float, as the kernel's FMUL
    return (int)p;
  };
  std::vector<int> first(kBuieRecords);
  for (int b = 0; b < kBuieBuckets; ++b) {
    float edge = 0.f;  // the smallest float the kernel maps to bucket b
    if (b > 0) {
      edge = (float)b / inv_bucket;
      while (bucket_of(edge) < b) edge = std::nextafter(edge, HUGE_VALF);
      while (bucket_of(std::nextafter(edge, 0.f)) >= b) edge = std::nextafter(edge, 0.f);
    }
    int lo = 0, hi = 1023;
    while (lo < hi) {  // largest i <= 1023 with cy[i] <= edge
      int mid = (lo + hi + 1) >> 1;
      if (cy[mid] <= edge) lo = mid;
      else hi = mid - 1;
    }
    first[b] = lo;
  }
  first[kBuieBuckets] = std::min(first[kBuieBuckets - 1] + 1, 1023);
  // the values of bucket b lie below bucket b + 1's smallest, so their
  // intervals run from first[b] to first[b + 1]: at most one step apart; the
  // last bucket's values lie below core, in intervals up to 1023
  for (int b = 0; b + 1 < kBuieBuckets; ++b)
    if (first[b + 1] - first[b] > 1) return false;
  if (first[kBuieBuckets - 1] < 1022) return false;
  t->host.resize(4 * (size_t)kBuieRecords);
  for (int b = 0; b < kBuieRecords; ++b) {
    const int i = first[b];
    float* r = t->host.data() + 4 * b;
    r[0] = cx[i];
    r[1] = cy[i];
    r[2] = sl[i];
    r[3] = i < 1023 ? cy[i + 1] : HUGE_VALF;  // the last interval is never left
  }
  t->inv_bucket = inv_bucket;
  t->csr = csr;
  // the largest angle the sampler returns: the aureole's end (u -> 1) or the
  // core's last node, computed as the kernel computes it, plus rounding
  const double core_max = cx[1024];
  const double aur_max = std::pow((double)(t->params[3] - t->params[2]) * t->params[4] + t->params[5],
                                  1.0 / ((double)t->params[1] + 1.0));
  t->within_alpha = std::max(core_max, aur_max) * 1e-3 * (1.0 + 1e-5) <= kSunAlphaMax;
  return true;
}

// The tracer's Buie inverse CDF on caller-provided uniforms (test hook,
// qmcrt_buie_sample_probe): the shared-memory staging and lookup of the
// trace kernels, reading only the sampler's scalars of `a`.
__global__ void buie_probe_kernel(const TraceArgs a, const float* u, int64_t n, float* theta) {
  __shared__ float4 s_tab[kBuieRecords];
  load_buie(a.buie, s_tab);
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    theta[i] = buie_theta_mrad(a, s_tab, u[i]);
}

static qmcrt_status ensure_buie(qmcrt_scene* s, float csr, cudaStream_t st) {
  if (!(csr > 0.f && csr < 1.f)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "csr must be in (0,1)");
  if (s->buie.csr == csr) return QMCRT_OK;
  if (!buie_bucket_table(csr, &s->buie))
    return set_error(QMCRT_ERR_INTERNAL, "Buie table: a bucket holds two interval boundaries");
  QM_CUDA(cudaMemcpyAsync(s->d_buie, s->buie.host.data(), s->buie.host.size() * sizeof(float),
                          cudaMemcpyHostToDevice, st));
  return QMCRT_OK;
}

void fill_trace_args(qmcrt_scene* s, const SunGeom& geo, const qmcrt_sun* sun, uint32_t quirks, TraceArgs* a) {
  double sd[3] = {sun->dir[0], sun->dir[1], sun->dir[2]};
  double l = std::sqrt(sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2]);
  for (int i = 0; i < 3; ++i) sd[i] /= l;
  // sun frame of local2world (global_function.cuh:14-52)
  double u[3], n[3] = {sd[0], sd[1], sd[2]}, v[3];
  if (std::fabs(n[0]) < 1e-6 && std::fabs(n[2]) < 1e-6) {
    double sg = (n[1] < 0 && !(quirks & QMCRT_QUIRK_ZENITH_FRAME)) ? -1.0 : 1.0;
    u[0] = 1; u[1] = 0; u[2] = 0;
    n[0] = 0; n[1] = sg; n[2] = 0;
    v[0] = 0; v[1] = 0; v[2] = sg;
  } else {
    double lu = std::sqrt(n[2] * n[2] + n[0] * n[0]);
    u[0] = n[2] / lu; u[1] = 0; u[2] = -n[0] / lu;
    v[0] = u[1] * n[2] - u[2] * n[1];
    v[1] = u[2] * n[0] - u[0] * n[2];
    v[2] = u[0] * n[1] - u[1] * n[0];
    double lv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int i = 0; i < 3; ++i) v[i] /= lv;
  }
  for (int i = 0; i < 3; ++i) {
    a->su[i] = u[i];
    a->sn[i] = n[i];
    a->sv[i] = v[i];
    a->sdir[i] = sd[i];
  }
  a->buie = s->d_buie;
  a->b_total = s->buie.params[3];
  a->b_core = s->buie.params[2];
  a->b_B = s->buie.params[4];
  a->b_C = s->buie.params[5];
  a->b_inv = 1 / (s->buie.params[1] + 1);  // scene_instance_process.cu:135
  a->b_inv_bucket = s->buie.inv_bucket;
  a->n_helio = s->n;
  a->frame = geo.frame;
  a->pos = s->d_pos;
  a->size = s->d_size;
  a->sigma = s->d_sigma;
  a->weight = s->d_helio_weight;
  a->crect = geo.cell_rect;
  a->cinfo = geo.cell_info;
  a->field_yr = geo.field_yr;
  for (int i = 0; i < 3; ++i) {
    a->gpos[i] = s->gpos[i];
    a->gcell[i] = s->gcell[i];
    a->ginv[i] = 1.0f / s->gcell[i];
    a->gdims[i] = s->gdims[i];
  }
  a->coarse_yr = s->fine_div > 1 ? geo.coarse_yr : nullptr;
  a->cand = geo.cand;
  a->cand_n = geo.cand_n;
  a->rect = geo.rect;
  a->cshift = 0;
  while ((1 << a->cshift) < s->fine_div) ++a->cshift;
  for (int i = 0; i < 3; ++i) {
    a->cdims[i] = s->gdims[i] >> a->cshift;
    a->ccell[i] = s->gcell[i] * (float)s->fine_div;
  }
  a->rtype = s->rg.type;
  for (int i = 0; i < 3; ++i) {
    a->rA[i] = s->rg.v0[i];
    a->rE1[i] = s->rg.v1[i] - s->rg.v0[i];
    a->rE2[i] = s->rg.v3[i] - s->rg.v0[i];
  }
  {
    const double* E1 = a->rE1;
    const double* E2 = a->rE2;
    double* N = a->rN;
    N[0] = E1[1] * E2[2] - E1[2] * E2[1];
    N[1] = E1[2] * E2[0] - E1[0] * E2[2];
    N[2] = E1[0] * E2[1] - E1[1] * E2[0];
    const double nn = N[0] * N[0] + N[1] * N[1] + N[2] * N[2];
    const double inn = nn > 0 ? 1.0 / nn : 0.0;
    a->rD1[0] = (E2[1] * N[2] - E2[2] * N[1]) * inn;
    a->rD1[1] = (E2[2] * N[0] - E2[0] * N[2]) * inn;
    a->rD1[2] = (E2[0] * N[1] - E2[1] * N[0]) * inn;
    a->rD2[0] = (N[1] * E1[2] - N[2] * E1[1]) * inn;
    a->rD2[1] = (N[2] * E1[0] - N[0] * E1[2]) * inn;
    a->rD2[2] = (N[0] * E1[1] - N[1] * E1[0]) * inn;
  }
  for (int i = 0; i < 5; ++i) a->cyl[i] = s->rg.cyl[i];
  a->cyl[5] = s->rg.cyl[4] > 0 ? 1.0 / s->rg.cyl[4] : 0.0;
  a->cyl_edge = s->d_cyl_edge;
  a->res_x = s->rg.res_x;
  a->res_y = s->rg.res_y;
  a->quirks = quirks;
  a->counts = s->d_counts;
  a->energy = s->d_energy;
  a->stats = s->d_stats;
}

// log2(v) when v is a power of two, else -1 (lets the kernel split ray ids with a shift)
static int pow2_shift(int v) {
  if (v <= 0 || (v & (v - 1))) return -1;
  int s = 0;
  while ((1 << s) < v) ++s;
  return s;
}

static qmcrt_status check_params(const qmcrt_trace_params* p) {
  if (!p) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "params is NULL");
  if (p->rays_per_point <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "rays_per_point must be positive");
  if (!(p->reflectivity >= 0.f && p->reflectivity <= 1.f))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "reflectivity must be in [0,1]");
  if (p->quirks & ~QMCRT_QUIRKS_REFERENCE) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "unknown quirk bits");
  if (p->deposit != QMCRT_DEPOSIT_NEAREST) return set_error(QMCRT_ERR_NOT_SUPPORTED, "bilinear deposition is only used by the adjoint");
  if (p->kernel_variant < 0 || p->kernel_variant > 5) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "kernel_variant must be 0..5");
  if (p->attenuation != QMCRT_ATTEN_NONE && p->attenuation != QMCRT_ATTEN_POLY_EXP)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "unknown attenuation mode");
  if (p->ray_end != 0 && p->ray_begin >= p->ray_end)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "ray range must have ray_begin < ray_end");
  return QMCRT_OK;
}

// The range [ray_begin, ray_end) of a trace of `total` rays (all of them when
// ray_end is 0), as 64-bit ray ids; run_and_finish splits it into launches
// that each stay between two multiples of 2^32.
static qmcrt_status apply_range(const qmcrt_trace_params* p, uint64_t total, TraceArgs* a) {
  a->rays = total;
  a->ray0 = 0;
  if (p->ray_end == 0) return QMCRT_OK;
  if (p->ray_end > total) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "ray_end is past the trace's last ray");
  a->ray0 = p->ray_begin;
  a->rays = p->ray_end;
  return QMCRT_OK;
}

// W/m^2 per unit of the raw energy map: DNI * S_sub * rho / N_c / S_rec
// (Gtest.cu:40-46); S_sub is folded into the per-point weights of Philox
// traces (weight_scale 1) and is point_spacing^2 for table traces.
static double flux_scale(const qmcrt_scene* s, const qmcrt_sun* sun, const qmcrt_trace_params* p,
                         double weight_scale) {
  return (double)sun->dni * p->reflectivity * weight_scale / ((double)p->rays_per_point * s->rg.pixel_area);
}

__global__ void scale_kernel(float* m, int64_t n, float k) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m[i] *= k;
}

// Philox rays of the corrected method test their heliostat's occluder
// candidates instead of walking the grid (variants 4 and 5 walk the grid; the
// lists leave out the ray's own heliostat, so not under QMCRT_QUIRK_SELF_HIT;
// vertical culling needs every rectangle registered in every cell it touches
// and the origin cell tested, so not under the two grid quirks or variant 2).
static bool uses_candidates(const qmcrt_scene* s, const qmcrt_trace_params* p, bool tables) {
  const bool cull = p->kernel_variant != 2 && !(p->quirks & (QMCRT_QUIRK_SKIP_ORIGIN_CELL | QMCRT_QUIRK_AABB_RADIUS));
  return cull && !tables && s->buie.within_alpha && !(p->quirks & QMCRT_QUIRK_SELF_HIT) && p->kernel_variant != 4 &&
         p->kernel_variant != 5;
}

static qmcrt_status run_and_finish(qmcrt_scene* s, const qmcrt_sun* sun, const qmcrt_trace_params* p, TraceArgs& a,
                                   bool tables, double weight_scale, const qmcrt_outputs* out,
                                   qmcrt_trace_stats* stats, cudaStream_t st) {
  int64_t res = (int64_t)s->rg.res_x * s->rg.res_y;
  const int zb = (int)std::min<int64_t>((res + 255) / 256, 2 * sm_count());
  QM_CUDA(launch_pdl(true, zero_maps_kernel, dim3(zb), dim3(256), 0, st, s->d_counts, s->d_energy, res, s->d_stats));
  bool records = out && (out->d_ray_flags || out->d_ray_pixel);
  if (out) {
    a.flags = out->d_ray_flags;
    a.pixel = out->d_ray_pixel;
  }
  // timing events on request only: an event between two kernels keeps the
  // second from starting while the first finishes (programmatic dependent
  // launch), about 10 % of the small field's step with every stage timed
  const bool t_trace = s->timing_stages & QMCRT_TIMING_TRACE, t_fin = s->timing_stages & QMCRT_TIMING_FINALIZE;
  if (t_trace) QM_CUDA(cudaEventRecord(s->ev[2], st));
  // vertical culling needs every rectangle registered in every cell it
  // touches and the origin cell tested: off under the two grid quirks
  // (level 2 adds the coarse level of a two-level grid)
  int cull = p->kernel_variant != 2 && !(p->quirks & (QMCRT_QUIRK_SKIP_ORIGIN_CELL | QMCRT_QUIRK_AABB_RADIUS));
  if (cull && a.coarse_yr && p->kernel_variant != 4) cull = 2;
  if (a.cand && uses_candidates(s, p, tables)) cull = 3;
  // one launch per block of 2^32 ray ids: a launch's threads carry the low
  // word of their ray id, the launch the high word (and the records pointers
  // its offset)
  for (uint64_t b = a.ray0; b < a.rays;) {
    const uint64_t hi = b >> 32, end = std::min<uint64_t>(a.rays, (hi + 1) << 32);
    TraceArgs sa = a;
    sa.ray_hi = (uint32_t)hi;
    sa.g_hi = a.rpp_shift >= 0 ? (uint32_t)((hi << 32) >> a.rpp_shift) : 0u;
    sa.ray0 = b - (hi << 32);
    sa.rays = end - (hi << 32);
    if (sa.flags) sa.flags += hi << 32;
    if (sa.pixel) sa.pixel += hi << 32;
    QM_CUDA(dispatch(sa, tables, records, stats != nullptr, cull, p->kernel_variant, st));
    b = end;
  }
  if (t_trace || t_fin) QM_CUDA(cudaEventRecord(s->ev[3], st));
  const double scale = flux_scale(s, sun, p, weight_scale);
  FinalizeArgs f{};
  f.res = res;
  f.counts = s->d_counts;
  f.energy = s->d_energy;
  f.out_counts = out ? out->d_counts : nullptr;
  f.out_energy = out ? out->d_energy : nullptr;
  f.out_flux = out ? out->d_flux : nullptr;
  f.scale = (float)scale;
  f.accumulate = p->accumulate;
  f.stats = s->d_stats;
  int fb = (int)std::min<int64_t>((res + 255) / 256, 4 * sm_count());
  QM_CUDA(launch_pdl(true, finalize_kernel, dim3(fb), dim3(256), 0, st, f));
  if (t_fin) QM_CUDA(cudaEventRecord(s->ev[4], st));
  s->timed |= (t_trace ? QMCRT_TIMING_TRACE : 0u) | (t_fin ? QMCRT_TIMING_FINALIZE : 0u);
  s->traced = true;
  if (stats) {
    unsigned long long h[16];
    int32_t flag = 0;
    QM_CUDA(cudaMemcpyAsync(h, s->d_stats, sizeof(h), cudaMemcpyDeviceToHost, st));
    QM_CUDA(cudaMemcpyAsync(&flag, s->d_flag, sizeof(flag), cudaMemcpyDeviceToHost, st));
    QM_CUDA(cudaStreamSynchronize(st));
    if (flag == 1) return set_error(QMCRT_ERR_INTERNAL, "grid registrations exceeded the scene's capacity");
    double tp, ie;
    std::memcpy(&tp, &h[8], sizeof(double));
    std::memcpy(&ie, &h[9], sizeof(double));
    stats->rays = h[0];
    stats->shadowed = h[1];
    stats->blocked = h[2];
    stats->hit = h[3];
    stats->offmap = h[4];
    stats->rect_tests = h[5];
    stats->dda_cells = h[6];
    stats->total_power = tp * sun->dni * p->reflectivity;
    stats->intercepted_power = ie * sun->dni * p->reflectivity * weight_scale / p->rays_per_point;
    stats->intercept_ratio = stats->total_power > 0 ? stats->intercepted_power / stats->total_power : 0.0;
  }
  return QMCRT_OK;
}

}  // namespace qm

extern "C" {

qmcrt_status qmcrt_trace(qmcrt_scene* s, const qmcrt_sun* sun, const qmcrt_trace_params* p, const qmcrt_outputs* out,
                         qmcrt_trace_stats* stats, void* stream) {
  if (!s || !sun) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  qmcrt_status e = check_params(p);
  if (e) return e;
  cudaStream_t st = (cudaStream_t)stream;
  if (!(sun->dni >= 0)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "dni must be non-negative");
  if ((e = ensure_buie(s, sun->csr, st))) return e;
  s->timed = 0;
  // a trace that tests candidates needs the grid only where a list overflows
  if ((e = ensure_sun(s, sun, p->quirks, st, !uses_candidates(s, p, false)))) return e;
  if ((e = ensure_points(s, p, st))) return e;
  TraceArgs a{};
  fill_trace_args(s, scene_geom(s), sun, p->quirks, &a);
  a.atten = p->attenuation;
  if ((e = apply_range(p, (uint64_t)s->points * (uint64_t)p->rays_per_point, &a))) return e;
  a.rpp = p->rays_per_point;
  a.rpp_shift = pow2_shift(a.rpp);
  philox_round_keys(make_uint2((uint32_t)p->seed, (uint32_t)(p->seed >> 32)), a.rk);
  a.item = p->item;
  a.point_xz = s->d_point_xz;
  a.point_helio = s->d_point_helio;
  if ((e = ensure_masks(s, st))) return e;
  a.point_mask = s->d_point_mask;
  a.point_origin = s->d_point_origin;
  return run_and_finish(s, sun, p, a, false, 1.0, out, stats, st);
}

qmcrt_status qmcrt_trace_tables(qmcrt_scene* s, const qmcrt_sun* sun, const qmcrt_table_inputs* t,
                                const qmcrt_trace_params* p, const qmcrt_outputs* out, qmcrt_trace_stats* stats,
                                void* stream) {
  if (!s || !sun || !t) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  qmcrt_status e = check_params(p);
  if (e) return e;
  if (!t->d_sun_local || !t->d_turb_local || !t->d_start || !t->d_point_xz || !t->d_point_helio || t->table_size <= 0 ||
      t->points <= 0 || t->rays_per_point <= 0 || t->rays_per_point != p->rays_per_point)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "incomplete table inputs");
  if ((uint64_t)t->points * (uint64_t)t->rays_per_point > 0xFFFFFFFFull)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "ray count must be below 2^32");
  cudaStream_t st = (cudaStream_t)stream;
  s->timed = 0;
  if ((e = ensure_sun(s, sun, p->quirks, st))) return e;
  TraceArgs a{};
  fill_trace_args(s, scene_geom(s), sun, p->quirks, &a);
  a.atten = p->attenuation;
  if ((e = apply_range(p, (uint64_t)t->points * (uint64_t)t->rays_per_point, &a))) return e;
  a.rpp = t->rays_per_point;
  a.rpp_shift = pow2_shift(a.rpp);
  a.point_xz = (const float2*)t->d_point_xz;
  a.point_helio = t->d_point_helio;
  a.sun_local = t->d_sun_local;
  a.turb_local = t->d_turb_local;
  a.T = t->table_size;
  a.start = t->d_start;
  a.weight = nullptr;
  // S_sub = point_spacing^2 (Gtest.cu:40)
  double ws = (double)p->point_spacing * p->point_spacing;
  return run_and_finish(s, sun, p, a, true, ws, out, stats, st);
}

qmcrt_status qmcrt_trace_host(qmcrt_scene* s, const qmcrt_field* field, const qmcrt_sun* sun,
                              const qmcrt_trace_params* p, uint32_t* h_counts, float* h_flux,
                              qmcrt_trace_stats* stats, void* stream) {
  if (!s || !sun || !p) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  qmcrt_status e;
  if (field && (e = qmcrt_scene_set_field(s, field, stream))) return e;
  qmcrt_outputs out{};
  out.d_flux = s->d_energy;  // flux in place of the raw energy map
  qmcrt_trace_params pp = *p;
  pp.accumulate = 0;
  if ((e = qmcrt_trace(s, sun, &pp, &out, stats, stream))) return e;
  int64_t res = (int64_t)s->rg.res_x * s->rg.res_y;
  if (h_counts) QM_CUDA(cudaMemcpyAsync(h_counts, s->d_counts, res * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (h_flux) QM_CUDA(cudaMemcpyAsync(h_flux, s->d_energy, res * sizeof(float), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaStreamSynchronize(st));
  return QMCRT_OK;
}

qmcrt_status qmcrt_buie_sample_probe(float csr, const float* d_u, int64_t n, float* d_theta_mrad, void* stream) {
  if (!d_u || !d_theta_mrad || n <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad probe arguments");
  if (!(csr > 0.f && csr < 1.f)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "csr must be in (0,1)");
  BuieTable t;
  if (!buie_bucket_table(csr, &t)) return set_error(QMCRT_ERR_INTERNAL, "Buie table: a bucket holds two interval boundaries");
  cudaStream_t st = (cudaStream_t)stream;
  TraceArgs a;
  std::memset(&a, 0, sizeof(a));
  a.b_total = t.params[3];
  a.b_core = t.params[2];
  a.b_B = t.params[4];
  a.b_C = t.params[5];
  a.b_inv = 1 / (t.params[1] + 1);
  a.b_inv_bucket = t.inv_bucket;
  float* d_tab = nullptr;
  QM_CUDA(cudaMalloc(&d_tab, t.host.size() * sizeof(float)));
  a.buie = d_tab;
  cudaError_t ce = cudaMemcpyAsync(d_tab, t.host.data(), t.host.size() * sizeof(float), cudaMemcpyHostToDevice, st);
  if (ce == cudaSuccess) {
    buie_probe_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4 * sm_count()), 256, 0, st>>>(a, d_u, n,
                                                                                                   d_theta_mrad);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  cudaFree(d_tab);
  if (ce != cudaSuccess) return cuda_error(ce, "Buie sample probe");
  return QMCRT_OK;
}

qmcrt_status qmcrt_results_host(qmcrt_scene* s, const qmcrt_field* field, const qmcrt_sun* sun,
                                const qmcrt_trace_params* p, const qmcrt_smooth_params* sm, uint32_t* h_counts,
                                float* h_flux, float* h_smoothed, qmcrt_trace_stats* stats, void* stream) {
  if (!s || !sun || !p) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (sm && sm->source != QMCRT_SMOOTH_COUNTS && sm->source != QMCRT_SMOOTH_ENERGY)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "unknown smoothing source");
  if (!sm && h_smoothed) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "h_smoothed needs smoothing parameters");
  cudaStream_t st = (cudaStream_t)stream;
  qmcrt_status e;
  if (field && (e = qmcrt_scene_set_field(s, field, stream))) return e;
  // the trace leaves the raw counts and energy in the scene's maps and the
  // scaled flux in d_map_flux
  qmcrt_outputs out{};
  out.d_flux = s->d_map_flux;
  qmcrt_trace_params pp = *p;
  pp.accumulate = 0;
  // (with `stats` the trace counts its events and synchronises)
  if ((e = qmcrt_trace(s, sun, &pp, &out, stats, stream))) return e;
  const int64_t res = (int64_t)s->rg.res_x * s->rg.res_y;
  if (sm) {
    if (sm->source == QMCRT_SMOOTH_COUNTS) {
      e = qmcrt_smooth_trimmed_u32(s->d_counts, s->d_map_smooth, s->rg.res_x, s->rg.res_y, sm->radius, sm->ratio,
                                   sm->method, stream);
    } else {
      // the reference smooths its raw image, then scales it (Gtest.cu:52-57)
      e = qmcrt_smooth_trimmed_f32(s->d_energy, s->d_map_smooth, s->rg.res_x, s->rg.res_y, sm->radius, sm->ratio,
                                   sm->method, stream);
      if (!e) {
        const int blocks = (int)std::min<int64_t>((res + 255) / 256, 4 * sm_count());
        scale_kernel<<<blocks, 256, 0, st>>>(s->d_map_smooth, res, (float)flux_scale(s, sun, p, 1.0));
        QM_CUDA(cudaGetLastError());
      }
    }
    if (e) return e;
  }
  if (h_counts) QM_CUDA(cudaMemcpyAsync(h_counts, s->d_counts, res * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (h_flux) QM_CUDA(cudaMemcpyAsync(h_flux, s->d_map_flux, res * sizeof(float), cudaMemcpyDeviceToHost, st));
  if (h_smoothed)
    QM_CUDA(cudaMemcpyAsync(h_smoothed, s->d_map_smooth, res * sizeof(float), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaStreamSynchronize(st));
  return QMCRT_OK;
}

}  // extern "C"
