// adjoint.cu — gradients of a flux-map loss with respect to each heliostat's
// 2D aim offset and 2D normal tilt.  No counterpart in the reference.
//
// Forward: the tracer with bilinear deposition of each ray's energy into the
// four pixels around its receiver hit, writing one visibility byte per ray
// (the tape).  Loss: L = sum_p (F_p - T_p)^2 for flux F and target T; the
// adjoint map G_p = dL/dE_p = 2 (F_p - T_p) * scale (E = raw energy map).
// Backward: per ray, the pathwise derivative of its deposit under the same
// random numbers, visibility held constant: the chain
//   theta -> mirror frame (u, n, v) -> origin, perturbed normal -> reflected
//   direction -> receiver (u, v) -> bilinear weights, and -> energy |s . n'|,
// with the frame's Jacobian per heliostat from FP64 dual numbers and the
// per-ray chain in FP32 tangents.  Rays past the tape's capacity recompute
// their visibility (two traversals) instead of reading it.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.hpp"
#include "trace.cuh"

using namespace qm;

namespace qm {
void fill_trace_args(qmcrt_scene* s, const SunGeom& geo, const qmcrt_sun* sun, uint32_t quirks, TraceArgs* a);

// 2 CTAs of 512 threads per SM (32 warps) at <= 64 registers: against 3 CTAs
// of 256 at 72 and 80 registers, the forward takes 12 % and the backward 4 %
// less time (the backward spills a little at 64 registers and still gains)
constexpr int kAdjThreads = 512;
constexpr int kAdjCtasPerSm = 2;
// up to 83.5 KB of tile (rows of 145) + 20 KB of Buie table: 2 CTAs per SM;
// a 128 x 128 map fits whole (forward 1.18 -> 1.07 ms against a 112^2 tile)
constexpr int kAdjTileMax = 144;

// ------------------------------------------------------------ dual numbers
// value + derivatives with respect to the 4 parameters of one heliostat
struct dual {
  double v, d[4];
};
__device__ __forceinline__ dual dc(double v) { return dual{v, {0, 0, 0, 0}}; }
__device__ __forceinline__ dual operator+(dual a, dual b) {
  return dual{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2], a.d[3] + b.d[3]}};
}
__device__ __forceinline__ dual operator-(dual a, dual b) {
  return dual{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2], a.d[3] - b.d[3]}};
}
__device__ __forceinline__ dual operator*(dual a, dual b) {
  dual r;
  r.v = a.v * b.v;
  for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
__device__ __forceinline__ dual operator/(dual a, dual b) {
  dual r;
  r.v = a.v / b.v;
  for (int k = 0; k < 4; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
  return r;
}
__device__ __forceinline__ dual dsqrt(dual a) {
  dual r;
  r.v = sqrt(a.v);
  for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] / (2.0 * r.v);
  return r;
}
struct dvec {
  dual x, y, z;
};
__device__ __forceinline__ dvec operator+(dvec a, dvec b) { return dvec{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ dvec operator-(dvec a, dvec b) { return dvec{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ dvec scale(dual s, dvec a) { return dvec{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ dual ddot(dvec a, dvec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ dvec dcross(dvec a, dvec b) {
  return dvec{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ dvec dnorm(dvec a) {
  dual l = dsqrt(ddot(a, a));
  return dvec{a.x / l, a.y / l, a.z / l};
}

struct JacArgs {
  int n;
  const float *pos, *aim, *normal_in, *tilt;
  double focus[3], sun[3], ew[3], eh[3];
  float* jac;  // [36 n]: d(u, n, v)/d(theta), row-major 9 x 4
};

// Jacobian of the mirror frame with respect to theta = (aim offset along the
// receiver width, along its height, extra tilt about u, about v), evaluated at
// theta = 0 with the aiming and tilt rule of the aim kernel (heliostat.cpp:51-58).
__global__ void frame_jacobian_kernel(JacArgs a) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= a.n) return;
  dvec n0;
  if (a.normal_in) {
    n0 = dnorm(dvec{dc(a.normal_in[3 * h]), dc(a.normal_in[3 * h + 1]), dc(a.normal_in[3 * h + 2])});
  } else {
    double t[3];
    for (int i = 0; i < 3; ++i) t[i] = a.aim ? (double)a.aim[3 * h + i] : a.focus[i];
    dvec aimp;
    dual* ap[3] = {&aimp.x, &aimp.y, &aimp.z};
    for (int i = 0; i < 3; ++i) *ap[i] = dual{t[i], {a.ew[i], a.eh[i], 0, 0}};
    dvec p{dc(a.pos[3 * h]), dc(a.pos[3 * h + 1]), dc(a.pos[3 * h + 2])};
    dvec r = dnorm(aimp - p);
    n0 = dnorm(r - dvec{dc(a.sun[0]), dc(a.sun[1]), dc(a.sun[2])});
  }
  // frame of the untilted normal, then the tilt (tx + theta2, tz + theta3)
  dvec u0 = dnorm(dvec{n0.z, dc(0), dc(0) - n0.x});
  dvec v0 = dnorm(dcross(u0, n0));
  dual tx = dual{a.tilt ? (double)a.tilt[2 * h] : 0.0, {0, 0, 1, 0}};
  dual tz = dual{a.tilt ? (double)a.tilt[2 * h + 1] : 0.0, {0, 0, 0, 1}};
  dvec n = dnorm(n0 + scale(tx, u0) + scale(tz, v0));
  dvec u = dnorm(dvec{n.z, dc(0), dc(0) - n.x});
  dvec v = dnorm(dcross(u, n));
  const dvec fr[3] = {u, n, v};
  float* J = a.jac + 36 * h;
  for (int b = 0; b < 3; ++b) {
    const dual* c[3] = {&fr[b].x, &fr[b].y, &fr[b].z};
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 4; ++k) J[(3 * b + i) * 4 + k] = (float)c[i]->d[k];
  }
}

struct AdjArgs {
  TraceArgs t;
  int tile, tile_r0, tile_c0;  // forward: block-private tile of tile x tile pixels at (row r0, col c0); 0: none
  double ew[3], eh[3];  // receiver width / height unit axes (flat receivers)
  // backward: the receiver edges and the sun direction in float, read from
  // the parameter space where they are used (no registers held across the ray loop)
  float e1f[3], e2f[3], sdf[3];
  uint8_t* tape;        // one visibility byte per ray
  unsigned long long* energy_fx;  // replay: the energy map in 2^-40 fixed point (exact sums in any order)
  uint64_t saved;       // rays with a byte in the tape
  const float* G;       // adjoint map (backward)
  const float* jac;     // frame Jacobians (backward)
  float* grad_aim;      // [2n]
  float* grad_tilt;     // [2n]
};

// Receiver hit with the continuous (u, v) (flat receivers): along E1 (rows)
// and E2 (columns), each in [0, 1]; t along the ray.  The plane form of the
// tracer's receiver_hit: t = ((A - o) . N) / (d . N) and the dual-edge
// coordinates of the hit's offset from A.
__device__ __forceinline__ bool receiver_uv(const TraceArgs& a, d3 o, d3 d, double* u, double* v, double* t) {
  const d3 N = mk(a.rN[0], a.rN[1], a.rN[2]);
  const double dn = dot(d, N);
  if (fabs(dn) < 1e-6) return false;
  const d3 ao = mk(a.rA[0], a.rA[1], a.rA[2]) - o;
  *t = dot(ao, N) * rcp_nr(dn);
  if (*t < 1e-6) return false;
  const d3 w = *t * d - ao;  // hit - A
  *u = dot(w, mk(a.rD1[0], a.rD1[1], a.rD1[2]));
  if (*u < 0 || *u > 1) return false;
  *v = dot(w, mk(a.rD2[0], a.rD2[1], a.rD2[2]));
  return *v >= 0 && *v <= 1;
}

// The receiver plane's (u, v) of the line o + t d, without the range tests:
// the same arithmetic as receiver_uv.  The replayed forward pass deposits a
// ray the tape marks as a hit wherever its (u, v) now falls.
__device__ __forceinline__ void receiver_plane_uv(const TraceArgs& a, d3 o, d3 d, double* u, double* v) {
  const d3 N = mk(a.rN[0], a.rN[1], a.rN[2]);
  const d3 ao = mk(a.rA[0], a.rA[1], a.rA[2]) - o;
  const d3 w = (dot(ao, N) * rcp_nr(dot(d, N))) * d - ao;
  *u = dot(w, mk(a.rD1[0], a.rD1[1], a.rD1[2]));
  *v = dot(w, mk(a.rD2[0], a.rD2[1], a.rD2[2]));
}

// Reflection geometry of one ray: the perturbed unit normal and reflected
// unit direction, and the lengths they had before normalising (for the
// derivative of the normalisation in the backward pass).  The forward pass
// keeps both unscaled and carries 1 / |np| for the energy.
struct Refl {
  d3 np, rd;
  double lnp, lr;
  double en;  // 1 / |np| as far as the energy needs it (np is not scaled in the forward pass)
};

// LENGTHS = false (the forward pass): rd keeps the length of the sun sample
// (1 to float rounding) and the lengths are not formed; the receiver's
// (u, v) and the visibility tests are scale-free in rd.
// The forward pass forms the reflection as the plain tracer does: a Philox
// perturbation in the orthonormal FP64 frame has q = |np|^2 = 1 + t with
// |t| < 2e-6, so 1 / q = 1 - t + t^2 (error below 1e-17) and 1 / |np| =
// 1.5 - q / 2 (error below 2e-12, for the float energy), and np stays
// unscaled.
template <bool LENGTHS = true>
__device__ __forceinline__ Refl reflect_ray(const RaySetup& R) {
  Refl g;
  const d3 npr = apply(R.fr, (double)R.tl.x, (double)R.tl.y, (double)R.tl.z);
  const double q = dot(npr, npr);
  if (LENGTHS) {
    const double iq = rsqrt_nr(q);
    g.np = iq * npr;
    g.en = 1.0;
    const d3 rr = R.ws - (2.0 * dot(R.ws, g.np)) * g.np;
    g.lnp = q * iq;
    const double q2 = dot(rr, rr), iq2 = rsqrt_nr(q2);
    g.rd = iq2 * rr;
    g.lr = q2 * iq2;
  } else {
    const double t = q - 1.0;
    const double k = -2.0 * dot(R.ws, npr) * fma(t, t - 1.0, 1.0);
    g.np = npr;
    g.en = fma(-0.5, q, 1.5);
    g.rd = mk(fma(k, npr.x, R.ws.x), fma(k, npr.y, R.ws.y), fma(k, npr.z, R.ws.z));
    g.lnp = g.lr = 1.0;
  }
  return g;
}

// Visibility and hit geometry of one ray (reflection, shadow, block,
// receiver).  The reflection comes first, as in the plain tracer, so the
// mirror frame is dead before the walks; the ray's energy |s . n'| w (the
// only use of the normal in the forward pass) is formed there too.
template <bool CULL, bool LENGTHS = true>
__device__ __forceinline__ bool ray_hits(const TraceArgs& a, const RaySetup& R, float fy0, float fy1, Refl* g,
                                         double* u, double* v, double* t, float* e = nullptr) {
  *g = reflect_ray<LENGTHS>(R);
  if (e) *e = (float)(fabs(g->np.x * a.sdir[0] + g->np.y * a.sdir[1] + g->np.z * a.sdir[2]) * g->en) * R.w;
  // with CULL (corrected mode) the heliostat's occluder candidates answer the
  // visibility questions (the grid walk where there are none)
  uint32_t nt = 0, nc = 0;
  const float3 of = R.of;
  const float3 sd = f3((float)-R.ws.x, (float)-R.ws.y, (float)-R.ws.z);
  if (CULL ? list_blocked<false>(a, R.h, 0, of, sd, fy0, fy1, nt, nc, R.reach.x)
           : dda_blocked<false, false>(a, of, sd, R.h, fy0, fy1, nt, nc))
    return false;
  if (CULL ? list_blocked<false>(a, R.h, 1, of, to_f(g->rd), fy0, fy1, nt, nc, R.reach.y)
           : dda_blocked<false, false>(a, of, to_f(g->rd), R.h, fy0, fy1, nt, nc))
    return false;
  return receiver_uv(a, R.o, g->rd, u, v, t);
}

// REPLAY: the visibility of every ray comes from the tape instead of the
// walks (qmcrt_adjoint_replay), and a ray the tape marks as a hit deposits
// wherever its (u, v) falls now, corners off the map dropped; the tape is
// only read.  The deposits are 64-bit fixed point with 2^-40 resolution,
// added with integer atomics: the sums are exact in any order, so the
// replayed loss is the same bit for bit from run to run.
// LEAN: a power-of-two count of rays per point and the point masks present
// (the plain tracer's lean ray setup).
template <bool CULL, bool REPLAY = false, bool LEAN = false>
__global__ void __launch_bounds__(kAdjThreads, kAdjCtasPerSm) adjoint_forward_kernel(const AdjArgs A) {
  __shared__ float4 s_tab[kBuieRecords];
  // block-private tile of the energy map: many heliostats aim at the same
  // spot, so global atomics on it would queue at the hot pixels
  extern __shared__ float s_tile[];
  // rows of the tile are T + 1 floats apart (an odd stride: hits in the same
  // column a few rows apart fall in different shared-memory banks)
  const int T = A.tile, TS = T + 1, r0 = A.tile_r0, c0 = A.tile_c0;
  const TraceArgs& a = A.t;
  for (int i = threadIdx.x; i < T * TS; i += blockDim.x) s_tile[i] = 0.f;
  load_buie(a.buie, s_tab);
  __syncthreads();
  const float fy0 = CULL ? from_ordered(__ldg(a.field_yr)) : 0.f, fy1 = CULL ? from_ordered(__ldg(a.field_yr + 1)) : 0.f;
  // chunks of consecutive rays taken grid-stride, as in the plain tracer;
  // i counts the rays of the range [ray0, rays) (ray0 + i is the ray id and
  // i its tape byte).  32-bit: the adjoint takes fewer than 2^32 rays.
  const uint32_t n = (uint32_t)(a.rays - a.ray0), ray0 = (uint32_t)a.ray0;
  const uint64_t chunk = (uint64_t)kChunkBlocks * blockDim.x, nch = ((uint64_t)n + chunk - 1) / chunk;
  for (uint64_t ch = blockIdx.x; ch < nch; ch += gridDim.x)
  for (uint32_t i = (uint32_t)(ch * chunk) + threadIdx.x, i1 = (uint32_t)min((ch + 1) * chunk, (uint64_t)n); i < i1;
       i += blockDim.x) {
    const uint64_t r64 = i;
    if (REPLAY && A.tape[r64] == 0) continue;
    RaySetup R;
    ray_setup<false, LEAN>(a, s_tab, ray0 + i, R, a.rk);
    Refl g;
    double u, v, t;
    float e;
    if (REPLAY) {
      g = reflect_ray<false>(R);
      e = (float)(fabs(g.np.x * a.sdir[0] + g.np.y * a.sdir[1] + g.np.z * a.sdir[2]) * g.en) * R.w;
      receiver_plane_uv(a, R.o, g.rd, &u, &v);
    } else {
      const bool hit = ray_hits<CULL, false>(a, R, fy0, fy1, &g, &u, &v, &t, &e);
      if (r64 < A.saved) A.tape[r64] = hit ? 1 : 0;
      if (!hit) continue;
    }
    float px = (float)(v * a.res_x) - 0.5f, py = (float)(u * a.res_y) - 0.5f;
    const float flx = floorf(px), fly = floorf(py);
    const int i0 = (int)flx, j0 = (int)fly;
    const float fx = px - flx, fy = py - fly;
    const float wgt[4] = {(1.f - fx) * (1.f - fy), fx * (1.f - fy), (1.f - fx) * fy, fx * fy};
    if (REPLAY) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int ci = i0 + (k & 1), cj = j0 + (k >> 1);
        if (ci < 0 || cj < 0 || ci >= a.res_x || cj >= a.res_y) continue;
        atomicAdd(A.energy_fx + cj * a.res_x + ci, __double2ull_rn((double)(e * wgt[k]) * 0x1p40));
      }
      continue;
    }
    if ((unsigned)(j0 - r0) < (unsigned)(T - 1) && (unsigned)(i0 - c0) < (unsigned)(T - 1)) {
      // all four corners in the tile (which lies inside the map): one check
      float* q = s_tile + (j0 - r0) * TS + (i0 - c0);
      atomicAdd(q, e * wgt[0]);
      atomicAdd(q + 1, e * wgt[1]);
      atomicAdd(q + TS, e * wgt[2]);
      atomicAdd(q + TS + 1, e * wgt[3]);
      continue;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      int ci = i0 + (k & 1), cj = j0 + (k >> 1);
      if (ci < 0 || cj < 0 || ci >= a.res_x || cj >= a.res_y) continue;
      if ((unsigned)(cj - r0) < (unsigned)T && (unsigned)(ci - c0) < (unsigned)T)
        atomicAdd(s_tile + (cj - r0) * TS + (ci - c0), e * wgt[k]);
      else
        atomicAdd(a.energy + cj * a.res_x + ci, e * wgt[k]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < T * T; i += blockDim.x) {
    const int tr = i / T, tc = i - tr * T;
    const float v = s_tile[tr * TS + tc];
    if (v != 0.f) atomicAdd(a.energy + (r0 + tr) * a.res_x + (c0 + tc), v);
  }
}

struct LossArgs {
  const float* energy;
  const float* target;
  float* flux;  // may be NULL
  float* G;
  float scale;
  int64_t res;
  double* loss;
};

__global__ void loss_kernel(LossArgs a) {
  double acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.res; i += (int64_t)gridDim.x * blockDim.x) {
    float f = a.energy[i] * a.scale;
    if (a.flux) a.flux[i] = f;
    float d = f - a.target[i];
    acc += (double)d * d;
    a.G[i] = 2.f * d * a.scale;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(a.loss, acc);
}

// The loss of a fixed-point energy map (the replay), in double throughout.
struct LossFxArgs {
  const unsigned long long* energy;
  const float* target;
  float* flux;  // may be NULL
  float* G;
  double scale;
  int64_t res;
  double* loss;
};

// One block of kLossThreads threads: every thread sums a fixed stride of the
// pixels and the block reduces the partial sums in a fixed tree, so the
// replayed loss is the same double from run to run.
constexpr int kLossThreads = 1024;
__global__ void __launch_bounds__(kLossThreads) loss_fx_kernel(LossFxArgs a) {
  __shared__ double part[kLossThreads / 32];
  double acc = 0;
  for (int64_t i = threadIdx.x; i < a.res; i += kLossThreads) {
    const double f = (double)a.energy[i] * 0x1p-40 * a.scale;
    if (a.flux) a.flux[i] = (float)f;
    const double d = f - (double)a.target[i];
    acc += d * d;
    a.G[i] = (float)(2.0 * d * a.scale);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = part[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) *a.loss = acc;
  }
}

__device__ __forceinline__ float3 fma3(float s, float3 a, float3 b) { return f3(s * a.x + b.x, s * a.y + b.y, s * a.z + b.z); }

// RECOMPUTE: the tape holds fewer rays than the trace (state_bytes_max), and
// the rays past it walk again for their visibility; without it the walks
// are compiled out.  Register pressure at the 64-register cap, measured on
// the differentiable field: 144 B of spills and 1.32 ms with the walks
// compiled in, 116 B and 1.27 ms without, 56 B and 1.21 ms once the
// receiver edges and sun direction are read in float from the parameter
// space instead of held in registers across the ray loop.
template <bool CULL, bool RECOMPUTE>
__global__ void __launch_bounds__(kAdjThreads, kAdjCtasPerSm) adjoint_backward_kernel(const AdjArgs A) {
  __shared__ float4 s_tab[kBuieRecords];
  const TraceArgs& a = A.t;
  load_buie(a.buie, s_tab);
  __syncthreads();
  const float fy0 = CULL ? from_ordered(__ldg(a.field_yr)) : 0.f, fy1 = CULL ? from_ordered(__ldg(a.field_yr + 1)) : 0.f;

  // Each warp takes segments of 256 consecutive rays (grid-stride over all
  // warps) and works only on the rays that contribute: those the tape marks
  // as hits, and every ray past the saved part of the tape (their visibility
  // is recomputed).  Lane i reads the tape bytes of rays 8i..8i+7 of the
  // segment; the selected rays are then handed out 32 per pass, lane j taking
  // the j-th one (a binary search over the lanes' prefix counts finds the lane
  // that owns it).  Lost rays cost nothing, and a segment's rays mostly share
  // a heliostat, so the warp reduction below stays uniform.
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  // rays of the range [ray0, rays), counted from ray0 (the tape's indexing)
  const uint64_t n = a.rays - a.ray0, nseg = (n + 255) / 256;
  for (uint64_t sg = (uint64_t)blockIdx.x * nwarps + (threadIdx.x >> 5); sg < nseg;
       sg += (uint64_t)gridDim.x * nwarps) {
    const uint64_t b0 = sg * 256 + 8 * lane;  // this lane's first ray (a multiple of 8)
    uint32_t m = 0;  // bit k: ray b0 + k is worked on
    if (b0 + 8 <= A.saved && b0 + 8 <= n) {
      const uint2 t8 = *reinterpret_cast<const uint2*>(A.tape + b0);  // 8-byte aligned
#pragma unroll
      for (int k = 0; k < 8; ++k) m |= (((k < 4 ? t8.x >> (8 * k) : t8.y >> (8 * (k - 4))) & 0xFFu) != 0u) << k;
    } else {
      for (int k = 0; k < 8; ++k) {
        const uint64_t r = b0 + k;
        if (r < n && (r >= A.saved || A.tape[r] != 0)) m |= 1u << k;
      }
    }
    const int cnt = __popc(m);
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int excl = incl - cnt, total = __shfl_sync(0xffffffffu, incl, 31);
  for (int base = 0; base < total; base += 32) {
    const int q = base + lane;
    int own = 0;  // the last lane whose prefix count is <= q
    for (int step = 16; step > 0; step >>= 1)
      if (__shfl_sync(0xffffffffu, excl, own + step) <= q) own += step;
    uint32_t mo = __shfl_sync(0xffffffffu, m, own);
    const int skip = q - __shfl_sync(0xffffffffu, excl, own);
    float gk[4] = {0.f, 0.f, 0.f, 0.f};
    int h = -1;
    if (q < total) {
      for (int i = 0; i < skip; ++i) mo &= mo - 1u;  // drop the lower selected rays
      const uint64_t r64 = sg * 256 + 8 * own + (__ffs(mo) - 1);
      const uint32_t ray = (uint32_t)(a.ray0 + r64);
      RaySetup R;
      ray_setup<false>(a, s_tab, ray, R, a.rk);
      h = R.h;
      bool hit;
      Refl g;
      double u = 0, v = 0, tr = 0;
      if (!RECOMPUTE || r64 < A.saved) {  // the tape says hit: rebuild the geometry without the traversals
        g = reflect_ray(R);
        hit = receiver_uv(a, R.o, g.rd, &u, &v, &tr);
      } else {
        hit = ray_hits<CULL>(a, R, fy0, fy1, &g, &u, &v, &tr);
      }
      if (hit) {
        // bilinear corners and the adjoint map there
        float px = (float)(v * a.res_x) - 0.5f, py = (float)(u * a.res_y) - 0.5f;
        const float flx = floorf(px), fly = floorf(py);
        const int i0 = (int)flx, j0 = (int)fly;
        const float fx = px - flx, fy = py - fly;
        float Gc[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          int ci = i0 + (k & 1), cj = j0 + (k >> 1);
          Gc[k] = (ci < 0 || cj < 0 || ci >= a.res_x || cj >= a.res_y) ? 0.f : __ldg(A.G + cj * a.res_x + ci);
        }
        const float gW = (1.f - fx) * (1.f - fy) * Gc[0] + fx * (1.f - fy) * Gc[1] + (1.f - fx) * fy * Gc[2] + fx * fy * Gc[3];
        const float gWx = (1.f - fy) * (Gc[1] - Gc[0]) + fy * (Gc[3] - Gc[2]);
        const float gWy = (1.f - fx) * (Gc[2] - Gc[0]) + fx * (Gc[3] - Gc[1]);
        // forward quantities in float
        const float3 npf = to_f(g.np), rdf = to_f(g.rd), wsf = to_f(R.ws);
        // the tangents are FP32: reciprocals to ~1e-12 (and 2 ulp below) suffice
        const float ilnp = (float)rcp_nr(g.lnp), ilr = (float)rcp_nr(g.lr);
        const float nws = dot(npf, wsf);
        const float3 sd = f3(A.sdf[0], A.sdf[1], A.sdf[2]);
        const float3 E1 = f3(A.e1f[0], A.e1f[1], A.e1f[2]), E2 = f3(A.e2f[0], A.e2f[1], A.e2f[2]);
        const float sdn = dot(sd, npf);
        const float e = fabsf(sdn) * R.w, sg = sdn < 0.f ? -1.f : 1.f;
        // t along the reflected ray to the receiver plane (for d(hit) = do + t dr)
        const float3 cr = cross(E2, rdf);
        const float iden = __fdividef(1.f, dot(E1, cr));
        const float t = (float)tr;
        const float x = R.xz.x, z = R.xz.y, hy = 0.5f * __ldg(a.size + 3 * h + 1);
        // Reverse mode through the ray: the loss's sensitivity to the ray's
        // frame components (c_u, c_n, c_v), then one product with the frame
        // Jacobian per parameter.  The chain, forward: origin
        // dO = x du + hy dn + z dv; normal dN = P_n(tl.x du + tl.y dn + tl.z dv) / |n'|;
        // reflection dR = P_r(-2 ((dN.ws) n + (n.ws) dN)) / |r'| (P: the
        // projections of the normalisations); hit b = dO + t dR, read along
        // the plane as du = (b . (E2 x r)) / det and dv = (b . (r x E1)) / det;
        // energy de = sgn(s.n) (s . dN) w; the loss term
        // de gW + e (gWx res_x dv + gWy res_y du).  Each step below is the
        // transpose of one of these.
        const float3 beta = (e * gWy * (float)a.res_y * iden) * cr + (e * gWx * (float)a.res_x * iden) * cross(rdf, E1);
        float3 rho = t * beta;                          // d/dR
        rho = ilr * (rho - dot(rdf, rho) * rdf);        // through r's normalisation
        float3 nu = -2.f * (dot(rho, npf) * wsf + nws * rho);  // d/dN from the reflection
        nu = fma3(gW * sg * R.w, sd, nu);               // and from the energy
        const float3 mu = ilnp * (nu - dot(npf, nu) * npf);  // through n's normalisation
        const float3 cu = fma3(x, beta, R.tl.x * mu), cn = fma3(hy, beta, R.tl.y * mu),
                     cv = fma3(z, beta, R.tl.z * mu);
        // the frame Jacobian, row-major [9][4]: row r holds d(frame component r)
        // for the 4 parameters, one float4 (144-byte records, 16-byte aligned;
        // the same heliostat for most of a warp: broadcast loads), read row by
        // row into the 4 products
        const float4* J = reinterpret_cast<const float4*>(A.jac) + 9 * h;
        const float c9[9] = {cu.x, cu.y, cu.z, cn.x, cn.y, cn.z, cv.x, cv.y, cv.z};
#pragma unroll
        for (int r = 0; r < 9; ++r) {
          const float4 jr = __ldg(J + r);
          gk[0] = fmaf(c9[r], jr.x, gk[0]);
          gk[1] = fmaf(c9[r], jr.y, gk[1]);
          gk[2] = fmaf(c9[r], jr.z, gk[2]);
          gk[3] = fmaf(c9[r], jr.w, gk[3]);
        }
      }
    }
    // one atomic per warp and parameter when the warp's rays share a heliostat
    const unsigned full = 0xffffffffu;
    const int h0 = __shfl_sync(full, h, 0);
    const bool uniform = __all_sync(full, h == h0 || h < 0);
    if (uniform && h0 >= 0) {
      for (int k = 0; k < 4; ++k)
        for (int o = 16; o > 0; o >>= 1) gk[k] += __shfl_down_sync(full, gk[k], o);
      if ((threadIdx.x & 31) == 0) {
        atomicAdd(A.grad_aim + 2 * h0, gk[0]);
        atomicAdd(A.grad_aim + 2 * h0 + 1, gk[1]);
        atomicAdd(A.grad_tilt + 2 * h0, gk[2]);
        atomicAdd(A.grad_tilt + 2 * h0 + 1, gk[3]);
      }
    } else if (h >= 0) {
      atomicAdd(A.grad_aim + 2 * h, gk[0]);
      atomicAdd(A.grad_aim + 2 * h + 1, gk[1]);
      atomicAdd(A.grad_tilt + 2 * h, gk[2]);
      atomicAdd(A.grad_tilt + 2 * h + 1, gk[3]);
    }
  }
  }
}

// Grid of a grid-stride adjoint kernel: as many CTAs as stay resident
// together (more would leave the last ones running nearly alone).
template <class K>
static int adj_blocks(K kernel, uint64_t rays, size_t smem = 0) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kAdjThreads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sms * per_sm, (rays + kAdjThreads - 1) / kAdjThreads));
}

}  // namespace qm

struct qmcrt_tape {
  qmcrt_scene* scene = nullptr;
  qmcrt_sun sun{};
  qmcrt_trace_params params{};
  qm::AdjArgs args{};
  qm::BuieTable buie;
  float* d_buie = nullptr;
  uint8_t* d_tape = nullptr;
  float* d_G = nullptr;
  float* d_jac = nullptr;
  double* d_loss = nullptr;
  float* d_energy = nullptr;
  unsigned long long* d_energy_fx = nullptr;  // replay: [res] fixed-point energy map
  bool cull = true;
  // rays of the traced range [args.t.ray0, args.t.rays): one tape byte each
  uint64_t count() const { return args.t.rays - args.t.ray0; }
  // capacities, so that a tape passed back to qmcrt_adjoint_forward reuses its buffers
  uint64_t cap_tape = 0;
  int64_t cap_res = 0;
  int cap_n = 0;
};

namespace qm {
// The tape's arguments against the scene's current geometry (after
// tape_geometry): the pointers and per-sun values the kernels read.
static AdjArgs tape_args(qmcrt_tape* t) {
  qmcrt_scene* s = t->scene;
  AdjArgs A = t->args;
  fill_trace_args(s, scene_geom(s), &t->sun, t->params.quirks, &A.t);
  A.t.buie = t->d_buie;
  A.t.b_total = t->buie.params[3];
  A.t.b_core = t->buie.params[2];
  A.t.b_B = t->buie.params[4];
  A.t.b_C = t->buie.params[5];
  A.t.b_inv = 1 / (t->buie.params[1] + 1);
  A.t.b_inv_bucket = t->buie.inv_bucket;
  if (!t->buie.within_alpha) { A.t.cand = nullptr; A.t.cand_n = nullptr; }
  A.t.rays = t->args.t.rays;
  A.t.ray0 = t->args.t.ray0;
  A.t.rpp = t->args.t.rpp;
  A.t.rpp_shift = t->args.t.rpp_shift;
  std::memcpy(A.t.rk, t->args.t.rk, sizeof(A.t.rk));
  A.t.item = t->args.t.item;
  A.t.point_xz = s->d_point_xz;
  A.t.point_helio = s->d_point_helio;
  A.t.point_mask = s->d_point_mask;
  A.t.point_origin = s->d_point_origin;
  A.t.energy = t->d_energy;
  return A;
}

// Flux, loss and adjoint map from the tape's energy map: flux = energy x
// DNI rho / (rays per point x pixel area) (Gtest.cu:40-46 with the map's
// pixel area), L = sum (flux - target)^2 and G = dL/d(energy).
static qmcrt_status tape_loss_pass(qmcrt_tape* t, const float* d_target, float* d_flux, double* loss, cudaStream_t st) {
  qmcrt_scene* s = t->scene;
  const int64_t res = (int64_t)s->rg.res_x * s->rg.res_y;
  QM_CUDA(cudaMemsetAsync(t->d_loss, 0, sizeof(double), st));
  LossArgs la{t->d_energy, d_target, d_flux, t->d_G,
              (float)((double)t->sun.dni * t->params.reflectivity /
                      ((double)t->params.rays_per_point * s->rg.pixel_area)),
              res, t->d_loss};
  loss_kernel<<<(unsigned)std::min<int64_t>((res + 255) / 256, 1024), 256, 0, st>>>(la);
  QM_CUDA(cudaGetLastError());
  if (loss) {
    QM_CUDA(cudaMemcpyAsync(loss, t->d_loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    QM_CUDA(cudaStreamSynchronize(st));
  }
  return QMCRT_OK;
}

static qmcrt_status tape_geometry(qmcrt_tape* t, cudaStream_t st) {
  qmcrt_scene* s = t->scene;
  qmcrt_status e;
  if ((e = ensure_sun(s, &t->sun, t->params.quirks, st))) return e;
  if ((e = ensure_points(s, &t->params, st))) return e;
  if ((e = ensure_masks(s, st))) return e;
  return QMCRT_OK;
}
}  // namespace qm

extern "C" {

qmcrt_status qmcrt_adjoint_forward(qmcrt_scene* s, const qmcrt_sun* sun, const qmcrt_trace_params* p,
                                   const float* d_target, uint64_t state_bytes_max, float* d_flux, double* loss,
                                   qmcrt_tape** tape, void* stream) {
  if (!s || !sun || !p || !d_target || !tape) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (*tape && (*tape)->scene != s) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "a tape is reused only on its own scene");
  if (s->rg.type != QMCRT_RECEIVER_FLAT) return set_error(QMCRT_ERR_NOT_SUPPORTED, "the adjoint needs a flat receiver");
  if (p->deposit != QMCRT_DEPOSIT_BILINEAR) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "the adjoint deposits bilinearly");
  if (p->point_mode != QMCRT_POINTS_POISSON || p->rays == 0 || p->rays > 0xFFFFFFFFull)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "the adjoint needs Poisson points and 0 < rays < 2^32");
  if (p->quirks & ~QMCRT_QUIRK_ZENITH_FRAME)
    return set_error(QMCRT_ERR_NOT_SUPPORTED, "the adjoint traces in corrected mode");
  if (p->attenuation != QMCRT_ATTEN_NONE)
    return set_error(QMCRT_ERR_NOT_SUPPORTED, "the adjoint has no attenuation term");
  if (p->ray_end != 0 && (p->ray_begin >= p->ray_end || p->ray_end > p->rays))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "ray range must have ray_begin < ray_end <= rays");
  if (!(sun->csr > 0.f && sun->csr < 1.f)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "csr must be in (0,1)");
  cudaStream_t st = (cudaStream_t)stream;
  // a tape from an earlier call keeps its buffers where they are large enough
  const bool fresh = *tape == nullptr;
  qmcrt_tape* t = fresh ? new qmcrt_tape() : *tape;
  auto fail = [&](qmcrt_status e) {
    if (fresh) qmcrt_tape_free(t);
    return e;
  };
  t->scene = s;
  t->sun = *sun;
  t->params = *p;
  qmcrt_status e;
  int64_t res = (int64_t)s->rg.res_x * s->rg.res_y;
  // the rays [ray_begin, ray_end) of the trace (all of them when ray_end is 0)
  const uint64_t r0 = p->ray_end ? p->ray_begin : 0, r1 = p->ray_end ? p->ray_end : p->rays, count = r1 - r0;
  uint64_t saved = state_bytes_max == 0 ? count : std::min<uint64_t>(count, state_bytes_max);
  cudaError_t ce = cudaSuccess;
  if (saved > t->cap_tape) {
    cudaFree(t->d_tape);
    t->d_tape = nullptr;
    t->cap_tape = 0;
    ce = cudaMalloc(&t->d_tape, std::max<uint64_t>(saved, 1));
    if (ce == cudaSuccess) t->cap_tape = saved;
  }
  if (ce == cudaSuccess && res > t->cap_res) {
    cudaFree(t->d_G);
    cudaFree(t->d_energy);
    t->d_G = t->d_energy = nullptr;
    t->cap_res = 0;
    ce = cudaMalloc(&t->d_G, res * sizeof(float));
    if (ce == cudaSuccess) ce = cudaMalloc(&t->d_energy, res * sizeof(float));
    if (ce == cudaSuccess) t->cap_res = res;
  }
  if (ce == cudaSuccess && s->n > t->cap_n) {
    cudaFree(t->d_jac);
    t->d_jac = nullptr;
    t->cap_n = 0;
    ce = cudaMalloc(&t->d_jac, 36 * (size_t)s->n * sizeof(float));
    if (ce == cudaSuccess) t->cap_n = s->n;
  }
  if (ce == cudaSuccess && !t->d_loss) ce = cudaMalloc(&t->d_loss, sizeof(double));
  if (ce == cudaSuccess && !t->d_buie) ce = cudaMalloc(&t->d_buie, 4 * (size_t)kBuieRecords * sizeof(float));
  if (ce != cudaSuccess) return fail(cuda_error(ce, "adjoint tape allocation"));
  if ((e = tape_geometry(t, st))) return fail(e);
  if (!buie_bucket_table(sun->csr, &t->buie))
    return fail(set_error(QMCRT_ERR_INTERNAL, "Buie table: a bucket holds two interval boundaries"));
  AdjArgs& A = t->args;
  fill_trace_args(s, scene_geom(s), sun, p->quirks, &A.t);
  A.t.buie = t->d_buie;
  A.t.b_total = t->buie.params[3];
  A.t.b_core = t->buie.params[2];
  A.t.b_B = t->buie.params[4];
  A.t.b_C = t->buie.params[5];
  A.t.b_inv = 1 / (t->buie.params[1] + 1);
  A.t.b_inv_bucket = t->buie.inv_bucket;
  if (!t->buie.within_alpha) { A.t.cand = nullptr; A.t.cand_n = nullptr; }  // walk the grid
  A.t.ray0 = r0;
  A.t.rays = r1;
  A.t.rpp = p->rays_per_point;
  A.t.rpp_shift = (A.t.rpp & (A.t.rpp - 1)) ? -1 : __builtin_ctz((unsigned)A.t.rpp);
  philox_round_keys(make_uint2((uint32_t)p->seed, (uint32_t)(p->seed >> 32)), A.t.rk);
  A.t.item = p->item;
  A.t.point_xz = s->d_point_xz;
  A.t.point_helio = s->d_point_helio;
  A.t.point_mask = s->d_point_mask;
  A.t.point_origin = s->d_point_origin;
  A.t.energy = t->d_energy;
  double l1 = 0, l2 = 0;
  for (int i = 0; i < 3; ++i) {
    A.ew[i] = s->rg.v3[i] - s->rg.v0[i];
    A.eh[i] = s->rg.v1[i] - s->rg.v0[i];
    l1 += A.ew[i] * A.ew[i];
    l2 += A.eh[i] * A.eh[i];
  }
  for (int i = 0; i < 3; ++i) {
    A.ew[i] /= std::sqrt(l1);
    A.eh[i] /= std::sqrt(l2);
  }
  A.tape = t->d_tape;
  A.saved = saved;
  A.G = t->d_G;
  A.jac = t->d_jac;
  // the tile: the map's central T x T pixels, T as large as keeps 2 CTAs
  // (with the 20 KB Buie table) on an SM
  A.tile = std::min({s->rg.res_x, s->rg.res_y, kAdjTileMax});
  A.tile_r0 = (s->rg.res_y - A.tile) / 2;
  A.tile_c0 = (s->rg.res_x - A.tile) / 2;
  const size_t tile_bytes = (size_t)A.tile * (A.tile + 1) * sizeof(float);  // rows T + 1 floats apart
  const bool lean = A.t.rpp_shift >= 0 && A.t.point_mask;
  auto fwd = lean ? adjoint_forward_kernel<true, false, true> : adjoint_forward_kernel<true>;
  QM_CUDA(cudaFuncSetAttribute(fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_bytes));
  const int blocks = adj_blocks(fwd, count, tile_bytes);
  *tape = t;  // from here on the caller owns it, also when a launch below fails
  QM_CUDA(cudaMemcpyAsync(t->d_buie, t->buie.host.data(), t->buie.host.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  QM_CUDA(cudaMemsetAsync(t->d_energy, 0, res * sizeof(float), st));
  fwd<<<blocks, kAdjThreads, tile_bytes, st>>>(A);
  QM_CUDA(cudaGetLastError());
  return qm::tape_loss_pass(t, d_target, d_flux, loss, st);
}

qmcrt_status qmcrt_adjoint_backward(qmcrt_tape* t, float* d_grad_aim, float* d_grad_tilt, void* stream) {
  if (!t || !d_grad_aim || !d_grad_tilt) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  qmcrt_scene* s = t->scene;
  qmcrt_status e;
  if ((e = tape_geometry(t, st))) return e;  // re-aims only if the scene moved on to another sun
  AdjArgs A = tape_args(t);
  A.grad_aim = d_grad_aim;
  A.grad_tilt = d_grad_tilt;
  for (int i = 0; i < 3; ++i) {
    A.e1f[i] = (float)A.t.rE1[i];
    A.e2f[i] = (float)A.t.rE2[i];
    A.sdf[i] = (float)A.t.sdir[i];
  }
  JacArgs j{};
  j.n = s->n;
  j.pos = s->d_pos;
  j.aim = s->has_aim ? s->d_aim : nullptr;
  j.normal_in = s->has_normal ? s->d_normal_in : nullptr;
  j.tilt = s->has_tilt ? s->d_tilt : nullptr;
  for (int i = 0; i < 3; ++i) {
    j.focus[i] = s->rg.focus[i];
    j.ew[i] = A.ew[i];
    j.eh[i] = A.eh[i];
  }
  double l = std::sqrt((double)t->sun.dir[0] * t->sun.dir[0] + (double)t->sun.dir[1] * t->sun.dir[1] +
                       (double)t->sun.dir[2] * t->sun.dir[2]);
  for (int i = 0; i < 3; ++i) j.sun[i] = t->sun.dir[i] / l;
  j.jac = t->d_jac;
  QM_CUDA(cudaMemsetAsync(d_grad_aim, 0, 2 * (size_t)s->n * sizeof(float), st));
  QM_CUDA(cudaMemsetAsync(d_grad_tilt, 0, 2 * (size_t)s->n * sizeof(float), st));
  frame_jacobian_kernel<<<(s->n + 127) / 128, 128, 0, st>>>(j);
  QM_CUDA(cudaGetLastError());
  if (A.saved < t->count())
    adjoint_backward_kernel<true, true><<<adj_blocks(adjoint_backward_kernel<true, true>, t->count()), kAdjThreads, 0, st>>>(A);
  else
    adjoint_backward_kernel<true, false><<<adj_blocks(adjoint_backward_kernel<true, false>, t->count()), kAdjThreads, 0, st>>>(A);
  QM_CUDA(cudaGetLastError());
  return QMCRT_OK;
}

qmcrt_status qmcrt_adjoint_replay(qmcrt_tape* t, const float* d_target, float* d_flux, double* loss, void* stream) {
  if (!t || !d_target) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (t->args.saved < t->count())
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "replay needs a tape that holds every ray (state_bytes_max 0)");
  cudaStream_t st = (cudaStream_t)stream;
  qmcrt_scene* s = t->scene;
  qmcrt_status e;
  if ((e = tape_geometry(t, st))) return e;  // the scene's current aim points and tilts
  AdjArgs A = tape_args(t);
  const int64_t res = (int64_t)s->rg.res_x * s->rg.res_y;
  if (!t->d_energy_fx) QM_CUDA(cudaMalloc(&t->d_energy_fx, t->cap_res * sizeof(unsigned long long)));
  A.energy_fx = t->d_energy_fx;
  A.tile = 0;  // every deposit a 64-bit integer atomic into the global map
  QM_CUDA(cudaMemsetAsync(t->d_energy_fx, 0, res * sizeof(unsigned long long), st));
  QM_CUDA(cudaMemsetAsync(t->d_loss, 0, sizeof(double), st));
  adjoint_forward_kernel<true, true>
      <<<adj_blocks(adjoint_forward_kernel<true, true>, t->count()), kAdjThreads, 0, st>>>(A);
  QM_CUDA(cudaGetLastError());
  const qmcrt_trace_params& p = t->params;
  LossFxArgs la{t->d_energy_fx, d_target, d_flux, t->d_G,
                (double)t->sun.dni * p.reflectivity / ((double)p.rays_per_point * s->rg.pixel_area), res, t->d_loss};
  loss_fx_kernel<<<1, kLossThreads, 0, st>>>(la);
  QM_CUDA(cudaGetLastError());
  if (loss) {
    QM_CUDA(cudaMemcpyAsync(loss, t->d_loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    QM_CUDA(cudaStreamSynchronize(st));
  }
  return QMCRT_OK;
}

qmcrt_status qmcrt_tape_energy(const qmcrt_tape* t, float* d_energy, void* stream) {
  if (!t || !d_energy) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  const int64_t res = (int64_t)t->scene->rg.res_x * t->scene->rg.res_y;
  QM_CUDA(cudaMemcpyAsync(d_energy, t->d_energy, res * sizeof(float), cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return QMCRT_OK;
}

qmcrt_status qmcrt_adjoint_loss(qmcrt_tape* t, const float* d_energy, const float* d_target, float* d_flux,
                                double* loss, void* stream) {
  if (!t || !d_target) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t res = (int64_t)t->scene->rg.res_x * t->scene->rg.res_y;
  if (d_energy && d_energy != t->d_energy)
    QM_CUDA(cudaMemcpyAsync(t->d_energy, d_energy, res * sizeof(float), cudaMemcpyDeviceToDevice, st));
  return qm::tape_loss_pass(t, d_target, d_flux, loss, st);
}

qmcrt_status qmcrt_tape_loss(qmcrt_tape* t, double* loss, void* stream) {
  if (!t || !loss) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  QM_CUDA(cudaMemcpyAsync(loss, t->d_loss, sizeof(double), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaStreamSynchronize(st));
  return QMCRT_OK;
}

qmcrt_status qmcrt_tape_free(qmcrt_tape* t) {
  if (!t) return QMCRT_OK;
  cudaFree(t->d_tape);
  cudaFree(t->d_G);
  cudaFree(t->d_jac);
  cudaFree(t->d_loss);
  cudaFree(t->d_energy);
  cudaFree(t->d_energy_fx);
  cudaFree(t->d_buie);
  delete t;
  return QMCRT_OK;
}

}  // extern "C"
