// trace.cuh — device side of the tracer: arguments, Buie sampling, the FP32
// any-hit tests (per-heliostat occluder candidates, or the 3D-DDA grid walk),
// the FP64 receiver intersection and the kernel.
#pragma once
#include <stdint.h>

#include "../../include/qmcrt.h"
#include "common.cuh"
#include "internal.hpp"

namespace qm {

constexpr int kTraceThreads = 256;
constexpr int kChunkBlocks = 16;    // rays per CTA chunk = kChunkBlocks x blockDim
constexpr int kPolyAtanCols = 32768;  // widest cylinder map the polynomial column estimate serves

struct TraceArgs {
  // sun: frame of local2world for the sun direction, and the direction
  double su[3], sn[3], sv[3], sdir[3];
  // Buie table in global memory (kBuieRecords records, one per bucket) and its scalars
  const float* buie;
  float b_total, b_core, b_B, b_C, b_inv, b_inv_bucket;
  // field
  const double* frame;  // [kFrameStride n] u, n, v, mirror centre
  const float* pos;
  const float* size;
  const float* sigma;
  const float* weight;  // [n] area per point; NULL -> 1
  // grid
  const float4* crect;
  const int4* cinfo;      // [cells] {first, end, ylo, yhi (float bits)}: the cell's run of crect
  // per-heliostat occluder candidates: for each heliostat and walk (shadow,
  // block) the candidates' rectangle records inline, and their counts
  // (> kCandCap: the list overflowed); NULL: walk the grid
  const float4* cand;   // [n][2][kCandCap][3]
  const int* cand_n;    // [n][2]
  // [points] candidates reachable from each point (shadow, block bits), and
  // the slope sigma and area weight of its heliostat (float bits); NULL: all
  // candidates, sigma and weight read per heliostat
  const uint4* point_mask;
  // [points] world coordinates of each point, w holding their float x and y
  // (Philox traces; table mode computes them)
  const double4* point_origin;
  const float4* rect;   // [3n] every heliostat's own rectangle record
  const int* field_yr;    // [2] height range of the field (order-preserving ints)
  float gpos[3], gcell[3], ginv[3];  // ginv = 1 / gcell
  int gdims[3];
  // two-level grid: each coarse cell covers 2^cshift fine cells per axis;
  // coarse_yr is the union of its fine cells' height ranges (NULL: one level)
  const float2* coarse_yr;
  int cshift;
  int cdims[3];
  float ccell[3];
  // receiver
  int rtype;
  double rA[3], rE1[3], rE2[3];
  // flat receiver as a plane: N = E1 x E2, and the dual edges D1 = (E2 x N) / |N|^2,
  // D2 = (N x E1) / |N|^2, so that w . D1 and w . D2 are the E1 and E2 coordinates
  // of an in-plane offset w
  double rN[3], rD1[3], rD2[3];
  double cyl[6];  // cylinder: bottom centre x, y, z, radius, height, 1 / height
  const double2* cyl_edge;  // cylinder: [res_x] (cos, sin) of each column's first edge, 2 pi k / res_x
  int res_x, res_y;
  // rays
  int n_helio;
  // Rays of one launch: ids ray_hi * 2^32 + [ray0, rays).  A launch never
  // crosses a multiple of 2^32, so a thread works with the low word of its
  // ray id; the high word is word 1 of the Philox counter, and g_hi the
  // point of ray ray_hi * 2^32 (power-of-two rays per point; 0 when ray_hi
  // is 0).
  uint64_t rays;
  uint64_t ray0;
  uint32_t ray_hi, g_hi;
  int rpp;
  int rpp_shift;  // log2(rpp) when rpp is a power of two, else -1
  uint2 rk[10];  // Philox round keys of the seed (philox_round_keys)
  uint32_t item;
  uint32_t quirks;
  const float2* point_xz;
  const int32_t* point_helio;
  // table mode
  const float* sun_local;
  const float* turb_local;
  int64_t T;
  const int32_t* start;
  // outputs
  uint32_t* counts;
  float* energy;
  uint8_t* flags;
  int32_t* pixel;
  unsigned long long* stats;
  int atten;  // QMCRT_ATTEN_*
};

// Atmospheric transmittance over the slant range d (m) from the mirror to the
// receiver: the formula eta_aAlpha carries, disabled, at
// rectgrid_raytracing.cu:120-127 (the reference returns 1).
__device__ __forceinline__ float atten_eta(int mode, float d) {
  if (mode != QMCRT_ATTEN_POLY_EXP) return 1.f;
  return d <= 1000.f ? 0.99331f - 0.0001176f * d + 1.97e-8f * d * d : expf(-0.0001106f * d);
}

// max_less_index (scene_instance_process.cu:98-113) over the table in smem:
// the largest i with cdf_y[i] <= value.
__device__ __forceinline__ int max_less_index(const float* cdf_y, float value) {
  int left = 0, right = 1024, mid;
  while (left <= right) {
    mid = (left + right) >> 1;
    float c = cdf_y[mid];
    if (value > c) left = mid + 1;
    else if (value < c) right = mid - 1;
    else return mid;
  }
  return right;
}

// Inverse CDF of the Buie sunshape (linear_interpolate, :115-137).  mrad.
// The interval index equals max_less_index's (the largest i with
// cdf_y[i] <= uu, at most 1023).  The table is staged per uniform bucket of
// [0, core): record b is {angle, cdf, slope, next interval's cdf} of the
// interval holding the bucket's smallest value.  A bucket holds at most one
// interval boundary, and past it lies the interval of record b + 1, so one
// compare picks between two records loaded together: no guide lookup, no
// scan and no branch (68.8 G rays/s on the mid field with record b + 1
// loaded only when needed, 69.2 G with both loaded; 67.6 G with the guide
// table and scan this replaced).
__device__ __forceinline__ float buie_theta_mrad(const TraceArgs& a, const float4* s_tab, float u) {
  float uu = u * a.b_total;
  if (uu < a.b_core) {
    const int b = min((int)(uu * a.b_inv_bucket), kBuieBuckets - 1);
    const float4 q0 = s_tab[b], q1 = s_tab[b + 1];
    const float4 q = uu >= q0.w ? q1 : q0;
    return (uu - q.y) * q.z + q.x;
  }
  // the aureole's analytic inverse (a few percent of the rays, but a warp
  // with one of them runs it): the hardware power, relative error ~2^-21,
  // moves the sample by ~1e-9 rad
  return __powf((uu - a.b_core) * a.b_B + a.b_C, a.b_inv);
}

// sin and cos of a small angle by their Taylor series in Horner form,
// x + x^3 (-1/6 + x^2/120) and 1 + x^2 (-1/2 + x^2/24): exact to float
// rounding for |x| < 0.05 (the first omitted terms are below 2e-11 relative).
// A Buie sample is at most 9.3 mrad (the aureole's end), so the sun sample
// always takes this form; sincos_small falls back to sincosf above 0.05.
__device__ __forceinline__ void sincos_taylor(float x, float* s, float* c) {
  const float x2 = x * x;
  *s = fmaf(x * x2, fmaf(x2, 1.f / 120.f, -1.f / 6.f), x);
  *c = fmaf(x2, fmaf(x2, 1.f / 24.f, -0.5f), 1.f);
}
__device__ __forceinline__ void sincos_small(float x, float* s, float* c) {
  if (fabsf(x) < 0.05f) sincos_taylor(x, s, c);
  else sincosf(x, s, c);
}

// Does the ray o + t d hit the parallelogram A, E1, E2 at t > eps?  The test
// of rayParallelogramIntersect (global_function.cuh:78-105) with the
// divisions by det folded into the comparisons.
__device__ __forceinline__ bool rect_hit(float4 r0, float4 r1, float4 r2, float3 o, float3 d) {
  float3 E1 = f3(r1.x, r1.y, r1.z), E2 = f3(r2.x, r2.y, r2.z);
  float3 T = f3(o.x - r0.x, o.y - r0.y, o.z - r0.z);
  float3 pv = cross(d, E2);
  float det = dot(E1, pv);
  if (fabsf(det) < kEps) return false;
  float sg = det < 0.f ? -1.f : 1.f, ad = fabsf(det);
  float un = dot(T, pv) * sg;
  if (un < 0.f || un > ad) return false;
  float3 qv = cross(T, E1);
  float vn = dot(d, qv) * sg;
  if (vn < 0.f || vn > ad) return false;
  float tn = dot(E2, qv) * sg;
  return tn >= kEps * ad;
}

// One grid cell (its run [b, e) of cell-major records): any rectangle other
// than `own` hit?
template <bool STATS>
__device__ __forceinline__ bool cell_hit(const TraceArgs& a, int b, int e, float3 o, float3 d, int own, bool selfhit,
                                         uint32_t& ntest) {
  for (int k = b; k < e; ++k) {
    float4 r0 = __ldg(a.crect + 3 * k);
    if (__float_as_int(r0.w) == own && !selfhit) continue;
    if (STATS) ++ntest;
    if (rect_hit(r0, __ldg(a.crect + 3 * k + 1), __ldg(a.crect + 3 * k + 2), o, d)) return true;
  }
  return false;
}

// |t / dir| with the reference's guard (absDivide, rectgrid_raytracing.cu:11-17)
__device__ __forceinline__ float abs_div(float t, float d) {
  return (d <= kEps && d >= -kEps) ? 2147483648.0f : fabsf(t / d);
}

__device__ __forceinline__ float from_ordered(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

// 3D-DDA any-hit (NotCollision, rectgrid_raytracing.cu:38-117).  The origin
// cell is tested first unless QMCRT_QUIRK_SKIP_ORIGIN_CELL.
// CULL (corrected mode only): a cell whose rectangles all lie above or below
// the ray's height over the cell's [t_in, t_out] is not tested, and the walk
// ends once the ray has left the field's height range.  With every rectangle
// registered in every cell it touches, a real hit is always found in the cell
// holding the hit point, whose height range contains that point, so the
// answer is unchanged.
// TWO (with CULL, two-level grid): the same test one level up — a coarse cell
// whose height range (the union of its fine cells') misses the ray's height
// over the coarse cell is stepped through without touching any fine cell.
// The fine walk itself is unchanged, so the set of cells that can hold a hit,
// and therefore the answer, is the single-level one.
template <bool STATS, bool CULL, bool TWO = false>
__device__ bool dda_blocked(const TraceArgs& a, float3 o, float3 d, int own, float fy0, float fy1, uint32_t& ntest,
                            uint32_t& ncell) {
  const bool selfhit = a.quirks & QMCRT_QUIRK_SELF_HIT;
  const int gx = a.gdims[0], gy = a.gdims[1], gz = a.gdims[2];
  float rx = o.x - a.gpos[0], ry = o.y - a.gpos[1], rz = o.z - a.gpos[2];
  int ix = min(max((int)floorf(rx * a.ginv[0]), 0), gx - 1);
  int iy = min(max((int)floorf(ry * a.ginv[1]), 0), gy - 1);
  int iz = min(max((int)floorf(rz * a.ginv[2]), 0), gz - 1);
  int sx = d.x >= 0.f ? 1 : -1, sy = d.y >= 0.f ? 1 : -1, sz = d.z >= 0.f ? 1 : -1;
  // calTMax and absDivide (rectgrid_raytracing.cu:3-17) with one reciprocal
  // per axis in place of the divisions
  const float big = 2147483648.0f;
  const bool px = fabsf(d.x) > kEps, py = fabsf(d.y) > kEps, pz = fabsf(d.z) > kEps;
  const float qx = px ? fabsf(__frcp_rn(d.x)) : 0.f, qy = py ? fabsf(__frcp_rn(d.y)) : 0.f,
              qz = pz ? fabsf(__frcp_rn(d.z)) : 0.f;
  float tx = px ? fabsf(d.x >= 0.f ? (float)(ix + 1) * a.gcell[0] - rx : rx - (float)ix * a.gcell[0]) * qx : big;
  float ty = py ? fabsf(d.y >= 0.f ? (float)(iy + 1) * a.gcell[1] - ry : ry - (float)iy * a.gcell[1]) * qy : big;
  float tz = pz ? fabsf(d.z >= 0.f ? (float)(iz + 1) * a.gcell[2] - rz : rz - (float)iz * a.gcell[2]) * qz : big;
  float dx = px ? a.gcell[0] * qx : big, dy = py ? a.gcell[1] * qy : big, dz = pz ? a.gcell[2] * qz : big;
  // true if the cell may hold a hit: the ray's height over [t0, t1], widened
  // by a margin far above FP32 error, meets the cell's rectangle heights
  auto may_hit = [&](int4 ci, float t0, float t1) -> bool {
    if (!CULL) return true;
    float ya = o.y + t0 * d.y, yb = o.y + t1 * d.y;
    float mg = 0.01f + 1e-5f * t1;
    return !(fmaxf(ya, yb) + mg < __int_as_float(ci.z) || fminf(ya, yb) - mg > __int_as_float(ci.w));
  };
  // whether the current coarse cell is stepped through, evaluated when the
  // walk enters a coarse cell; its exit along each axis is that axis' next
  // fine crossing plus the fine cells left in the coarse cell
  bool cskip = false;
  const int cm = TWO ? (1 << a.cshift) - 1 : 0;
  auto coarse_eval = [&](float t0) {
    const int cs = a.cshift;
    int cc = ((ix >> cs) * a.cdims[1] + (iy >> cs)) * a.cdims[2] + (iz >> cs);
    float ex = tx + dx * (float)(sx > 0 ? cm - (ix & cm) : (ix & cm));
    float ey = ty + dy * (float)(sy > 0 ? cm - (iy & cm) : (iy & cm));
    float ez = tz + dz * (float)(sz > 0 ? cm - (iz & cm) : (iz & cm));
    float t1 = fminf(ex, fminf(ey, ez));
    float2 yr = __ldg(a.coarse_yr + cc);
    float ya = o.y + t0 * d.y, yb = o.y + t1 * d.y;
    float mg = 0.05f + 1e-4f * t1;
    cskip = fmaxf(ya, yb) + mg < yr.x || fminf(ya, yb) - mg > yr.y;
  };
  if (TWO) coarse_eval(0.f);
  if (!(a.quirks & QMCRT_QUIRK_SKIP_ORIGIN_CELL)) {
    if (!TWO || !cskip) {
      const int4 ci = __ldg(a.cinfo + ((ix * gy + iy) * gz + iz));
      if (may_hit(ci, 0.f, fminf(tx, fminf(ty, tz)))) {
        if (STATS) ++ncell;
        if (cell_hit<STATS>(a, ci.x, ci.y, o, d, own, selfhit, ntest)) return true;
      }
    }
  }
  for (int guard = gx + gy + gz + 2; guard > 0; --guard) {
    float tin;
    bool cross = false;  // the step entered a new coarse cell
    if (tx < ty) {
      if (tx < tz) {
        ix += sx;
        if (ix >= gx || ix < 0) return false;
        tin = tx;
        tx += dx;
        if (TWO) cross = (ix & cm) == (sx > 0 ? 0 : cm);
      } else {
        iz += sz;
        if (iz >= gz || iz < 0) return false;
        tin = tz;
        tz += dz;
        if (TWO) cross = (iz & cm) == (sz > 0 ? 0 : cm);
      }
    } else {
      if (ty < tz) {
        iy += sy;
        if (iy >= gy || iy < 0) return false;
        tin = ty;
        ty += dy;
        if (TWO) cross = (iy & cm) == (sy > 0 ? 0 : cm);
      } else {
        iz += sz;
        if (iz >= gz || iz < 0) return false;
        tin = tz;
        tz += dz;
        if (TWO) cross = (iz & cm) == (sz > 0 ? 0 : cm);
      }
    }
    if (CULL) {
      float y = o.y + tin * d.y, mg = 0.01f + 1e-5f * tin;
      if ((d.y > 0.f && y - mg > fy1) || (d.y < 0.f && y + mg < fy0)) return false;  // left the mirror layer
    }
    if (TWO) {
      if (cross) coarse_eval(tin);
      if (cskip) continue;
    }
    const int4 ci = __ldg(a.cinfo + ((ix * gy + iy) * gz + iz));
    if (!may_hit(ci, tin, fminf(tx, fminf(ty, tz)))) continue;
    if (STATS) ++ncell;
    if (cell_hit<STATS>(a, ci.x, ci.y, o, d, own, selfhit, ntest)) return true;
  }
  return false;
}

// Any-hit over heliostat h's occluder candidates for one walk (which = 0:
// toward the sun, 1: after the reflection).  Every heliostat a ray of h can
// meet is in the list, so the answer is the grid walk's; all lanes of a warp
// share h, so they run the same candidates with broadcast loads.  A list that
// overflowed, or no lists (cand_n NULL), falls back to the grid walk.
// reach: the candidates the ray's point can reach (bit j: list entry j), from
// the per-point masks; every bit set when there are none.
// A point mask is either all ones (no masks, a list that overflowed, or
// every candidate reachable) or holds only bits below the list's count, as the
// mask pass writes them; so a mask of 0 needs no list at all and only an
// all-ones mask needs the list's count.
template <bool STATS>
__device__ __forceinline__ bool list_blocked(const TraceArgs& a, int h, int which, float3 o, float3 d, float fy0,
                                             float fy1, uint32_t& ntest, uint32_t& ncell, uint32_t reach) {
  if (reach == 0u) return false;
  uint32_t bits = reach;
  if (reach == 0xffffffffu) {
    const int m = a.cand_n ? __ldg(a.cand_n + 2 * h + which) : kCandCap + 1;  // no lists: walk
    if (m > kCandCap) return dda_blocked<STATS, true>(a, o, d, h, fy0, fy1, ntest, ncell);
    bits = m == 32 ? 0xffffffffu : (1u << m) - 1u;
  }
  const float4* L = a.cand + (size_t)(2 * h + which) * (kCandCap * 3);
  while (bits) {  // the same bits on every lane of a warp (one point)
    const int i = __ffs(bits) - 1;
    bits &= bits - 1u;
    if (STATS) ++ntest;
    if (rect_hit(__ldg(L + 3 * i), __ldg(L + 3 * i + 1), __ldg(L + 3 * i + 2), o, d)) return true;
  }
  return false;
}

// Receiver intersection in FP64; returns true on a hit and the pixel index
// (-1 when the hit falls outside the map, QMCRT_QUIRK_PIXEL_EDGE only).
// RT: the receiver type when known at compile time (QMCRT_RECEIVER_*), -1
// to read it from the arguments.
// LEAN: QMCRT_QUIRK_PIXEL_EDGE is off (the pixel is clamped to the map).
template <int RT = -1, bool LEAN = false>
__device__ __forceinline__ bool receiver_hit(const TraceArgs& a, d3 o, d3 d, int& pix, double* t_out = nullptr) {
  double u, v = 0.0;
  int col = -1;  // set directly by the cylinder
  if (RT < 0 ? a.rtype == QMCRT_RECEIVER_CYLINDER : RT == QMCRT_RECEIVER_CYLINDER) {
    double ox = o.x - a.cyl[0], oz = o.z - a.cyl[2], R = a.cyl[3], H = a.cyl[4];
    double qa = d.x * d.x + d.z * d.z;
    if (qa < 1e-18) return false;
    double qb = ox * d.x + oz * d.z, qc = ox * ox + oz * oz - R * R;
    double disc = qb * qb - qa * qc;
    if (disc < 0) return false;
    // sqrt(disc) = disc / sqrt(disc) and one reciprocal of qa for both roots
    // (relative errors ~1e-12: picometres at the receiver)
    const double sq = disc > 1e-300 ? disc * rsqrt_nr(disc) : 0.0, iqa = rcp_nr(qa);
    double t = (-qb - sq) * iqa;
    double y = o.y + t * d.y - a.cyl[1];
    if (t < 1e-6 || y < 0 || y > H) {
      t = (-qb + sq) * iqa;
      y = o.y + t * d.y - a.cyl[1];
      if (t < 1e-6 || y < 0 || y > H) return false;
    }
    if (t_out) *t_out = t;
    u = y * a.cyl[5];
    // column = floor(phi / 2 pi * res_x), phi = atan2(Z, X) in [0, 2 pi):
    // a single-precision angle picks a column within one of the right one;
    // the signs of the hit's FP64 cross products with that column's edges
    // (directions at 2 pi k / res_x) settle it.  Both edges lie within two
    // columns of the hit, where sign(cos a Z - sin a X) = sign(sin(phi - a)).
    // The angle: atan of the octant ratio q = min/max of |X|, |Z| as
    // q (c0 + c1 q^2 + c2 q^4 + c3 q^6), a minimax fit of atan on [0, 1]
    // (Lawson-weighted least squares on 4001 Chebyshev nodes), largest error
    // 8.2e-5 rad in float arithmetic, then the octant and quadrant folds.
    // The estimate stays within one column while 2 pi / res_x exceeds twice
    // that error, up to 38 000 columns; wider maps take atan2f.
    const double X = ox + t * d.x, Z = oz + t * d.z;
    const float xf = (float)X, zf = (float)Z;
    float pf;
    if (a.res_x <= kPolyAtanCols) {
      const float ax = fabsf(xf), az = fabsf(zf);
      const float q = __fdividef(fminf(ax, az), fmaxf(ax, az)), q2 = q * q;
      pf = q * fmaf(fmaf(fmaf(-0.0389864407f, q2, 0.146264359f), q2, -0.321174920f), q2, 0.999213815f);
      if (az > ax) pf = 1.57079633f - pf;
      if (xf < 0.f) pf = 3.14159265f - pf;
      if (zf < 0.f) pf = 6.28318531f - pf;
    } else {
      pf = atan2f(zf, xf);
      if (pf < 0.f) pf += 6.28318531f;
    }
    int c = min(max((int)(pf * (float)a.res_x * 0.159154943f), 0), a.res_x - 1);
    const double2 e0 = __ldg(a.cyl_edge + c);
    if (e0.x * Z - e0.y * X < 0.0) {
      c = c == 0 ? a.res_x - 1 : c - 1;
    } else {
      const int c1 = c + 1 == a.res_x ? 0 : c + 1;
      const double2 e1 = __ldg(a.cyl_edge + c1);
      if (e1.x * Z - e1.y * X >= 0.0) c = c1;
    }
    col = c;
  } else {
    // the parallelogram test of rayParallelogramIntersect (global_function.cuh:78-105)
    // in plane form: its determinant E1 . (d x E2) is -d . N, t = ((A - o) . N) / (d . N),
    // and (u, v) are the dual-edge coordinates of the hit's offset from A
    const d3 N = mk(a.rN[0], a.rN[1], a.rN[2]);
    const double dn = dot(d, N);
    if (fabs(dn) < 1e-6) return false;
    const d3 ao = mk(a.rA[0], a.rA[1], a.rA[2]) - o;
    const double t = dot(ao, N) * rcp_nr(dn);
    if (t < 1e-6) return false;
    const d3 w = t * d - ao;  // hit - A
    u = dot(w, mk(a.rD1[0], a.rD1[1], a.rD1[2]));
    if (u < 0 || u > 1) return false;
    v = dot(w, mk(a.rD2[0], a.rD2[1], a.rD2[2]));
    if (v < 0 || v > 1) return false;
    if (t_out) *t_out = t;
  }
  int row = (int)(u * a.res_y);  // rectgrid_raytracing.cu:144
  if (col < 0) col = (int)(v * a.res_x);
  if (!LEAN && (a.quirks & QMCRT_QUIRK_PIXEL_EDGE)) {
    if (row >= a.res_y || col >= a.res_x) {
      pix = -1;
      return true;
    }
  } else {
    row = min(row, a.res_y - 1);
    col = min(col, a.res_x - 1);
  }
  pix = row * a.res_x + col;
  return true;
}

__device__ __forceinline__ d3 rnorm(d3 a) {
  double r = rsqrt_nr(dot(a, a));
  return r * a;
}

struct RayCounters {
  uint32_t ray = 0, sh = 0, bl = 0, hit = 0, off = 0, test = 0, cell = 0;
};

// Deposit into the global maps with plain atomics.
struct GlobalDeposit {
  uint32_t* counts;
  float* energy;
  __device__ __forceinline__ void operator()(int pix, float e) const {
    red_add(counts + pix, 1u);
    red_add(energy + pix, e);
  }
};

// Load the Buie table's bucket records into shared memory (all threads): one
// {angle, cdf, slope, next cdf} record per uniform bucket of the core CDF,
// of the interval holding the bucket's smallest value (kBuieRecords of them).
__device__ __forceinline__ void load_buie(const float* buie, float4* s_tab) {
  const float4* rec = reinterpret_cast<const float4*>(buie);  // kBuieRecords 16-byte records
  for (int i = threadIdx.x; i < kBuieRecords; i += blockDim.x) s_tab[i] = __ldg(rec + i);
}

// Everything a ray needs before its traversals: heliostat, local point,
// mirror frame, origin, the sun sample (local and world) and the local
// perturbation of the normal.
struct RaySetup {
  int h;
  float2 xz;
  uint2 reach;  // candidate masks of the ray's point (shadow, block)
  frame64 fr;
  d3 o;
  float3 of;  // o rounded to float
  float3 sl, tl;
  d3 ws;
  float w;
};

// Sun sample and slope-error perturbation of ray `ray` from Philox (seed,
// ray id): theta from the Buie inverse CDF, phi uniform; slope theta
// Gaussian (Box-Muller), phi uniform (set_samplelights, set_perturbation).
// rk: the seed's Philox round keys (a.rk, or a copy the caller holds in
// faster memory).
// The stages of philox_samples: the Philox block of a ray, and the two
// directions from that block and the ray's Buie angle (mrad).
__device__ __forceinline__ uint4 ray_block(const TraceArgs& a, uint32_t ray, const uint2* rk) {
  return philox4x32_10_rk(make_uint4(ray, a.ray_hi, a.item, kTagTrace), rk);
}
__device__ __forceinline__ void sample_dirs(uint4 r, float th_mrad, float sigma, float3* sl, float3* tl) {
  const float th = th_mrad * 1e-3f;
  float st, ct, sp, cp;
  // The azimuths and the Box-Muller log use the hardware approximations
  // (__sincosf, __logf: absolute errors near 2^-21): they scale milliradian
  // polar angles, so a direction moves by ~1e-9 rad, far below FP32 rounding
  // of the geometry that follows.
  sincos_taylor(th, &st, &ct);  // th <= 9.3 mrad
  __sincosf(6.28318531f * u23f(r.y), &sp, &cp);
  *sl = f3(st * cp, ct, st * sp);  // angle2xyz (global_function.cuh:175-180)
  // the Box-Muller radius with the hardware square root (relative error
  // ~2^-22, a slope angle moves by ~1e-9 rad)
  float rad;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(rad) : "f"(-2.f * __logf(u23f(r.z))));
  float z = rad * __cosf(6.28318531f * u23f(r.w));
  float ths = sigma * z;
  // the slope azimuth from the words' top bytes (the uniforms above use bits 0-22)
  uint32_t extra = __byte_perm(__byte_perm(r.x, r.y, 0x0073u), __byte_perm(r.z, r.w, 0x0073u), 0x5410u);
  sincos_small(ths, &st, &ct);
  __sincosf(6.28318531f * u23f(extra), &sp, &cp);
  *tl = f3(st * cp, ct, st * sp);
}

// Sun sample and slope-error perturbation of ray `ray` from Philox (seed,
// ray id): theta from the Buie inverse CDF, phi uniform; slope theta
// Gaussian (Box-Muller), phi uniform (set_samplelights, set_perturbation).
// rk: the seed's Philox round keys (a.rk, or a copy the caller holds in
// faster memory).
__device__ __forceinline__ void philox_samples(const TraceArgs& a, const float4* s_tab, uint32_t ray,
                                               float sigma, float3* sl, float3* tl, const uint2* rk) {
  const uint4 r = ray_block(a, ray, rk);
  sample_dirs(r, buie_theta_mrad(a, s_tab, u23f(r.x)), sigma, sl, tl);
}

// Returns false for a ray to skip (table mode with an out-of-range heliostat id).
// LEAN (Philox traces only): a power-of-two count of rays per point and the
// per-point mask records present, so neither is tested per ray.
template <bool TABLES, bool LEAN = false>
__device__ __forceinline__ bool ray_setup(const TraceArgs& a, const float4* s_tab, uint32_t ray,
                                          RaySetup& R, const uint2* rk) {
  const uint32_t g = (LEAN || a.rpp_shift >= 0) ? a.g_hi + (ray >> a.rpp_shift) : ray / (uint32_t)a.rpp;
  const uint32_t j = ray - g * (uint32_t)a.rpp;  // table mode (ray_hi 0)
  const int h = __ldg(a.point_helio + g);
  if (TABLES && (h < 0 || h >= a.n_helio)) return false;  // caller-provided ids: never index out of range
  R.h = h;
  R.xz = __ldg(a.point_xz + g);
  float sigma_h = 0.f;
  if (LEAN || a.point_mask) {
    const uint4 pm = __ldg(a.point_mask + g);
    R.reach = make_uint2(pm.x, pm.y);
    sigma_h = __uint_as_float(pm.z);
    R.w = __uint_as_float(pm.w);
  } else {
    R.reach = make_uint2(0xffffffffu, 0xffffffffu);
    if (!TABLES) {
      sigma_h = __ldg(a.sigma + h);
      R.w = a.weight ? __ldg(a.weight + h) : 1.f;
    }
  }
  // the frame axes (16-byte aligned record) as 16-byte loads
  const double2* F = reinterpret_cast<const double2*>(a.frame + kFrameStride * h);
  const double2 q0 = __ldg(F), q1 = __ldg(F + 1), q2 = __ldg(F + 2), q3 = __ldg(F + 3), q4 = __ldg(F + 4);
  R.fr.u = mk(q0.x, q0.y, q1.x);
  R.fr.n = mk(q1.y, q2.x, q2.y);
  R.fr.v = mk(q3.x, q3.y, q4.x);
  if (TABLES) {  // origin: the mirror centre plus the point's in-plane offset
    const double2 q5 = __ldg(F + 5);
    R.o = mk(q4.y, q5.x, q5.y) + (double)R.xz.x * R.fr.u + (double)R.xz.y * R.fr.v;
    R.of = to_f(R.o);
  } else {  // the same, computed once per point and sun by the mask pass
    const double2* O = reinterpret_cast<const double2*>(a.point_origin + g);  // 32-byte records
    const double2 oa = __ldg(O), ob = __ldg(O + 1);
    R.o = mk(oa.x, oa.y, ob.x);
    R.of = f3(__int_as_float(__double2loint(ob.y)), __int_as_float(__double2hiint(ob.y)), (float)ob.x);
  }
  if (TABLES) {
    R.w = 1.f;
    // (start + j) mod T, kept in [0, T) for any caller-provided start
    int64_t ia = (((int64_t)__ldg(a.start + g) + j) % a.T + a.T) % a.T;
    // the reference's index restarts at each heliostat's launch
    int64_t gp = (a.quirks & QMCRT_QUIRK_PREV_PERTURB) && g > 0 && __ldg(a.point_helio + g - 1) == R.h ? g - 1 : g;
    int64_t ib = (((int64_t)__ldg(a.start + gp) + j) % a.T + a.T) % a.T;
    R.sl = f3(__ldg(a.sun_local + 3 * ia), __ldg(a.sun_local + 3 * ia + 1), __ldg(a.sun_local + 3 * ia + 2));
    R.tl = f3(__ldg(a.turb_local + 3 * ib), __ldg(a.turb_local + 3 * ib + 1), __ldg(a.turb_local + 3 * ib + 2));
  } else {
    philox_samples(a, s_tab, ray, sigma_h, &R.sl, &R.tl, rk);
  }
  // world sample (local2world(sample, sun_dir)), incident direction
  const float3 sl = R.sl;
  R.ws = mk(sl.x * a.su[0] + sl.y * a.sn[0] + sl.z * a.sv[0], sl.x * a.su[1] + sl.y * a.sn[1] + sl.z * a.sv[1],
            sl.x * a.su[2] + sl.y * a.sn[2] + sl.z * a.sv[2]);
  return true;
}

// One ray: the body of map_tracing (rectgrid_raytracing.cu:164-195).
// CULL: 0 no culling, 1 vertical culling, 2 vertical culling on both levels
// of a two-level grid, 3 the per-heliostat occluder candidates (Philox
// sampling only: their cones bound the sampler's directions).
// LEAN (Philox traces only): power-of-two rays per point, per-point masks,
// no attenuation and no QMCRT_QUIRK_PIXEL_EDGE, so none of them is tested
// per ray.
template <bool TABLES, bool RECORDS, bool STATS, int CULL, class Dep, int RT = -1, bool LEAN = false>
__device__ __forceinline__ void trace_ray(const TraceArgs& a, const float4* s_tab, uint32_t ray,
                                          float fy0, float fy1, RayCounters& c, const Dep& deposit,
                                          const uint2* rk) {
  RaySetup R;
  if (!ray_setup<TABLES, LEAN>(a, s_tab, ray, R, rk)) {
    if (RECORDS) {
      if (a.flags) a.flags[ray] = 0;
      if (a.pixel) a.pixel[ray] = -1;
    }
    return;
  }
  const int h = R.h;
  const d3 o = R.o, ws = R.ws;
  // perturbed normal, reflected direction (i - 2 n (n.i)) and energy first,
  // so that the mirror frame is dead before the walks.  The reflection keeps
  // the length of ws (1 to float rounding of the sample), and nothing that
  // uses rd depends on its length beyond that: the receiver's (u, v), the
  // rectangle tests and the walk's cell order are scale-free, the slant range
  // for attenuation moves by ~1e-7 relative; so rd is not renormalised.
  const d3 npu = apply(R.fr, (double)R.tl.x, (double)R.tl.y, (double)R.tl.z);
  const double nn = dot(npu, npu);
  d3 rd;
  float e;  // calEnergy (rectgrid_raytracing.cu:129-133)
  if (TABLES) {  // caller tables may hold vectors of any length
    const d3 np = rsqrt_nr(nn) * npu;
    rd = ws - (2.0 * dot(ws, np)) * np;
    e = (float)fabs(np.x * a.sdir[0] + np.y * a.sdir[1] + np.z * a.sdir[2]) * R.w;
  } else {
    // A Philox perturbation is a unit vector to float rounding and the frame
    // is orthonormal in FP64, so nn = 1 + t with |t| < 2e-6.  Then
    // 1 / nn = 1 - t + t^2 to within t^3 (below 1e-17), and 1 / sqrt(nn) =
    // 1.5 - nn / 2 to within 3 t^2 / 8 (below 2e-12, for the float energy):
    // no square root or reciprocal, and the normal is never scaled.
    const double t = nn - 1.0;
    const double k = -2.0 * dot(ws, npu) * fma(t, t - 1.0, 1.0);
    rd = mk(fma(k, npu.x, ws.x), fma(k, npu.y, ws.y), fma(k, npu.z, ws.z));
    e = (float)(fabs(npu.x * a.sdir[0] + npu.y * a.sdir[1] + npu.z * a.sdir[2]) * fma(-0.5, nn, 1.5)) * R.w;
  }
  uint8_t flag = 0;
  int pix = -1;
  double th = 0.0;
  // The walks' FP32 origin and directions are formed only for a walk that
  // runs: a point mask of 0 (most points) skips its walk, and with it five to
  // seven FP64-to-FP32 conversions on the XU pipe.
  auto of = [&]() { return TABLES ? R.of : f3(R.of.x, R.of.y, (float)o.z); };
  auto sdir = [&]() { return f3((float)-ws.x, (float)-ws.y, (float)-ws.z); };
  bool shadowed, blocked = false;
  if (CULL == 3) {
    shadowed = R.reach.x != 0u && list_blocked<STATS>(a, h, 0, of(), sdir(), fy0, fy1, c.test, c.cell, R.reach.x);
    if (!shadowed)
      blocked = R.reach.y != 0u && list_blocked<STATS>(a, h, 1, of(), to_f(rd), fy0, fy1, c.test, c.cell, R.reach.y);
  } else {
    shadowed = dda_blocked<STATS, (CULL > 0), (CULL == 2)>(a, of(), sdir(), h, fy0, fy1, c.test, c.cell);
    if (!shadowed) blocked = dda_blocked<STATS, (CULL > 0), (CULL == 2)>(a, of(), to_f(rd), h, fy0, fy1, c.test, c.cell);
  }
  if (shadowed) {
    flag = QMCRT_RAY_SHADOWED;
  } else if (blocked) {
    flag = QMCRT_RAY_BLOCKED;
  } else if (receiver_hit<RT, LEAN>(a, o, rd, pix, &th)) {
    flag = QMCRT_RAY_HIT;
    if (pix < 0) flag |= QMCRT_RAY_OFFMAP;
    else deposit(pix, !LEAN && a.atten ? e * atten_eta(a.atten, (float)th) : e);  // times eta(t) (:147)
  }
  if (RECORDS) {
    if (a.flags) a.flags[ray] = flag;
    if (a.pixel) a.pixel[ray] = pix;
  }
  if (STATS) {
    ++c.ray;
    c.sh += (flag & QMCRT_RAY_SHADOWED) != 0;
    c.bl += (flag & QMCRT_RAY_BLOCKED) != 0;
    c.hit += (flag & QMCRT_RAY_HIT) != 0;
    c.off += (flag & QMCRT_RAY_OFFMAP) != 0;
  }
}

// Warp-reduce the counters and add them to stats[0..6].
__device__ __forceinline__ void flush_counters(const RayCounters& c, unsigned long long* stats) {
  unsigned long long v[7] = {c.ray, c.sh, c.bl, c.hit, c.off, c.test, c.cell};
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    unsigned long long x = v[k];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(stats + k, x);
  }
}

// The plain tracer: one grid-stride pass over the rays of one trace.  RT:
// the receiver type, or -1 to read it from the arguments; LEAN: as trace_ray.
template <bool TABLES, bool RECORDS, bool STATS, int CULL, int MINB = 1, int RT = -1, bool LEAN = false>
__global__ void __launch_bounds__(kTraceThreads, MINB) trace_kernel(const TraceArgs a) {
  pdl_wait();
  __shared__ float4 s_tab[kBuieRecords];
  const float fy0 = CULL ? from_ordered(__ldg(a.field_yr)) : 0.f, fy1 = CULL ? from_ordered(__ldg(a.field_yr + 1)) : 0.f;
  if (!TABLES) {
    load_buie(a.buie, s_tab);
    __syncthreads();
  }
  RayCounters c;
  const GlobalDeposit dep{a.counts, a.energy};
  // chunks of kChunkBlocks x 256 consecutive rays (16 sample points at 256
  // rays per point) taken grid-stride: a CTA stays on one heliostat for most
  // of a chunk, so its frame and candidates stay in L1, and the chunks are
  // small enough to keep the SMs evenly loaded
  const uint64_t chunk = (uint64_t)kChunkBlocks * blockDim.x,
                 nch = (a.rays - a.ray0 + chunk - 1) / chunk;
  for (uint64_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    // the low words of the chunk's ray ids (the launch stays below 2^32)
    const uint64_t b64 = a.ray0 + ch * chunk;
    const uint32_t base = (uint32_t)b64, len = (uint32_t)(min(b64 + chunk, a.rays) - b64);
    for (uint32_t j = threadIdx.x; j < len; j += blockDim.x)
      trace_ray<TABLES, RECORDS, STATS, CULL, GlobalDeposit, RT, LEAN>(a, s_tab, base + j, fy0, fy1, c, dep, a.rk);
  }
  if (STATS) flush_counters(c, a.stats);
}

}  // namespace qm
