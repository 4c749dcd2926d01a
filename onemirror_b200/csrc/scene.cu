// scene.cu — scene lifetime, heliostat aiming, GPU grid build and
// micro-heliostat sample points.
//
// Replaces, on the GPU: set_helio_content + RectangleHelio::CRotate
// (scene_instance_process.cpp:24-35, heliostat.cpp:16-58), the host CSR build
// RectGrid::Cinit/CGridHelioMatch (grid.cpp:3-83) and the micro-point
// generators set_microhelio_centers / set_possion_microhelio_centers
// (steps_for_raytracing.cu:67-158).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "internal.hpp"

using namespace qm;

namespace qm {

// --------------------------------------------------------------- aiming
struct AimArgs {
  int n;
  const float *pos, *size, *aim, *normal_in, *tilt;
  double focus[3];
  double sun[3];
  uint32_t quirks;
  double* normal;
  double* frame;
  float4* rect;
  int4* cellbox;
  int32_t* cell_count;
  float gpos[3], gcell[3];
  int gdims[3];
  double* power;
};

__device__ __forceinline__ d3 nrm3(d3 a) {
  double l = sqrt(dot(a, a));
  return mk(a.x / l, a.y / l, a.z / l);
}

// local2world frame (global_function.cuh:14-52)
__device__ __forceinline__ frame64 frame_of(d3 n, uint32_t quirks) {
  frame64 f;
  if (fabs(n.x) < 1e-6 && fabs(n.z) < 1e-6) {
    double s = (n.y < 0 && !(quirks & QMCRT_QUIRK_ZENITH_FRAME)) ? -1.0 : 1.0;
    f.u = mk(1, 0, 0);
    f.n = mk(0, s, 0);
    f.v = mk(0, 0, s);
    return f;
  }
  f.n = n;
  f.u = nrm3(mk(n.z, 0, -n.x));  // (0,1,0) x n
  f.v = nrm3(cross(f.u, n));
  return f;
}

// Clears the per-sun registration counts of the grid cells and the field's
// total power before aim_kernel adds to them (one launch in place of two
// memsets, so that it joins the chain of kernels launched with programmatic
// dependent launch), and resets the grid's control words.
//
// The grid of a sun's geometry is built on demand.  Philox traces test
// occluder candidates and walk the grid only where a candidate list
// overflowed, so for them the build (scan, fill, cell records) runs only if
// cand_kernel finds an overflowing list.  ctl[0]: the grid is needed (forced
// by the host, or an overflowing list); ctl[1]: the grid of this geometry is
// built; ctl[2]: the build sequence now in the stream builds it (decided by
// the single-CTA scan pass, read by the passes after it).  The registration
// counts stay untouched until the scan runs, so a later trace that needs the
// grid can still build it (grid_demand_kernel, then the same passes).
__global__ void zero_geom_kernel(int32_t* cell_count, int64_t cells, double* power, int* ctl, int force) {
  pdl_wait();
  pdl_trigger();
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t i = i0; i < cells; i += (int64_t)gridDim.x * blockDim.x) cell_count[i] = 0;
  if (i0 == 0) {
    *power = 0.0;
    ctl[0] = force;
    ctl[1] = 0;
    ctl[2] = 0;
  }
}

// Marks the grid of the current geometry as needed, before its build passes
// run again for a trace that walks the grid (they build it if no build ran yet).
__global__ void grid_demand_kernel(int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (threadIdx.x == 0) ctl[0] = 1;
}

// The single-CTA decision of a build sequence (all threads of the CTA): build
// if the grid is needed and not built yet; published in ctl[2] for the passes
// after this one.
__device__ __forceinline__ bool grid_build_decide(int* ctl) {
  __shared__ int s_go;
  if (threadIdx.x == 0) {
    const int go = ctl[0] != 0 && ctl[1] == 0;
    ctl[2] = go;
    if (go) ctl[1] = 1;
    s_go = go;
  }
  __syncthreads();
  return s_go != 0;
}

__global__ void aim_kernel(AimArgs a) {
  pdl_wait();
  pdl_trigger();
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  double pw = 0;
  if (h < a.n) {
    d3 p = mk(a.pos[3 * h], a.pos[3 * h + 1], a.pos[3 * h + 2]);
    d3 n;
    if (a.normal_in) {
      n = nrm3(mk(a.normal_in[3 * h], a.normal_in[3 * h + 1], a.normal_in[3 * h + 2]));
    } else {
      d3 t = a.aim ? mk(a.aim[3 * h], a.aim[3 * h + 1], a.aim[3 * h + 2])
                   : mk(a.focus[0], a.focus[1], a.focus[2]);
      d3 r = nrm3(t - p);
      n = nrm3(r - mk(a.sun[0], a.sun[1], a.sun[2]));  // heliostat.cpp:51-58
    }
    frame64 f = frame_of(n, a.quirks);
    if (a.tilt) {
      n = nrm3(n + a.tilt[2 * h] * f.u + a.tilt[2 * h + 1] * f.v);
      f = frame_of(n, a.quirks);
    }
    a.normal[3 * h] = n.x;
    a.normal[3 * h + 1] = n.y;
    a.normal[3 * h + 2] = n.z;
    double* fr = a.frame + kFrameStride * h;
    fr[0] = f.u.x; fr[1] = f.u.y; fr[2] = f.u.z;
    fr[3] = f.n.x; fr[4] = f.n.y; fr[5] = f.n.z;
    fr[6] = f.v.x; fr[7] = f.v.y; fr[8] = f.v.z;
    double sx = a.size[3 * h], sy = a.size[3 * h + 1], sz = a.size[3 * h + 2];
    const d3 c = p + (sy / 2) * f.n;  // the mirror centre: sample points are c + u x + v z
    fr[9] = c.x; fr[10] = c.y; fr[11] = c.z;
    // Cset_localvertex + Cset_worldvertex (heliostat.cpp:30-49): v0, v1, v3
    d3 v0 = p + apply(f, -sx / 2, sy / 2, -sz / 2);
    d3 v1 = p + apply(f, -sx / 2, sy / 2, sz / 2);
    d3 v3 = p + apply(f, sx / 2, sy / 2, -sz / 2);
    d3 e1 = v1 - v0, e2 = v3 - v0;
    a.rect[3 * h] = make_float4((float)v0.x, (float)v0.y, (float)v0.z, __int_as_float(h));
    a.rect[3 * h + 1] = make_float4((float)e1.x, (float)e1.y, (float)e1.z, 0.f);
    a.rect[3 * h + 2] = make_float4((float)e2.x, (float)e2.y, (float)e2.z, 0.f);
    // cells covered (CGridHelioMatch grid.cpp:47-61)
    int lo[3], hi[3];
    if (a.quirks & QMCRT_QUIRK_AABB_RADIUS) {
      float fx = a.size[3 * h], fy = a.size[3 * h + 1], fz = a.size[3 * h + 2];
      float radius = sqrtf(__fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)), __fmul_rn(fz, fz)))) / 2;
      for (int i = 0; i < 3; ++i) {
        float pc = a.pos[3 * h + i];
        int l = (int)(__fsub_rn(__fsub_rn(pc, radius), a.gpos[i]) / a.gcell[i]);
        int u = (int)(__fsub_rn(__fadd_rn(pc, radius), a.gpos[i]) / a.gcell[i]);
        lo[i] = min(max(l, 0), a.gdims[i] - 1);
        hi[i] = min(max(u, 0), a.gdims[i] - 1);
      }
    } else {
      d3 v2 = v1 + e2;
      double c[4][3] = {{v0.x, v0.y, v0.z}, {v1.x, v1.y, v1.z}, {v2.x, v2.y, v2.z}, {v3.x, v3.y, v3.z}};
      for (int i = 0; i < 3; ++i) {
        double mn = c[0][i], mx = c[0][i];
        for (int k = 1; k < 4; ++k) {
          mn = fmin(mn, c[k][i]);
          mx = fmax(mx, c[k][i]);
        }
        int l = (int)floor((mn - (double)a.gpos[i]) / (double)a.gcell[i]);
        int u = (int)floor((mx - (double)a.gpos[i]) / (double)a.gcell[i]);
        lo[i] = min(max(l, 0), a.gdims[i] - 1);
        hi[i] = min(max(u, 0), a.gdims[i] - 1);
      }
    }
    a.cellbox[2 * h] = make_int4(lo[0], lo[1], lo[2], 0);
    a.cellbox[2 * h + 1] = make_int4(hi[0], hi[1], hi[2], 0);
    for (int x = lo[0]; x <= hi[0]; ++x)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int z = lo[2]; z <= hi[2]; ++z)
          atomicAdd(&a.cell_count[((int64_t)x * a.gdims[1] + y) * a.gdims[2] + z], 1);
    // Gtest.cu:29: |n . sun| * A
    pw = fabs(dot(n, mk(a.sun[0], a.sun[1], a.sun[2]))) * sx * sz;
  }
  for (int o = 16; o > 0; o >>= 1) pw += __shfl_down_sync(0xffffffffu, pw, o);
  if ((threadIdx.x & 31) == 0 && pw != 0) atomicAdd(a.power, pw);
}

// Exclusive scan of cell_count into cell_start (one CTA of 1024 threads,
// each scanning a contiguous run), then zero cell_count for the fill cursor.
__global__ void __launch_bounds__(1024) scan_kernel(int32_t* count, int32_t* start, int64_t cells,
                                                    int64_t cap, int32_t* flag, int* field_yr, int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (!grid_build_decide(ctl)) return;
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  if (t == 0) {  // empty height range for cell_finish_kernel's atomicMin/Max
    field_yr[0] = 0x7F7FFFFF;                        // ordered(+FLT_MAX)
    field_yr[1] = (int)(0xFF7FFFFFu ^ 0x7FFFFFFFu);  // ordered(-FLT_MAX)
  }
  int64_t per = (cells + 1023) / 1024;
  int64_t b = t * per, e = min(cells, b + per);
  int64_t s = 0;
  for (int64_t i = b; i < e; ++i) s += count[i];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int64_t v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int64_t run = part[t] - s;
  for (int64_t i = b; i < e; ++i) {
    start[i] = (int32_t)min(run, cap);
    run += count[i];
    count[i] = 0;
  }
  if (t == 1023) {
    start[cells] = (int32_t)min(part[1023], cap);
    if (part[1023] > cap) atomicExch(flag, 1);
  }
}

// The same scan over many CTAs for large grids (one CTA reads its cells
// with one thread per 4 consecutive cells; the single-CTA scan above walks
// 216 000 cells of the 12.5 m grid of a 10 000-heliostat field in 0.29 ms).
// Pass 1: each CTA's tile of kScanTile cells, its tile-local exclusive
// prefix into start and its total into part.
__global__ void __launch_bounds__(1024) scan_tiles_kernel(const int32_t* count, int32_t* start, int64_t cells,
                                                          int64_t* part, const int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (!(ctl[0] != 0 && ctl[1] == 0)) return;  // the decision scan_parts_kernel takes next
  __shared__ int64_t warp_sum[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t b = (int64_t)blockIdx.x * kScanTile + 4 * t;
  int32_t c[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) c[k] = b + k < cells ? count[b + k] : 0;
  const int64_t sum = (int64_t)c[0] + c[1] + c[2] + c[3];
  int64_t incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_sum[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int64_t x = warp_sum[lane];
    int64_t xi = x;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t v = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += v;
    }
    warp_sum[lane] = xi - x;  // the warps' exclusive prefix
    if (lane == 31) part[blockIdx.x] = xi;
  }
  __syncthreads();
  int64_t run = warp_sum[w] + incl - sum;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (b + k < cells) {
      start[b + k] = (int32_t)min(run, (int64_t)INT32_MAX);
      run += c[k];
    }
}

// Pass 2 (one CTA): exclusive scan of the tiles' totals in place, the grid's
// total into start[cells] (clamped to the capacity, flag set past it), and
// the empty height range for cell_finish_kernel.
__global__ void __launch_bounds__(1024) scan_parts_kernel(int64_t* part, int64_t tiles, int32_t* start,
                                                          int64_t cells, int64_t cap, int32_t* flag, int* field_yr,
                                                          int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (!grid_build_decide(ctl)) return;
  __shared__ int64_t acc[1024];
  const int t = threadIdx.x;
  if (t == 0) {
    field_yr[0] = 0x7F7FFFFF;                        // ordered(+FLT_MAX)
    field_yr[1] = (int)(0xFF7FFFFFu ^ 0x7FFFFFFFu);  // ordered(-FLT_MAX)
  }
  const int64_t per = (tiles + 1023) / 1024, b = t * per, e = min(tiles, b + per);
  int64_t sum = 0;
  for (int64_t i = b; i < e; ++i) sum += part[i];
  acc[t] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int64_t v = t >= o ? acc[t - o] : 0;
    __syncthreads();
    acc[t] += v;
    __syncthreads();
  }
  int64_t run = acc[t] - sum;
  for (int64_t i = b; i < e; ++i) {
    const int64_t x = part[i];
    part[i] = run;
    run += x;
  }
  if (t == 1023) {
    start[cells] = (int32_t)min(acc[1023], cap);
    if (acc[1023] > cap) atomicExch(flag, 1);
  }
}

// Pass 3: each cell's start = its tile's offset + its tile-local prefix
// (clamped to the capacity); the count is zeroed for the fill cursor.
__global__ void scan_add_kernel(int32_t* count, int32_t* start, int64_t cells, const int64_t* part, int64_t cap,
                                const int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (!ctl[2]) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cells) return;
  start[i] = (int32_t)min(part[i / kScanTile] + start[i], cap);
  count[i] = 0;
}

__global__ void fill_kernel(int n, const int4* cellbox, const int32_t* start, int32_t* cursor,
                            int32_t* entries, int gy, int gz, int64_t cap, const int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (!ctl[2]) return;
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= n) return;
  int4 lo = cellbox[2 * h], hi = cellbox[2 * h + 1];
  for (int x = lo.x; x <= hi.x; ++x)
    for (int y = lo.y; y <= hi.y; ++y)
      for (int z = lo.z; z <= hi.z; ++z) {
        int64_t c = ((int64_t)x * gy + y) * gz + z;
        int slot = atomicAdd(&cursor[c], 1);
        int64_t k = (int64_t)start[c] + slot;
        if (k < start[c + 1] && k < cap) entries[k] = h;
      }
}

// float -> int with the same order (for atomicMin/Max on floats)
__device__ __forceinline__ int ordered(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}

// Sort each cell's list ascending (the reference's push_back order,
// grid.cpp:36-44), lay the rectangles out cell-major, and write each cell's
// record {first, end, ylo, yhi}: its run of rectangles and their height range
// (for the traversal's vertical culling; one 16-byte load per DDA step), and
// the height range of the whole field.
// One thread per cell (large grids, most of whose cells are empty): the
// cell's ids sorted in place by insertion, then as the warp-per-cell kernel
// below.
__global__ void cell_finish_kernel(int64_t cells, const int32_t* start, int32_t* entries,
                                   const float4* rect, float4* cell_rect, int4* cell_info, int* field_yr,
                                   const int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (!ctl[2]) return;
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cells) return;
  int b = start[c], e = start[c + 1];
  for (int i = b + 1; i < e; ++i) {
    int v = entries[i], j = i - 1;
    while (j >= b && entries[j] > v) {
      entries[j + 1] = entries[j];
      --j;
    }
    entries[j + 1] = v;
  }
  float ylo = 3.0e38f, yhi = -3.0e38f;
  for (int i = b; i < e; ++i) {
    int h = entries[i];
    float4 r0 = rect[3 * h], r1 = rect[3 * h + 1], r2 = rect[3 * h + 2];
    cell_rect[3 * (int64_t)i] = r0;
    cell_rect[3 * (int64_t)i + 1] = r1;
    cell_rect[3 * (int64_t)i + 2] = r2;
    float y0 = r0.y, y1 = r0.y + r1.y, y2 = r0.y + r2.y, y3 = r0.y + r1.y + r2.y;
    ylo = fminf(ylo, fminf(fminf(y0, y1), fminf(y2, y3)));
    yhi = fmaxf(yhi, fmaxf(fmaxf(y0, y1), fmaxf(y2, y3)));
  }
  cell_info[c] = make_int4(b, e, __float_as_int(ylo), __float_as_int(yhi));
  if (e > b) {
    atomicMin(field_yr, ordered(ylo));
    atomicMax(field_yr + 1, ordered(yhi));
  }
}

// One warp per cell: the cell's heliostat ids in ascending order (the
// reference's push_back order, grid.cpp:53-83), its cell-major rectangle
// records, its 16-byte cell record {first, end, ylo, yhi} and the field's
// height range.  A cell's ids are distinct, so each id's position is the
// number of smaller ids in the cell: every lane ranks up to kCellRankMax / 32
// ids against all of the cell's ids (cached loads), the warp writes them in
// order.  Larger cells (none in the bench's fields) sort on one lane.
constexpr int kCellRankMax = 128;
__global__ void cell_finish_warp_kernel(int64_t cells, const int32_t* start, int32_t* entries,
                                   const float4* rect, float4* cell_rect, int4* cell_info, int* field_yr,
                                   const int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (!ctl[2]) return;
  const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= cells) return;  // whole warps leave together
  const int b = start[c], e = start[c + 1], k = e - b;
  if (k <= kCellRankMax) {
    int v[kCellRankMax / 32], r[kCellRankMax / 32];
#pragma unroll
    for (int q = 0; q < kCellRankMax / 32; ++q) {
      const int i = b + lane + 32 * q;
      v[q] = i < e ? entries[i] : 0;
      r[q] = 0;
    }
    for (int m = b; m < e; ++m) {
      const int x = entries[m];
#pragma unroll
      for (int q = 0; q < kCellRankMax / 32; ++q) r[q] += x < v[q];
    }
    __syncwarp();  // every lane has read the cell's ids before any is overwritten
#pragma unroll
    for (int q = 0; q < kCellRankMax / 32; ++q)
      if (b + lane + 32 * q < e) entries[b + r[q]] = v[q];
  } else if (lane == 0) {
    for (int i = b + 1; i < e; ++i) {
      int x = entries[i], j = i - 1;
      while (j >= b && entries[j] > x) {
        entries[j + 1] = entries[j];
        --j;
      }
      entries[j + 1] = x;
    }
  }
  __syncwarp();
  float ylo = 3.0e38f, yhi = -3.0e38f;
  for (int i = b + lane; i < e; i += 32) {
    const int h = entries[i];
    const float4 r0 = rect[3 * h], r1 = rect[3 * h + 1], r2 = rect[3 * h + 2];
    cell_rect[3 * (int64_t)i] = r0;
    cell_rect[3 * (int64_t)i + 1] = r1;
    cell_rect[3 * (int64_t)i + 2] = r2;
    const float y0 = r0.y, y1 = r0.y + r1.y, y2 = r0.y + r2.y, y3 = r0.y + r1.y + r2.y;
    ylo = fminf(ylo, fminf(fminf(y0, y1), fminf(y2, y3)));
    yhi = fmaxf(yhi, fmaxf(fmaxf(y0, y1), fmaxf(y2, y3)));
  }
  for (int o = 16; o > 0; o >>= 1) {
    ylo = fminf(ylo, __shfl_xor_sync(0xffffffffu, ylo, o));
    yhi = fmaxf(yhi, __shfl_xor_sync(0xffffffffu, yhi, o));
  }
  if (lane == 0) {
    cell_info[c] = make_int4(b, e, __float_as_int(ylo), __float_as_int(yhi));
    if (e > b) {
      atomicMin(field_yr, ordered(ylo));
      atomicMax(field_yr + 1, ordered(yhi));
    }
  }
}

// Height range of each coarse cell of a two-level grid: the union of the
// ranges of its div^3 fine cells (empty cells contribute nothing).
__global__ void coarse_finish_kernel(int64_t coarse_cells, int div, int3 cdims, int gy, int gz, const int4* cell_info,
                                     float2* coarse_yr, const int* ctl) {
  pdl_wait();
  pdl_trigger();
  if (!ctl[2]) return;
  int64_t cc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cc >= coarse_cells) return;
  int cz = (int)(cc % cdims.z), cy = (int)((cc / cdims.z) % cdims.y), cx = (int)(cc / ((int64_t)cdims.z * cdims.y));
  float ylo = 3.0e38f, yhi = -3.0e38f;
  for (int x = cx * div; x < (cx + 1) * div; ++x)
    for (int y = cy * div; y < (cy + 1) * div; ++y)
      for (int z = cz * div; z < (cz + 1) * div; ++z) {
        int4 r = cell_info[((int64_t)x * gy + y) * gz + z];
        ylo = fminf(ylo, __int_as_float(r.z));
        yhi = fmaxf(yhi, __int_as_float(r.w));
      }
  coarse_yr[cc] = make_float2(ylo, yhi);
}

// Occluder candidates of each heliostat's rays (corrected mode, Philox
// sampling): every heliostat k whose bounding sphere some ray of heliostat h
// can reach on its way to the sun (shadow) or after reflection (block).  A
// ray starts within R_h of h's centre and leaves inside a cone about the
// walk's axis: the sun axis widened by the largest Buie angle for shadow
// rays; the nominal reflection widened by that angle plus twice the largest
// slope deviation (zmax sigma: the Box-Muller deviate of 24-bit uniforms is at
// most 5.89 in magnitude) for block rays.  Once every ray of the cone rises, a
// sphere entirely below the lowest ray of the cone is out of reach too.
struct CandArgs {
  int n;
  const float *pos, *size, *sigma;
  const double* frame;
  double sun[3];      // incident direction, unit
  double sun_alpha;   // largest angle of a sun sample from the sun axis (rad)
  double shadow_tan, shadow_rise;  // the shadow cone (the same for every heliostat): tan of its half-angle, rise
  double zmax;        // largest |z| of the slope deviate, in units of sigma
  const float4* rect;  // [3n] every heliostat's rectangle record
  float4* cand;        // [n][2][kCandCap][3] the candidates' records, inline
  int* cand_n;        // [n][2]
  const CandBuckets* buckets;    // centre buckets of the field (header)
  const int32_t* bucket_start;   // [nbx * nbz + 1]
  const int32_t* bucket_ids;     // [n]
  int* grid_ctl;  // the geometry's grid control words: word 0 set when a list overflows (NULL: none)
};

__device__ __forceinline__ double bound_radius(const float* size, int h) {
  double x = size[3 * h], y = size[3 * h + 1], z = size[3 * h + 2];
  return 0.5 * sqrt(x * x + y * y + z * z) + 0.01;  // + 1 cm for FP32 rounding of records and origins
}

// Can a ray from within Rh of ch, leaving within angle atan(tan_a) of the
// unit axis d, meet the sphere (ck, Rk)?  At axial distance t a ray is at most
// Rh + (t + Rh) tan_a from the axis; rays rise at least dymin per unit length.
__device__ __forceinline__ bool cone_reaches(d3 ch, double Rh, d3 d, double tan_a, double dymin, d3 ck, double Rk) {
  const d3 q = ck - ch;
  const double t = dot(q, d), rr = Rh + Rk;
  if (t < -rr) return false;
  const d3 v = q - t * d;
  const double lim = rr + (fmax(t, 0.0) + rr) * tan_a;
  if (dot(v, v) > lim * lim) return false;
  if (dymin > 1e-3 && t - Rk > Rh + (ck.y + Rk - (ch.y - Rh)) / dymin) return false;
  return true;
}

// Second, tighter test for a pair that passed cone_reaches: the two mirrors'
// parallelograms (corners from the FP32 rectangle records, widened by mu for
// their rounding) projected along the cone axis d onto the plane across it.
// A ray from a point p of mirror h meeting a point q of mirror k travels
// (q - p).d >= 0 along d and at most (q - p).d tan(alpha) across it, so the
// projections can be at most rho = (max_k a - min_h a) tan(alpha) apart
// (a = axial coordinate).  A separating axis of the two projected
// parallelograms with a larger gap rules the pair out; the axes tried are the
// projected edge normals (an axis that degenerates is skipped, which only
// keeps the pair).
__device__ bool sat_reaches(const float4* rh, const float4* rk, d3 d, double tan_a) {
  const double mu = 0.01;
  d3 e1 = fabs(d.x) < 0.9 ? mk(1, 0, 0) : mk(0, 1, 0);
  e1 = e1 - dot(e1, d) * d;
  e1 = (1.0 / sqrt(dot(e1, e1))) * e1;
  const d3 e2 = cross(d, e1);
  double px[2][4], py[2][4], amin_h = 1e300, amax_k = -1e300;
  double ex[2][2], ey[2][2];
  for (int m = 0; m < 2; ++m) {
    const float4* r = m ? rk : rh;
    const d3 A = mk(r[0].x, r[0].y, r[0].z), E1 = mk(r[1].x, r[1].y, r[1].z), E2 = mk(r[2].x, r[2].y, r[2].z);
    const d3 c[4] = {A, A + E1, A + E2, A + E1 + E2};
    for (int i = 0; i < 4; ++i) {
      const double ax = dot(c[i], d);
      if (m) amax_k = fmax(amax_k, ax);
      else amin_h = fmin(amin_h, ax);
      px[m][i] = dot(c[i], e1);
      py[m][i] = dot(c[i], e2);
    }
    ex[m][0] = dot(E1, e1); ey[m][0] = dot(E1, e2);
    ex[m][1] = dot(E2, e1); ey[m][1] = dot(E2, e2);
  }
  const double da = amax_k - amin_h + 2.0 * mu;
  if (da < 0.0) return false;  // k lies wholly behind h along every ray
  const double rho = da * tan_a + 2.0 * mu;
  for (int m = 0; m < 2; ++m)
    for (int j = 0; j < 2; ++j) {
      double nx = -ey[m][j], ny = ex[m][j];
      const double l = sqrt(nx * nx + ny * ny);
      if (!(l > 1e-9)) continue;
      nx /= l;
      ny /= l;
      double lo[2] = {1e300, 1e300}, hi[2] = {-1e300, -1e300};
      for (int q = 0; q < 2; ++q)
        for (int i = 0; i < 4; ++i) {
          const double v = px[q][i] * nx + py[q][i] * ny;
          lo[q] = fmin(lo[q], v);
          hi[q] = fmax(hi[q], v);
        }
      if (lo[1] - hi[0] > rho || lo[0] - hi[1] > rho) return false;
    }
  return true;
}

// The cone of one walk of heliostat h: axis d, tan of its half-angle, and
// the rise per unit length of its lowest ray, sin(asin(d.y) - alpha) (<= 1e-3:
// it does not rise).  all: the half-angle is too wide for a cone (slope
// errors of ~0.13 rad and more); every heliostat is a candidate.
struct Cone {
  d3 d;
  double tan_a, rise;
  bool all;
};

__device__ __forceinline__ Cone walk_cone(const CandArgs& a, int h, int walk) {
  const d3 s = mk(a.sun[0], a.sun[1], a.sun[2]);
  if (walk == 0) return Cone{mk(-s.x, -s.y, -s.z), a.shadow_tan, a.shadow_rise, false};
  const double* F = a.frame + kFrameStride * h;
  const d3 nh = mk(F[3], F[4], F[5]);
  const d3 db = s - (2.0 * dot(s, nh)) * nh;
  const double ab = a.sun_alpha + 2.0 * a.zmax * (double)a.sigma[h] + 1e-6;
  if (!(ab < 1.2)) return Cone{db, 0.0, 0.0, true};
  double sa, ca;
  sincos(ab, &sa, &ca);
  const double y = fmin(fmax(db.y, -1.0), 1.0);
  return Cone{db, sa / ca, y * ca - sqrt(fmax(1.0 - y * y, 0.0)) * sa, false};
}

// Each lane tests its heliostat k (k < 0: none) against heliostat h's cone;
// the passing ones are appended to list L in lane order.  Returns the updated
// count, which may pass kCandCap (only the first kCandCap records are kept).
__device__ __forceinline__ int cand_take(const CandArgs& a, int k, int h, d3 ch, double Rh, const Cone& c, float4* L,
                                         int cnt) {
  const int lane = threadIdx.x & 31;
  bool r = false;
  if (k >= 0 && k != h) {
    const d3 ck = mk(a.pos[3 * k], a.pos[3 * k + 1], a.pos[3 * k + 2]);
    r = c.all || (cone_reaches(ch, Rh, c.d, c.tan_a, c.rise, ck, bound_radius(a.size, k)) &&
                  sat_reaches(a.rect + 3 * h, a.rect + 3 * k, c.d, c.tan_a));
  }
  const unsigned m = __ballot_sync(0xffffffffu, r);
  if (r) {
    const int slot = cnt + __popc(m & ((1u << lane) - 1u));
    if (slot < kCandCap)
      for (int j = 0; j < 3; ++j) L[3 * slot + j] = a.rect[3 * k + j];
  }
  return cnt + __popc(m);
}

__device__ __forceinline__ int clamp_bucket(double v, int nb) { return (int)fmin(fmax(floor(v), 0.0), nb - 1.0); }

// The candidates of one walk of heliostat h, searched over the centre
// buckets the cone can reach.  A k accepted by cone_reaches lies at axial
// distance t in [-(Rh + Rk), Rh + Rk + (ck.y + Rk - ch.y + Rh) / rise] and
// within Rh + Rk + (t + Rh + Rk) tan_a of the axis, so its centre projects
// onto (x, z) within rad of the projected axis segment [t0, t1] (bounded
// with the field's largest Rk and ck.y + Rk; 5 cm added for rounding).  Per
// bucket row, the part of the segment within rad of the row's z-strip gives
// the x-range of buckets, one contiguous run of ids.  A cone that does not
// rise has no axial bound and visits every bucket.  The lanes take one row
// each (32 rows at a time), and the rows' runs are then tested as one list,
// 32 ids at a time: each lane finds the row of its id by a binary search over
// the rows' exclusive prefix sums.
__device__ int cand_search(const CandArgs& a, const CandBuckets& B, int h, d3 ch, double Rh, const Cone& c,
                           float4* L) {
  const int lane = threadIdx.x & 31;
  const double rr = Rh + B.rmax;
  const bool bounded = !c.all && c.rise > 1e-3;
  double rad = 0.0, p0x = 0.0, p0z = 0.0, dx = 0.0, dz = 0.0;
  int bz0 = 0, bz1 = B.nbz - 1;
  if (bounded) {
    const double t0 = -rr, t1 = rr + (B.ytop - ch.y + Rh) / c.rise;
    rad = rr + (fmax(t1, 0.0) + rr) * c.tan_a + 0.05;
    p0x = ch.x + t0 * c.d.x;
    p0z = ch.z + t0 * c.d.z;
    dx = (t1 - t0) * c.d.x;
    dz = (t1 - t0) * c.d.z;
    bz0 = clamp_bucket((fmin(p0z, p0z + dz) - rad - B.z0) * B.inv, B.nbz);
    bz1 = clamp_bucket((fmax(p0z, p0z + dz) + rad - B.z0) * B.inv, B.nbz);
  }
  const double bsz = 1.0 / B.inv;
  int cnt = 0;
  for (int rb = bz0; rb <= bz1; rb += 32) {
    const int bz = rb + lane;
    int s0 = 0, len = 0;
    if (bz <= bz1) {
      int bx0 = 0, bx1 = B.nbx - 1;
      bool any = true;
      if (bounded) {
        const double zs0 = B.z0 + bz * bsz - rad, zs1 = B.z0 + (bz + 1) * bsz + rad;
        double ta = 0.0, tb = 1.0;
        if (fabs(dz) > 1e-12) {
          ta = (zs0 - p0z) / dz;
          tb = (zs1 - p0z) / dz;
          if (ta > tb) {
            const double t = ta;
            ta = tb;
            tb = t;
          }
          ta = fmax(ta, 0.0);
          tb = fmin(tb, 1.0);
          any = ta <= tb;
        } else {
          any = p0z >= zs0 && p0z <= zs1;
        }
        const double xa = p0x + ta * dx, xb = p0x + tb * dx;
        bx0 = clamp_bucket((fmin(xa, xb) - rad - B.x0) * B.inv, B.nbx);
        bx1 = clamp_bucket((fmax(xa, xb) + rad - B.x0) * B.inv, B.nbx);
      }
      if (any) {
        s0 = __ldg(a.bucket_start + bz * B.nbx + bx0);
        len = __ldg(a.bucket_start + bz * B.nbx + bx1 + 1) - s0;
      }
    }
    int incl = len;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int excl = incl - len, total = __shfl_sync(0xffffffffu, incl, 31);
    for (int base = 0; base < total; base += 32) {
      const int idx = base + lane;
      int r = 0;  // the last row whose exclusive prefix is <= idx
      for (int step = 16; step > 0; step >>= 1)
        if (__shfl_sync(0xffffffffu, excl, r + step) <= idx) r += step;
      const int rs0 = __shfl_sync(0xffffffffu, s0, r), rex = __shfl_sync(0xffffffffu, excl, r);
      const int k = idx < total ? __ldg(a.bucket_ids + rs0 + idx - rex) : -1;
      cnt = cand_take(a, k, h, ch, Rh, c, L, cnt);
    }
  }
  return cnt;
}

// One warp per (heliostat, walk): the shadow (walk 0) or block (walk 1)
// candidates.  EXHAUSTIVE tests every other heliostat (the O(n^2)
// definition, kept as the check of the bucket search); otherwise the bucket
// search, which finds the same set.
template <bool EXHAUSTIVE>
__global__ void __launch_bounds__(128) cand_kernel(CandArgs a) {
  pdl_wait();
  pdl_trigger();
  const int w = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (w >= 2 * a.n) return;  // w is uniform across the warp
  const int h = w >> 1, walk = w & 1;
  const d3 ch = mk(a.pos[3 * h], a.pos[3 * h + 1], a.pos[3 * h + 2]);
  const double Rh = bound_radius(a.size, h);
  const Cone c = walk_cone(a, h, walk);
  float4* L = a.cand + (int64_t)(2 * h + walk) * kCandCap * 3;
  int cnt = 0;
  if (EXHAUSTIVE) {
    for (int b = 0; b < a.n; b += 32) {
      const int k = b + (int)(threadIdx.x & 31);
      cnt = cand_take(a, k < a.n ? k : -1, h, ch, Rh, c, L, cnt);
    }
  } else {
    cnt = cand_search(a, *a.buckets, h, ch, Rh, c, L);
  }
  if ((threadIdx.x & 31) == 0) {
    a.cand_n[2 * h + walk] = cnt;
    if (cnt > kCandCap && a.grid_ctl) a.grid_ctl[0] = 1;  // its rays walk the grid: build it
  }
}

// ---------------------------------------------------- per-point candidate masks
// A heliostat's candidate list holds every heliostat that some ray of ANY of
// its sample points can reach.  From one point the rays leave within the same
// cone (the apex now the point itself), so most of the list is out of reach:
// bit j of a point's mask is set when candidate j of its heliostat's list can
// be reached from that point, and its rays test only those candidates.
struct MaskArgs {
  int64_t points;
  const float2* point_xz;
  const int32_t* point_helio;
  const double* frame;  // [kFrameStride n] u, n, v, mirror centre
  const float4* cand;
  const int* cand_n;
  const float* sigma;
  const float* weight;  // [n] mirror area per point (NULL: 1)
  double sun[3];
  double shadow_tan, sun_alpha, zmax;
  uint4* mask;      // [points] shadow bits, block bits, slope sigma and area weight of the point's heliostat
  double4* origin;  // [points] the point in world coordinates (the rays' origin); w: float x, y
};

// Can a ray from point p, leaving within atan(tan_a) of the unit axis d, meet
// the parallelogram of rectangle record r?  The hit q satisfies (q - p).d >= 0
// and lies at most (q - p).d tan_a across the axis from p, so the
// parallelogram's projection across d must come within (largest axial
// distance) tan_a of p's; a projected edge normal that separates them by more
// rules the pair out.  The corner is taken relative to p in FP64 and the rest
// runs in FP32 (lengths of at most a few hundred metres: ~1e-5 m of rounding);
// 2 cm of slack covers that and the FP32 rounding of the ray's origin,
// direction and rectangle test.  e1, e2: unit vectors across d.
__device__ bool point_reaches(d3 p, const float4* r, float3 d, float3 e1, float3 e2, float tan_a) {
  const float mu = 0.02f;
  const float4 r0 = r[0], r1 = r[1], r2 = r[2];
  const float3 A = f3((float)((double)r0.x - p.x), (float)((double)r0.y - p.y), (float)((double)r0.z - p.z));
  const float3 E1 = f3(r1.x, r1.y, r1.z), E2 = f3(r2.x, r2.y, r2.z);
  // axial and cross-axis coordinates of A, E1, E2 (the corners are A, A + E1, A + E2, A + E1 + E2)
  const float aA = dot(A, d), a1 = dot(E1, d), a2 = dot(E2, d);
  const float amax = aA + fmaxf(a1, 0.f) + fmaxf(a2, 0.f);
  if (amax < -mu) return false;  // wholly behind the point
  const float rho = (fmaxf(amax, 0.f) + mu) * tan_a + mu;
  const float xA = dot(A, e1), x1 = dot(E1, e1), x2 = dot(E2, e1);
  const float yA = dot(A, e2), y1 = dot(E1, e2), y2 = dot(E2, e2);
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const float ex = j ? x2 : x1, ey = j ? y2 : y1;
    const float l2 = ex * ex + ey * ey;
    if (!(l2 > 1e-12f)) continue;
    const float il = rsqrtf(l2), nx = -ey * il, ny = ex * il;
    // the corners' coordinates along (nx, ny): A's plus either edge's or both
    const float c0 = xA * nx + yA * ny, d1 = x1 * nx + y1 * ny, d2 = x2 * nx + y2 * ny;
    const float lo = c0 + fminf(d1, 0.f) + fminf(d2, 0.f), hi = c0 + fmaxf(d1, 0.f) + fmaxf(d2, 0.f);
    if (lo > rho || hi < -rho) return false;  // the point projects to 0
  }
  return true;
}

__global__ void __launch_bounds__(256) point_mask_kernel(MaskArgs a) {
  pdl_wait();
  pdl_trigger();
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.points) return;
  const int h = a.point_helio[g];
  const float2 xz = a.point_xz[g];
  const double* F = a.frame + kFrameStride * h;
  const d3 u = mk(F[0], F[1], F[2]), n = mk(F[3], F[4], F[5]), v = mk(F[6], F[7], F[8]);
  const d3 p = mk(F[9], F[10], F[11]) + (double)xz.x * u + (double)xz.y * v;
  // the spare 8 bytes carry the float x and y the walks use (low, high word)
  a.origin[g] = make_double4(p.x, p.y, p.z, __hiloint2double(__float_as_int((float)p.y), __float_as_int((float)p.x)));
  const d3 s = mk(a.sun[0], a.sun[1], a.sun[2]);
  uint32_t bits[2] = {0u, 0u};
  for (int w = 0; w < 2; ++w) {
    const int m = a.cand_n[2 * h + w];
    if (m > kCandCap) {  // the rays walk the grid
      bits[w] = 0xffffffffu;
      continue;
    }
    d3 dd;
    double tan_a;
    if (w == 0) {
      dd = mk(-s.x, -s.y, -s.z);
      tan_a = a.shadow_tan;
    } else {
      dd = s - (2.0 * dot(s, n)) * n;
      const double ab = a.sun_alpha + 2.0 * a.zmax * (double)a.sigma[h] + 1e-6;
      if (!(ab < 1.2)) {  // no cone bounds the block rays: every candidate
        bits[w] = m == 32 ? 0xffffffffu : (1u << m) - 1u;
        continue;
      }
      tan_a = tanf((float)ab);  // relative error ~1e-7, far inside the 1e-4 rounding-up below
    }
    dd = rsqrt_nr(dot(dd, dd)) * dd;
    const float3 d = f3((float)dd.x, (float)dd.y, (float)dd.z);
    float3 e1 = fabsf(d.x) < 0.9f ? f3(1.f, 0.f, 0.f) : f3(0.f, 1.f, 0.f);
    e1 = e1 - dot(e1, d) * d;
    e1 = rsqrtf(dot(e1, e1)) * e1;
    const float3 e2 = cross(d, e1);
    const float ta = (float)tan_a * 1.0001f;  // rounded up
    const float4* L = a.cand + (int64_t)(2 * h + w) * kCandCap * 3;
    for (int j = 0; j < m; ++j)
      if (point_reaches(p, L + 3 * j, d, e1, e2, ta)) bits[w] |= 1u << j;
  }
  // the rays also take their heliostat's slope error and area weight from here
  a.mask[g] = make_uint4(bits[0], bits[1], __float_as_uint(a.sigma[h]), __float_as_uint(a.weight ? a.weight[h] : 1.f));
}

// ------------------------------------------------------------ points
struct PoissonArgs {
  int n;
  const float* size;
  int64_t q, rem;
  int64_t Rq, R2, cq, nb;
  uint2 key;
  int64_t max_batches;
  int2* point_q;
  float2* point_xz;
  int32_t* point_helio;
  int32_t* flag;
};

// Sequential dart throwing on a 2^-16 m lattice with exact integer distance
// tests: 32 candidates per batch (one per lane, Philox), accepted in lane
// order against every earlier point.  One warp per heliostat, background grid
// of cell r/sqrt(2) in shared memory (at most one point per cell).
__global__ void __launch_bounds__(32) poisson_kernel(PoissonArgs a) {
  extern __shared__ int32_t sgrid[];
  const int h = blockIdx.x, lane = threadIdx.x;
  const int64_t P = a.q + (h < a.rem ? 1 : 0);
  const int64_t base = (int64_t)h * a.q + min((int64_t)h, a.rem);
  const float sx = a.size[3 * h], sz = a.size[3 * h + 2];
  const int64_t W = (int64_t)((double)sx * 65536.0), H = (int64_t)((double)sz * 65536.0);
  const int64_t gx = (W + a.cq - 1) / a.cq, gz = (H + a.cq - 1) / a.cq;
  for (int64_t i = lane; i < gx * gz; i += 32) sgrid[i] = -1;
  __syncwarp();
  int64_t got = 0;
  for (int64_t b = 0; b < a.max_batches && got < P; ++b) {
    uint64_t cid = (uint64_t)b * 32 + lane;
    uint4 w = philox4x32_10(make_uint4((uint32_t)h, (uint32_t)cid, (uint32_t)(cid >> 32), kTagPoisson), a.key);
    int64_t ix = (int64_t)(((uint64_t)w.x * (uint64_t)W) >> 32);
    int64_t iz = (int64_t)(((uint64_t)w.y * (uint64_t)H) >> 32);
    int64_t cx = ix / a.cq, cz = iz / a.cq;
    bool ok = true;
    for (int64_t dx = -a.nb; dx <= a.nb && ok; ++dx)
      for (int64_t dz = -a.nb; dz <= a.nb && ok; ++dz) {
        int64_t x = cx + dx, z = cz + dz;
        if (x < 0 || z < 0 || x >= gx || z >= gz) continue;
        int k = sgrid[x * gz + z];
        if (k < 0) continue;
        int2 pq = a.point_q[base + k];
        int64_t ddx = pq.x - ix, ddz = pq.y - iz;
        if (ddx * ddx + ddz * ddz < a.R2) ok = false;
      }
    for (int l = 0; l < 32 && got < P; ++l) {
      unsigned m = __ballot_sync(0xffffffffu, ok);
      if (!((m >> l) & 1u)) continue;
      int64_t lx = __shfl_sync(0xffffffffu, ix, l), lz = __shfl_sync(0xffffffffu, iz, l);
      if (lane == l) {
        sgrid[cx * gz + cz] = (int32_t)got;
        a.point_q[base + got] = make_int2((int)ix, (int)iz);
      }
      if (lane > l && ok) {
        int64_t ddx = lx - ix, ddz = lz - iz;
        if (ddx * ddx + ddz * ddz < a.R2) ok = false;
      }
      ++got;
    }
    __syncwarp();
  }
  if (got < P) {
    if (lane == 0) atomicExch(a.flag, 2);
    return;
  }
  for (int64_t k = lane; k < P; k += 32) {
    int2 pq = a.point_q[base + k];
    float x = (float)pq.x * (1.0f / 65536.0f), z = (float)pq.y * (1.0f / 65536.0f);
    a.point_xz[base + k] = make_float2(__fsub_rn(x, 0.5f * sx), __fsub_rn(z, 0.5f * sz));
    a.point_helio[base + k] = h;
  }
}

// Regular grid of cell centres (map_microhelio_centers, steps_for_raytracing.cu:4-22).
__global__ void grid_points_kernel(int n, const float* size, float pl, const int64_t* base,
                                   float2* xz, int32_t* helio) {
  int h = blockIdx.x;
  float sx = size[3 * h], sz = size[3 * h + 2];
  int rows = (int)(sz / pl), cols = (int)(sx / pl);
  for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
    int r = i / cols, c = i % cols;
    float x = __fsub_rn(__fadd_rn(__fmul_rn((float)c, pl), pl / 2), sx / 2);
    float z = __fsub_rn(__fadd_rn(__fmul_rn((float)r, pl), pl / 2), sz / 2);
    xz[base[h] + i] = make_float2(x, z);
    helio[base[h] + i] = h;
  }
}

__global__ void weight_kernel(int n, const float* size, int64_t q, int64_t rem, int mode, float pl,
                              float* w) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= n) return;
  if (mode == QMCRT_POINTS_GRID) {
    w[h] = pl * pl;  // Gtest.cu:40: S_sub = helio_pixel_length^2
  } else {
    int64_t P = q + (h < rem ? 1 : 0);
    w[h] = (float)((double)size[3 * h] * (double)size[3 * h + 2] / (double)P);
  }
}

// ------------------------------------------------------------ helpers
template <class T>
static qmcrt_status dev_alloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  QM_CUDA(cudaMalloc((void**)p, count * sizeof(T)));
  return QMCRT_OK;
}
template <class T>
static void dev_free(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

static int64_t cells_in_box(const float gpos[3], const float gcell[3], const int gdims[3], const double lo[3],
                            const double hi[3]) {
  int64_t c = 1;
  for (int i = 0; i < 3; ++i) {
    int a = (int)std::floor((lo[i] - gpos[i]) / gcell[i]);
    int b = (int)std::floor((hi[i] - gpos[i]) / gcell[i]);
    a = std::min(std::max(a, 0), gdims[i] - 1);
    b = std::min(std::max(b, 0), gdims[i] - 1);
    c *= (b - a + 1);
  }
  return c;
}

static qmcrt_status check_field(const qmcrt_field* f) {
  if (!f || f->n <= 0 || !f->pos || !f->size) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "field needs n > 0, pos and size");
  for (int h = 0; h < f->n; ++h) {
    for (int i = 0; i < 3; ++i)
      if (!std::isfinite(f->pos[3 * h + i])) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "non-finite heliostat position");
    if (!(f->size[3 * h] > 0) || !(f->size[3 * h + 2] > 0) || !(f->size[3 * h + 1] >= 0) ||
        f->size[3 * h] > 1000.f || f->size[3 * h + 2] > 1000.f)
      return set_error(QMCRT_ERR_INVALID_ARGUMENT, "heliostat size must be positive and below 1000 m");
    float sg = f->slope_sigma ? f->slope_sigma[h] : f->sigma;
    if (!(sg >= 0) || sg > 0.5f) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "slope error must be in [0, 0.5] rad");
  }
  return QMCRT_OK;
}

// Bucket the heliostat centres on a 2D grid over (x, z) for the candidate
// search: bucket size max(2 R_max, sqrt(area / n)) (about one centre per
// bucket, never smaller than a mirror), grown until the table fits its
// capacity; ids ascending within each bucket (a stable counting sort).  The
// bucket of a centre is floor((x - x0) / size) clamped to the grid, the same
// double arithmetic the device search uses.
static qmcrt_status build_buckets(qmcrt_scene* s, const qmcrt_field* f, cudaStream_t st) {
  const int n = f->n;
  CandBuckets& B = s->h_buckets;
  double xmin = 1e300, xmax = -1e300, zmin = 1e300, zmax = -1e300, rmax = 0.0, ytop = -1e300;
  for (int h = 0; h < n; ++h) {
    const double x = f->pos[3 * h], y = f->pos[3 * h + 1], z = f->pos[3 * h + 2];
    const double sx = f->size[3 * h], sy = f->size[3 * h + 1], sz = f->size[3 * h + 2];
    const double r = 0.5 * std::sqrt(sx * sx + sy * sy + sz * sz) + 0.01;  // bound_radius on the device
    xmin = std::min(xmin, x); xmax = std::max(xmax, x);
    zmin = std::min(zmin, z); zmax = std::max(zmax, z);
    rmax = std::max(rmax, r);
    ytop = std::max(ytop, y + r);
  }
  const double area = std::max((xmax - xmin) * (zmax - zmin), 1.0);
  double size = std::max(2.0 * rmax, std::sqrt(area / n));
  int64_t nbx = 1, nbz = 1;
  for (int it = 0; it < 200; ++it, size *= 1.25) {
    nbx = (int64_t)std::floor((xmax - xmin) / size) + 1;
    nbz = (int64_t)std::floor((zmax - zmin) / size) + 1;
    if (nbx * nbz <= s->bucket_cap) break;
  }
  if (nbx * nbz > s->bucket_cap) return set_error(QMCRT_ERR_INTERNAL, "candidate bucket grid does not fit");
  B.x0 = xmin;
  B.z0 = zmin;
  B.inv = 1.0 / size;
  B.nbx = (int)nbx;
  B.nbz = (int)nbz;
  B.ytop = ytop + 0.01;
  B.rmax = rmax + 0.01;
  const int64_t nb = nbx * nbz;
  auto bucket_of = [&](int h) {
    const double bx = std::floor((f->pos[3 * h] - B.x0) * B.inv), bz = std::floor((f->pos[3 * h + 2] - B.z0) * B.inv);
    const int ix = (int)std::min(std::max(bx, 0.0), (double)(nbx - 1));
    const int iz = (int)std::min(std::max(bz, 0.0), (double)(nbz - 1));
    return (int64_t)iz * nbx + ix;
  };
  s->h_bucket_start.assign(nb + 1, 0);
  for (int h = 0; h < n; ++h) s->h_bucket_start[bucket_of(h) + 1]++;
  for (int64_t b = 0; b < nb; ++b) s->h_bucket_start[b + 1] += s->h_bucket_start[b];
  std::vector<int32_t> fill(s->h_bucket_start.begin(), s->h_bucket_start.end() - 1);
  s->h_bucket_ids.assign(n, 0);
  for (int h = 0; h < n; ++h) s->h_bucket_ids[fill[bucket_of(h)]++] = h;
  // pageable sources: each copy returns once its source is staged
  QM_CUDA(cudaMemcpyAsync(s->d_buckets, &s->h_buckets, sizeof(CandBuckets), cudaMemcpyHostToDevice, st));
  QM_CUDA(cudaMemcpyAsync(s->d_bucket_start, s->h_bucket_start.data(), (nb + 1) * sizeof(int32_t),
                          cudaMemcpyHostToDevice, st));
  QM_CUDA(cudaMemcpyAsync(s->d_bucket_ids, s->h_bucket_ids.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  return QMCRT_OK;
}

__global__ void fill_value_kernel(float* p, int n, float v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

qmcrt_status upload_field(qmcrt_scene* s, const qmcrt_field* f, cudaStream_t st) {
  size_t n = (size_t)f->n;
  QM_CUDA(cudaMemcpyAsync(s->d_pos, f->pos, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st));
  QM_CUDA(cudaMemcpyAsync(s->d_size, f->size, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st));
  if (f->aim) QM_CUDA(cudaMemcpyAsync(s->d_aim, f->aim, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st));
  if (f->normal) QM_CUDA(cudaMemcpyAsync(s->d_normal_in, f->normal, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st));
  if (f->tilt) QM_CUDA(cudaMemcpyAsync(s->d_tilt, f->tilt, 2 * n * sizeof(float), cudaMemcpyHostToDevice, st));
  if (f->slope_sigma) {
    QM_CUDA(cudaMemcpyAsync(s->d_sigma, f->slope_sigma, n * sizeof(float), cudaMemcpyHostToDevice, st));
  } else {  // one sigma for the field: written on the device (no host staging, no wait)
    fill_value_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s->d_sigma, (int)n, f->sigma);
    QM_CUDA(cudaGetLastError());
  }
  // sample points depend only on the mirror sizes (and the trace parameters)
  bool sizes_changed = s->h_size.size() != 3 * n || std::memcmp(s->h_size.data(), f->size, 3 * n * sizeof(float)) != 0;
  bool moved = sizes_changed || s->h_pos.size() != 3 * n ||
               std::memcmp(s->h_pos.data(), f->pos, 3 * n * sizeof(float)) != 0;
  s->h_pos.assign(f->pos, f->pos + 3 * n);
  s->h_size.assign(f->size, f->size + 3 * n);
  s->ytop = -3.0e38f;
  for (size_t h = 0; h < n; ++h) {
    const float* z = f->size + 3 * h;
    s->ytop = std::max(s->ytop, f->pos[3 * h + 1] + 0.5f * std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]));
  }
  if (moved) {
    qmcrt_status e = build_buckets(s, f, st);
    if (e) return e;
  }
  s->field_version++;
  if (sizes_changed) s->points_key = PointsKey{};
  return QMCRT_OK;
}

qmcrt_status ensure_sun(qmcrt_scene* s, const qmcrt_sun* sun, uint32_t quirks, cudaStream_t st, bool need_grid) {
  SunKey k;
  std::memcpy(k.dir, sun->dir, sizeof(k.dir));
  k.quirks = quirks & (QMCRT_QUIRK_AABB_RADIUS | QMCRT_QUIRK_ZENITH_FRAME);
  k.field_version = s->field_version;
  if (k == s->sun_key) return need_grid ? ensure_grid(s, st) : QMCRT_OK;
  double sd[3] = {sun->dir[0], sun->dir[1], sun->dir[2]};
  double l = std::sqrt(sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2]);
  if (!(l > 0) || !std::isfinite(l)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "sun direction is zero or not finite");
  for (int i = 0; i < 3; ++i) sd[i] /= l;
  const bool timed = s->timing_stages & QMCRT_TIMING_SETUP;
  if (timed) QM_CUDA(cudaEventRecord(s->ev[0], st));
  qmcrt_status e = launch_sun_geom(s, scene_geom(s), sd, k.quirks, st, true, need_grid);
  if (e) return e;
  s->grid_forced = need_grid;
  if (timed) {
    QM_CUDA(cudaEventRecord(s->ev[1], st));
    s->timed |= QMCRT_TIMING_SETUP;
  }
  s->sun_key = k;
  std::memcpy(s->sun_unit, sd, sizeof(sd));
  s->geom_version++;
  return QMCRT_OK;
}

qmcrt_status launch_point_masks(const qmcrt_scene* s, const SunGeom& g, const double sun[3], const float2* xz,
                                const int32_t* helio, const float* weight, int64_t points, uint4* mask,
                                double4* origin, cudaStream_t st, bool pdl) {
  if (points <= 0) return QMCRT_OK;
  MaskArgs m{};
  m.points = points;
  m.point_xz = xz;
  m.point_helio = helio;
  m.frame = g.frame;
  m.cand = g.cand;
  m.cand_n = g.cand_n;
  m.sigma = s->d_sigma;
  m.weight = weight;
  for (int i = 0; i < 3; ++i) m.sun[i] = sun[i];
  m.shadow_tan = std::tan(kSunAlphaMax + 1e-6);
  m.sun_alpha = kSunAlphaMax;
  m.zmax = kSlopeZMax;
  m.mask = mask;
  m.origin = origin;
  QM_CUDA(launch_pdl(pdl, point_mask_kernel, dim3((unsigned)((points + 255) / 256)), dim3(256), 0, st, m));
  return QMCRT_OK;
}

qmcrt_status ensure_masks(qmcrt_scene* s, cudaStream_t st) {
  if (s->mask_geom == s->geom_version && s->mask_points == s->points_version) return QMCRT_OK;
  if (s->mask_cap < s->points) {
    dev_free(s->d_point_mask);
    dev_free(s->d_point_origin);
    s->mask_cap = 0;
    qmcrt_status e = dev_alloc(&s->d_point_mask, (size_t)s->points);
    if (!e) e = dev_alloc(&s->d_point_origin, (size_t)s->points);
    if (e) return e;
    s->mask_cap = s->points;
  }
  qmcrt_status e = launch_point_masks(s, scene_geom(s), s->sun_unit, s->d_point_xz, s->d_point_helio,
                                      s->d_helio_weight, s->points, s->d_point_mask, s->d_point_origin, st, true);
  if (e) return e;
  s->mask_geom = s->geom_version;
  s->mask_points = s->points_version;
  return QMCRT_OK;
}

SunGeom scene_geom(qmcrt_scene* s) {
  SunGeom g;
  g.normal = s->d_normal;
  g.frame = s->d_frame;
  g.rect = s->d_rect;
  g.cellbox = s->d_cellbox;
  g.cell_count = s->d_cell_count;
  g.cell_start = s->d_cell_start;
  g.entries = s->d_entries;
  g.cell_rect = s->d_cell_rect;
  g.cell_info = s->d_cell_info;
  g.coarse_yr = s->d_coarse_yr;
  g.scan_part = s->d_scan_part;
  g.cand = s->d_cand;
  g.cand_n = s->d_cand_n;
  g.field_yr = s->d_field_yr;
  g.power = reinterpret_cast<double*>(s->d_stats + 8);
  g.grid_ctl = s->d_grid_ctl;
  return g;
}

qmcrt_status alloc_sun_geom(const qmcrt_scene* s, SunGeom* g) {
  size_t n = (size_t)s->n;
  qmcrt_status e;
#define GALLOC(p, c)                    \
  if ((e = dev_alloc(&(p), (c)))) {     \
    free_sun_geom(g);                   \
    return e;                           \
  }
  GALLOC(g->normal, 3 * n);
  GALLOC(g->frame, kFrameStride * n);
  GALLOC(g->rect, 3 * n);
  GALLOC(g->cellbox, 2 * n);
  GALLOC(g->cell_count, (size_t)s->cells);
  GALLOC(g->cell_start, (size_t)s->cells + 1);
  GALLOC(g->entries, (size_t)s->entry_cap);
  GALLOC(g->cell_rect, 3 * (size_t)s->entry_cap);
  GALLOC(g->cell_info, (size_t)s->cells);
  if (s->coarse_cells) GALLOC(g->coarse_yr, (size_t)s->coarse_cells);
  if (s->cells > kScanOneCtaMax) GALLOC(g->scan_part, (size_t)((s->cells + kScanTile - 1) / kScanTile));
  GALLOC(g->cand, 2 * 3 * kCandCap * n);
  GALLOC(g->cand_n, 2 * n);
  GALLOC(g->field_yr, 2);
  GALLOC(g->power, 1);
  GALLOC(g->grid_ctl, 4);
#undef GALLOC
  return QMCRT_OK;
}

void free_sun_geom(SunGeom* g) {
  dev_free(g->normal); dev_free(g->frame); dev_free(g->rect); dev_free(g->cellbox); dev_free(g->cell_count);
  dev_free(g->cell_start); dev_free(g->entries); dev_free(g->cell_rect); dev_free(g->cell_info); dev_free(g->field_yr);
  dev_free(g->coarse_yr); dev_free(g->cand); dev_free(g->cand_n); dev_free(g->power); dev_free(g->scan_part); dev_free(g->grid_ctl);
}

// Occluder candidates of every heliostat of scene s for the (normalised) sun,
// from the aimed frames and rectangle records, into cand / cand_n.
static qmcrt_status launch_cand(const qmcrt_scene* s, const double* frame, const float4* rect, const double sun[3],
                                bool exhaustive, float4* cand, int* cand_n, cudaStream_t st, bool pdl = false,
                                int* grid_ctl = nullptr) {
  CandArgs ca{};
  ca.n = s->n;
  ca.pos = s->d_pos;
  ca.size = s->d_size;
  ca.sigma = s->d_sigma;
  ca.frame = frame;
  for (int i = 0; i < 3; ++i) ca.sun[i] = sun[i];
  ca.sun_alpha = kSunAlphaMax;
  ca.zmax = kSlopeZMax;
  {
    const double as = kSunAlphaMax + 1e-6, y = std::min(std::max(-sun[1], -1.0), 1.0);
    ca.shadow_tan = std::tan(as);
    ca.shadow_rise = y * std::cos(as) - std::sqrt(std::max(1.0 - y * y, 0.0)) * std::sin(as);
  }
  ca.rect = rect;
  ca.cand = cand;
  ca.cand_n = cand_n;
  ca.buckets = s->d_buckets;
  ca.bucket_start = s->d_bucket_start;
  ca.bucket_ids = s->d_bucket_ids;
  ca.grid_ctl = grid_ctl;
  if (exhaustive)
    QM_CUDA(launch_pdl(pdl, cand_kernel<true>, dim3((2 * s->n + 3) / 4), dim3(128), 0, st, ca));
  else
    QM_CUDA(launch_pdl(pdl, cand_kernel<false>, dim3((2 * s->n + 3) / 4), dim3(128), 0, st, ca));
  return QMCRT_OK;
}

// Aim every heliostat for the sun (normalised) and rebuild the grid into g:
// stream-ordered kernels only, so the sequence can be captured in a graph.
// The grid build passes of geometry g (scan, fill, cell records, coarse
// ranges); they build the grid only if its control words say it is needed and
// not built yet.
static qmcrt_status launch_grid(const qmcrt_scene* s, const SunGeom& g, cudaStream_t st, bool pdl) {
  if (s->cells <= kScanOneCtaMax) {
    QM_CUDA(launch_pdl(pdl, scan_kernel, dim3(1), dim3(1024), 0, st, g.cell_count, g.cell_start, s->cells,
                       s->entry_cap, s->d_flag, g.field_yr, g.grid_ctl));
  } else {
    const int64_t tiles = (s->cells + kScanTile - 1) / kScanTile;
    QM_CUDA(launch_pdl(pdl, scan_tiles_kernel, dim3((unsigned)tiles), dim3(1024), 0, st, g.cell_count, g.cell_start,
                       s->cells, g.scan_part, (const int*)g.grid_ctl));
    QM_CUDA(launch_pdl(pdl, scan_parts_kernel, dim3(1), dim3(1024), 0, st, g.scan_part, tiles, g.cell_start,
                       s->cells, s->entry_cap, s->d_flag, g.field_yr, g.grid_ctl));
    QM_CUDA(launch_pdl(pdl, scan_add_kernel, dim3((unsigned)((s->cells + 255) / 256)), dim3(256), 0, st,
                       g.cell_count, g.cell_start, s->cells, g.scan_part, s->entry_cap, (const int*)g.grid_ctl));
  }
  QM_CUDA(launch_pdl(pdl, fill_kernel, dim3((s->n + 127) / 128), dim3(128), 0, st, s->n, g.cellbox, g.cell_start,
                     g.cell_count, g.entries, s->gdims[1], s->gdims[2], s->entry_cap, (const int*)g.grid_ctl));
  // a warp per cell on small grids (few cells, many ids each), a thread per
  // cell on large ones (mostly empty cells): 13.2 -> 4.4 us on the small
  // field, and 6.8 us instead of 77 us on the large field's 176 000 cells
  if (s->cells <= kCellWarpMax)
    QM_CUDA(launch_pdl(pdl, cell_finish_warp_kernel, dim3((unsigned)((s->cells + 7) / 8)), dim3(256), 0, st,
                       s->cells, g.cell_start, g.entries, g.rect, g.cell_rect, g.cell_info, g.field_yr,
                       (const int*)g.grid_ctl));
  else
    QM_CUDA(launch_pdl(pdl, cell_finish_kernel, dim3((unsigned)((s->cells + 255) / 256)), dim3(256), 0, st,
                       s->cells, g.cell_start, g.entries, g.rect, g.cell_rect, g.cell_info, g.field_yr,
                       (const int*)g.grid_ctl));
  QM_CUDA(cudaGetLastError());
  if (s->coarse_cells) {
    int3 cd = make_int3(s->gdims[0] / s->fine_div, s->gdims[1] / s->fine_div, s->gdims[2] / s->fine_div);
    QM_CUDA(launch_pdl(pdl, coarse_finish_kernel, dim3((unsigned)((s->coarse_cells + 127) / 128)), dim3(128), 0, st,
                       s->coarse_cells, s->fine_div, cd, s->gdims[1], s->gdims[2], (const int4*)g.cell_info,
                       g.coarse_yr, (const int*)g.grid_ctl));
  }
  return QMCRT_OK;
}

qmcrt_status launch_sun_geom(const qmcrt_scene* s, const SunGeom& g, const double sun[3], uint32_t quirks,
                             cudaStream_t st, bool pdl, bool force_grid) {
  AimArgs a{};
  a.n = s->n;
  a.pos = s->d_pos;
  a.size = s->d_size;
  a.aim = s->has_aim ? s->d_aim : nullptr;
  a.normal_in = s->has_normal ? s->d_normal_in : nullptr;
  a.tilt = s->has_tilt ? s->d_tilt : nullptr;
  std::memcpy(a.focus, s->rg.focus, sizeof(a.focus));
  for (int i = 0; i < 3; ++i) a.sun[i] = sun[i];
  a.quirks = quirks & (QMCRT_QUIRK_AABB_RADIUS | QMCRT_QUIRK_ZENITH_FRAME);
  a.normal = g.normal;
  a.frame = g.frame;
  a.rect = g.rect;
  a.cellbox = g.cellbox;
  a.cell_count = g.cell_count;
  std::memcpy(a.gpos, s->gpos, sizeof(a.gpos));
  std::memcpy(a.gcell, s->gcell, sizeof(a.gcell));
  std::memcpy(a.gdims, s->gdims, sizeof(a.gdims));
  a.power = g.power;
  QM_CUDA(launch_pdl(pdl, zero_geom_kernel, dim3((unsigned)std::min<int64_t>((s->cells + 255) / 256, 592)), dim3(256), 0,
                     st, g.cell_count, s->cells, g.power, g.grid_ctl, force_grid ? 1 : 0));
  QM_CUDA(launch_pdl(pdl, aim_kernel, dim3((s->n + 127) / 128), dim3(128), 0, st, a));
  qmcrt_status e = launch_cand(s, g.frame, g.rect, sun, false, g.cand, g.cand_n, st, pdl, g.grid_ctl);
  if (e) return e;
  return launch_grid(s, g, st, pdl);
}

// Build the grid of the scene's current geometry if the trace that built the
// geometry left it unbuilt (no candidate list overflowed).
qmcrt_status ensure_grid(qmcrt_scene* s, cudaStream_t st) {
  if (s->grid_forced || !s->geom_version) return QMCRT_OK;
  const SunGeom g = scene_geom(s);
  QM_CUDA(launch_pdl(true, grid_demand_kernel, dim3(1), dim3(32), 0, st, g.grid_ctl));
  qmcrt_status e = launch_grid(s, g, st, true);
  if (e) return e;
  s->grid_forced = true;
  return QMCRT_OK;
}

qmcrt_status ensure_points(qmcrt_scene* s, const qmcrt_trace_params* p, cudaStream_t st) {
  PointsKey k;
  k.seed = p->seed;
  k.rays = p->rays;
  k.rpp = p->rays_per_point;
  k.mode = p->point_mode;
  k.spacing = p->point_spacing;
  if (k == s->points_key) return QMCRT_OK;
  if (p->rays_per_point <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "rays_per_point must be positive");
  int64_t total = 0;
  std::vector<int64_t> base;
  if (p->point_mode == QMCRT_POINTS_GRID) {
    if (!(p->point_spacing > 0)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "grid points need a pixel length");
    base.resize(s->n);
    for (int h = 0; h < s->n; ++h) {
      base[h] = total;
      int rows = (int)(s->h_size[3 * h + 2] / p->point_spacing), cols = (int)(s->h_size[3 * h] / p->point_spacing);
      total += (int64_t)rows * cols;
    }
  } else if (p->point_mode == QMCRT_POINTS_POISSON) {
    if (p->rays == 0 || p->rays % (uint64_t)p->rays_per_point != 0)
      return set_error(QMCRT_ERR_INVALID_ARGUMENT, "rays must be a positive multiple of rays_per_point");
    total = (int64_t)(p->rays / (uint64_t)p->rays_per_point);
    if (total < s->n) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "fewer points than heliostats");
    if (!(p->point_spacing > 0)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "Poisson points need a minimum spacing");
  } else {
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "unknown point mode");
  }
  // points are 32-bit ids; rays reach 2^32 and beyond only with a power-of-two
  // count per point, which splits a ray id into its point with a shift
  const bool pow2 = (p->rays_per_point & (p->rays_per_point - 1)) == 0;
  if (total <= 0 || total > 0x7FFFFFFFll || (!pow2 && (uint64_t)total * (uint64_t)p->rays_per_point > 0xFFFFFFFFull))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT,
                     "points must be in [1, 2^31); rays below 2^32 unless rays_per_point is a power of two");
  if (total > s->points_cap) {
    dev_free(s->d_point_xz);
    dev_free(s->d_point_helio);
    qmcrt_status e = dev_alloc(&s->d_point_xz, total);
    if (e) return e;
    e = dev_alloc(&s->d_point_helio, total);
    if (e) return e;
    s->points_cap = total;
  }
  int64_t q = total / s->n, rem = total % s->n;
  QM_CUDA(cudaMemsetAsync(s->d_flag, 0, sizeof(int32_t), st));
  if (p->point_mode == QMCRT_POINTS_GRID) {
    int64_t* d_base = nullptr;
    qmcrt_status e = dev_alloc(&d_base, s->n);
    if (e) return e;
    QM_CUDA(cudaMemcpyAsync(d_base, base.data(), s->n * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    grid_points_kernel<<<s->n, 256, 0, st>>>(s->n, s->d_size, p->point_spacing, d_base, s->d_point_xz, s->d_point_helio);
    cudaError_t le = cudaGetLastError();
    cudaStreamSynchronize(st);
    cudaFree(d_base);
    if (le != cudaSuccess) return cuda_error(le, "grid_points_kernel");
  } else {
    PoissonArgs a{};
    a.n = s->n;
    a.size = s->d_size;
    a.q = q;
    a.rem = rem;
    a.Rq = (int64_t)((double)p->point_spacing * 65536.0);
    if (a.Rq < 1) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "Poisson spacing below 2^-16 m");
    a.R2 = a.Rq * a.Rq;
    int64_t cq = (int64_t)std::sqrt((double)(a.R2 / 2));
    while (cq * cq > a.R2 / 2) --cq;
    while ((cq + 1) * (cq + 1) <= a.R2 / 2) ++cq;
    a.cq = std::max<int64_t>(cq, 1);
    a.nb = (a.Rq + a.cq - 1) / a.cq;
    a.key = make_uint2((uint32_t)p->seed ^ kPoissonKey0, (uint32_t)(p->seed >> 32) ^ kPoissonKey1);
    a.max_batches = (64 * (q + 1) + 1023) / 32 + 32;
    int2* d_q = nullptr;
    qmcrt_status e = dev_alloc(&d_q, total);
    if (e) return e;
    a.point_q = d_q;
    a.point_xz = s->d_point_xz;
    a.point_helio = s->d_point_helio;
    a.flag = s->d_flag;
    int64_t smem = 0;
    for (int h = 0; h < s->n; ++h) {
      int64_t W = (int64_t)((double)s->h_size[3 * h] * 65536.0), H = (int64_t)((double)s->h_size[3 * h + 2] * 65536.0);
      int64_t g = ((W + a.cq - 1) / a.cq) * ((H + a.cq - 1) / a.cq);
      smem = std::max(smem, g * (int64_t)sizeof(int32_t));
    }
    if (smem > 200 * 1024) {
      cudaFree(d_q);
      return set_error(QMCRT_ERR_INVALID_ARGUMENT, "Poisson spacing too small for the heliostat size (background grid over 200 KB)");
    }
    if (smem > 48 * 1024) QM_CUDA(cudaFuncSetAttribute(poisson_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    poisson_kernel<<<s->n, 32, (size_t)smem, st>>>(a);
    cudaError_t le = cudaGetLastError();
    int32_t flag = 0;
    cudaError_t ce = cudaMemcpyAsync(&flag, s->d_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    cudaError_t se = cudaStreamSynchronize(st);
    cudaFree(d_q);
    if (le != cudaSuccess) return cuda_error(le, "poisson_kernel");
    if (ce != cudaSuccess) return cuda_error(ce, "poisson flag copy");
    if (se != cudaSuccess) return cuda_error(se, "poisson sync");
    if (flag == 2)
      return set_error(QMCRT_ERR_SAMPLING, "Poisson-disk spacing too large for the requested points per heliostat");
  }
  weight_kernel<<<(s->n + 127) / 128, 128, 0, st>>>(s->n, s->d_size, q, rem, p->point_mode, p->point_spacing,
                                                     s->d_helio_weight);
  QM_CUDA(cudaGetLastError());
  s->points = total;
  s->points_key = k;
  s->points_version++;
  return QMCRT_OK;
}

}  // namespace qm

extern "C" {

qmcrt_status qmcrt_scene_create(const qmcrt_field* field, const qmcrt_receiver* recv, const qmcrt_grid_params* grid,
                                qmcrt_scene** out) {
  if (!out) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  qmcrt_status e = check_field(field);
  if (e) return e;
  if (!recv || !grid) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "receiver and grid are required");
  for (int i = 0; i < 3; ++i)
    if (!(grid->cell[i] > 0)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "grid cell sizes must be positive");
  qmcrt_scene* s = new qmcrt_scene();
  s->n = field->n;
  s->recv = *recv;
  s->gp = *grid;
  e = receiver_setup(*recv, &s->rg);
  if (e) { delete s; return e; }
  s->has_aim = field->aim != nullptr;
  s->has_normal = field->normal != nullptr;
  s->has_tilt = field->tilt != nullptr;
  // grid bounds: union of pos +- |size|/2 (any orientation) and of the
  // reference's registration cube, plus margin (RectGrid::Cinit grid.cpp:3-8)
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  std::vector<double> rad(s->n);
  for (int h = 0; h < s->n; ++h) {
    double sx = field->size[3 * h], sy = field->size[3 * h + 1], sz = field->size[3 * h + 2];
    double r = 0.5 * std::sqrt(sx * sx + sy * sy + sz * sz);
    double rq = std::sqrt(std::sqrt(sx * sx + sy * sy + sz * sz)) / 2.0;
    rad[h] = std::max(r, rq) + 1e-3;
    for (int i = 0; i < 3; ++i) {
      lo[i] = std::min(lo[i], field->pos[3 * h + i] - std::max(r, rq));
      hi[i] = std::max(hi[i], field->pos[3 * h + i] + std::max(r, rq));
    }
  }
  // two-level grid: the coarse dims cover the bounds, the fine grid (the one
  // that holds the registrations) has fine_div cells per coarse cell per axis
  const int div = grid->fine_div > 1 ? grid->fine_div : 1;
  if (div != 1 && div != 2 && div != 4 && div != 8) {
    delete s;
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "fine_div must be 0, 1, 2, 4 or 8");
  }
  for (int i = 0; i < 3; ++i) {
    int cd;
    if (grid->explicit_bounds) {
      s->gpos[i] = grid->origin[i];
      cd = std::max(1, (int)std::ceil((double)grid->extent[i] / grid->cell[i]));
    } else {
      float g = (float)(lo[i] - grid->margin);
      s->gpos[i] = g;
      cd = std::max(1, (int)std::ceil(((hi[i] + grid->margin) - (double)g) / grid->cell[i]));
    }
    s->gcell[i] = grid->cell[i] / (float)div;  // exact: div is a power of two
    s->gdims[i] = cd * div;
  }
  s->cells = (int64_t)s->gdims[0] * s->gdims[1] * s->gdims[2];
  s->coarse_cells = div > 1 ? s->cells / ((int64_t)div * div * div) : 0;
  // explicit bounds must contain every heliostat centre: a walk ends at the
  // grid's edge, so an occluder outside it would never be tested (the
  // reference indexes its cell vectors out of range there, grid.cpp:36-44)
  if (grid->explicit_bounds)
    for (int h = 0; h < s->n; ++h)
      for (int i = 0; i < 3; ++i) {
        double p = field->pos[3 * h + i], g0 = s->gpos[i], g1 = g0 + (double)s->gdims[i] * s->gcell[i];
        if (!(p >= g0 && p < g1)) {
          delete s;
          return set_error(QMCRT_ERR_INVALID_ARGUMENT,
                           "heliostat " + std::to_string(h) + " lies outside the explicit grid bounds");
        }
      }
  if (s->cells > (int64_t)64 * 1024 * 1024) {
    delete s;
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "grid has more than 2^26 cells; use larger cells");
  }
  int64_t cap = 0;
  for (int h = 0; h < s->n; ++h) {
    double l3[3], h3[3];
    for (int i = 0; i < 3; ++i) {
      l3[i] = field->pos[3 * h + i] - rad[h];
      h3[i] = field->pos[3 * h + i] + rad[h];
    }
    cap += cells_in_box(s->gpos, s->gcell, s->gdims, l3, h3);
  }
  s->entry_cap = cap;
  if (cap > 0x7FFFFFFF) { delete s; return set_error(QMCRT_ERR_INVALID_ARGUMENT, "grid registrations exceed 2^31"); }
  s->fine_div = div;
  size_t n = (size_t)s->n;
  size_t res = (size_t)recv->res_x * recv->res_y;
#define ALLOC(p, c)              \
  do {                           \
    e = dev_alloc(&(p), (c));    \
    if (e) goto fail;            \
  } while (0)
  {
    int dev = 0;
    cudaGetDevice(&dev);
    s->device = dev;
  }
  ALLOC(s->d_pos, 3 * n);
  ALLOC(s->d_size, 3 * n);
  if (s->has_aim) ALLOC(s->d_aim, 3 * n);
  if (s->has_normal) ALLOC(s->d_normal_in, 3 * n);
  if (s->has_tilt) ALLOC(s->d_tilt, 2 * n);
  ALLOC(s->d_sigma, n);
  ALLOC(s->d_normal, 3 * n);
  ALLOC(s->d_frame, kFrameStride * n);
  ALLOC(s->d_rect, 3 * n);
  ALLOC(s->d_cellbox, 2 * n);
  ALLOC(s->d_cell_count, (size_t)s->cells);
  ALLOC(s->d_cell_start, (size_t)s->cells + 1);
  ALLOC(s->d_entries, (size_t)cap);
  ALLOC(s->d_cell_rect, 3 * (size_t)cap);
  ALLOC(s->d_cell_info, (size_t)s->cells);
  if (s->coarse_cells) ALLOC(s->d_coarse_yr, (size_t)s->coarse_cells);
  if (s->cells > kScanOneCtaMax) ALLOC(s->d_scan_part, (size_t)((s->cells + kScanTile - 1) / kScanTile));
  ALLOC(s->d_cand, 2 * 3 * kCandCap * n);
  ALLOC(s->d_cand_n, 2 * n);
  s->bucket_cap = 4 * (int64_t)n + 64;
  ALLOC(s->d_buckets, 1);
  ALLOC(s->d_bucket_start, (size_t)s->bucket_cap + 1);
  ALLOC(s->d_bucket_ids, n);
  ALLOC(s->d_field_yr, 2);
  ALLOC(s->d_grid_ctl, 4);
  if (recv->type == QMCRT_RECEIVER_CYLINDER) {
    ALLOC(s->d_cyl_edge, (size_t)recv->res_x);
    std::vector<double2> edge(recv->res_x);
    for (int k = 0; k < recv->res_x; ++k) {
      const double a = 2.0 * 3.141592653589793 * k / recv->res_x;
      edge[k] = make_double2(std::cos(a), std::sin(a));
    }
    cudaError_t ce = cudaMemcpy(s->d_cyl_edge, edge.data(), edge.size() * sizeof(double2), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) { e = cuda_error(ce, "cylinder column edges"); goto fail; }
  }
  ALLOC(s->d_helio_weight, n);
  ALLOC(s->d_flag, 1);
  ALLOC(s->d_counts, res);
  ALLOC(s->d_energy, res);
  ALLOC(s->d_map_flux, res);
  ALLOC(s->d_map_smooth, res);
  ALLOC(s->d_stats, 16);
  ALLOC(s->d_buie, 4 * kBuieRecords);  // one record per bucket of the Buie table
#undef ALLOC
  for (int i = 0; i < 5; ++i) {
    cudaError_t ce = cudaEventCreate(&s->ev[i]);
    if (ce != cudaSuccess) { e = cuda_error(ce, "cudaEventCreate"); goto fail; }
  }
  e = upload_field(s, field, 0);
  if (e) goto fail;
  {
    cudaError_t ce = cudaMemset(s->d_flag, 0, sizeof(int32_t));
    if (ce == cudaSuccess) ce = cudaMemset(s->d_stats, 0, 16 * sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) { e = cuda_error(ce, "scene init"); goto fail; }
  }
  *out = s;
  return QMCRT_OK;
fail:
  qmcrt_scene_destroy(s);
  return e;
}

qmcrt_status qmcrt_scene_destroy(qmcrt_scene* s) {
  if (!s) return QMCRT_OK;
  dev_free(s->d_pos); dev_free(s->d_size); dev_free(s->d_aim); dev_free(s->d_normal_in);
  dev_free(s->d_sigma); dev_free(s->d_tilt); dev_free(s->d_normal); dev_free(s->d_frame);
  dev_free(s->d_rect); dev_free(s->d_cellbox); dev_free(s->d_cell_count); dev_free(s->d_cell_start);
  dev_free(s->d_entries); dev_free(s->d_cell_rect); dev_free(s->d_cell_info); dev_free(s->d_coarse_yr); dev_free(s->d_scan_part); dev_free(s->d_cand); dev_free(s->d_cand_n); dev_free(s->d_field_yr); dev_free(s->d_grid_ctl);
  dev_free(s->d_buckets); dev_free(s->d_bucket_start); dev_free(s->d_bucket_ids); dev_free(s->d_cyl_edge);
  dev_free(s->d_point_mask); dev_free(s->d_point_origin); dev_free(s->d_point_xz); dev_free(s->d_point_helio);
  dev_free(s->d_helio_weight); dev_free(s->d_flag); dev_free(s->d_counts); dev_free(s->d_energy);
  dev_free(s->d_map_flux); dev_free(s->d_map_smooth); dev_free(s->d_stats); dev_free(s->d_buie);
  for (int i = 0; i < 5; ++i)
    if (s->ev[i]) cudaEventDestroy(s->ev[i]);
  delete s;
  return QMCRT_OK;
}

qmcrt_status qmcrt_scene_timing(qmcrt_scene* s, qmcrt_timing* t) {
  if (!s || !t) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!s->traced) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "no trace recorded on this scene yet");
  if (!(s->timed & (QMCRT_TIMING_TRACE | QMCRT_TIMING_FINALIZE)))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT,
                     "the last trace timed no stage (enable the trace or finalize stage with qmcrt_scene_set_timing)");
  QM_CUDA(cudaEventSynchronize(s->ev[(s->timed & QMCRT_TIMING_FINALIZE) ? 4 : 3]));
  t->setup_ms = t->trace_kernel_ms = t->finalize_ms = -1.f;
  if (s->timed & QMCRT_TIMING_SETUP) QM_CUDA(cudaEventElapsedTime(&t->setup_ms, s->ev[0], s->ev[1]));
  if (s->timed & QMCRT_TIMING_TRACE) QM_CUDA(cudaEventElapsedTime(&t->trace_kernel_ms, s->ev[2], s->ev[3]));
  if (s->timed & QMCRT_TIMING_FINALIZE) QM_CUDA(cudaEventElapsedTime(&t->finalize_ms, s->ev[3], s->ev[4]));
  return QMCRT_OK;
}

qmcrt_status qmcrt_scene_set_timing(qmcrt_scene* s, uint32_t stages) {
  if (!s) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "scene is NULL");
  if (stages & ~(uint32_t)QMCRT_TIMING_ALL) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "unknown timing stage bits");
  s->timing_stages = stages;
  return QMCRT_OK;
}

qmcrt_status qmcrt_scene_set_field(qmcrt_scene* s, const qmcrt_field* f, void* stream) {
  if (!s) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "scene is NULL");
  qmcrt_status e = check_field(f);
  if (e) return e;
  if (f->n != s->n) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "field size differs from the scene's");
  if ((f->aim != nullptr) != s->has_aim || (f->normal != nullptr) != s->has_normal || (f->tilt != nullptr) != s->has_tilt)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "field must provide the same optional arrays as at creation");
  for (int h = 0; h < s->n; ++h)
    for (int i = 0; i < 3; ++i)
      if (f->pos[3 * h + i] != s->h_pos[3 * h + i] || f->size[3 * h + i] != s->h_size[3 * h + i]) {
        // positions/sizes define the grid bounds; they may move only within them
        float r = 0.5f * std::sqrt(f->size[3 * h] * f->size[3 * h] + f->size[3 * h + 1] * f->size[3 * h + 1] +
                                   f->size[3 * h + 2] * f->size[3 * h + 2]);
        if (f->pos[3 * h + i] - r < s->gpos[i] || f->pos[3 * h + i] + r > s->gpos[i] + s->gdims[i] * s->gcell[i] ||
            f->size[3 * h + i] > s->h_size[3 * h + i])
          return set_error(QMCRT_ERR_INVALID_ARGUMENT, "a heliostat moved outside the scene's grid; create a new scene");
      }
  return upload_field(s, f, (cudaStream_t)stream);
}

qmcrt_status qmcrt_scene_set_sun(qmcrt_scene* s, const qmcrt_sun* sun, uint32_t quirks, void* stream) {
  if (!s || !sun) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  return ensure_sun(s, sun, quirks, (cudaStream_t)stream);
}

qmcrt_status qmcrt_scene_grid_info(qmcrt_scene* s, qmcrt_grid_info* info) {
  if (!s || !info) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::memcpy(info->origin, s->gpos, sizeof(info->origin));
  std::memcpy(info->cell, s->gcell, sizeof(info->cell));
  std::memcpy(info->dims, s->gdims, sizeof(info->dims));
  info->cells = s->cells;
  int32_t tot = 0;
  if (!s->grid_forced && s->geom_version) {
    // the grid of a candidate trace's geometry may be unbuilt: build it on the
    // default stream once the device is idle (the trace's stream is not known)
    QM_CUDA(cudaDeviceSynchronize());
    qmcrt_status e = ensure_grid(s, 0);
    if (e) return e;
  }
  if (s->d_cell_start) QM_CUDA(cudaMemcpy(&tot, s->d_cell_start + s->cells, sizeof(int32_t), cudaMemcpyDeviceToHost));
  info->entries = tot;
  info->fine_div = s->fine_div;
  return QMCRT_OK;
}

qmcrt_status qmcrt_scene_read_grid(qmcrt_scene* s, int32_t* h_start, int32_t* h_entries, void* stream) {
  if (!s || !h_start) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  qmcrt_status e = ensure_grid(s, st);  // the grid of a candidate trace's geometry may be unbuilt
  if (e) return e;
  QM_CUDA(cudaMemcpyAsync(h_start, s->d_cell_start, (s->cells + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaStreamSynchronize(st));
  if (h_entries && h_start[s->cells] > 0)
    QM_CUDA(cudaMemcpyAsync(h_entries, s->d_entries, (size_t)h_start[s->cells] * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaStreamSynchronize(st));
  return QMCRT_OK;
}

qmcrt_status qmcrt_scene_read_geometry(qmcrt_scene* s, double* h_normals, double* h_vertices, void* stream) {
  if (!s) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "scene is NULL");
  cudaStream_t st = (cudaStream_t)stream;
  if (h_normals) QM_CUDA(cudaMemcpyAsync(h_normals, s->d_normal, 3 * (size_t)s->n * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (h_vertices) {
    std::vector<double> fr(kFrameStride * (size_t)s->n);
    QM_CUDA(cudaMemcpyAsync(fr.data(), s->d_frame, fr.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    QM_CUDA(cudaStreamSynchronize(st));
    for (int h = 0; h < s->n; ++h) {
      const double* f = fr.data() + kFrameStride * h;
      double sx = s->h_size[3 * h], sy = s->h_size[3 * h + 1], sz = s->h_size[3 * h + 2];
      const double loc[3][3] = {{-sx / 2, sy / 2, -sz / 2}, {-sx / 2, sy / 2, sz / 2}, {sx / 2, sy / 2, -sz / 2}};
      for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 3; ++i)
          h_vertices[9 * h + 3 * k + i] =
              loc[k][0] * f[i] + loc[k][1] * f[3 + i] + loc[k][2] * f[6 + i] + s->h_pos[3 * h + i];
    }
  }
  QM_CUDA(cudaStreamSynchronize(st));
  return QMCRT_OK;
}

static_assert(kCandCap == QMCRT_CAND_CAP, "candidate capacity of the C-ABI");

qmcrt_status qmcrt_scene_read_candidates(qmcrt_scene* s, int32_t exhaustive, int32_t* h_counts, int32_t* h_ids,
                                         void* stream) {
  if (!s || !h_counts) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (s->sun_key.field_version != s->field_version)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "no sun set for the current field (qmcrt_scene_set_sun)");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)s->n;
  float4* cand = s->d_cand;
  int* cand_n = s->d_cand_n;
  float4* tc = nullptr;
  int* tn = nullptr;
  if (exhaustive) {
    qmcrt_status e = dev_alloc(&tc, 2 * 3 * kCandCap * n);
    if (!e) e = dev_alloc(&tn, 2 * n);
    double sd[3] = {s->sun_key.dir[0], s->sun_key.dir[1], s->sun_key.dir[2]};
    const double l = std::sqrt(sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2]);
    for (int i = 0; i < 3; ++i) sd[i] /= l;  // as ensure_sun normalised it
    if (!e) e = launch_cand(s, s->d_frame, s->d_rect, sd, true, tc, tn, st);
    if (e) {
      dev_free(tc);
      dev_free(tn);
      return e;
    }
    cand = tc;
    cand_n = tn;
  }
  std::vector<float4> rec(h_ids ? 2 * 3 * kCandCap * n : 0);
  cudaError_t ce = cudaMemcpyAsync(h_counts, cand_n, 2 * n * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess && h_ids)
    ce = cudaMemcpyAsync(rec.data(), cand, rec.size() * sizeof(float4), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  dev_free(tc);
  dev_free(tn);
  if (ce != cudaSuccess) return cuda_error(ce, "qmcrt_scene_read_candidates");
  if (h_ids)
    for (size_t l = 0; l < 2 * n; ++l)
      for (int j = 0; j < kCandCap; ++j)
        if (j < h_counts[l]) std::memcpy(h_ids + l * kCandCap + j, &rec[(l * kCandCap + j) * 3].w, sizeof(int32_t));
        else h_ids[l * kCandCap + j] = -1;
  return QMCRT_OK;
}

qmcrt_status qmcrt_scene_sample_points(qmcrt_scene* s, const qmcrt_trace_params* p, int64_t* points_out, void* stream) {
  if (!s || !p) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  qmcrt_status e = ensure_points(s, p, (cudaStream_t)stream);
  if (e) return e;
  if (points_out) *points_out = s->points;
  return QMCRT_OK;
}

qmcrt_status qmcrt_scene_read_points(qmcrt_scene* s, float* h_point_q, int32_t* h_point_helio, void* stream) {
  if (!s) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "scene is NULL");
  if (s->points <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "no points sampled yet");
  cudaStream_t st = (cudaStream_t)stream;
  if (h_point_q) QM_CUDA(cudaMemcpyAsync(h_point_q, s->d_point_xz, (size_t)s->points * sizeof(float2), cudaMemcpyDeviceToHost, st));
  if (h_point_helio) QM_CUDA(cudaMemcpyAsync(h_point_helio, s->d_point_helio, (size_t)s->points * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaStreamSynchronize(st));
  return QMCRT_OK;
}

}  // extern "C"

// ------------------------------------------------- points without allocation
// Scratch for qmcrt_sample_points_noalloc: the lattice coordinates of accepted
// points, a copy of the mirror sizes and the sampler's error flag.  It lives in
// every context that loads this library, for the life of the process.
namespace qm {

struct NoAllocScratch {
  int2 lattice[QMCRT_NOALLOC_MAX_POINTS];
  float size[3 * QMCRT_NOALLOC_MAX_HELIOSTATS];
  int32_t flag;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of the scratch on the current device.  Host code cannot use
// the symbol itself as a device address, so every call asks the runtime for
// it (cudaGetSymbolAddress, cheap next to the call's synchronisation): no
// process-wide cache that could go stale when a context is torn down and
// re-created (cudaDeviceReset) or race between host threads.
static qmcrt_status noalloc_scratch(NoAllocScratch** out) {
  void* p = nullptr;
  QM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  *out = (NoAllocScratch*)p;
  return QMCRT_OK;
}

}  // namespace qm

extern "C" qmcrt_status qmcrt_sample_points_noalloc(const float* h_size, int32_t n, int64_t total_points, float spacing,
                                                    uint64_t seed, float* d_point_xz, int32_t* d_point_helio,
                                                    void* stream) {
  if (!h_size || !d_point_xz || !d_point_helio) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (n <= 0 || n > QMCRT_NOALLOC_MAX_HELIOSTATS)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "n must be in [1, QMCRT_NOALLOC_MAX_HELIOSTATS = 16384]");
  if (total_points < n || total_points > QMCRT_NOALLOC_MAX_POINTS)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT,
                     "total_points must be in [n, QMCRT_NOALLOC_MAX_POINTS = 1048576] for the allocation-free sampler");
  if (!(spacing > 0)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "Poisson points need a minimum spacing");
  for (int h = 0; h < n; ++h)
    if (!(h_size[3 * h] > 0) || !(h_size[3 * h + 2] > 0) || h_size[3 * h] > 1000.f || h_size[3 * h + 2] > 1000.f)
      return set_error(QMCRT_ERR_INVALID_ARGUMENT, "heliostat size must be positive and below 1000 m");
  NoAllocScratch* scr = nullptr;
  qmcrt_status e = noalloc_scratch(&scr);
  if (e) return e;
  cudaStream_t st = (cudaStream_t)stream;
  PoissonArgs a{};
  // addresses inside the device array, computed without dereferencing it on the host
  char* base = reinterpret_cast<char*>(scr);
  int2* lattice = reinterpret_cast<int2*>(base + offsetof(NoAllocScratch, lattice));
  float* dsize = reinterpret_cast<float*>(base + offsetof(NoAllocScratch, size));
  int32_t* dflag = reinterpret_cast<int32_t*>(base + offsetof(NoAllocScratch, flag));
  a.n = n;
  a.size = dsize;
  a.q = total_points / n;
  a.rem = total_points % n;
  a.Rq = (int64_t)((double)spacing * 65536.0);
  if (a.Rq < 1) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "Poisson spacing below 2^-16 m");
  a.R2 = a.Rq * a.Rq;
  int64_t cq = (int64_t)std::sqrt((double)(a.R2 / 2));
  while (cq * cq > a.R2 / 2) --cq;
  while ((cq + 1) * (cq + 1) <= a.R2 / 2) ++cq;
  a.cq = std::max<int64_t>(cq, 1);
  a.nb = (a.Rq + a.cq - 1) / a.cq;
  a.key = make_uint2((uint32_t)seed ^ kPoissonKey0, (uint32_t)(seed >> 32) ^ kPoissonKey1);
  a.max_batches = (64 * (a.q + 1) + 1023) / 32 + 32;
  a.point_q = lattice;
  a.point_xz = (float2*)d_point_xz;
  a.point_helio = d_point_helio;
  a.flag = dflag;
  int64_t smem = 0;
  for (int h = 0; h < n; ++h) {
    int64_t W = (int64_t)((double)h_size[3 * h] * 65536.0), H = (int64_t)((double)h_size[3 * h + 2] * 65536.0);
    smem = std::max(smem, ((W + a.cq - 1) / a.cq) * ((H + a.cq - 1) / a.cq) * (int64_t)sizeof(int32_t));
  }
  if (smem > 200 * 1024)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT,
                     "Poisson spacing too small for the heliostat size (background grid over 200 KB)");
  if (smem > 48 * 1024) QM_CUDA(cudaFuncSetAttribute(poisson_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // the flag must start at zero; the lattice is written before it is read
  QM_CUDA(cudaMemsetAsync(dflag, 0, sizeof(int32_t), st));
  QM_CUDA(cudaMemcpyAsync(dsize, h_size, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st));
  poisson_kernel<<<n, 32, (size_t)smem, st>>>(a);
  QM_CUDA(cudaGetLastError());
  int32_t flag = 0;
  QM_CUDA(cudaMemcpyAsync(&flag, dflag, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  QM_CUDA(cudaStreamSynchronize(st));
  if (flag == 2)
    return set_error(QMCRT_ERR_SAMPLING, "Poisson-disk spacing too large for the requested points per heliostat");
  return QMCRT_OK;
}
