// internal.hpp — host-side state behind the qmcrt C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/qmcrt.h"
#include "common.cuh"

namespace qm {

// Thread-local last-error message; set_error returns its status for chaining.
qmcrt_status set_error(qmcrt_status s, const std::string& msg);
qmcrt_status cuda_error(cudaError_t e, const char* what);

#define QM_CUDA(call)                                         \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::qm::cuda_error(e_, #call); \
  } while (0)

// Receiver geometry computed on the host in double (receiver.cpp:24-118).
struct ReceiverGeom {
  int type = 0;
  double v0[3], v1[3], v3[3];  // flat: parallelogram corners (v2 = v1 + v3 - v0)
  double focus[3];
  double cyl[5];  // cylinder: cx, y0, cz, radius, height
  int res_x = 0, res_y = 0;
  double pixel_area = 0;
};

// Buie sunshape table (1025 + 1025 + 1024 floats) and its scalars.
// Launch `kernel` on `st`, with programmatic stream serialization when `pdl`
// (the kernel then starts while its predecessor in the stream finishes, and
// waits for it in pdl_wait()).
template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? at : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Buie table staging: uniform buckets over the core CDF, each holding at
// most one boundary of the table's 1024 intervals (checked when the table is
// built), and one interval record per bucket plus one past the last.
constexpr int kBuieBuckets = 2048;
constexpr int kBuieRecords = kBuieBuckets + 1;

struct BuieTable {
  float csr = -1.f;
  std::vector<float> host;  // one {angle, cdf, slope, next cdf} record per bucket (kBuieRecords)
  float params[6];          // k, gamma, core, total, B, C
  float inv_bucket = 0;     // buckets per unit of CDF
  bool within_alpha = false; // every sample lies within kSunAlphaMax of the sun axis
};

// The Buie table of `csr` in the kernels' staging layout (one interval
// record per uniform bucket of the core CDF) and its scalars; false if a
// bucket would hold two interval boundaries.
bool buie_bucket_table(float csr, BuieTable* t);

// Build the table exactly as set_samplelights does (float arithmetic).
void buie_build(float csr, float* cdf_x, float* cdf_y, float* slope, float params[6]);

// Receiver geometry from the C description.
qmcrt_status receiver_setup(const qmcrt_receiver& r, ReceiverGeom* g);

// Device geometry of a field for one sun position: aimed normals and frames,
// rectangle records and the grid CSR.  A scene owns one; a batch owns one per
// (field, sun) item.
// Largest angle of a Buie sun sample from the sun axis (rad): the aureole
// ends at 9.3 mrad for every CSR; the host checks each table against it.
constexpr double kSunAlphaMax = 9.31e-3;
// Largest |z| of the slope-error deviate sqrt(-2 ln u1) cos(2 pi u2) with
// 23-bit uniforms (u1 >= 2^-24): 5.77, in units of sigma.
constexpr double kSlopeZMax = 6.0;

// Heliostat centres bucketed on a 2D grid over (x, z), rebuilt on the host
// whenever the field is uploaded: the candidate search visits only the
// buckets a cone can reach.  The header lives in device memory so that a
// captured graph reads the current field's values.
struct CandBuckets {
  double x0, z0, inv;  // grid origin (smallest centre x, z) and 1 / bucket size
  int nbx, nbz;        // buckets along x and z; bucket (bx, bz) is bz * nbx + bx
  double ytop;         // largest centre height + bounding radius over the field
  double rmax;         // largest bounding radius (half-diagonal + 1 cm)
};

// The grid's cell-count scan: one CTA up to kScanOneCtaMax cells, above that
// tiles of kScanTile cells, one CTA each.
constexpr int64_t kScanOneCtaMax = 65536;
constexpr int kScanTile = 4096;
constexpr int64_t kCellWarpMax = 16384;  // grids up to this many cells finish with a warp per cell

struct SunGeom {
  double* normal = nullptr;      // [3n]
  double* frame = nullptr;       // [kFrameStride n] u, n, v, mirror centre
  float4* rect = nullptr;        // [3n] A(v0)+id, E1, E2
  int4* cellbox = nullptr;       // [2n]
  int32_t* cell_count = nullptr; // [cells]
  int32_t* cell_start = nullptr; // [cells+1]
  int32_t* entries = nullptr;    // [entry_cap]
  float4* cell_rect = nullptr;   // [3*entry_cap]
  int4* cell_info = nullptr;     // [cells] first, end, ylo bits, yhi bits
  float2* coarse_yr = nullptr;   // [coarse_cells] two-level grid only
  int64_t* scan_part = nullptr;  // [cells / kScanTile] tile totals of the multi-CTA scan (large grids only)
  float4* cand = nullptr;        // [n][2][kCandCap][3] rectangle records of each heliostat's shadow / block candidates
  int* cand_n = nullptr;         // [n][2] their counts (> kCandCap: too many, the rays walk the grid)
  int* field_yr = nullptr;       // [2]
  double* power = nullptr;       // [1] sum |n . sun| * A
  int* grid_ctl = nullptr;       // [4] the grid's build control words (zero_geom_kernel, scene.cu)
};

struct PointsKey {
  uint64_t seed = 0, rays = 0;
  int rpp = 0, mode = -1;
  float spacing = 0;
  bool operator==(const PointsKey& o) const {
    return seed == o.seed && rays == o.rays && rpp == o.rpp && mode == o.mode && spacing == o.spacing;
  }
};

struct SunKey {
  float dir[3] = {0, 0, 0};
  uint32_t quirks = 0xFFFFFFFFu;
  uint64_t field_version = ~0ull;
  bool operator==(const SunKey& o) const {
    return dir[0] == o.dir[0] && dir[1] == o.dir[1] && dir[2] == o.dir[2] && quirks == o.quirks &&
           field_version == o.field_version;
  }
};

}  // namespace qm

struct qmcrt_scene {
  int device = 0;
  int n = 0;
  uint64_t field_version = 0;
  bool has_aim = false, has_normal = false, has_tilt = false;
  std::vector<float> h_pos, h_size;
  float ytop = 0.f;  // highest point any mirror can reach (centre + half-diagonal)
  // centre buckets of the candidate search (host copies stay alive for the async uploads)
  int64_t bucket_cap = 0;                    // capacity of the bucket table (buckets)
  qm::CandBuckets h_buckets{};
  std::vector<int32_t> h_bucket_start, h_bucket_ids;
  qm::CandBuckets* d_buckets = nullptr;      // [1]
  int32_t* d_bucket_start = nullptr;         // [bucket_cap + 1] first index of each bucket in d_bucket_ids
  int32_t* d_bucket_ids = nullptr;           // [n] heliostat ids by bucket, ascending within a bucket
  qmcrt_receiver recv{};
  qm::ReceiverGeom rg;
  qmcrt_grid_params gp{};

  // grid: bounds fixed per scene (orientation-independent sphere bounds)
  float gpos[3], gcell[3];
  int gdims[3];
  int64_t cells = 0, entry_cap = 0;
  int fine_div = 1;
  int64_t coarse_cells = 0;  // fine_div > 1: cells of the coarse level

  // device field
  float *d_pos = nullptr, *d_size = nullptr, *d_aim = nullptr, *d_normal_in = nullptr;
  float *d_sigma = nullptr, *d_tilt = nullptr;
  // per-sun geometry
  double* d_normal = nullptr;   // [3n]
  double* d_frame = nullptr;    // [kFrameStride n] u, n, v, mirror centre
  float4* d_rect = nullptr;     // [3n] A(v0)+id, E1, E2 (float)
  int4* d_cellbox = nullptr;    // [2n] lo, hi cell indices per heliostat
  int32_t* d_cell_count = nullptr;  // [cells]
  int32_t* d_cell_start = nullptr;  // [cells+1]
  int32_t* d_entries = nullptr;     // [entry_cap]
  float4* d_cell_rect = nullptr;    // [3*entry_cap] cell-major rectangle records
  int4* d_cell_info = nullptr;      // [cells] run of each cell's rectangles and their height range
  float2* d_coarse_yr = nullptr;    // [coarse_cells] the same per coarse cell (two-level grid)
  int64_t* d_scan_part = nullptr;   // [cells / kScanTile] tile totals of the multi-CTA scan (large grids only)
  double2* d_cyl_edge = nullptr;    // cylinder receivers: [res_x] direction of each column's first edge
  float4* d_cand = nullptr;         // [n][2][kCandCap][3] occluder candidates' rectangle records (shadow, block)
  int* d_cand_n = nullptr;          // [n][2]
  int* d_field_yr = nullptr;        // [2] height range of the field (order-preserving ints)
  int* d_grid_ctl = nullptr;        // [4] grid build control words of the current geometry
  bool grid_forced = false;         // the current geometry's grid is built (or being built) in the stream
  qm::SunKey sun_key;

  // points
  qm::PointsKey points_key;
  int64_t points = 0, points_cap = 0;
  // per-point candidate masks, rebuilt when the sun geometry or the points change
  uint64_t geom_version = 0, points_version = 0, mask_geom = ~0ull, mask_points = ~0ull;
  double sun_unit[3] = {0, 0, 0};   // the normalised sun direction of the current geometry
  int64_t mask_cap = 0;
  uint4* d_point_mask = nullptr;     // [points] (shadow, block) candidate bits, slope sigma, area weight
  double4* d_point_origin = nullptr; // [points] the points in world coordinates for the current sun
  float2* d_point_xz = nullptr;
  int32_t* d_point_helio = nullptr;
  float* d_helio_weight = nullptr;  // [n] mirror area per point
  int32_t* d_flag = nullptr;        // device error flag for setup kernels

  // maps and statistics
  uint32_t* d_counts = nullptr;
  float* d_energy = nullptr;
  float* d_map_flux = nullptr;    // [res] qmcrt_results_host: the flux map
  float* d_map_smooth = nullptr;  // [res] qmcrt_results_host: the smoothed map
  unsigned long long* d_stats = nullptr;  // [16]

  // sunshape
  qm::BuieTable buie;
  float* d_buie = nullptr;

  // stage timing of the last trace: [0,1] setup, [2,3] trace kernel, [3,4]
  // finalize; timing_stages (QMCRT_TIMING_*) says which stages record their
  // events, timed those the last trace recorded
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  uint32_t timing_stages = 0;
  uint32_t timed = 0;
  bool traced = false;
};

namespace qm {
// The scene's own per-sun buffers as a SunGeom.
SunGeom scene_geom(qmcrt_scene* s);
// Allocate / free a SunGeom sized for scene s.
qmcrt_status alloc_sun_geom(const qmcrt_scene* s, SunGeom* g);
void free_sun_geom(SunGeom* g);
// Enqueue aiming + grid build of scene s for the (normalised) sun direction
// into g.  pdl: launch the kernels with programmatic stream serialization
// (each starts while the one before it finishes; not inside graph captures).
// force_grid false: the grid is built only if a candidate list overflows (the
// traces that test candidates walk the grid only there).
qmcrt_status launch_sun_geom(const qmcrt_scene* s, const SunGeom& g, const double sun[3], uint32_t quirks,
                             cudaStream_t st, bool pdl = false, bool force_grid = true);
// The scene's sun geometry for `sun`, rebuilt when the sun, the quirks that
// shape it or the field changed; need_grid: the caller walks the grid (table
// traces, quirk modes, grid-walk variants), so it is built whatever the
// candidate lists hold.
qmcrt_status ensure_sun(qmcrt_scene* s, const qmcrt_sun* sun, uint32_t quirks, cudaStream_t st, bool need_grid = true);
// Build the current geometry's grid if it was left unbuilt.
qmcrt_status ensure_grid(qmcrt_scene* s, cudaStream_t st);
qmcrt_status ensure_points(qmcrt_scene* s, const qmcrt_trace_params* p, cudaStream_t st);
// Per-point candidate masks of `points` points (xz, helio) for geometry g of
// scene s and the (normalised) sun, into mask, and the points' world
// coordinates (the rays' origins) into origin.
qmcrt_status launch_point_masks(const qmcrt_scene* s, const SunGeom& g, const double sun[3], const float2* xz,
                                const int32_t* helio, const float* weight, int64_t points, uint4* mask, double4* origin,
                                cudaStream_t st, bool pdl = false);
// The scene's masks for its current sun and points (rebuilt when stale).
qmcrt_status ensure_masks(qmcrt_scene* s, cudaStream_t st);
}  // namespace qm
