/*
 * qmcrt.h — C-ABI of the B200 heliostat-field Monte Carlo ray tracer.
 *
 * Plain C, plain pointers and sizes, status-code returns, no exits.  Every
 * entry point here replaces one call on the hot path of the reference
 * (youxianru11/onemirror, Hu_smooth/ClassedSunRay); each declaration cites the
 * reference interface it stands in for.
 *
 * Conventions
 *  - World frame as in the reference driver (main.cpp:71-73): x = east,
 *    y = up, z = south.  The sun direction is the INCIDENT direction (from the
 *    sun toward the ground), as SunRay::sun_dir_ (sunray.h:41).
 *  - A heliostat is a flat rectangle (RectangleHelio, heliostat.cuh:38-61):
 *    size = (width along local x, thickness, height along local z); the mirror
 *    plane sits at local y = thickness/2.
 *  - Pointers named d_* are device pointers on the current device; h_* are
 *    host pointers.  Everything else is host memory read during the call.
 *  - Work is enqueued on the caller's `stream` (a cudaStream_t passed as
 *    void*, NULL = legacy default stream).  Calls that return host values
 *    synchronise that stream and say so.
 *  - Errors: every call returns qmcrt_status; qmcrt_last_error() gives a
 *    thread-local message for the last failure.  The reference exits the
 *    process on any CUDA error (utils.h:13-22); this library never does.
 */
#ifndef QMCRT_H_
#define QMCRT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QMCRT_ABI_VERSION 1

typedef enum qmcrt_status {
  QMCRT_OK = 0,
  QMCRT_ERR_INVALID_ARGUMENT = 1, /* bad size, null pointer, out-of-range parameter */
  QMCRT_ERR_CUDA = 2,             /* a CUDA runtime call failed */
  QMCRT_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed */
  QMCRT_ERR_NOT_SUPPORTED = 4,    /* feature/receiver type not available */
  QMCRT_ERR_TIMEOUT = 5,          /* a bounded device-side wait expired */
  QMCRT_ERR_SAMPLING = 6,         /* Poisson-disk sampling could not place the requested points */
  QMCRT_ERR_INTERNAL = 7
} qmcrt_status;

/* Reference behaviours that differ from the corrected method.  Each bit makes
 * the tracer (and the oracle) reproduce one reference quirk exactly. */
enum {
  /* 3D-DDA steps before it tests, so the origin cell is never tested
   * (rectgrid_raytracing.cu:70-114). */
  QMCRT_QUIRK_SKIP_ORIGIN_CELL = 1u << 0,
  /* Grid registration uses the cube of half-side sqrt(|size|)/2 around the
   * heliostat centre (grid.cpp:55-59) instead of the rectangle's bounding box. */
  QMCRT_QUIRK_AABB_RADIUS = 1u << 1,
  /* The ray's own heliostat is not excluded; only t > 1e-6 rejects the
   * self-hit (global_function.cuh:101-102). */
  QMCRT_QUIRK_SELF_HIT = 1u << 2,
  /* Table mode: the perturbation of a heliostat's point l uses the start
   * offset of its point max(l-1, 0) (rectgrid_raytracing.cu:183-184; the
   * reference launches map_tracing per heliostat, so l restarts at each one). */
  QMCRT_QUIRK_PREV_PERTURB = 1u << 3,
  /* local2world returns its input unchanged whenever the aligned normal is
   * parallel to y, also for -y (global_function.cuh:29-30). */
  QMCRT_QUIRK_ZENITH_FRAME = 1u << 4,
  /* Pixel index int(u*res) without clamping: u == 1 lands one row/column past
   * the map (rectgrid_raytracing.cu:144); such hits are counted, not written. */
  QMCRT_QUIRK_PIXEL_EDGE = 1u << 5,
  QMCRT_QUIRKS_REFERENCE = 0x3Fu
};

/* Receiver kinds (receiver.cuh:66-143). */
enum { QMCRT_RECEIVER_FLAT = 0, QMCRT_RECEIVER_CYLINDER = 1 };

/* Micro-heliostat sample point layouts (heliostat.cuh:6-10). */
enum { QMCRT_POINTS_POISSON = 0, QMCRT_POINTS_GRID = 1 };

/* Flux deposition: nearest pixel (reference) or bilinear (adjoint). */
enum { QMCRT_DEPOSIT_NEAREST = 0, QMCRT_DEPOSIT_BILINEAR = 1 };

/* Atmospheric attenuation eta(d) of a ray's energy over its slant range d (m)
 * from the mirror to the receiver hit (eta_aAlpha, rectgrid_raytracing.cu:120-127). */
enum {
  QMCRT_ATTEN_NONE = 0,    /* eta = 1: what the reference computes */
  QMCRT_ATTEN_POLY_EXP = 1 /* the formula the reference carries disabled: d <= 1000 m:
                              0.99331 - 1.176e-4 d + 1.97e-8 d^2, else exp(-1.106e-4 d) */
};

/* Trimmed-mean definitions (image_smooth.cu:10-58). */
enum {
  QMCRT_TRIM_SORTED = 0, /* exact order statistics: drop the k lowest and k highest */
  QMCRT_TRIM_HEAPS = 1   /* the reference's two-heap stream, else-if chain included */
};

/* Per-ray record flags (parity mode). */
enum {
  QMCRT_RAY_SHADOWED = 1u << 0, /* hit another heliostat on the way from the sun */
  QMCRT_RAY_BLOCKED = 1u << 1,  /* reflected ray hit another heliostat */
  QMCRT_RAY_HIT = 1u << 2,      /* reflected ray hit the receiver */
  QMCRT_RAY_OFFMAP = 1u << 3    /* receiver hit whose pixel fell outside the map (quirk) */
};

/* Heliostat field, structure of arrays, n heliostats.
 * Replaces vector<Heliostat*> (solar_scene.h:217) built by
 * SceneFileProc::SceneFileRead (scene_file_proc.cpp:41-286). */
typedef struct qmcrt_field {
  int32_t n;
  const float* pos;         /* [3n] mirror centre */
  const float* size;        /* [3n] width, thickness, height */
  const float* aim;         /* [3n] aim point; NULL: the receiver's focus centre */
  const float* normal;      /* [3n] fixed normal (Heliostat::CRotate(dir), heliostat.cpp:23-28);
                               NULL: aimed as the sun/target bisector (heliostat.cpp:51-58) */
  const float* slope_sigma; /* [n] Gaussian slope error in rad; NULL: use `sigma` */
  float sigma;              /* default slope error (common_var.cpp:18 uses 1 mrad) */
  const float* tilt;        /* [2n] extra normal tilt (rad) about local x and z; NULL: none */
} qmcrt_field;

/* Receiver (RectangleReceiver receiver.cuh:66-101, receiver.cpp:24-118;
 * CylinderReceiver receiver.cuh:103-122, a stub in the reference). */
typedef struct qmcrt_receiver {
  int32_t type;     /* QMCRT_RECEIVER_* */
  float pos[3];     /* flat: box centre; cylinder: centre of the bottom circle */
  float size[3];    /* flat: width (x), height (y), depth (z); cylinder: radius, height, unused */
  float normal[3];  /* flat: facing direction, rotated about y only (receiver.cpp:85-97) */
  int32_t face;     /* flat: face index 0..3 (receiver.cpp:30-83) */
  int32_t res_x;    /* map columns (flat: along width; cylinder: around the circumference) */
  int32_t res_y;    /* map rows (along height) */
} qmcrt_receiver;

/* Uniform grid over the field (RectGrid grid.h:25-48).  The bounds are taken
 * from the field (plus `margin`) unless `explicit_bounds` is set.
 * Two-level grid (fine_div = 2, 4 or 8): `cell` is the coarse cell; the
 * heliostats are registered in fine cells of cell / fine_div, and each coarse
 * cell keeps the height range of its fine cells so that the traversal can
 * step through a coarse cell without visiting its fine cells.  The grid
 * reported by qmcrt_scene_grid_info is the fine one. */
typedef struct qmcrt_grid_params {
  float cell[3];         /* cell size in m (RectGrid::interval_); the coarse cell when fine_div > 1 */
  float margin;          /* added around the field's bounding box, m */
  int32_t explicit_bounds;
  float origin[3];       /* used when explicit_bounds: RectGrid::pos_ */
  float extent[3];       /* used when explicit_bounds: RectGrid::size_ */
  int32_t fine_div;      /* 0 or 1: one level; 2, 4 or 8: two-level grid, each coarse cell split into fine_div^3 */
} qmcrt_grid_params;

/* Sun (SunRay sunray.h:3-50). */
typedef struct qmcrt_sun {
  float dir[3]; /* incident direction, normalised inside (scene_instance_process.cu:8) */
  float dni;    /* W/m^2 */
  float csr;    /* circumsolar ratio of the Buie sunshape */
} qmcrt_sun;

/* What one trace does (replaces the per-heliostat loop of
 * results_with_given_normal, Gtest.cu:10-63). */
typedef struct qmcrt_trace_params {
  uint64_t seed;           /* Philox key; every ray is a function of (seed, ray id) */
  uint64_t rays;           /* total rays; must be a multiple of rays_per_point (Poisson).  2^32 rays and more
                              need a power-of-two rays_per_point (fewer than 2^31 points); the adjoint and
                              batches take fewer than 2^32 */
  int32_t rays_per_point;  /* rays per micro-heliostat point (reference: 2048) */
  int32_t point_mode;      /* QMCRT_POINTS_* */
  float point_spacing;     /* Poisson: minimum spacing in m; GRID: pixel length in m */
  float reflectivity;      /* rho (common_var.cpp:19 uses 0.88) */
  uint32_t quirks;         /* QMCRT_QUIRK_* */
  int32_t deposit;         /* QMCRT_DEPOSIT_* */
  int32_t accumulate;      /* 0: zero the output maps first; 1: add into them */
  int32_t kernel_variant;  /* 0 or 1: default (fastest: Philox rays test their heliostat's occluder
                              candidates); 2: grid walk without vertical culling (every cell on the path
                              tested); 3: the production kernel without its 4-CTA register cap;
                              4: grid walk, a two-level grid on its fine level only; 5: grid walk */
  uint32_t item;           /* Philox stream (counter word 2): distinct items give independent ray sets
                              (shards of one trace, items of a batch) */
  int32_t attenuation;     /* QMCRT_ATTEN_*: atmospheric transmittance of the mirror-to-receiver leg */
  uint64_t ray_begin;      /* trace only the rays [ray_begin, ray_end) of the full set: the same
                              rays, points and deposits as the whole trace restricted to them (rays
                              are numbered point-major and points by heliostat, so one heliostat's
                              rays are one range: the reference's per-heliostat launches,
                              ray_tracing.cu:23-27); ray_end = 0: all rays.  Statistics count the
                              range's rays; total_power stays the whole field's. */
  uint64_t ray_end;
} qmcrt_trace_params;

/* Device outputs of a trace.  Any pointer may be NULL. */
typedef struct qmcrt_outputs {
  uint32_t* d_counts;      /* [res_y*res_x] rays per pixel (exact integer) */
  float* d_energy;         /* [res_y*res_x] sum of |sun . n_perturbed| * area-per-point (raw) */
  float* d_flux;           /* [res_y*res_x] W/m^2 = energy * DNI * rho / (rays_per_point * pixel area) */
  uint8_t* d_ray_flags;    /* [rays] QMCRT_RAY_* per ray */
  int32_t* d_ray_pixel;    /* [rays] row*res_x + col, -1 if no receiver hit */
} qmcrt_outputs;

/* Scalars of a trace (filled only when requested; the call then synchronises). */
typedef struct qmcrt_trace_stats {
  uint64_t rays;
  uint64_t shadowed;
  uint64_t blocked;
  uint64_t hit;
  uint64_t offmap;
  uint64_t rect_tests;      /* rectangle tests in both traversals */
  uint64_t dda_cells;       /* cells visited in both traversals */
  double total_power;       /* sum_h |n_h . sun| * DNI * A_h * rho, W (Gtest.cu:29,44) */
  double intercepted_power; /* sum over the map of flux * pixel area, W */
  double intercept_ratio;   /* intercepted / total (image_save.cpp:26-48) */
} qmcrt_trace_stats;

/* Table-mode inputs (device), the sampling structure of the reference kernel
 * map_tracing (rectgrid_raytracing.cu:155-196): ray j of point m takes sun
 * sample (start[m]+j) mod table_size and perturbation (start[m']+j) mod
 * table_size (m' = m, or max(m-1,0) with QMCRT_QUIRK_PREV_PERTURB). */
typedef struct qmcrt_table_inputs {
  const float* d_sun_local;  /* [3T] unit vectors, y-up local frame (set_samplelights) */
  const float* d_turb_local; /* [3T] unit vectors, y-up local frame (set_perturbation) */
  int64_t table_size;        /* T (reference: 128*2048) */
  const int32_t* d_start;    /* [points] start offsets (set_microhelio_groups) */
  const float* d_point_xz;   /* [2*points] local (x, z) of each point, m, mirror-centred */
  const int32_t* d_point_helio; /* [points] heliostat of each point */
  int64_t points;
  int32_t rays_per_point;
} qmcrt_table_inputs;

/* Grid summary (of the fine grid when the grid has two levels). */
typedef struct qmcrt_grid_info {
  float origin[3];
  float cell[3];
  int32_t dims[3];    /* a multiple of fine_div on every axis */
  int64_t cells;
  int64_t entries; /* CSR entries (heliostat registrations) */
  int32_t fine_div;
} qmcrt_grid_info;

/* Radial-staggered field layout generator (scene front-end). */
typedef struct qmcrt_layout_params {
  int32_t n;               /* heliostats wanted */
  float helio_w, helio_h;  /* mirror width, height (m) */
  float thickness;         /* mirror thickness (m) */
  float r_min, r_max;      /* ring radii (m) */
  float az_center_deg;     /* centre of the field's azimuth span (0 = north), degrees */
  float az_span_deg;       /* span; 360 = surround field */
  float spacing;           /* minimum centre spacing (m); 0 = auto to fill r_max */
  float jitter;            /* uniform jitter amplitude on x and z (m) */
  float mount_height;      /* mirror centre height above ground (m) */
  uint64_t seed;
} qmcrt_layout_params;

/* A faceted paraboloid heliostat (SceneFileProc::SceneFileRead,
 * scene_file_proc.cpp:288-341): rows x cols flat square facets of side
 * `facet` whose centres sit on the paraboloid y = x^2/a^2 + z^2/b^2 of the
 * heliostat's local frame at pitch facet + gap, each canted to the
 * paraboloid's normal (-2x/a^2, 1, -2z/b^2) there.  The local frame is
 * (e1, n, e1 x n) with n the heliostat normal and e1 horizontal; it is placed
 * at `centre`.  Every facet is one rectangle with a given normal in a
 * qmcrt_field.  The reference's own scene: a = b (its arguments A, B),
 * 3 x 3 facets of sqrt(2)/3 m, gap 0.1 m, thickness 0.1 m. */
typedef struct qmcrt_facet_params {
  float a, b;            /* paraboloid coefficients (m) */
  float normal[3];       /* heliostat normal (mirrorNormal), unit */
  float centre[3];       /* world position of the paraboloid's vertex */
  int32_t rows, cols;    /* facets along local z and x */
  float facet;           /* facet side (m) */
  float gap;             /* gap between facets (m) */
  float thickness;       /* facet thickness (m) */
  int32_t reference_frame; /* 1: the reference's e1 = (n.z, 0, -n.x) / sqrt(n.x^2 + n.y^2), which is not a unit
                              vector in general (scene_file_proc.cpp:300-316); 0: e1 normalised */
} qmcrt_facet_params;

typedef struct qmcrt_scene qmcrt_scene;
typedef struct qmcrt_tape qmcrt_tape;
typedef struct qmcrt_batch qmcrt_batch;

/* ------------------------------------------------------------------ info */
const char* qmcrt_version(void);
const char* qmcrt_status_string(qmcrt_status s);
/* The thread-local message of the last failure (named qmcrt_last_error_string
 * in earlier designs of this boundary). */
const char* qmcrt_last_error(void);

/* --------------------------------------------------- host-side helpers
 * Pure host code; these need no GPU. */

/* Sun incident direction from elevation/azimuth (degrees, azimuth from north
 * clockwise), the convention of main.cpp:71-73. */
qmcrt_status qmcrt_sun_direction(float elevation_deg, float azimuth_deg, float dir_out[3]);

/* Sun position for a site: solar declination (degrees) of day `day_of_year`
 * by Cooper's formula, and elevation / azimuth (degrees, azimuth from north
 * clockwise) for latitude, declination and hour angle (15 degrees per hour from
 * solar noon, negative in the morning).  Stands in for the NREL SPA call of the
 * reference driver (main.cpp:62-73). */
float qmcrt_solar_declination(int32_t day_of_year);
qmcrt_status qmcrt_solar_position(float latitude_deg, float declination_deg, float hour_angle_deg,
                                  float* elevation_deg, float* azimuth_deg);

/* Buie sunshape inverse-CDF table, built exactly as
 * SceneProcessor::set_samplelights (scene_instance_process.cu:163-200) builds
 * it: 1024 trapezoids on [0, 4.65] mrad plus the analytic aureole to 9.3 mrad.
 * params_out = {k, gamma, core_area, total_area, B, C}. */
qmcrt_status qmcrt_buie_table(float csr, float* cdf_x /*[1025]*/, float* cdf_y /*[1025]*/,
                              float* slope /*[1024]*/, float params_out[6]);

/* Radial-staggered layout: writes up to `capacity` heliostat centres. */
qmcrt_status qmcrt_layout_radial_staggered(const qmcrt_layout_params* p, float* h_pos,
                                           int32_t capacity, int32_t* n_out);

/* Facets of one paraboloid heliostat into h_pos / h_size / h_normal [3 x
 * rows x cols] (row-major over local z then x, as the reference lists them);
 * *n_out = rows x cols.  Normals are unit length. */
qmcrt_status qmcrt_layout_paraboloid_facets(const qmcrt_facet_params* p, float* h_pos, float* h_size, float* h_normal,
                                            int32_t capacity, int32_t* n_out);

/* Parse a reference .scn scene file (scene_file_proc.cpp:41-286) into
 * caller-visible arrays.  Call once with h_pos == NULL to get the counts. */
qmcrt_status qmcrt_scn_parse(const char* path, qmcrt_receiver* recv_out,
                             qmcrt_grid_params* grid_out, float* h_pos, float* h_size,
                             int32_t capacity, int32_t* n_out);

/* Result files, host buffers, the reference's text formats
 * (ImageSaver::savetxt, image_save.cpp:5-48).  The map is [height][width] as
 * the tracer writes it; both writers go from its last row to its first (the
 * receiver's top edge first) and treat values below 1e-6 as zero.
 * append != 0 appends, as the reference does (it opens with ios::app).
 *
 * Flux map (image_save.cpp:5-24): one line per row, every value followed by
 * ','; zero as "0", others in fixed notation with `precision` decimals. */
qmcrt_status qmcrt_write_flux_csv(const char* path, const float* h_map, int32_t width, int32_t height,
                                  int32_t precision, int32_t append);

/* Intercept ratio (image_save.cpp:26-48): the float sum of the map's values
 * (in the file's order) divided by total_energy, written with 6 significant
 * digits and a newline.  path may be NULL to get *ratio_out only. */
qmcrt_status qmcrt_write_intercept_ratio(const char* path, const float* h_map, int32_t width, int32_t height,
                                         float total_energy, int32_t append, float* ratio_out);

/* -------------------------------------------------------------- scenes
 * A scene owns the device copy of the field, receiver and grid.  Replaces
 * SolarScene (solar_scene.h:19-50) plus SceneProcessor::set_*_content
 * (scene_instance_process.h:5-26). */
qmcrt_status qmcrt_scene_create(const qmcrt_field* field, const qmcrt_receiver* recv,
                                const qmcrt_grid_params* grid, qmcrt_scene** out);
qmcrt_status qmcrt_scene_destroy(qmcrt_scene* scene);

/* Upload a new field (same n) from host memory; h2d copies on `stream`. */
qmcrt_status qmcrt_scene_set_field(qmcrt_scene* scene, const qmcrt_field* field, void* stream);

/* Aim the heliostats for `sun` and rebuild the grid on the GPU.  Replaces
 * set_helio_content + set_grid_content (scene_instance_process.cpp:4-35)
 * and RectGrid::CGridHelioMatch (grid.cpp:47-83). */
qmcrt_status qmcrt_scene_set_sun(qmcrt_scene* scene, const qmcrt_sun* sun, uint32_t quirks,
                                 void* stream);

/* The grid's bounds and its CSR entry count.  When the last trace left its
 * geometry's grid unbuilt (see qmcrt_scene_read_grid), this waits for the
 * device to be idle and builds it on the default stream.  Syncs. */
qmcrt_status qmcrt_scene_grid_info(qmcrt_scene* scene, qmcrt_grid_info* info);

/* Copy the grid CSR to host (cells+1 offsets, entries heliostat ids).  The
 * geometry of a trace that tests occluder candidates builds its grid only if a
 * candidate list overflows; this call (and qmcrt_scene_grid_info) builds it
 * first when it was left unbuilt.  Syncs. */
qmcrt_status qmcrt_scene_read_grid(qmcrt_scene* scene, int32_t* h_cell_start, int32_t* h_entries,
                                   void* stream);

/* Copy per-heliostat geometry (double): normals [3n] and vertices v0,v1,v3
 * [9n] (RectangleHelio::Cget_vertex, heliostat.cuh:45-50).  Syncs. */
qmcrt_status qmcrt_scene_read_geometry(qmcrt_scene* scene, double* h_normals, double* h_vertices,
                                       void* stream);

/* Copy the occluder candidates of the current sun (no reference
 * counterpart; they replace the grid walk of NotCollision,
 * rectgrid_raytracing.cu:38-117, for Philox traces): h_counts [2n] holds
 * each heliostat's shadow and block candidate counts (above QMCRT_CAND_CAP:
 * the rays walk the grid), h_ids [2n*QMCRT_CAND_CAP] (may be NULL) their
 * heliostat ids, -1 past the count.  exhaustive = 1 recomputes them by testing every pair instead
 * of the bucket search (same sets; the order within a list may differ).
 * Needs a sun set for the current field.  Syncs. */
#define QMCRT_CAND_CAP 32
qmcrt_status qmcrt_scene_read_candidates(qmcrt_scene* scene, int32_t exhaustive, int32_t* h_counts,
                                         int32_t* h_ids, void* stream);

/* Micro-heliostat sample points for (seed, rays, rays_per_point, mode,
 * spacing) (set_possion_microhelio_centers steps_for_raytracing.cu:105-158,
 * set_microhelio_centers :67-103).  Cached in the scene.  points_out: count. */
qmcrt_status qmcrt_scene_sample_points(qmcrt_scene* scene, const qmcrt_trace_params* params,
                                       int64_t* points_out, void* stream);

/* Copy the cached points: local (x, z) in m relative to the mirror centre
 * ([2*points] floats; Poisson points lie on a 2^-16 m lattice from the mirror
 * corner) and their heliostat ids.  Syncs. */
qmcrt_status qmcrt_scene_read_points(qmcrt_scene* scene, float* h_point_xz, int32_t* h_point_helio,
                                     void* stream);

/* Poisson-disk sample points without allocating device memory.
 *
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code running under another allocator's ownership (a host application that
 * owns every device buffer), a real-time loop that may not allocate, or a
 * plugin whose memory budget is fixed at load time.  The same points as
 * qmcrt_scene_sample_points + qmcrt_scene_read_points for the same sizes,
 * total_points, spacing and seed, written to caller-owned device outputs.
 *
 * Inputs: h_size [3n] host mirror sizes; outputs: d_point_xz [2*total_points]
 * and d_point_helio [total_points], device.  Its working memory is one
 * file-scope __device__ array that every GPU loading this library holds until
 * the process exits: room for QMCRT_NOALLOC_MAX_POINTS points and
 * QMCRT_NOALLOC_MAX_HELIOSTATS heliostats (about 8.2 MB); larger requests are
 * rejected with QMCRT_ERR_INVALID_ARGUMENT.  Each call finds that array's
 * device address on the current device before it launches.  All calls share
 * the array, so calls that overlap on the GPU (different streams or host
 * threads at the same time) race; serialise them.  Synchronises `stream` to
 * read the sampler's status.  After any status other than QMCRT_OK the
 * outputs are undefined: a sampling failure leaves some heliostats' points
 * written and others not.  A later successful call overwrites all of them. */
#define QMCRT_NOALLOC_MAX_POINTS 1048576
#define QMCRT_NOALLOC_MAX_HELIOSTATS 16384
qmcrt_status qmcrt_sample_points_noalloc(const float* h_size, int32_t n, int64_t total_points, float spacing,
                                         uint64_t seed, float* d_point_xz, int32_t* d_point_helio, void* stream);

/* ------------------------------------------------------------- tracing */

/* One full trace: aim, grid, points (cached), Philox sampling, shadow and
 * block traversal, receiver deposition, flux scaling.  Replaces
 * results_with_given_normal's loop over recthelio_ray_tracing
 * (Gtest.cu:21-46, recthelio_tracing.cpp:46-80, ray_tracing.cu:3-32).
 * If `stats` is not NULL the call synchronises `stream` and fills it. */
qmcrt_status qmcrt_trace(qmcrt_scene* scene, const qmcrt_sun* sun, const qmcrt_trace_params* params,
                         const qmcrt_outputs* out, qmcrt_trace_stats* stats, void* stream);

/* Parity mode: the same traversal fed by caller-provided sample tables
 * (the inputs of map_tracing, rectgrid_raytracing.cu:155-162).  Rays are
 * numbered point-major (ray = point*rays_per_point + j).  Named
 * qmcrt_trace_records in earlier designs of this boundary. */
qmcrt_status qmcrt_trace_tables(qmcrt_scene* scene, const qmcrt_sun* sun,
                                const qmcrt_table_inputs* tables, const qmcrt_trace_params* params,
                                const qmcrt_outputs* out, qmcrt_trace_stats* stats, void* stream);

/* End-to-end call on host buffers: upload the field (NULL: keep the scene's),
 * trace, download the maps.  h_counts / h_flux may be NULL.  Synchronises. */
qmcrt_status qmcrt_trace_host(qmcrt_scene* scene, const qmcrt_field* field, const qmcrt_sun* sun,
                              const qmcrt_trace_params* params, uint32_t* h_counts, float* h_flux,
                              qmcrt_trace_stats* stats, void* stream);

/* Which map qmcrt_results_host smooths. */
enum {
  QMCRT_SMOOTH_COUNTS = 0, /* the integer count map (exact with QMCRT_TRIM_SORTED) */
  QMCRT_SMOOTH_ENERGY = 1  /* the raw energy image, then scaled to W/m^2, as Gtest.cu:49-57 does */
};

/* Trimmed-mean smoothing of one result map (ImageSmoother::image_smooth
 * arguments, image_smooth.cuh:20-22). */
typedef struct qmcrt_smooth_params {
  int32_t radius; /* window half-size, 0..7 (Gtest.cu:50 uses 5) */
  float ratio;    /* fraction dropped at each end, [0, 0.5) (Gtest.cu:51 uses 0.02) */
  int32_t method; /* QMCRT_TRIM_* */
  int32_t source; /* QMCRT_SMOOTH_* */
} qmcrt_smooth_params;

/* One sun position end to end on host buffers: the work of
 * results_with_given_normal (Gtest.cu:10-63) without its file output.
 * Uploads the field (NULL: keep the scene's), traces, scales the flux map,
 * smooths the map `smooth` names (NULL: no smoothing) and downloads the
 * results: h_counts [res] counts, h_flux [res] W/m^2 (the non-smoothed
 * result), h_smoothed [res] the smoothed map (smoothed counts, or W/m^2 for
 * QMCRT_SMOOTH_ENERGY).  Any output pointer may be NULL.  Synchronises. */
qmcrt_status qmcrt_results_host(qmcrt_scene* scene, const qmcrt_field* field, const qmcrt_sun* sun,
                                const qmcrt_trace_params* params, const qmcrt_smooth_params* smooth,
                                uint32_t* h_counts, float* h_flux, float* h_smoothed, qmcrt_trace_stats* stats,
                                void* stream);

/* ------------------------------------------------------------ batching
 * No counterpart in the reference (it launches and synchronises once per
 * heliostat per sun position, ray_tracing.cu:23-27).  Many (field, sun)
 * items traced by ONE persistent kernel that takes ray chunks from a global
 * work counter, the whole pass (aiming, grids, tracing, flux scaling)
 * replayable as one captured CUDA graph.  Item i traces the same rays as
 * qmcrt_trace with params.item = i, so its count map equals that trace's. */
typedef struct qmcrt_batch_item {
  int32_t scene;   /* index into the scenes array */
  qmcrt_sun sun;
} qmcrt_batch_item;

typedef struct qmcrt_batch_tuning {
  int32_t chunk_rays;   /* rays per work unit (multiple of 256) */
  int32_t ctas_per_sm;  /* resident CTAs per SM of the persistent grid (1..4) */
  int32_t tile;         /* 0, 32 or 48: side of the CTA-private shared-memory flux tile */
  float ms;             /* autotune: device time of the trace pass with this tuning */
} qmcrt_batch_tuning;

/* Items must use corrected-mode traversal (no SKIP_ORIGIN_CELL / AABB_RADIUS
 * quirks) and nearest deposition; every item traces params->rays rays.
 * qmcrt_batch_create is the qmcrt_batch_plan of earlier designs of this
 * boundary. */
qmcrt_status qmcrt_batch_create(qmcrt_scene* const* scenes, int32_t n_scenes, const qmcrt_batch_item* items,
                                int32_t n_items, const qmcrt_trace_params* params, qmcrt_batch** out);
qmcrt_status qmcrt_batch_destroy(qmcrt_batch* batch);
/* Time candidate tunings on the first items and keep the fastest. Syncs. */
qmcrt_status qmcrt_batch_autotune(qmcrt_batch* batch, qmcrt_batch_tuning* chosen, void* stream);
qmcrt_status qmcrt_batch_set_tuning(qmcrt_batch* batch, const qmcrt_batch_tuning* tuning);
/* Enqueue the whole pass on `stream` (no graph). */
qmcrt_status qmcrt_batch_run(qmcrt_batch* batch, void* stream);
/* Capture the pass into a CUDA graph (replaces any earlier graph). */
qmcrt_status qmcrt_batch_capture(qmcrt_batch* batch);
/* Replay the captured graph on `stream`. */
qmcrt_status qmcrt_batch_launch(qmcrt_batch* batch, void* stream);
/* Device pointers of an item's maps (valid until destroy). */
qmcrt_status qmcrt_batch_maps(qmcrt_batch* batch, int32_t item, uint32_t** d_counts, float** d_flux);
/* Copy an item's maps to host and fill its totals.  Syncs. */
qmcrt_status qmcrt_batch_read(qmcrt_batch* batch, int32_t item, uint32_t* h_counts, float* h_flux,
                              qmcrt_trace_stats* stats, void* stream);

/* ------------------------------------------------------------- adjoint
 * No counterpart in the reference.  Gradient of the flux-map loss
 * L = sum_p (F_p - T_p)^2 (F in W/m^2, bilinear deposition) with respect to
 * each heliostat's aim offset (along the receiver's width and height axes, m)
 * and extra normal tilt (about the mirror's local u and v axes, rad), at the
 * scene's current aim points and tilts.  Pathwise derivative under the same
 * random numbers; shadow/block/receiver visibility held constant.
 *
 * qmcrt_adjoint_forward traces params->rays rays, or the range
 * [ray_begin, ray_end) of them (params->deposit must be
 * QMCRT_DEPOSIT_BILINEAR, flat receiver, corrected mode), keeps one
 * visibility byte per traced ray for at most state_bytes_max rays (0 = all;
 * rays past the cap recompute their visibility in the backward pass), writes
 * the flux map to d_flux (may be NULL) and, if `loss` is not NULL,
 * synchronises and returns L.  qmcrt_adjoint_backward writes d_grad_aim [2n]
 * and d_grad_tilt [2n] (device): the gradient of L through the rays the tape
 * traced.
 * Sharded over GPUs (one ray range per rank): each rank runs the forward on
 * its range, the ranks sum their energy maps (qmcrt_tape_energy, then an
 * all-reduce), each passes the sum to qmcrt_adjoint_loss, runs the backward,
 * and the ranks sum their gradients.  The loss and the summed gradients are
 * those of one GPU tracing every ray, to float rounding.
 * `tape` is in/out: *tape == NULL makes a new tape; a tape returned by an
 * earlier call on the same scene is reused, its device buffers kept where
 * they are large enough (an optimisation loop then allocates nothing after
 * its first step).  Reuse it on the stream it last ran on, or after that
 * stream has finished with it. */
qmcrt_status qmcrt_adjoint_forward(qmcrt_scene* scene, const qmcrt_sun* sun, const qmcrt_trace_params* params,
                                   const float* d_target, uint64_t state_bytes_max, float* d_flux, double* loss,
                                   qmcrt_tape** tape, void* stream);
qmcrt_status qmcrt_adjoint_backward(qmcrt_tape* tape, float* d_grad_aim, float* d_grad_tilt, void* stream);
/* The forward pass again at the scene's current aim points and tilts (after
 * qmcrt_scene_set_field), with every ray's visibility taken from `tape`
 * instead of traced: a ray the tape marks as a hit deposits wherever its
 * receiver-plane (u, v) falls now (corners off the map dropped), the others
 * deposit nothing.  This is the estimator whose derivative the backward pass
 * computes, so its central differences check the gradient without the jumps
 * that visibility changes add to those of the full loss.  The tape must hold
 * every ray (state_bytes_max 0) and is only read; like a forward pass, the
 * call leaves its loss and adjoint map in the tape for a following backward
 * pass.  The replay deposits in 64-bit fixed point (2^-40) and forms the loss
 * in double, so its loss is the same bit for bit from run to run.  Writes
 * d_flux (may be NULL) and, if `loss` is not NULL, synchronises and returns L. */
qmcrt_status qmcrt_adjoint_replay(qmcrt_tape* tape, const float* d_target, float* d_flux, double* loss,
                                  void* stream);
/* Copy the tape's energy map (the forward's deposits before flux scaling,
 * [res_y x res_x] floats) to d_energy (device). */
qmcrt_status qmcrt_tape_energy(const qmcrt_tape* tape, float* d_energy, void* stream);
/* Re-form the flux map, the loss and the adjoint map the backward pass reads
 * from d_energy (an energy map of the tape's layout, e.g. the sum of the
 * ranks' maps of one sharded trace; NULL: the tape's own), against d_target.
 * Writes d_flux (may be NULL) and, if `loss` is not NULL, synchronises and
 * returns L. */
qmcrt_status qmcrt_adjoint_loss(qmcrt_tape* tape, const float* d_energy, const float* d_target, float* d_flux,
                                double* loss, void* stream);
qmcrt_status qmcrt_tape_loss(qmcrt_tape* tape, double* loss, void* stream);
qmcrt_status qmcrt_tape_free(qmcrt_tape* tape);

/* ----------------------------------------------------------- smoothing
 * Trimmed-mean smoothing over a (2r+1)^2 window clipped at the border,
 * k = int(cnt * ratio) values dropped at each end (ImageSmoother::image_smooth,
 * image_smooth.cu:60-115).  d_in and d_out must not overlap.  One entry point
 * per map type (the single qmcrt_smooth_trimmed of earlier designs of this
 * boundary). */
qmcrt_status qmcrt_smooth_trimmed_u32(const uint32_t* d_in, float* d_out, int32_t width,
                                      int32_t height, int32_t radius, float ratio, int32_t method,
                                      void* stream);
qmcrt_status qmcrt_smooth_trimmed_f32(const float* d_in, float* d_out, int32_t width,
                                      int32_t height, int32_t radius, float ratio, int32_t method,
                                      void* stream);

/* Stage timing (no counterpart in the reference).  Off by default: a timed
 * stage records a CUDA event on the call's stream before and after it, and an
 * event between two kernels keeps the second from starting while the first
 * finishes (the kernels of a trace use programmatic dependent launch), which
 * cost about a tenth of the small field's step with every stage timed. */
enum {
  QMCRT_TIMING_TRACE = 1,    /* the trace kernel launches */
  QMCRT_TIMING_SETUP = 2,    /* aiming, occluder candidates and grid build, when the sun changed */
  QMCRT_TIMING_FINALIZE = 4, /* flux scaling and the copy to the outputs */
  QMCRT_TIMING_ALL = 7
};
/* Which stages the scene's later traces time (QMCRT_TIMING_* bits; 0: none). */
qmcrt_status qmcrt_scene_set_timing(qmcrt_scene* scene, uint32_t stages);

/* Device time of the stages of the last qmcrt_trace / qmcrt_trace_tables on
 * this scene, from the CUDA events it recorded on the call's stream; -1 for a
 * stage it did not time (setup_ms also when that trace reused the cached
 * geometry).  QMCRT_ERR_INVALID_ARGUMENT if it timed neither the trace kernel
 * nor the finalize stage.  Waits for the last trace to finish. */
typedef struct qmcrt_timing {
  float setup_ms;
  float trace_kernel_ms;
  float finalize_ms;
} qmcrt_timing;
qmcrt_status qmcrt_scene_timing(qmcrt_scene* scene, qmcrt_timing* timing);

/* ------------------------------------------------------------ probes */

/* FP32 FMA issue-rate probe for the roofline: `iters` dependent FMA chains
 * per thread on every SM.  Writes a sink value (device) and returns the FLOP
 * count of one launch in *flops. */
qmcrt_status qmcrt_fp32_peak_probe(float* d_sink, int32_t iters, double* flops, void* stream);

/* Philox4x32-10 block for a counter/key (test hook for the in-kernel RNG).
 * Writes n blocks (4 words each) for counters ctr0 + i (word 0 incremented). */
qmcrt_status qmcrt_philox_blocks(const uint32_t ctr0[4], const uint32_t key[2], int64_t n,
                                 uint32_t* d_out, void* stream);

/* The tracer's double-precision reciprocal and reciprocal square root (the
 * receiver determinant, the perturbed normal's length) on n device values
 * (test hook): d_rcp[i] = 1/x, d_rsqrt[i] = 1/sqrt(x); either may be NULL. */
qmcrt_status qmcrt_fp64_recip_probe(const double* d_x, int64_t n, double* d_rcp, double* d_rsqrt, void* stream);

/* The tracer's Buie inverse CDF (the sun sample's polar angle, mrad) on n
 * device uniforms in [0, 1) (test hook): the table of `csr` staged and
 * looked up as the trace kernels do.  Synchronises. */
qmcrt_status qmcrt_buie_sample_probe(float csr, const float* d_u, int64_t n, float* d_theta_mrad, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QMCRT_H_ */
