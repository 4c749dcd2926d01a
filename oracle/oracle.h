/*
 * oracle.h — FP64 CPU restatement of the reference heliostat-field ray tracer.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product library never links or calls it.
 *
 * Parity pinning: the reference ships no tests and no golden vectors.  The
 * pieces of the reference that are host-callable (vector math, the
 * parallelogram test, the Buie table builder, max_less_index, the heap
 * classes) are compiled from the reference sources by oracle/Makefile into
 * oracle/_ref and checked against this restatement by tests/test_oracle_pins.py
 * through golden vectors in tests/golden/.  The device-only traversal
 * (NotCollision, rectgrid_raytracing.cu:38-117) is pinned by analytic
 * known-answer cases and by brute-force traversal.
 *
 * Each function cites the reference file:line it follows (paths relative to
 * Hu_smooth/ClassedSunRay/).
 */
#ifndef QMCRT_ORACLE_H_
#define QMCRT_ORACLE_H_
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Quirk bits: identical values to QMCRT_QUIRK_* in include/qmcrt.h. */
#define ORC_QUIRK_SKIP_ORIGIN_CELL (1u << 0)
#define ORC_QUIRK_AABB_RADIUS (1u << 1)
#define ORC_QUIRK_SELF_HIT (1u << 2)
#define ORC_QUIRK_PREV_PERTURB (1u << 3)
#define ORC_QUIRK_ZENITH_FRAME (1u << 4)
#define ORC_QUIRK_PIXEL_EDGE (1u << 5)

#define ORC_RAY_SHADOWED 1u
#define ORC_RAY_BLOCKED 2u
#define ORC_RAY_HIT 4u
#define ORC_RAY_OFFMAP 8u

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Buie table exactly as set_samplelights builds it (float arithmetic,
 * scene_instance_process.cu:56-96,163-200).  params = {k, gamma, core, total, B, C}. */
void orc_buie_table(float csr, float* cdf_x, float* cdf_y, float* slope, float params[6]);

/* max_less_index (scene_instance_process.cu:98-113) on the float table. */
int orc_max_less_index(const float* cdf_y, double value, int n);

/* Inverse CDF (linear_interpolate, scene_instance_process.cu:115-137) in
 * double, from a uniform u in (0,1).  Returns theta in mrad. */
double orc_buie_sample(double u, const float* cdf_x, const float* cdf_y, const float* slope,
                       const float params[6]);

/* local2world (global_function.cuh:14-52) in double. */
void orc_local2world(const double d[3], const double n[3], uint32_t quirks, double out[3]);

/* Scene as the oracle sees it (all double unless noted). */
typedef struct orc_scene {
  int n;
  const float* pos;    /* [3n] */
  const float* size;   /* [3n] */
  const float* sigma;  /* [n] slope error (rad) */
  double* normal;      /* [3n] (filled by orc_scene_aim) */
  double* frame;       /* [9n] u, n, v per heliostat */
  double* vert;        /* [9n] v0, v1, v3 per heliostat */
  /* receiver (flat) */
  int recv_type;
  double recv_v[12];   /* v0..v3 */
  double recv_focus[3];
  int res_x, res_y;
  double cyl[5];       /* cylinder: cx, y0, cz, radius, height */
  /* grid */
  double gpos[3], gcell[3];
  int gdims[3];
  const int32_t* cell_start; /* [cells+1] */
  const int32_t* entries;
  int fine_div;              /* reserved */
} orc_scene;

/* Heliostat normals, frames and vertices for a sun direction (heliostat.cpp:30-62).
 * aim == NULL: aim at the receiver focus centre; normal_in != NULL: fixed normals.
 * tilt != NULL: n <- normalize(n + tx*u + tz*v) in the untilted frame. */
void orc_scene_aim(orc_scene* s, const double sun_dir[3], const float* aim, const float* normal_in,
                   const float* tilt, uint32_t quirks);

/* Flat receiver vertices (receiver.cpp:24-118). */
void orc_receiver_flat(orc_scene* s, const float pos[3], const float size[3], const float normal[3],
                       int face, int res_x, int res_y);

/* Cylindrical receiver (unrolled map: columns = azimuth, rows = height). */
void orc_receiver_cylinder(orc_scene* s, const float pos[3], float radius, float height, int res_x,
                           int res_y);

/* Grid bounds from the field: union of pos +- |size|/2 plus margin; dims = ceil(extent/cell)
 * (RectGrid::Cinit grid.cpp:3-8). */
void orc_grid_bounds(const float* pos, const float* size, int n, const float cell[3], float margin,
                     double gpos[3], int gdims[3]);

/* CSR cell -> heliostats (CGridHelioMatch grid.cpp:25-83).  Returns entries;
 * call with cell_start/entries NULL to count.  Conservative boxes unless
 * ORC_QUIRK_AABB_RADIUS. */
int64_t orc_grid_build(const orc_scene* s, uint32_t quirks, int32_t* cell_start, int32_t* entries);

/* Ray vs parallelogram (rayParallelogramIntersect global_function.cuh:78-105), double. */
int orc_ray_parallelogram(const double o[3], const double d[3], const double A[3], const double B[3],
                          const double C[3], double* t, double* u, double* v);

/* 3D-DDA any-hit (NotCollision rectgrid_raytracing.cu:38-117).  Returns 1 if
 * the ray hits another heliostat.  counters: [0] rect tests, [1] cells tested. */
int orc_dda_blocked(const orc_scene* s, const double o[3], const double d[3], int own,
                    uint32_t quirks, uint64_t counters[2]);

/* Same question answered by testing every heliostat (no grid). */
int orc_brute_blocked(const orc_scene* s, const double o[3], const double d[3], int own,
                      uint32_t quirks);

/* Receiver hit (receiver_drawing rectgrid_raytracing.cu:135-153):
 * returns 1 on hit and fills pixel (row*res_x+col, or -1 if off the map). */
int orc_receiver_hit(const orc_scene* s, const double o[3], const double d[3], uint32_t quirks,
                     int32_t* pixel, double* t_out);

/* Sample points.  Poisson: sequential dart throwing on a 2^-16 m lattice
 * with min spacing r, candidates in batches of 32 (Philox), accepted in
 * order; GRID: cell centres of pixel length pl (map_microhelio_centers
 * steps_for_raytracing.cu:4-22).  Writes float2 (x, z) mirror-centred and the
 * heliostat of each point.  Returns 0, or -1-h if heliostat h could not get
 * its points. */
int orc_points_poisson(const float* size, int n, int64_t total_points, float spacing,
                       uint64_t seed, float* xz, int32_t* helio);
int64_t orc_points_grid(const float* size, int n, float pl, float* xz, int32_t* helio);

typedef struct orc_trace_cfg {
  double sun_dir[3];
  double dni, rho;
  const float* cdf_x; const float* cdf_y; const float* slope; const float* bparams;
  uint64_t seed;
  uint32_t item;
  int64_t rays;
  int rays_per_point;
  const float* point_xz;  /* [2*points] */
  const int32_t* point_helio;
  const double* helio_weight; /* [n] area per point (Philox mode) */
  uint32_t quirks;
  int threads;            /* OpenMP threads (0 = all) */
  int64_t ray_begin, ray_end; /* sub-range to trace (end=0: all) */
  int deposit;            /* 0 nearest, 1 bilinear */
  int atten;              /* 0: eta = 1; 1: eta(d) of rectgrid_raytracing.cu:120-127 (disabled there) */
} orc_trace_cfg;

typedef struct orc_trace_out {
  uint8_t* flags;     /* [rays] or NULL (indexed ray - ray_begin) */
  int32_t* pixel;     /* [rays] or NULL */
  uint32_t* counts;   /* [res] or NULL */
  double* energy;     /* [res] or NULL */
  uint64_t stats[7];  /* rays, shadowed, blocked, hit, offmap, rect_tests, dda_cells */
} orc_trace_out;

/* Full Philox-mode pipeline of the GPU tracer, in double. */
void orc_trace_philox(const orc_scene* s, const orc_trace_cfg* c, orc_trace_out* out);

/* Table mode: the sampling structure of map_tracing
 * (rectgrid_raytracing.cu:164-196). */
void orc_trace_tables(const orc_scene* s, const orc_trace_cfg* c, const float* sun_local,
                      const float* turb_local, int64_t table_size, const int32_t* start,
                      int64_t points, orc_trace_out* out);

/* Per-ray sample of the Philox pipeline (for sampler tests): sun local
 * direction and perturbation local direction, double. */
void orc_ray_samples(const orc_trace_cfg* c, double sigma, uint64_t ray, double sun_local[3],
                     double turb_local[3]);

/* FP64 adjoint of the bilinear-deposition loss L = sum_p (scale*E_p - T_p)^2.
 * Forward: visibility with the scene's current geometry, bilinear deposit of
 * |sun . n'| * w at the receiver hit.  Gradient with respect to theta_h =
 * (aim offset along ew, along eh, extra tilt about u, about v) of every
 * heliostat: for each visible ray, central differences (step fd_h) of that
 * ray's value sum_c G_c e W_c, where G = dL/dE, with its random numbers and
 * visibility fixed -- the pathwise derivative, computed without the analytic
 * chain.  aim / normal_in / tilt0 as in orc_scene_aim.  energy [res],
 * grad [4n] (aim_w, aim_h, tilt_u, tilt_v per heliostat). */
void orc_adjoint(const orc_scene* s, const orc_trace_cfg* c, const float* aim, const float* normal_in,
                 const float* tilt0, const double ew[3], const double eh[3], const double* target, double scale,
                 double fd_h, double* energy, double* loss, double* grad);

/* Trimmed mean (trimmed_mean image_smooth.cu:10-58, heap.cuh:9-212).
 * method 0: sorted order statistics; 1: the reference's two-heap stream. */
void orc_smooth_u32(const uint32_t* in, float* out, int w, int h, int radius, float ratio,
                    int method);
void orc_smooth_f32(const float* in, float* out, int w, int h, int radius, float ratio, int method);

#ifdef __cplusplus
}
#endif
#endif
