/*
 * oracle.c — FP64 CPU restatement of the reference tracer.  TEST
 * INFRASTRUCTURE ONLY (see oracle.h): the checker for the CUDA path, never a
 * product code path.  Compiled with -ffp-contract=off so float replicas round
 * exactly as written.
 */
#include "oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPS 1e-6 /* global_constant.h:7 */
#define TAG_TRACE 0x51A7u
#define TAG_POISSON 0x9015u
#define POISSON_Q 65536.0 /* lattice: 2^-16 m */

/* ------------------------------------------------------------ Philox */
void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* the tracer's uniform: (k + 0.5) 2^-23, k the top 23 bits of the Philox word */
/* the ray sampler's uniform: (k + 0.5) 2^-23 with k the low 23 bits of w (u23f) */
static inline double u23(uint32_t w) { return ((double)(w & 0x7FFFFFu) + 0.5) * (1.0 / 8388608.0); }

/* ------------------------------------------------------------ Buie */
static float buie_core(float theta) {
  /* sunshape_intensity: 0.326*theta is a double product (scene_instance_process.cu:59) */
  return cosf((float)(0.326 * (double)theta)) / cosf((float)(0.308 * (double)theta));
}
static float buie_aureole_int(float theta, float k, float gamma) {
  /* inter_larger_465_intensity (scene_instance_process.cu:62-66) */
  return expf(k) / (gamma + 1) * powf(theta, gamma + 1);
}

void orc_buie_table(float csr, float* cdf_x, float* cdf_y, float* slope, float params[6]) {
  const int num_group = 1024;
  const float upper_lm = 4.65f;
  float k = 0.9f * logf(13.5f * csr) * powf(csr, -0.3f);
  float gamma = 2.2f * logf(0.52f * csr) * powf(csr, 0.43f) - 0.1f;
  float v465_930 = buie_aureole_int(9.3f, k, gamma) - buie_aureole_int(upper_lm, k, gamma);
  /* parameters_generate (scene_instance_process.cu:73-96) */
  float len = upper_lm / (float)num_group;
  float x = 0.0f;
  cdf_x[0] = 0.0f;
  cdf_y[0] = 0.0f;
  float hist_pre = buie_core(x), hist_cur, sub;
  for (int i = 1; i <= num_group; ++i) {
    x += len;
    hist_cur = buie_core(x);
    sub = (hist_pre + hist_cur) * len / 2.0f;
    cdf_x[i] = x;
    cdf_y[i] = sub + cdf_y[i - 1];
    slope[i - 1] = len / sub;
    hist_pre = hist_cur;
  }
  float core = cdf_y[num_group];
  params[0] = k;
  params[1] = gamma;
  params[2] = core;
  params[3] = core + v465_930;               /* A */
  params[4] = (gamma + 1) / expf(k);         /* B */
  params[5] = powf(4.65f, gamma + 1);        /* C */
}

int orc_max_less_index(const float* cdf_y, double value, int n) {
  int left = 0, right = n, mid;
  while (left <= right) {
    mid = (left + right) >> 1;
    if (value > (double)cdf_y[mid]) left = mid + 1;
    else if (value < (double)cdf_y[mid]) right = mid - 1;
    else return mid;
  }
  return right;
}

double orc_buie_sample(double u, const float* cdf_x, const float* cdf_y, const float* slope,
                       const float p[6]) {
  double uu = u * (double)p[3];
  if (uu < (double)p[2]) {
    int id = orc_max_less_index(cdf_y, uu, 1024);
    return (uu - (double)cdf_y[id]) * (double)slope[id] + (double)cdf_x[id];
  }
  return pow((uu - (double)p[2]) * (double)p[4] + (double)p[5], 1.0 / ((double)p[1] + 1.0));
}

/* ------------------------------------------------------------ vectors */
static inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void cross3(const double* a, const double* b, double* o) {
  double x = a[1] * b[2] - a[2] * b[1], y = a[2] * b[0] - a[0] * b[2], z = a[0] * b[1] - a[1] * b[0];
  o[0] = x; o[1] = y; o[2] = z;
}
static inline void normalize3(double* a) {
  double l = sqrt(dot3(a, a));
  a[0] /= l; a[1] /= l; a[2] /= l;
}
static inline void sub3(const double* a, const double* b, double* o) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }

/* frame of local2world: u = normalize(Y x n), v = normalize(u x n) (global_function.cuh:41-44) */
static void frame_of(const double n[3], uint32_t quirks, double f[9]) {
  if (fabs(n[0]) < ORC_EPS && fabs(n[2]) < ORC_EPS) {
    double s = (n[1] < 0 && !(quirks & ORC_QUIRK_ZENITH_FRAME)) ? -1.0 : 1.0;
    f[0] = 1; f[1] = 0; f[2] = 0;
    f[3] = 0; f[4] = s; f[5] = 0;
    f[6] = 0; f[7] = 0; f[8] = s;
    return;
  }
  double Y[3] = {0, 1, 0}, u[3], v[3];
  cross3(Y, n, u);
  normalize3(u);
  cross3(u, n, v);
  normalize3(v);
  f[0] = u[0]; f[1] = u[1]; f[2] = u[2];
  f[3] = n[0]; f[4] = n[1]; f[5] = n[2];
  f[6] = v[0]; f[7] = v[1]; f[8] = v[2];
}
static inline void apply_frame(const double f[9], const double d[3], double o[3]) {
  o[0] = d[0] * f[0] + d[1] * f[3] + d[2] * f[6];
  o[1] = d[0] * f[1] + d[1] * f[4] + d[2] * f[7];
  o[2] = d[0] * f[2] + d[1] * f[5] + d[2] * f[8];
}

void orc_local2world(const double d[3], const double n[3], uint32_t quirks, double out[3]) {
  double f[9];
  frame_of(n, quirks, f);
  apply_frame(f, d, out);
}

/* ------------------------------------------------------------ scene */
void orc_scene_aim(orc_scene* s, const double sun_in[3], const float* aim, const float* normal_in,
                   const float* tilt, uint32_t quirks) {
  double sun[3] = {sun_in[0], sun_in[1], sun_in[2]};
  normalize3(sun);
  for (int h = 0; h < s->n; ++h) {
    double p[3] = {s->pos[3 * h], s->pos[3 * h + 1], s->pos[3 * h + 2]};
    double n[3];
    if (normal_in) {
      n[0] = normal_in[3 * h]; n[1] = normal_in[3 * h + 1]; n[2] = normal_in[3 * h + 2];
      normalize3(n); /* Cset_normal(dir) heliostat.cpp:60-63 */
    } else {
      double a[3];
      if (aim) { a[0] = aim[3 * h]; a[1] = aim[3 * h + 1]; a[2] = aim[3 * h + 2]; }
      else { a[0] = s->recv_focus[0]; a[1] = s->recv_focus[1]; a[2] = s->recv_focus[2]; }
      double r[3];
      sub3(a, p, r);
      normalize3(r);
      sub3(r, sun, n); /* bisector, heliostat.cpp:51-58 */
      normalize3(n);
    }
    double f[9];
    if (tilt) {
      frame_of(n, quirks, f);
      double tx = tilt[2 * h], tz = tilt[2 * h + 1];
      for (int i = 0; i < 3; ++i) n[i] = n[i] + tx * f[i] + tz * f[6 + i];
      normalize3(n);
    }
    frame_of(n, quirks, f);
    memcpy(s->normal + 3 * h, n, sizeof(n));
    memcpy(s->frame + 9 * h, f, sizeof(f));
    double sx = s->size[3 * h], sy = s->size[3 * h + 1], sz = s->size[3 * h + 2];
    /* Cset_localvertex heliostat.cpp:30-36; v0, v1, v3 */
    double lv[3][3] = {{-sx / 2, sy / 2, -sz / 2}, {-sx / 2, sy / 2, sz / 2}, {sx / 2, sy / 2, -sz / 2}};
    for (int k = 0; k < 3; ++k) {
      double w[3];
      apply_frame(f, lv[k], w);
      s->vert[9 * h + 3 * k + 0] = w[0] + p[0];
      s->vert[9 * h + 3 * k + 1] = w[1] + p[1];
      s->vert[9 * h + 3 * k + 2] = w[2] + p[2];
    }
  }
}

/* rotateY (global_function.cuh:61-74); 1-cos^2 clamped at 0 */
static void rotate_y(const double o[3], const double a[3], const double b[3], double r[3]) {
  double c[3];
  cross3(a, b, c);
  double dir = c[1] > 0 ? 1.0 : -1.0;
  double cs = dot3(a, b);
  double t = 1 - cs * cs;
  double sn = dir * sqrt(t > 0 ? t : 0);
  r[0] = cs * o[0] + sn * o[2];
  r[1] = o[1];
  r[2] = -sn * o[0] + cs * o[2];
}

void orc_receiver_flat(orc_scene* s, const float pos[3], const float size[3], const float normal[3],
                       int face, int res_x, int res_y) {
  double x = size[0] / 2.0, y = size[1] / 2.0, z = size[2] / 2.0;
  double lv[4][3];
  double ln[3] = {0, 0, 0};
  switch (face) { /* receiver.cpp:30-83 */
    case 1:
      ln[0] = 1;
      lv[0][0] = x; lv[0][1] = -y; lv[0][2] = z;   lv[1][0] = x; lv[1][1] = y; lv[1][2] = z;
      lv[2][0] = x; lv[2][1] = y; lv[2][2] = -z;   lv[3][0] = x; lv[3][1] = -y; lv[3][2] = -z;
      break;
    case 2:
      ln[2] = -1;
      lv[0][0] = x; lv[0][1] = -y; lv[0][2] = -z;  lv[1][0] = x; lv[1][1] = y; lv[1][2] = -z;
      lv[2][0] = -x; lv[2][1] = y; lv[2][2] = -z;  lv[3][0] = -x; lv[3][1] = -y; lv[3][2] = -z;
      break;
    case 3:
      ln[0] = -1;
      lv[0][0] = -x; lv[0][1] = -y; lv[0][2] = -z; lv[1][0] = -x; lv[1][1] = y; lv[1][2] = -z;
      lv[2][0] = -x; lv[2][1] = y; lv[2][2] = z;   lv[3][0] = -x; lv[3][1] = -y; lv[3][2] = z;
      break;
    default:
      ln[2] = 1;
      lv[0][0] = -x; lv[0][1] = -y; lv[0][2] = z;  lv[1][0] = -x; lv[1][1] = y; lv[1][2] = z;
      lv[2][0] = x; lv[2][1] = y; lv[2][2] = z;    lv[3][0] = x; lv[3][1] = -y; lv[3][2] = z;
      break;
  }
  double nn[3] = {normal[0], normal[1], normal[2]};
  normalize3(nn);
  for (int k = 0; k < 4; ++k) {
    double r[3];
    rotate_y(lv[k], ln, nn, r);
    s->recv_v[3 * k + 0] = r[0] + pos[0];
    s->recv_v[3 * k + 1] = r[1] + pos[1];
    s->recv_v[3 * k + 2] = r[2] + pos[2];
  }
  for (int i = 0; i < 3; ++i) s->recv_focus[i] = (s->recv_v[i] + s->recv_v[6 + i]) / 2;
  s->recv_type = 0;
  s->res_x = res_x;
  s->res_y = res_y;
}

void orc_receiver_cylinder(orc_scene* s, const float pos[3], float radius, float height, int res_x,
                           int res_y) {
  s->recv_type = 1;
  s->cyl[0] = pos[0]; s->cyl[1] = pos[1]; s->cyl[2] = pos[2];
  s->cyl[3] = radius; s->cyl[4] = height;
  s->recv_focus[0] = pos[0];
  s->recv_focus[1] = (double)pos[1] + height / 2.0;
  s->recv_focus[2] = pos[2];
  s->res_x = res_x;
  s->res_y = res_y;
}

/* ------------------------------------------------------------ grid */
void orc_grid_bounds(const float* pos, const float* size, int n, const float cell[3], float margin,
                     double gpos[3], int gdims[3]) {
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int h = 0; h < n; ++h) {
    double sx = size[3 * h], sy = size[3 * h + 1], sz = size[3 * h + 2];
    double r = 0.5 * sqrt(sx * sx + sy * sy + sz * sz);
    double rq = sqrt(sqrt(sx * sx + sy * sy + sz * sz)) / 2.0; /* quirk box (grid.cpp:55-57) */
    if (rq > r) r = rq;
    for (int i = 0; i < 3; ++i) {
      double a = pos[3 * h + i] - r, b = pos[3 * h + i] + r;
      if (a < lo[i]) lo[i] = a;
      if (b > hi[i]) hi[i] = b;
    }
  }
  for (int i = 0; i < 3; ++i) {
    float g = (float)(lo[i] - margin);
    gpos[i] = g;
    double ext = (hi[i] + margin) - (double)g;
    int d = (int)ceil(ext / (double)cell[i]);
    gdims[i] = d < 1 ? 1 : d;
  }
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static void helio_cell_box(const orc_scene* s, int h, uint32_t quirks, int lo[3], int hi[3]) {
  if (quirks & ORC_QUIRK_AABB_RADIUS) {
    /* CGridHelioMatch (grid.cpp:53-61) + boxIntersect (grid.cpp:25-45), float */
    float sx = s->size[3 * h], sy = s->size[3 * h + 1], sz = s->size[3 * h + 2];
    float diag = sqrtf(sx * sx + sy * sy + sz * sz);
    float radius = sqrtf(diag) / 2;
    for (int i = 0; i < 3; ++i) {
      float gp = (float)s->gpos[i], gc = (float)s->gcell[i];
      float mn = s->pos[3 * h + i] - radius, mx = s->pos[3 * h + i] + radius;
      int a = (int)((mn - gp) / gc), b = (int)((mx - gp) / gc);
      lo[i] = clampi(a, 0, s->gdims[i] - 1);
      hi[i] = clampi(b, 0, s->gdims[i] - 1);
    }
    return;
  }
  const double* v = s->vert + 9 * h;
  double c[4][3];
  for (int i = 0; i < 3; ++i) {
    c[0][i] = v[i]; c[1][i] = v[3 + i]; c[2][i] = v[6 + i];
    c[3][i] = v[3 + i] + v[6 + i] - v[i];
  }
  for (int i = 0; i < 3; ++i) {
    double mn = c[0][i], mx = c[0][i];
    for (int k = 1; k < 4; ++k) { if (c[k][i] < mn) mn = c[k][i]; if (c[k][i] > mx) mx = c[k][i]; }
    int a = (int)floor((mn - s->gpos[i]) / s->gcell[i]);
    int b = (int)floor((mx - s->gpos[i]) / s->gcell[i]);
    lo[i] = clampi(a, 0, s->gdims[i] - 1);
    hi[i] = clampi(b, 0, s->gdims[i] - 1);
  }
}

int64_t orc_grid_build(const orc_scene* s, uint32_t quirks, int32_t* cell_start, int32_t* entries) {
  int64_t cells = (int64_t)s->gdims[0] * s->gdims[1] * s->gdims[2];
  int64_t total = 0;
  int32_t* cnt = (int32_t*)calloc((size_t)cells, sizeof(int32_t));
  for (int h = 0; h < s->n; ++h) {
    int lo[3], hi[3];
    helio_cell_box(s, h, quirks, lo, hi);
    for (int x = lo[0]; x <= hi[0]; ++x)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int z = lo[2]; z <= hi[2]; ++z) {
          int64_t c = ((int64_t)x * s->gdims[1] + y) * s->gdims[2] + z; /* grid.cpp:40 */
          cnt[c]++;
          total++;
        }
  }
  if (cell_start && entries) {
    cell_start[0] = 0;
    for (int64_t c = 0; c < cells; ++c) cell_start[c + 1] = cell_start[c] + cnt[c];
    memset(cnt, 0, (size_t)cells * sizeof(int32_t));
    for (int h = 0; h < s->n; ++h) { /* ascending id per cell, as the reference's push_back */
      int lo[3], hi[3];
      helio_cell_box(s, h, quirks, lo, hi);
      for (int x = lo[0]; x <= hi[0]; ++x)
        for (int y = lo[1]; y <= hi[1]; ++y)
          for (int z = lo[2]; z <= hi[2]; ++z) {
            int64_t c = ((int64_t)x * s->gdims[1] + y) * s->gdims[2] + z;
            entries[cell_start[c] + cnt[c]++] = h;
          }
    }
  }
  free(cnt);
  return total;
}

/* ------------------------------------------------------------ tracing */
int orc_ray_parallelogram(const double o[3], const double d[3], const double A[3], const double B[3],
                          const double C[3], double* t, double* u, double* v) {
  double E1[3], E2[3], pv[3], T[3], qv[3];
  sub3(B, A, E1);
  sub3(C, A, E2);
  cross3(d, E2, pv);
  double det = dot3(E1, pv);
  if (fabs(det) < ORC_EPS) return 0;
  double inv = 1.0 / det;
  sub3(o, A, T);
  *u = dot3(T, pv) * inv;
  if (*u < 0 || *u > 1) return 0;
  cross3(T, E1, qv);
  *v = dot3(d, qv) * inv;
  if (*v < 0 || *v > 1) return 0;
  *t = dot3(E2, qv) * inv;
  if (*t < ORC_EPS) return 0;
  return 1;
}

static int cell_hit(const orc_scene* s, int64_t c, const double o[3], const double d[3], int own,
                    uint32_t quirks, uint64_t* ctr) {
  if (ctr) ctr[1]++;
  for (int32_t e = s->cell_start[c]; e < s->cell_start[c + 1]; ++e) {
    int h = s->entries[e];
    if (h == own && !(quirks & ORC_QUIRK_SELF_HIT)) continue;
    if (ctr) ctr[0]++;
    const double* v = s->vert + 9 * h;
    double t, u, w;
    if (orc_ray_parallelogram(o, d, v, v + 3, v + 6, &t, &u, &w)) return 1;
  }
  return 0;
}

static inline double tmax_init(double dir, double interval, int idx, double cur) {
  return dir >= 0 ? (double)(idx + 1) * interval - cur : cur - (double)idx * interval; /* calTMax */
}
static inline double abs_divide(double num, double den) {
  if (den <= ORC_EPS && den >= -ORC_EPS) return (double)INT_MAX; /* absDivide */
  return fabs(num / den);
}

int orc_dda_blocked(const orc_scene* s, const double o[3], const double d[3], int own,
                    uint32_t quirks, uint64_t ctr[2]) {
  int idx[3], step[3];
  double rel[3], tmax[3], tdel[3];
  for (int i = 0; i < 3; ++i) {
    rel[i] = o[i] - s->gpos[i];
    idx[i] = clampi((int)floor(rel[i] / s->gcell[i]), 0, s->gdims[i] - 1);
    step[i] = d[i] >= 0 ? 1 : -1;
    tmax[i] = abs_divide(tmax_init(d[i], s->gcell[i], idx[i], rel[i]), d[i]);
    tdel[i] = abs_divide(s->gcell[i], d[i]);
  }
  const int gy = s->gdims[1], gz = s->gdims[2];
  if (!(quirks & ORC_QUIRK_SKIP_ORIGIN_CELL)) {
    if (cell_hit(s, ((int64_t)idx[0] * gy + idx[1]) * gz + idx[2], o, d, own, quirks, ctr)) return 1;
  }
  int guard = s->gdims[0] + s->gdims[1] + s->gdims[2] + 2;
  while (guard-- > 0) {
    int a;
    if (tmax[0] < tmax[1]) a = (tmax[0] < tmax[2]) ? 0 : 2;
    else a = (tmax[1] < tmax[2]) ? 1 : 2;
    idx[a] += step[a];
    if (idx[a] >= s->gdims[a] || idx[a] < 0) return 0;
    tmax[a] += tdel[a];
    if (cell_hit(s, ((int64_t)idx[0] * gy + idx[1]) * gz + idx[2], o, d, own, quirks, ctr)) return 1;
  }
  return 0;
}

int orc_brute_blocked(const orc_scene* s, const double o[3], const double d[3], int own,
                      uint32_t quirks) {
  for (int h = 0; h < s->n; ++h) {
    if (h == own && !(quirks & ORC_QUIRK_SELF_HIT)) continue;
    const double* v = s->vert + 9 * h;
    double t, u, w;
    if (orc_ray_parallelogram(o, d, v, v + 3, v + 6, &t, &u, &w)) return 1;
  }
  return 0;
}

/* unrolled cylinder: nearest intersection with the lateral surface,
 * column = azimuth atan2(dz, dx) in [0, 2pi), row = height fraction */
static int cylinder_hit(const orc_scene* s, const double o[3], const double d[3], double* t_out,
                        double* u_out, double* v_out) {
  double cx = s->cyl[0], y0 = s->cyl[1], cz = s->cyl[2], R = s->cyl[3], H = s->cyl[4];
  double ox = o[0] - cx, oz = o[2] - cz;
  double a = d[0] * d[0] + d[2] * d[2];
  if (a < 1e-18) return 0;
  double b = ox * d[0] + oz * d[2];
  double c = ox * ox + oz * oz - R * R;
  double disc = b * b - a * c;
  if (disc < 0) return 0;
  double sq = sqrt(disc);
  double ts[2] = {(-b - sq) / a, (-b + sq) / a};
  for (int i = 0; i < 2; ++i) {
    double t = ts[i];
    if (t < ORC_EPS) continue;
    double y = o[1] + t * d[1] - y0;
    if (y < 0 || y > H) continue;
    double px = ox + t * d[0], pz = oz + t * d[2];
    double phi = atan2(pz, px);
    if (phi < 0) phi += 2 * M_PI;
    *t_out = t;
    *u_out = y / H;
    *v_out = phi / (2 * M_PI);
    return 1;
  }
  return 0;
}

int orc_receiver_hit(const orc_scene* s, const double o[3], const double d[3], uint32_t quirks,
                     int32_t* pixel, double* t_out) {
  double t, u, v;
  int hit;
  if (s->recv_type == 1) {
    hit = cylinder_hit(s, o, d, &t, &u, &v);
  } else {
    hit = orc_ray_parallelogram(o, d, s->recv_v, s->recv_v + 3, s->recv_v + 9, &t, &u, &v);
  }
  if (!hit) return 0;
  if (t_out) *t_out = t;
  int row = (int)(u * s->res_y), col = (int)(v * s->res_x); /* rectgrid_raytracing.cu:144 */
  if (quirks & ORC_QUIRK_PIXEL_EDGE) {
    if (row >= s->res_y || col >= s->res_x) { *pixel = -1; return 1; }
  } else {
    if (row >= s->res_y) row = s->res_y - 1;
    if (col >= s->res_x) col = s->res_x - 1;
  }
  *pixel = row * s->res_x + col;
  return 1;
}

/* atmospheric transmittance over the slant range d (m): eta_aAlpha's
 * formula, commented out in the reference (rectgrid_raytracing.cu:120-127) */
static double orc_eta(int mode, double d) {
  if (mode != 1) return 1.0;
  return d <= 1000.0 ? 0.99331 - 0.0001176 * d + 1.97e-8 * d * d : exp(-0.0001106 * d);
}

static inline void angle2xyz(double theta, double phi, double o[3]) {
  /* global_function.cuh:175-180 */
  o[0] = sin(theta) * cos(phi);
  o[1] = cos(theta);
  o[2] = sin(theta) * sin(phi);
}

void orc_ray_samples(const orc_trace_cfg* c, double sigma, uint64_t ray, double sun_local[3],
                     double turb_local[3]) {
  uint32_t ctr[4] = {(uint32_t)ray, (uint32_t)(ray >> 32), c->item, TAG_TRACE};
  uint32_t key[2] = {(uint32_t)c->seed, (uint32_t)(c->seed >> 32)};
  uint32_t w[4];
  orc_philox4x32_10(ctr, key, w);
  double th = orc_buie_sample(u23(w[0]), c->cdf_x, c->cdf_y, c->slope, c->bparams) / 1000.0;
  angle2xyz(th, 2.0 * M_PI * u23(w[1]), sun_local);
  double z = sqrt(-2.0 * log(u23(w[2]))) * cos(2.0 * M_PI * u23(w[3]));
  /* the slope azimuth from the words' top bytes (the other uniforms use bits 0-22) */
  uint32_t extra = (w[0] >> 24) | ((w[1] >> 24) << 8) | ((w[2] >> 24) << 16) | (w[3] & 0xFF000000u);
  angle2xyz(sigma * z, 2.0 * M_PI * u23(extra), turb_local);
}

/* one ray given its local samples; the body of map_tracing
 * (rectgrid_raytracing.cu:168-195) */
static void trace_one(const orc_scene* s, const orc_trace_cfg* c, const double sunf[9],
                      const double sun_dir[3], int h, const float xz[2], const double sl[3],
                      const double tl[3], double weight, uint8_t* flag, int32_t* pix, double* e_out,
                      uint64_t* ctr, double* uv_out) {
  const double* f = s->frame + 9 * h;
  double lp[3] = {(double)xz[0], (double)s->size[3 * h + 1] / 2.0, (double)xz[1]};
  double o[3];
  apply_frame(f, lp, o);
  o[0] += s->pos[3 * h]; o[1] += s->pos[3 * h + 1]; o[2] += s->pos[3 * h + 2];
  double ws[3], dir[3];
  apply_frame(sunf, sl, ws);
  dir[0] = -ws[0]; dir[1] = -ws[1]; dir[2] = -ws[2];
  *flag = 0;
  *pix = -1;
  *e_out = 0;
  if (orc_dda_blocked(s, o, dir, h, c->quirks, ctr)) { *flag = ORC_RAY_SHADOWED; return; }
  double np[3];
  apply_frame(f, tl, np);
  normalize3(np);
  double di = dot3(ws, np);
  double r[3] = {ws[0] - 2 * di * np[0], ws[1] - 2 * di * np[1], ws[2] - 2 * di * np[2]};
  normalize3(r);
  if (orc_dda_blocked(s, o, r, h, c->quirks, ctr)) { *flag = ORC_RAY_BLOCKED; return; }
  double t;
  int32_t p;
  if (!orc_receiver_hit(s, o, r, c->quirks, &p, &t)) return;
  *flag = ORC_RAY_HIT;
  if (p < 0) { *flag |= ORC_RAY_OFFMAP; return; }
  *pix = p;
  *e_out = fabs(dot3(sun_dir, np)) * weight * orc_eta(c->atten, t); /* calEnergy rectgrid_raytracing.cu:129-133, eta :147 */
  (void)uv_out;
}

static void sun_frame(const orc_trace_cfg* c, double sd[3], double f[9]) {
  sd[0] = c->sun_dir[0]; sd[1] = c->sun_dir[1]; sd[2] = c->sun_dir[2];
  normalize3(sd);
  frame_of(sd, c->quirks, f);
}

static void accumulate_maps(const orc_scene* s, orc_trace_out* out, uint32_t** tc, double** te,
                            int nt) {
  int64_t res = (int64_t)s->res_x * s->res_y;
  for (int t = 0; t < nt; ++t) {
    if (out->counts)
      for (int64_t i = 0; i < res; ++i) out->counts[i] += tc[t][i];
    if (out->energy)
      for (int64_t i = 0; i < res; ++i) out->energy[i] += te[t][i];
    free(tc[t]);
    free(te[t]);
  }
}

static void trace_driver(const orc_scene* s, const orc_trace_cfg* c, const float* sun_local,
                         const float* turb_local, int64_t T, const int32_t* start,
                         orc_trace_out* out) {
  double sd[3], sf[9];
  sun_frame(c, sd, sf);
  int64_t r0 = c->ray_begin, r1 = c->ray_end > 0 ? c->ray_end : c->rays;
  int nt = 1;
#ifdef _OPENMP
  nt = c->threads > 0 ? c->threads : omp_get_max_threads();
#endif
  int64_t res = (int64_t)s->res_x * s->res_y;
  uint32_t** tc = (uint32_t**)calloc((size_t)nt, sizeof(uint32_t*));
  double** te = (double**)calloc((size_t)nt, sizeof(double*));
  uint64_t* st = (uint64_t*)calloc((size_t)nt * 8, sizeof(uint64_t));
  for (int t = 0; t < nt; ++t) {
    tc[t] = (uint32_t*)calloc((size_t)res, sizeof(uint32_t));
    te[t] = (double*)calloc((size_t)res, sizeof(double));
  }
#ifdef _OPENMP
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
#endif
  for (int64_t ray = r0; ray < r1; ++ray) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    int64_t m = ray / c->rays_per_point;
    int64_t j = ray % c->rays_per_point;
    int h = c->point_helio[m];
    double sl[3], tl[3], w;
    if (sun_local) {
      int64_t a = (start[m] + j) % T;
      /* rectgrid_raytracing.cu:183 in per-heliostat launches
       * (recthelio_tracing.cpp:46-80): the local index restarts at each
       * heliostat, so its points 0 and 1 both use point 0's offset */
      int64_t mp = m;
      if ((c->quirks & ORC_QUIRK_PREV_PERTURB) && m > 0 && c->point_helio[m - 1] == c->point_helio[m]) mp = m - 1;
      int64_t b = (start[mp] + j) % T;
      for (int i = 0; i < 3; ++i) { sl[i] = sun_local[3 * a + i]; tl[i] = turb_local[3 * b + i]; }
      w = 1.0;
    } else {
      orc_ray_samples(c, (double)s->sigma[h], (uint64_t)ray, sl, tl);
      w = c->helio_weight ? c->helio_weight[h] : 1.0;
    }
    uint8_t fl;
    int32_t px;
    double e;
    uint64_t ctr[2] = {0, 0};
    trace_one(s, c, sf, sd, h, c->point_xz + 2 * m, sl, tl, w, &fl, &px, &e, ctr, NULL);
    if (out->flags) out->flags[ray - r0] = fl;
    if (out->pixel) out->pixel[ray - r0] = px;
    uint64_t* my = st + 8 * tid;
    my[0]++;
    if (fl & ORC_RAY_SHADOWED) my[1]++;
    if (fl & ORC_RAY_BLOCKED) my[2]++;
    if (fl & ORC_RAY_HIT) my[3]++;
    if (fl & ORC_RAY_OFFMAP) my[4]++;
    my[5] += ctr[0];
    my[6] += ctr[1];
    if (px >= 0) {
      tc[tid][px] += 1;
      te[tid][px] += e;
    }
  }
  memset(out->stats, 0, sizeof(out->stats));
  for (int t = 0; t < nt; ++t)
    for (int k = 0; k < 7; ++k) out->stats[k] += st[8 * t + k];
  free(st);
  accumulate_maps(s, out, tc, te, nt);
  free(tc);
  free(te);
}

void orc_trace_philox(const orc_scene* s, const orc_trace_cfg* c, orc_trace_out* out) {
  trace_driver(s, c, NULL, NULL, 0, NULL, out);
}

void orc_trace_tables(const orc_scene* s, const orc_trace_cfg* c, const float* sun_local,
                      const float* turb_local, int64_t T, const int32_t* start, int64_t points,
                      orc_trace_out* out) {
  (void)points;
  trace_driver(s, c, sun_local, turb_local, T, start, out);
}

/* ------------------------------------------------------------ points */
int64_t orc_points_grid(const float* size, int n, float pl, float* xz, int32_t* helio) {
  int64_t g = 0;
  for (int h = 0; h < n; ++h) {
    float sx = size[3 * h], sz = size[3 * h + 2];
    /* set_microhelio_centers (steps_for_raytracing.cu:74-82), 1x1 facets */
    int rows = (int)(sz / pl), cols = (int)(sx / pl);
    for (int r = 0; r < rows; ++r)
      for (int cc = 0; cc < cols; ++cc) {
        if (xz) {
          float x = (float)cc * pl;
          x = x + pl / 2;
          x = x - sx / 2;
          float z = (float)r * pl;
          z = z + pl / 2;
          z = z - sz / 2;
          xz[2 * g] = x;
          xz[2 * g + 1] = z;
          helio[g] = h;
        }
        ++g;
      }
  }
  return g;
}

static int64_t isqrt64(int64_t v) {
  int64_t r = (int64_t)sqrt((double)v);
  while (r * r > v) --r;
  while ((r + 1) * (r + 1) <= v) ++r;
  return r;
}

int orc_points_poisson(const float* size, int n, int64_t total_points, float spacing,
                       uint64_t seed, float* xz, int32_t* helio) {
  int64_t q = total_points / n, rem = total_points % n;
  int64_t base = 0;
  int64_t Rq = (int64_t)((double)spacing * POISSON_Q);
  int64_t R2 = Rq * Rq;
  int64_t cq = isqrt64(R2 / 2);
  if (cq < 1) cq = 1;
  int64_t nb = (Rq + cq - 1) / cq;
  uint32_t key[2] = {(uint32_t)seed ^ 0x5A17C0DEu, (uint32_t)(seed >> 32) ^ 0x0B5E55EDu};
  for (int h = 0; h < n; ++h) {
    int64_t P = q + (h < rem ? 1 : 0);
    float sx = size[3 * h], sz = size[3 * h + 2];
    int64_t W = (int64_t)((double)sx * POISSON_Q), H = (int64_t)((double)sz * POISSON_Q);
    int64_t gx = (W + cq - 1) / cq, gz = (H + cq - 1) / cq;
    int32_t* grid = (int32_t*)malloc((size_t)(gx * gz) * sizeof(int32_t));
    for (int64_t i = 0; i < gx * gz; ++i) grid[i] = -1;
    int64_t* px = (int64_t*)malloc((size_t)(P > 0 ? P : 1) * 2 * sizeof(int64_t));
    int64_t got = 0;
    int64_t max_batches = (64 * P + 1023) / 32 + 32;
    for (int64_t b = 0; b < max_batches && got < P; ++b) {
      for (int lane = 0; lane < 32 && got < P; ++lane) {
        uint32_t ctr[4] = {(uint32_t)h, (uint32_t)(b * 32 + lane), (uint32_t)((b * 32 + lane) >> 32), TAG_POISSON};
        uint32_t w[4];
        orc_philox4x32_10(ctr, key, w);
        int64_t ix = (int64_t)(((uint64_t)w[0] * (uint64_t)W) >> 32);
        int64_t iz = (int64_t)(((uint64_t)w[1] * (uint64_t)H) >> 32);
        int64_t cx = ix / cq, cz = iz / cq;
        int ok = 1;
        for (int64_t dx = -nb; dx <= nb && ok; ++dx)
          for (int64_t dz = -nb; dz <= nb && ok; ++dz) {
            int64_t x = cx + dx, z = cz + dz;
            if (x < 0 || z < 0 || x >= gx || z >= gz) continue;
            int32_t k = grid[x * gz + z];
            if (k < 0) continue;
            int64_t ddx = px[2 * k] - ix, ddz = px[2 * k + 1] - iz;
            if (ddx * ddx + ddz * ddz < R2) ok = 0;
          }
        if (!ok) continue;
        grid[cx * gz + cz] = (int32_t)got;
        px[2 * got] = ix;
        px[2 * got + 1] = iz;
        ++got;
      }
    }
    if (got < P) { free(grid); free(px); return -1 - h; }
    for (int64_t k = 0; k < P; ++k) {
      if (xz) {
        float x = (float)px[2 * k] * (1.0f / 65536.0f);
        float z = (float)px[2 * k + 1] * (1.0f / 65536.0f);
        xz[2 * (base + k)] = x - 0.5f * sx;
        xz[2 * (base + k) + 1] = z - 0.5f * sz;
      }
      if (helio) helio[base + k] = h;
    }
    base += P;
    free(grid);
    free(px);
  }
  return 0;
}

/* ------------------------------------------------------------ smoothing */
/* Heap (heap.cuh:9-127) with elements[1..numElems-1]; cmp: larger / smaller */
typedef struct { int num, max; float* e; int is_max; } orc_heap;
static inline int hcmp(const orc_heap* hp, float a, float b) { return hp->is_max ? (a > b) : (a < b); }
static void heap_insert(orc_heap* hp, float el) {
  if (hp->num == hp->max) return;
  int i = hp->num++;
  for (; i != 1 && hcmp(hp, el, hp->e[i / 2]); i /= 2) hp->e[i] = hp->e[i / 2];
  hp->e[i] = el;
}
static void heap_delete_and_insert(orc_heap* hp, float el) {
  if (hp->num == 1) return;
  int i = 1, c;
  for (; 2 * i < hp->num;) {
    c = (2 * i + 1 >= hp->num || hcmp(hp, hp->e[2 * i], hp->e[2 * i + 1])) ? 2 * i : 2 * i + 1;
    if (hcmp(hp, hp->e[c], el)) { hp->e[i] = hp->e[c]; i = c; }
    else break;
  }
  hp->e[i] = el;
}
static float heap_sum(const orc_heap* hp) {
  float s = 0.0f;
  for (int i = 1; i < hp->num; ++i) s += hp->e[i];
  return s;
}

static int cmp_u32(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : (x > y);
}
static int cmp_f32(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  return x < y ? -1 : (x > y);
}

static void smooth_heaps_at(const float* in, int w, int h, int x, int y, int radius, float ratio,
                            float* out, float* scratch) {
  int lx = x - radius >= 0 ? x - radius : 0, ly = y - radius >= 0 ? y - radius : 0;
  int rx = x + radius < w ? x + radius : w - 1, ry = y + radius < h ? y + radius : h - 1;
  int cnt = (rx - lx + 1) * (ry - ly + 1);
  int k = (int)((float)cnt * ratio);
  orc_heap mx = {1, k + 1, scratch, 1}, mn = {1, k + 1, scratch + k + 2, 0};
  float value = 0.0f;
  for (int r = ly; r <= ry; ++r)
    for (int c = lx; c <= rx; ++c) {
      float cur = in[(int64_t)r * w + c];
      value += cur;
      if (mx.num != mx.max) { heap_insert(&mx, cur); heap_insert(&mn, cur); }
      else if (mx.num > 1 && cur < mx.e[1]) heap_delete_and_insert(&mx, cur);
      else if (mn.num > 1 && cur > mn.e[1]) heap_delete_and_insert(&mn, cur);
    }
  out[(int64_t)y * w + x] = (value - heap_sum(&mx) - heap_sum(&mn)) / (float)(cnt - 2 * k);
}

void orc_smooth_f32(const float* in, float* out, int w, int h, int radius, float ratio, int method) {
  int win = (2 * radius + 1) * (2 * radius + 1);
#ifdef _OPENMP
#pragma omp parallel
#endif
  {
    float* buf = (float*)malloc((size_t)(2 * win + 8) * sizeof(float));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        if (method == 1) { smooth_heaps_at(in, w, h, x, y, radius, ratio, out, buf); continue; }
        int lx = x - radius >= 0 ? x - radius : 0, ly = y - radius >= 0 ? y - radius : 0;
        int rx = x + radius < w ? x + radius : w - 1, ry = y + radius < h ? y + radius : h - 1;
        int cnt = 0;
        for (int r = ly; r <= ry; ++r)
          for (int c = lx; c <= rx; ++c) buf[cnt++] = in[(int64_t)r * w + c];
        int k = (int)((float)cnt * ratio);
        qsort(buf, (size_t)cnt, sizeof(float), cmp_f32);
        double sum = 0;
        for (int i = k; i < cnt - k; ++i) sum += buf[i];
        out[(int64_t)y * w + x] = (float)(sum / (double)(cnt - 2 * k));
      }
    free(buf);
  }
}

void orc_smooth_u32(const uint32_t* in, float* out, int w, int h, int radius, float ratio,
                    int method) {
  if (method == 1) {
    int64_t n = (int64_t)w * h;
    float* f = (float*)malloc((size_t)n * sizeof(float));
    for (int64_t i = 0; i < n; ++i) f[i] = (float)in[i];
    orc_smooth_f32(f, out, w, h, radius, ratio, 1);
    free(f);
    return;
  }
  int win = (2 * radius + 1) * (2 * radius + 1);
#ifdef _OPENMP
#pragma omp parallel
#endif
  {
    uint32_t* buf = (uint32_t*)malloc((size_t)(win + 8) * sizeof(uint32_t));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        int lx = x - radius >= 0 ? x - radius : 0, ly = y - radius >= 0 ? y - radius : 0;
        int rx = x + radius < w ? x + radius : w - 1, ry = y + radius < h ? y + radius : h - 1;
        int cnt = 0;
        for (int r = ly; r <= ry; ++r)
          for (int c = lx; c <= rx; ++c) buf[cnt++] = in[(int64_t)r * w + c];
        int k = (int)((float)cnt * ratio);
        qsort(buf, (size_t)cnt, sizeof(uint32_t), cmp_u32);
        uint64_t sum = 0;
        for (int i = k; i < cnt - k; ++i) sum += buf[i];
        out[(int64_t)y * w + x] = (float)sum / (float)(cnt - 2 * k);
      }
    free(buf);
  }
}

/* ------------------------------------------------------------ adjoint */
/* Heliostat frame for parameters th = (aim offset along ew, along eh, extra
 * tilt about u0, about v0), following orc_scene_aim. */
static void adj_frame(const orc_scene* s, int h, const double sun[3], const float* aim, const float* normal_in,
                      const float* tilt0, const double ew[3], const double eh[3], const double th[4], double f[9]) {
  double p[3] = {s->pos[3 * h], s->pos[3 * h + 1], s->pos[3 * h + 2]};
  double n[3];
  if (normal_in) {
    n[0] = normal_in[3 * h]; n[1] = normal_in[3 * h + 1]; n[2] = normal_in[3 * h + 2];
    normalize3(n);
  } else {
    double a[3], r[3];
    for (int i = 0; i < 3; ++i) a[i] = (aim ? (double)aim[3 * h + i] : s->recv_focus[i]) + th[0] * ew[i] + th[1] * eh[i];
    sub3(a, p, r);
    normalize3(r);
    sub3(r, sun, n);
    normalize3(n);
  }
  double tx = (tilt0 ? (double)tilt0[2 * h] : 0.0) + th[2], tz = (tilt0 ? (double)tilt0[2 * h + 1] : 0.0) + th[3];
  if (tilt0 || th[2] != 0.0 || th[3] != 0.0) {
    double f0[9];
    frame_of(n, 0, f0);
    for (int i = 0; i < 3; ++i) n[i] = n[i] + tx * f0[i] + tz * f0[6 + i];
    normalize3(n);
  }
  frame_of(n, 0, f);
}

/* origin, perturbed normal and reflected direction of a ray for frame f */
static void adj_ray(const orc_scene* s, int h, const double f[9], const float xz[2], const double ws[3],
                    const double tl[3], double o[3], double np[3], double r[3]) {
  double lp[3] = {(double)xz[0], (double)s->size[3 * h + 1] / 2.0, (double)xz[1]};
  apply_frame(f, lp, o);
  o[0] += s->pos[3 * h]; o[1] += s->pos[3 * h + 1]; o[2] += s->pos[3 * h + 2];
  apply_frame(f, tl, np);
  normalize3(np);
  double di = dot3(ws, np);
  for (int i = 0; i < 3; ++i) r[i] = ws[i] - 2 * di * np[i];
  normalize3(r);
}

/* receiver-plane coordinates (u along v1-v0, v along v3-v0), no bounds */
static void adj_plane_uv(const orc_scene* s, const double o[3], const double d[3], double* u, double* v) {
  double E1[3], E2[3], T[3], pv[3], qv[3];
  sub3(s->recv_v + 3, s->recv_v, E1);
  sub3(s->recv_v + 9, s->recv_v, E2);
  cross3(d, E2, pv);
  double inv = 1.0 / dot3(E1, pv);
  sub3(o, s->recv_v, T);
  *u = dot3(T, pv) * inv;
  cross3(T, E1, qv);
  *v = dot3(d, qv) * inv;
}

/* sum over the bilinear corners of map[c] * W_c (corners off the map add 0) */
static double adj_bilinear(const orc_scene* s, double u, double v, const double* map, double* w4, int* c4) {
  double px = v * s->res_x - 0.5, py = u * s->res_y - 0.5;
  double i0 = floor(px), j0 = floor(py), fx = px - i0, fy = py - j0;
  double w[4] = {(1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy};
  double acc = 0;
  for (int k = 0; k < 4; ++k) {
    int ci = (int)i0 + (k & 1), cj = (int)j0 + (k >> 1);
    int ok = ci >= 0 && cj >= 0 && ci < s->res_x && cj < s->res_y;
    if (w4) { w4[k] = w[k]; c4[k] = ok ? cj * s->res_x + ci : -1; }
    if (ok && map) acc += map[cj * s->res_x + ci] * w[k];
  }
  return acc;
}

void orc_adjoint(const orc_scene* s, const orc_trace_cfg* c, const float* aim, const float* normal_in,
                 const float* tilt0, const double ew[3], const double eh[3], const double* target, double scale,
                 double fd_h, double* energy, double* loss, double* grad) {
  double sd[3], sf[9];
  sun_frame(c, sd, sf);
  int nt = 1;
#ifdef _OPENMP
  nt = c->threads > 0 ? c->threads : omp_get_max_threads();
#endif
  int64_t res = (int64_t)s->res_x * s->res_y;
  int64_t rays = c->ray_end > 0 ? c->ray_end : c->rays;
  uint8_t* vis = (uint8_t*)calloc((size_t)rays, 1);
  double* te = (double*)calloc((size_t)nt * res, sizeof(double));
  /* forward: visibility with the scene's geometry, bilinear deposit */
#ifdef _OPENMP
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
#endif
  for (int64_t ray = 0; ray < rays; ++ray) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    int64_t m = ray / c->rays_per_point;
    int h = c->point_helio[m];
    double sl[3], tl[3], ws[3], dir[3], o[3], np[3], r[3];
    orc_ray_samples(c, (double)s->sigma[h], (uint64_t)ray, sl, tl);
    apply_frame(sf, sl, ws);
    adj_ray(s, h, s->frame + 9 * h, c->point_xz + 2 * m, ws, tl, o, np, r);
    dir[0] = -ws[0]; dir[1] = -ws[1]; dir[2] = -ws[2];
    if (orc_dda_blocked(s, o, dir, h, 0, NULL)) continue;
    if (orc_dda_blocked(s, o, r, h, 0, NULL)) continue;
    double t, u, v;
    if (!orc_ray_parallelogram(o, r, s->recv_v, s->recv_v + 3, s->recv_v + 9, &t, &u, &v)) continue;
    vis[ray] = 1;
    double e = fabs(dot3(sd, np)) * (c->helio_weight ? c->helio_weight[h] : 1.0);
    double w4[4];
    int c4[4];
    adj_bilinear(s, u, v, NULL, w4, c4);
    for (int k = 0; k < 4; ++k)
      if (c4[k] >= 0) te[(int64_t)tid * res + c4[k]] += e * w4[k];
  }
  for (int64_t i = 0; i < res; ++i) {
    double acc = 0;
    for (int t = 0; t < nt; ++t) acc += te[(int64_t)t * res + i];
    energy[i] = acc;
  }
  double L = 0;
  double* G = (double*)malloc((size_t)res * sizeof(double));
  for (int64_t i = 0; i < res; ++i) {
    double d = scale * energy[i] - target[i];
    L += d * d;
    G[i] = 2.0 * d * scale;
  }
  *loss = L;
  /* backward: per-ray central differences of sum_c G_c e W_c */
  double* tg = (double*)calloc((size_t)nt * 4 * s->n, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
#endif
  for (int64_t ray = 0; ray < rays; ++ray) {
    if (!vis[ray]) continue;
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    int64_t m = ray / c->rays_per_point;
    int h = c->point_helio[m];
    double w = c->helio_weight ? c->helio_weight[h] : 1.0;
    double sl[3], tl[3], ws[3];
    orc_ray_samples(c, (double)s->sigma[h], (uint64_t)ray, sl, tl);
    apply_frame(sf, sl, ws);
    for (int k = 0; k < 4; ++k) {
      double val[2];
      /* tilts move the hit ~1000x more per unit than aim offsets: a smaller
       * step keeps the difference away from the bilinear weights' kinks */
      const double step = k < 2 ? fd_h : fd_h * 1e-3;
      for (int sgn = 0; sgn < 2; ++sgn) {
        double th[4] = {0, 0, 0, 0}, f[9], o[3], np[3], r[3], u, v;
        th[k] = sgn ? -step : step;
        adj_frame(s, h, sd, aim, normal_in, tilt0, ew, eh, th, f);
        adj_ray(s, h, f, c->point_xz + 2 * m, ws, tl, o, np, r);
        adj_plane_uv(s, o, r, &u, &v);
        val[sgn] = fabs(dot3(sd, np)) * w * adj_bilinear(s, u, v, G, NULL, NULL);
      }
      tg[((int64_t)tid * s->n + h) * 4 + k] += (val[0] - val[1]) / (2.0 * step);
    }
  }
  for (int64_t i = 0; i < 4 * (int64_t)s->n; ++i) {
    double acc = 0;
    for (int t = 0; t < nt; ++t) acc += tg[(int64_t)t * 4 * s->n + i];
    grad[i] = acc;
  }
  free(tg);
  free(G);
  free(te);
  free(vis);
}
