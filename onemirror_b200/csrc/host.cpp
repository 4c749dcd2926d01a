// host.cpp — host-only parts of the C-ABI: error strings, sun direction,
// Buie table builder, receiver geometry, radial-staggered layout generator
// and the .scn scene-file parser.  None of these touch the GPU.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "internal.hpp"

namespace qm {

static thread_local std::string g_last_error;

qmcrt_status set_error(qmcrt_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

qmcrt_status cuda_error(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a sticky launch error so later calls can report their own
  if (e == cudaErrorMemoryAllocation) return set_error(QMCRT_ERR_OUT_OF_MEMORY, m);
  return set_error(QMCRT_ERR_CUDA, m);
}

// sunshape_intensity (scene_instance_process.cu:56-60): the constants multiply
// a float by a double literal, so the product is formed in double.
static float buie_core(float theta) {
  return cosf((float)(0.326 * (double)theta)) / cosf((float)(0.308 * (double)theta));
}
// inter_larger_465_intensity (scene_instance_process.cu:62-66)
static float buie_aureole(float theta, float k, float gamma) {
  return expf(k) / (gamma + 1) * powf(theta, gamma + 1);
}

void buie_build(float csr, float* cdf_x, float* cdf_y, float* slope, float params[6]) {
  const int groups = 1024;
  const float upper = 4.65f;
  // k and gamma of the Buie model (scene_instance_process.cu:171-172)
  float k = 0.9f * logf(13.5f * csr) * powf(csr, -0.3f);
  float gamma = 2.2f * logf(0.52f * csr) * powf(csr, 0.43f) - 0.1f;
  float tail = buie_aureole(9.3f, k, gamma) - buie_aureole(upper, k, gamma);
  // trapezoid CDF of the core (parameters_generate, :73-96)
  float step = upper / (float)groups;
  float x = 0.0f, prev = buie_core(x);
  cdf_x[0] = 0.0f;
  cdf_y[0] = 0.0f;
  for (int i = 1; i <= groups; ++i) {
    x += step;
    float cur = buie_core(x);
    float area = (prev + cur) * step / 2.0f;
    cdf_x[i] = x;
    cdf_y[i] = area + cdf_y[i - 1];
    slope[i - 1] = step / area;
    prev = cur;
  }
  float core = cdf_y[groups];
  params[0] = k;
  params[1] = gamma;
  params[2] = core;
  params[3] = core + tail;             // A (:198)
  params[4] = (gamma + 1) / expf(k);   // B (:199)
  params[5] = powf(4.65f, gamma + 1);  // C (:200)
}

static void nrm(double* a) {
  double l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  a[0] /= l;
  a[1] /= l;
  a[2] /= l;
}

qmcrt_status receiver_setup(const qmcrt_receiver& r, ReceiverGeom* g) {
  if (r.res_x <= 0 || r.res_y <= 0 || (int64_t)r.res_x * r.res_y > (1 << 26))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "receiver resolution out of range");
  g->type = r.type;
  g->res_x = r.res_x;
  g->res_y = r.res_y;
  if (r.type == QMCRT_RECEIVER_CYLINDER) {
    if (!(r.size[0] > 0) || !(r.size[1] > 0))
      return set_error(QMCRT_ERR_INVALID_ARGUMENT, "cylinder radius/height must be positive");
    g->cyl[0] = r.pos[0];
    g->cyl[1] = r.pos[1];
    g->cyl[2] = r.pos[2];
    g->cyl[3] = r.size[0];
    g->cyl[4] = r.size[1];
    g->focus[0] = r.pos[0];
    g->focus[1] = (double)r.pos[1] + r.size[1] / 2.0;
    g->focus[2] = r.pos[2];
    double circ = 2.0 * M_PI * r.size[0];
    g->pixel_area = (circ / r.res_x) * ((double)r.size[1] / r.res_y);
    return QMCRT_OK;
  }
  if (r.type != QMCRT_RECEIVER_FLAT)
    return set_error(QMCRT_ERR_NOT_SUPPORTED, "receiver type not supported");
  if (r.face < 0 || r.face > 3) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "receiver face must be 0..3");
  double x = r.size[0] / 2.0, y = r.size[1] / 2.0, z = r.size[2] / 2.0;
  // local corners and normals per face (receiver.cpp:30-83)
  double lv[4][3], ln[3] = {0, 0, 0};
  const double faces[4][4][3] = {
      {{-x, -y, z}, {-x, y, z}, {x, y, z}, {x, -y, z}},
      {{x, -y, z}, {x, y, z}, {x, y, -z}, {x, -y, -z}},
      {{x, -y, -z}, {x, y, -z}, {-x, y, -z}, {-x, -y, -z}},
      {{-x, -y, -z}, {-x, y, -z}, {-x, y, z}, {-x, -y, z}}};
  const double lnorm[4][3] = {{0, 0, 1}, {1, 0, 0}, {0, 0, -1}, {-1, 0, 0}};
  std::memcpy(lv, faces[r.face], sizeof(lv));
  std::memcpy(ln, lnorm[r.face], sizeof(ln));
  double nn[3] = {r.normal[0], r.normal[1], r.normal[2]};
  if (nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2] <= 0)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "receiver normal is zero");
  nrm(nn);
  // rotateY (global_function.cuh:61-74); 1 - cos^2 clamped at 0
  double cy = ln[2] * nn[0] - ln[0] * nn[2];
  double dir = cy > 0 ? 1.0 : -1.0;
  double cs = ln[0] * nn[0] + ln[1] * nn[1] + ln[2] * nn[2];
  double t = 1 - cs * cs;
  double sn = dir * std::sqrt(t > 0 ? t : 0);
  double w[4][3];
  for (int k = 0; k < 4; ++k) {
    w[k][0] = cs * lv[k][0] + sn * lv[k][2] + r.pos[0];
    w[k][1] = lv[k][1] + r.pos[1];
    w[k][2] = -sn * lv[k][0] + cs * lv[k][2] + r.pos[2];
  }
  for (int i = 0; i < 3; ++i) {
    g->v0[i] = w[0][i];
    g->v1[i] = w[1][i];
    g->v3[i] = w[3][i];
    g->focus[i] = (w[0][i] + w[2][i]) / 2;  // Cset_focuscenter (receiver.cpp:47-50)
  }
  double e1 = 0, e2 = 0;
  for (int i = 0; i < 3; ++i) {
    e1 += (w[1][i] - w[0][i]) * (w[1][i] - w[0][i]);
    e2 += (w[3][i] - w[0][i]) * (w[3][i] - w[0][i]);
  }
  g->pixel_area = (std::sqrt(e2) / r.res_x) * (std::sqrt(e1) / r.res_y);
  return QMCRT_OK;
}

// Host Philox for the layout jitter (same generator as the kernels).
static void philox_host(uint32_t c0, uint32_t c1, uint64_t seed, uint32_t out[4]) {
  uint4 r = philox4x32_10(make_uint4(c0, c1, 0, 0x1A70u), make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
  out[3] = r.w;
}

struct Slot {
  double r, az;
  int ring;
};

// Rings of staggered positions at centre spacing s over [r_min, r_max].
static void layout_slots(const qmcrt_layout_params& p, double s, std::vector<Slot>* out, int64_t stop_at) {
  out->clear();
  const double span = std::min(360.0, std::max(1.0, (double)p.az_span_deg)) * M_PI / 180.0;
  const double c = p.az_center_deg * M_PI / 180.0;
  const bool full = p.az_span_deg >= 360.0f;
  const double dr = s * std::sqrt(3.0) / 2.0;
  int ring = 0;
  for (double r = p.r_min; r <= p.r_max + 1e-9; r += dr, ++ring) {
    int m = (int)std::floor(span * r / s);
    if (m < 1) continue;
    double step = span / m;
    double off = (ring & 1) ? 0.5 : 0.0;
    for (int i = 0; i < m; ++i) {
      double a = full ? c + (i + off) * step : c - span / 2 + (i + 0.25 + 0.5 * off) * step;
      out->push_back({r, a, ring});
    }
    if (stop_at > 0 && (int64_t)out->size() >= stop_at) return;
  }
}

}  // namespace qm

using namespace qm;

extern "C" {

const char* qmcrt_version(void) { return "qmcrt-b200 1.0 (sm_100a)"; }

const char* qmcrt_last_error(void) { return g_last_error.c_str(); }

const char* qmcrt_status_string(qmcrt_status s) {
  switch (s) {
    case QMCRT_OK: return "ok";
    case QMCRT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case QMCRT_ERR_CUDA: return "CUDA error";
    case QMCRT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case QMCRT_ERR_NOT_SUPPORTED: return "not supported";
    case QMCRT_ERR_TIMEOUT: return "device wait timed out";
    case QMCRT_ERR_SAMPLING: return "sample placement failed";
    case QMCRT_ERR_INTERNAL: return "internal error";
  }
  return "unknown status";
}

qmcrt_status qmcrt_sun_direction(float elevation_deg, float azimuth_deg, float dir_out[3]) {
  if (!dir_out) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "dir_out is NULL");
  if (!(elevation_deg > -90.f && elevation_deg <= 90.f))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "elevation out of range");
  // main.cpp:71-73 with zenith = 90 - elevation
  double zen = (90.0 - elevation_deg) * M_PI / 180.0, az = azimuth_deg * M_PI / 180.0;
  dir_out[0] = (float)(-std::sin(zen) * std::sin(az));
  dir_out[1] = (float)(-std::cos(zen));
  dir_out[2] = (float)(std::sin(zen) * std::cos(az));
  return QMCRT_OK;
}

float qmcrt_solar_declination(int32_t day_of_year) {
  // Cooper (1969): 23.45 deg * sin(360 deg * (284 + n) / 365)
  return (float)(23.45 * std::sin(2.0 * M_PI * (284.0 + day_of_year) / 365.0));
}

qmcrt_status qmcrt_solar_position(float latitude_deg, float declination_deg, float hour_angle_deg,
                                  float* elevation_deg, float* azimuth_deg) {
  if (!elevation_deg || !azimuth_deg) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL output");
  if (!(std::fabs(latitude_deg) <= 90.f) || !(std::fabs(declination_deg) <= 23.5f))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "latitude or declination out of range");
  const double d2r = M_PI / 180.0;
  double phi = latitude_deg * d2r, dec = declination_deg * d2r, h = hour_angle_deg * d2r;
  // spherical astronomy: sin(el) = sin(phi) sin(dec) + cos(phi) cos(dec) cos(h)
  double se = std::sin(phi) * std::sin(dec) + std::cos(phi) * std::cos(dec) * std::cos(h);
  se = std::max(-1.0, std::min(1.0, se));
  double el = std::asin(se);
  // azimuth from north, clockwise: east in the morning (h < 0), west after noon
  double ca = (std::sin(dec) - se * std::sin(phi)) / std::max(1e-12, std::cos(el) * std::cos(phi));
  ca = std::max(-1.0, std::min(1.0, ca));
  double az = std::acos(ca);
  if (h > 0) az = 2.0 * M_PI - az;
  *elevation_deg = (float)(el / d2r);
  *azimuth_deg = (float)(az / d2r);
  return QMCRT_OK;
}

qmcrt_status qmcrt_buie_table(float csr, float* cdf_x, float* cdf_y, float* slope, float params_out[6]) {
  if (!cdf_x || !cdf_y || !slope || !params_out)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL output");
  if (!(csr > 0.f && csr < 1.f)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "csr must be in (0,1)");
  buie_build(csr, cdf_x, cdf_y, slope, params_out);
  return QMCRT_OK;
}

qmcrt_status qmcrt_layout_radial_staggered(const qmcrt_layout_params* p, float* h_pos, int32_t capacity,
                                           int32_t* n_out) {
  if (!p || !n_out) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (p->n <= 0 || !(p->helio_w > 0) || !(p->helio_h > 0) || !(p->r_min > 0) || !(p->r_max >= p->r_min))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad layout parameters");
  double diag = std::sqrt((double)p->helio_w * p->helio_w + (double)p->helio_h * p->helio_h);
  double smin = diag * 1.05 + 2.0 * p->jitter;
  double s = p->spacing;
  std::vector<Slot> slots;
  if (s <= 0) {
    // largest spacing whose rings still hold n positions
    layout_slots(*p, smin, &slots, p->n);
    if ((int64_t)slots.size() < p->n)
      return set_error(QMCRT_ERR_INVALID_ARGUMENT, "field radius too small for n heliostats");
    double lo = smin, hi = smin * 64;
    for (int it = 0; it < 60; ++it) {
      double mid = 0.5 * (lo + hi);
      layout_slots(*p, mid, &slots, p->n);
      if ((int64_t)slots.size() >= p->n) lo = mid;
      else hi = mid;
    }
    s = lo;
  } else if (s < smin) {
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "spacing below heliostat diagonal");
  }
  layout_slots(*p, s, &slots, 0);
  if ((int64_t)slots.size() < p->n)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "field radius too small for n heliostats");
  // inner rings first; within the last ring used, positions nearest the span centre
  int last_ring = slots[p->n - 1].ring;
  std::vector<Slot> pick;
  std::vector<Slot> edge;
  for (const Slot& sl : slots) {
    if (sl.ring < last_ring) pick.push_back(sl);
    else if (sl.ring == last_ring) edge.push_back(sl);
  }
  const double c = p->az_center_deg * M_PI / 180.0;
  std::stable_sort(edge.begin(), edge.end(), [c](const Slot& a, const Slot& b) {
    double da = std::fabs(std::remainder(a.az - c, 2 * M_PI)), db = std::fabs(std::remainder(b.az - c, 2 * M_PI));
    return da < db;
  });
  for (size_t i = 0; pick.size() < (size_t)p->n && i < edge.size(); ++i) pick.push_back(edge[i]);
  *n_out = p->n;
  if (!h_pos) return QMCRT_OK;
  if (capacity < p->n) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "capacity too small");
  for (int i = 0; i < p->n; ++i) {
    uint32_t w[4];
    philox_host((uint32_t)i, 0, p->seed, w);
    double jx = (u24f(w[0]) * 2.0 - 1.0) * p->jitter, jz = (u24f(w[1]) * 2.0 - 1.0) * p->jitter;
    // azimuth from north clockwise; x = east, z = south
    h_pos[3 * i + 0] = (float)(pick[i].r * std::sin(pick[i].az) + jx);
    h_pos[3 * i + 1] = p->mount_height;
    h_pos[3 * i + 2] = (float)(-pick[i].r * std::cos(pick[i].az) + jz);
  }
  return QMCRT_OK;
}

// .scn reader (SceneFileProc::SceneFileRead, scene_file_proc.cpp:41-286):
// keywords ground/ngrid, Recv <type> {pos,size,norm,face,end},
// Grid <type> {pos,size,inter,n,type,end}, then gap/matrix/helio lines where
// each `helio x y z` line is followed by a size line.  Only grid 0 and the
// first receiver are used, as in the reference driver (Gtest.cu:12-13).
qmcrt_status qmcrt_scn_parse(const char* path, qmcrt_receiver* recv_out, qmcrt_grid_params* grid_out,
                             float* h_pos, float* h_size, int32_t capacity, int32_t* n_out) {
  if (!path || !n_out) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::ifstream f(path);
  if (!f) return set_error(QMCRT_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  enum { NONE, GROUND, RECV, GRID, HELIO } mode = NONE;
  qmcrt_receiver rv{};
  bool have_recv = false, in_recv = false;
  qmcrt_grid_params gp{};
  bool have_grid = false;
  int declared = -1;
  bool gap_set = false, matrix_set = false;
  std::vector<float> pos, size;
  std::string line;
  int lineno = 0;
  while (std::getline(f, line)) {
    ++lineno;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty() || line[0] == '#') continue;
    std::stringstream ls(line);
    std::string head;
    ls >> head;
    if (head.empty()) continue;
    if (head == "ground") { mode = GROUND; continue; }
    if (head == "Recv") {
      mode = RECV;
      int t = 0;
      ls >> t;
      if (t != 0 && t != 1)
        return set_error(QMCRT_ERR_NOT_SUPPORTED, "line " + std::to_string(lineno) + ": receiver type not supported");
      in_recv = !have_recv;
      if (in_recv) {
        rv = qmcrt_receiver{};
        rv.type = t;
      }
      continue;
    }
    if (head == "Grid") {
      mode = GRID;
      int t = 0;
      ls >> t;
      if (t != 0) return set_error(QMCRT_ERR_NOT_SUPPORTED, "line " + std::to_string(lineno) + ": grid type not supported");
      if (have_grid) return set_error(QMCRT_ERR_NOT_SUPPORTED, "more than one grid");
      gap_set = matrix_set = false;
      continue;
    }
    switch (mode) {
      case RECV:
        if (!in_recv) break;
        if (head == "pos") ls >> rv.pos[0] >> rv.pos[1] >> rv.pos[2];
        else if (head == "size") ls >> rv.size[0] >> rv.size[1] >> rv.size[2];
        else if (head == "norm") ls >> rv.normal[0] >> rv.normal[1] >> rv.normal[2];
        else if (head == "face") ls >> rv.face;
        else if (head == "end") { have_recv = true; in_recv = false; }
        break;
      case GRID:
        if (head == "pos") { ls >> gp.origin[0] >> gp.origin[1] >> gp.origin[2]; gp.explicit_bounds = 1; }
        else if (head == "size") ls >> gp.extent[0] >> gp.extent[1] >> gp.extent[2];
        else if (head == "inter") ls >> gp.cell[0] >> gp.cell[1] >> gp.cell[2];
        else if (head == "n") ls >> declared;
        else if (head == "type") { int ht; ls >> ht; if (ht != 0) return set_error(QMCRT_ERR_NOT_SUPPORTED, "heliostat type not supported"); }
        else if (head == "end") { have_grid = true; mode = HELIO; }
        break;
      case HELIO:
        if (head == "gap") gap_set = true;
        else if (head == "matrix") {
          int r = 0, c = 0;
          ls >> r >> c;
          if (r != 1 || c != 1) return set_error(QMCRT_ERR_NOT_SUPPORTED, "facet matrices other than 1x1 are not supported");
          matrix_set = true;
        } else if (head == "helio") {
          if (!gap_set || !matrix_set)
            return set_error(QMCRT_ERR_INVALID_ARGUMENT, "line " + std::to_string(lineno) + ": gap and matrix must precede helio");
          float x, y, z;
          if (!(ls >> x >> y >> z)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "line " + std::to_string(lineno) + ": bad helio position");
          std::string sl;
          if (!std::getline(f, sl)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "missing heliostat size line");
          ++lineno;
          std::stringstream ss(sl);
          float sx, sy, sz;
          if (!(ss >> sx >> sy >> sz)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "line " + std::to_string(lineno) + ": bad helio size");
          pos.insert(pos.end(), {x, y, z});
          size.insert(size.end(), {sx, sy, sz});
        }
        break;
      default:
        break;
    }
  }
  if (!have_recv) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "no receiver in scene file");
  if (!have_grid) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "no grid in scene file");
  int n = (int)(pos.size() / 3);
  if (declared >= 0 && declared != n)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "grid declares " + std::to_string(declared) + " heliostats, file has " + std::to_string(n));
  *n_out = n;
  if (recv_out) {
    *recv_out = rv;
    // receiver resolution: size * (1/pixel_length) with the default 0.01 m
    // (scene_instance_process.cpp:15-19, receiver.cpp:19-23)
    if (recv_out->res_x == 0) recv_out->res_x = (int)(rv.size[0] * 100.0f);
    if (recv_out->res_y == 0) recv_out->res_y = (int)(rv.size[1] * 100.0f);
  }
  if (grid_out) *grid_out = gp;
  if (h_pos || h_size) {
    if (capacity < n) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "capacity too small");
    if (h_pos) std::memcpy(h_pos, pos.data(), pos.size() * sizeof(float));
    if (h_size) std::memcpy(h_size, size.data(), size.size() * sizeof(float));
  }
  return QMCRT_OK;
}

// ------------------------------------------------------------ faceted heliostat
qmcrt_status qmcrt_layout_paraboloid_facets(const qmcrt_facet_params* p, float* h_pos, float* h_size, float* h_normal,
                                            int32_t capacity, int32_t* n_out) {
  if (!p || !n_out) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!(p->a > 0) || !(p->b > 0) || p->rows < 1 || p->cols < 1 || !(p->facet > 0) || !(p->gap >= 0) ||
      !(p->thickness >= 0))
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "paraboloid facets need a, b, facet > 0, rows, cols >= 1, gap >= 0");
  const int64_t n = (int64_t)p->rows * p->cols;
  if (n > 0x7FFFFFFF) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "too many facets");
  *n_out = (int32_t)n;
  if (!h_pos && !h_size && !h_normal) return QMCRT_OK;
  if (capacity < n) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "capacity too small");
  double nv[3] = {p->normal[0], p->normal[1], p->normal[2]};
  const double ln = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
  if (!(ln > 0)) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "heliostat normal is zero");
  if (!p->reference_frame)
    for (double& c : nv) c /= ln;
  // horizontal axis e1 (scene_file_proc.cpp:300-316): the reference divides
  // (n.z, 0, -n.x) by sqrt(n.x^2 + n.y^2); the corrected frame by its length
  double e1[3];
  const double t = p->reference_frame ? std::sqrt(nv[0] * nv[0] + nv[1] * nv[1]) : std::sqrt(nv[0] * nv[0] + nv[2] * nv[2]);
  if (nv[2] > 0 && t > 0) {
    e1[0] = nv[2] / t; e1[1] = 0; e1[2] = -nv[0] / t;
  } else if (nv[2] < 0 && t > 0) {
    e1[0] = -nv[2] / t; e1[1] = 0; e1[2] = nv[0] / t;
  } else {
    e1[0] = 0; e1[1] = 0; e1[2] = 1;
  }
  // third axis e1 x n (:317-319)
  const double e2[3] = {e1[1] * nv[2] - e1[2] * nv[1], e1[2] * nv[0] - e1[0] * nv[2], e1[0] * nv[1] - e1[1] * nv[0]};
  const double pitch = (double)p->facet + p->gap, a2 = (double)p->a * p->a, b2 = (double)p->b * p->b;
  int64_t k = 0;
  for (int r = 0; r < p->rows; ++r)
    for (int c = 0; c < p->cols; ++c, ++k) {
      // facet centre on the paraboloid (:289-297) and its normal (:325-327)
      const double x = (c - 0.5 * (p->cols - 1)) * pitch, z = (r - 0.5 * (p->rows - 1)) * pitch;
      const double y = x * x / a2 + z * z / b2;
      const double ln_[3] = {-2.0 * x / a2, 1.0, -2.0 * z / b2};
      double w[3], m[3];
      for (int i = 0; i < 3; ++i) {
        w[i] = x * e1[i] + y * nv[i] + z * e2[i] + p->centre[i];
        m[i] = ln_[0] * e1[i] + ln_[1] * nv[i] + ln_[2] * e2[i];
      }
      const double lm = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
      for (int i = 0; i < 3; ++i) {
        if (h_pos) h_pos[3 * k + i] = (float)w[i];
        if (h_normal) h_normal[3 * k + i] = (float)(m[i] / lm);
      }
      if (h_size) {
        h_size[3 * k] = p->facet;
        h_size[3 * k + 1] = p->thickness;
        h_size[3 * k + 2] = p->facet;
      }
    }
  return QMCRT_OK;
}

// ------------------------------------------------------------ result files
// The map is [height][width], row 0 at the receiver's v0 edge; both writers
// walk it from the last row to the first (the top of the receiver first), as
// ImageSaver::savetxt does (image_save.cpp:10-22).  Values below 1e-6 count as
// zero (Epsilon, global_constant.h:6).

static qmcrt_status open_out(const char* path, int32_t append, FILE** f) {
  *f = std::fopen(path, append ? "a" : "w");
  if (!*f) return set_error(QMCRT_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  return QMCRT_OK;
}

qmcrt_status qmcrt_write_flux_csv(const char* path, const float* h_map, int32_t width, int32_t height,
                                  int32_t precision, int32_t append) {
  if (!path || !h_map || width <= 0 || height <= 0 || precision < 0 || precision > 30)
    return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad flux file arguments");
  FILE* f;
  qmcrt_status e = open_out(path, append, &f);
  if (e) return e;
  for (int r = height - 1; r >= 0; --r) {
    const float* row = h_map + (size_t)r * width;
    for (int c = 0; c < width; ++c) {
      if ((double)row[c] < 1e-6) std::fputs("0,", f);
      else std::fprintf(f, "%.*f,", precision, (double)row[c]);
    }
    std::fputc('\n', f);
  }
  bool bad = std::ferror(f) != 0;
  if (std::fclose(f) != 0 || bad) return set_error(QMCRT_ERR_INVALID_ARGUMENT, std::string("write failed: ") + path);
  return QMCRT_OK;
}

qmcrt_status qmcrt_write_intercept_ratio(const char* path, const float* h_map, int32_t width, int32_t height,
                                         float total_energy, int32_t append, float* ratio_out) {
  if (!h_map || width <= 0 || height <= 0) return set_error(QMCRT_ERR_INVALID_ARGUMENT, "bad intercept arguments");
  // float accumulation in the file's order (image_save.cpp:29-45)
  float in = 0.0f;
  for (int r = height - 1; r >= 0; --r) {
    const float* row = h_map + (size_t)r * width;
    for (int c = 0; c < width; ++c)
      if (!((double)row[c] < 1e-6)) in += row[c];
  }
  float ratio = in / total_energy;
  if (ratio_out) *ratio_out = ratio;
  if (!path) return QMCRT_OK;
  FILE* f;
  qmcrt_status e = open_out(path, append, &f);
  if (e) return e;
  std::fprintf(f, "%g\n", (double)ratio);  // ostream's default: 6 significant digits
  bool bad = std::ferror(f) != 0;
  if (std::fclose(f) != 0 || bad) return set_error(QMCRT_ERR_INVALID_ARGUMENT, std::string("write failed: ") + path);
  return QMCRT_OK;
}

}  // extern "C"
