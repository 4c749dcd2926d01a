// harness.cu — test harness of the drop-in results_with_given_normal
// (results_with_given_normal.cu).  TEST INFRASTRUCTURE ONLY.
//
// The reference builds its SolarScene from a .scn file in solar_scene.cpp,
// which does not compile here (scene_file_proc.h declares an enumerator
// `norm` that collides with CUDA's norm()).  This harness supplies the two
// members of SolarScene that the drop-in's callers need, a constructor and a
// destructor, and builds the scene from arrays with the reference's own
// classes: RectangleHelio::CRotate (heliostat.cpp:23-28), RectGrid::Cinit
// and CGridHelioMatch (grid.cpp:3-83), RectangleReceiver::CInit
// (receiver.cpp:24-33) and SunRay (sunray.h).  extern "C" entry points let
// ctypes drive the drop-in.
#include <cstdint>
#include <string>
#include <vector>

#include "Gtest.cuh"
#include "grid.h"
#include "heliostat.cuh"
#include "qmcrt.h"
#include "receiver.cuh"
#include "sunray.h"

int qmcrt_results_for_scene(SolarScene& solar_scene, const qmcrt_smooth_params* smooth, uint64_t seed,
                            std::vector<float>& flux, std::vector<float>& smoothed, std::vector<uint32_t>* counts,
                            qmcrt_trace_stats* stats);

// the members solar_scene.cpp would define; the scene content belongs to
// ArrayScene below, which frees it with its concrete types (the reference's
// classes have no virtual destructors)
SolarScene::SolarScene() : sunray_(nullptr) {}
SolarScene::~SolarScene() {}

namespace {

struct ArrayScene : public SolarScene {
  std::vector<RectangleHelio*> own_helios;
  RectGrid* own_grid = nullptr;
  RectangleReceiver* own_recv = nullptr;
  ArrayScene() : SolarScene() {}
  ~ArrayScene() {
    if (own_recv) own_recv->CClear();
    delete own_recv;
    if (own_grid) own_grid->CClear();
    delete own_grid;
    for (RectangleHelio* h : own_helios) delete h;
    delete sunray_;
  }
};

float3 f3(const float* p) { return make_float3(p[0], p[1], p[2]); }

ArrayScene* make_scene(int n, const float* pos, const float* size, const float* normal, const float* gpos,
                       const float* gsize, const float* ginter, const float* rpos, const float* rsize,
                       const float* rnorm, int rface, int geometry_info, float helio_pixel, const float* sun_dir,
                       float dni, float csr, float sigma, int lights) {
  solarenergy::helio_pixel_length = helio_pixel;
  solarenergy::disturb_std = sigma;
  solarenergy::reflected_rate = 0.88f;
  ArrayScene* s = new ArrayScene();
  for (int i = 0; i < n; ++i) {
    RectangleHelio* h = new RectangleHelio();
    h->pos_ = f3(pos + 3 * i);
    h->size_ = f3(size + 3 * i);
    h->row_col_ = make_int2(1, 1);
    h->gap_ = make_float2(0, 0);
    h->Cset_pixel_length(helio_pixel);
    h->CRotate(f3(normal + 3 * i));
    s->own_helios.push_back(h);
    s->heliostats.push_back(h);
  }
  RectGrid* g = new RectGrid();
  s->own_grid = g;
  g->type_ = 0;
  g->helio_type_ = 0;
  g->start_helio_pos_ = 0;
  g->num_helios_ = n;
  g->pos_ = f3(gpos);
  g->size_ = f3(gsize);
  g->interval_ = f3(ginter);
  g->Cinit();
  g->CGridHelioMatch(s->heliostats);
  s->grid0s.push_back(g);
  RectangleReceiver* r = new RectangleReceiver();
  s->own_recv = r;
  r->type_ = 0;
  r->pos_ = f3(rpos);
  r->size_ = f3(rsize);
  r->normal_ = f3(rnorm);
  r->face_num_ = rface;
  r->CInit(geometry_info);
  s->receivers.push_back(r);
  s->sunray_ = new SunRay(normalize(f3(sun_dir)), 128, lights, dni, csr);
  return s;
}

}  // namespace

extern "C" {

// The drop-in's traced results for a scene built from arrays: counts,
// flux (W/m^2) and the smoothed map (radius, ratio, method, source as
// qmcrt_smooth_params), and the resolution.  normals_out [3n] and sun_out
// [3] receive the heliostat normals and sun direction as the reference's
// objects hold them (RectangleHelio::CRotate and the harness normalise in
// float), which is what the drop-in passes on.  Returns the qmcrt status.
int dropin_results(int n, const float* pos, const float* size, const float* normal, const float* gpos,
                   const float* gsize, const float* ginter, const float* rpos, const float* rsize, const float* rnorm,
                   int rface, int geometry_info, float helio_pixel, const float* sun_dir, float dni, float csr,
                   float sigma, int lights, unsigned long long seed, int radius, float ratio, int method, int source,
                   uint32_t* h_counts, float* h_flux, float* h_smoothed, int* res_out, double* stats_out,
                   float* normals_out, float* sun_out) {
  ArrayScene* s = make_scene(n, pos, size, normal, gpos, gsize, ginter, rpos, rsize, rnorm, rface, geometry_info,
                             helio_pixel, sun_dir, dni, csr, sigma, lights);
  for (int i = 0; i < n; ++i) {
    const float3 q = s->heliostats[i]->normal_;
    normals_out[3 * i] = q.x;
    normals_out[3 * i + 1] = q.y;
    normals_out[3 * i + 2] = q.z;
  }
  sun_out[0] = s->sunray_->sun_dir_.x;
  sun_out[1] = s->sunray_->sun_dir_.y;
  sun_out[2] = s->sunray_->sun_dir_.z;
  const qmcrt_smooth_params sm = {radius, ratio, method, source};
  std::vector<float> flux, smoothed;
  std::vector<uint32_t> counts;
  qmcrt_trace_stats st = {};
  int rc = qmcrt_results_for_scene(*s, &sm, seed, flux, smoothed, &counts, &st);
  res_out[0] = s->receivers[0]->resolution_.x;
  res_out[1] = s->receivers[0]->resolution_.y;
  if (rc == 0) {
    std::copy(counts.begin(), counts.end(), h_counts);
    std::copy(flux.begin(), flux.end(), h_flux);
    std::copy(smoothed.begin(), smoothed.end(), h_smoothed);
    stats_out[0] = (double)st.rays;
    stats_out[1] = (double)st.hit;
    stats_out[2] = st.total_power;
    stats_out[3] = st.intercept_ratio;
  }
  delete s;
  return rc;
}

// results_with_given_normal itself on a scene built from arrays, writing the
// reference's two result files to the given paths.
int dropin_results_with_given_normal(int n, const float* pos, const float* size, const float* normal,
                                     const float* gpos, const float* gsize, const float* ginter, const float* rpos,
                                     const float* rsize, const float* rnorm, int rface, int geometry_info,
                                     float helio_pixel, const float* sun_dir, float dni, float csr, float sigma,
                                     int lights, const char* nonsmooth_path, const char* smooth_path) {
  ArrayScene* s = make_scene(n, pos, size, normal, gpos, gsize, ginter, rpos, rsize, rnorm, rface, geometry_info,
                             helio_pixel, sun_dir, dni, csr, sigma, lights);
  solarenergy::result_save_nonsmooth_path = nonsmooth_path;
  solarenergy::result_save_smooth_path = smooth_path;
  results_with_given_normal(*s, nullptr);
  delete s;
  return 0;
}

}  // extern "C"
