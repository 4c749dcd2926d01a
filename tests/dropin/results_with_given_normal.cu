// results_with_given_normal.cu — the reference's per-sun-position call
// (Gtest.cu:10-63) re-implemented on this library, as a maintainer of the
// reference would drop it in: the same signature, the reference's own scene
// objects (SolarScene, RectGrid, RectangleReceiver, Heliostat, SunRay) as
// input and the reference's own result writer (ImageSaver::savetxt) as
// output.  The per-heliostat loop of cuRAND tables, micro-points and
// map_tracing launches (Gtest.cu:21-35) becomes one qmcrt scene and one
// qmcrt_results_host call (trace, flux scaling, smoothing).
//
// It compiles against the reference's headers (include path: the reference's
// ClassedSunRay directory and this repository's include/) and links
// libqmcrt.so; oracle/ref.mk builds it with a test harness into
// oracle/_ref/libdropin.so, and tests/test_gpu_dropin.py runs it.
#include <iostream>
#include <vector>

#include "Gtest.cuh"
#include "grid.h"
#include "heliostat.cuh"
#include "image_save.h"
#include "qmcrt.h"
#include "receiver.cuh"
#include "sunray.h"

// The reference scene's field, receiver and grid as qmcrt descriptions,
// traced once for its sun: the flux map (W/m^2, Gtest.cu:40-46), the map
// `smooth` names after smoothing (Gtest.cu:49-57), and, when not NULL, the
// integer counts and the trace statistics.  Returns the qmcrt status.
int qmcrt_results_for_scene(SolarScene& solar_scene, const qmcrt_smooth_params* smooth, uint64_t seed,
                            std::vector<float>& flux, std::vector<float>& smoothed, std::vector<uint32_t>* counts,
                            qmcrt_trace_stats* stats) {
  RectGrid* grid = dynamic_cast<RectGrid*>(solar_scene.grid0s[0]);
  RectangleReceiver* recv = dynamic_cast<RectangleReceiver*>(solar_scene.receivers[0]);
  const int n = grid->num_helios_;

  // field: SoA copies of the reference's Heliostat objects (heliostat.cuh:13-27)
  std::vector<float> pos(3 * n), size(3 * n), nrm(3 * n);
  for (int i = 0; i < n; ++i) {
    Heliostat* h = solar_scene.heliostats[grid->start_helio_pos_ + i];
    const float3 p = h->pos_, s = h->size_, q = h->normal_;
    pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z;
    size[3 * i] = s.x; size[3 * i + 1] = s.y; size[3 * i + 2] = s.z;
    nrm[3 * i] = q.x; nrm[3 * i + 1] = q.y; nrm[3 * i + 2] = q.z;
  }
  qmcrt_field field = {};
  field.n = n;
  field.pos = pos.data();
  field.size = size.data();
  field.normal = nrm.data();               // the normals main.cpp set (CRotate)
  field.sigma = solarenergy::disturb_std;  // common_var.cpp:18

  qmcrt_receiver rc = {};
  rc.type = QMCRT_RECEIVER_FLAT;
  rc.pos[0] = recv->pos_.x; rc.pos[1] = recv->pos_.y; rc.pos[2] = recv->pos_.z;
  rc.size[0] = recv->size_.x; rc.size[1] = recv->size_.y; rc.size[2] = recv->size_.z;
  rc.normal[0] = recv->normal_.x; rc.normal[1] = recv->normal_.y; rc.normal[2] = recv->normal_.z;
  rc.face = recv->face_num_;
  rc.res_x = recv->resolution_.x;
  rc.res_y = recv->resolution_.y;

  qmcrt_grid_params gp = {};
  gp.cell[0] = grid->interval_.x; gp.cell[1] = grid->interval_.y; gp.cell[2] = grid->interval_.z;
  gp.explicit_bounds = 1;
  gp.origin[0] = grid->pos_.x; gp.origin[1] = grid->pos_.y; gp.origin[2] = grid->pos_.z;
  gp.extent[0] = grid->size_.x; gp.extent[1] = grid->size_.y; gp.extent[2] = grid->size_.z;

  qmcrt_scene* scene = nullptr;
  qmcrt_status st = qmcrt_scene_create(&field, &rc, &gp, &scene);
  if (st != QMCRT_OK) {
    std::cerr << "qmcrt_scene_create: " << qmcrt_last_error() << std::endl;  // no exit(1): the caller decides
    return st;
  }
  const SunRay* s = solar_scene.sunray_;
  qmcrt_sun sun = {{s->sun_dir_.x, s->sun_dir_.y, s->sun_dir_.z}, s->dni_, s->csr_};
  qmcrt_trace_params tp = {};
  tp.seed = seed;                                    // every ray reproducible from (seed, ray id)
  tp.rays_per_point = s->num_sunshape_lights_per_group_;
  tp.point_mode = QMCRT_POINTS_GRID;                 // heliostat.cuh:23 default
  tp.point_spacing = solarenergy::helio_pixel_length;
  tp.reflectivity = solarenergy::reflected_rate;
  tp.quirks = 0;                                     // or QMCRT_QUIRKS_REFERENCE for the reference's traversal

  const size_t res = (size_t)rc.res_x * rc.res_y;
  flux.assign(res, 0.0f);
  smoothed.assign(res, 0.0f);
  if (counts) counts->assign(res, 0u);
  st = qmcrt_results_host(scene, nullptr, &sun, &tp, smooth, counts ? counts->data() : nullptr, flux.data(),
                          smooth ? smoothed.data() : nullptr, stats, nullptr);
  if (st != QMCRT_OK) std::cerr << "qmcrt_results_host: " << qmcrt_last_error() << std::endl;
  qmcrt_scene_destroy(scene);
  return st;
}

void results_with_given_normal(SolarScene& solar_scene, float3* normals) {
  (void)normals;  // unused, as in the reference (its set_helio_content call is commented out)
  RectGrid* grid = dynamic_cast<RectGrid*>(solar_scene.grid0s[0]);
  Receiver* recv = dynamic_cast<RectangleReceiver*>(solar_scene.receivers[0]);
  // total energy on the mirrors, as Gtest.cu:29,39-44 sums it
  const float Id = solar_scene.sunray_->dni_;
  float totalEnergy = 0.0f;
  for (int i = 0; i < grid->num_helios_; ++i) {
    Heliostat* h = solar_scene.heliostats[i + grid->start_helio_pos_];
    totalEnergy += fabsf(dot(h->normal_, solar_scene.sunray_->sun_dir_) * Id * h->size_.x * h->size_.z);
  }
  const float Srec = recv->pixel_length_ * recv->pixel_length_;
  totalEnergy *= solarenergy::reflected_rate / Srec;

  // smoothing as Gtest.cu:49-57: radius 5, 2 % trimmed, the reference's heaps,
  // on the raw image, then scaled to W/m^2
  const qmcrt_smooth_params sm = {5, 0.02f, QMCRT_TRIM_HEAPS, QMCRT_SMOOTH_ENERGY};
  std::vector<float> flux, smoothed;
  if (qmcrt_results_for_scene(solar_scene, &sm, 2018, flux, smoothed, nullptr, nullptr) != QMCRT_OK) return;
  ImageSaver::savetxt(solarenergy::result_save_nonsmooth_path, recv->resolution_.x, recv->resolution_.y, flux.data(),
                      totalEnergy);
  ImageSaver::savetxt(solarenergy::result_save_smooth_path, recv->resolution_.x, recv->resolution_.y,
                      smoothed.data(), totalEnergy);
}
