// ref_harness.cu — drives the REFERENCE's own code (compiled from its sources
// where they lie by oracle/ref.mk into oracle/_ref/libref.so) so the oracle
// and the CUDA path can be pinned against it.  TEST INFRASTRUCTURE ONLY.
//
// Host-callable pieces (run anywhere): local2world, rayParallelogramIntersect,
// angle2xyz, rotateY (global_function.cuh), the Buie table builder
// samplelights::parameters_generate and max_less_index
// (scene_instance_process.cu), the Max_heap/Min_heap classes (heap.cuh) and
// RectangleHelio::CRotate (heliostat.cpp), and the result writers
// ImageSaver::savetxt (image_save.cpp).
// Device pieces (need a GPU): RectGrid::CGridHelioMatch (grid.cpp),
// ImageSmoother::image_smooth (image_smooth.cu), and the tracing kernel
// map_tracing through ray_tracing (ray_tracing.cu) with caller-given tables.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <vector>

#include "global_function.cuh"
#include "grid.h"
#include "heap.cuh"
#include "heliostat.cuh"
#include "image_save.h"
#include "image_smooth.cuh"
#include "random_generator.h"
#include "ray_tracing.h"
#include "receiver.cuh"
#include "recthelio_tracing.h"
#include "scene_instance_process.h"
#include "steps_for_raytracing.h"
#include "sunray.h"

// defined by the reference's main.cpp, which is not linked here
curandGenerator_t* RandomGenerator::gen;

namespace samplelights {
float2* parameters_generate(float* h_k, int num_group, float k, float gamma, float upper_lm);
__host__ __device__ int max_less_index(float2* d_cdf, float value, size_t n);
float inter_larger_465_intensity(float theta, const float& k, const float& gamma);
}  // namespace samplelights

static float3 f3p(const float* p) { return make_float3(p[0], p[1], p[2]); }
static void put(float* o, float3 v) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
}

extern "C" {

// ---------------------------------------------------------------- host
void ref_local2world(const float* d, const float* n, float* out) { put(out, global_func::local2world(f3p(d), f3p(n))); }

int ref_ray_parallelogram(const float* o, const float* d, const float* A, const float* B, const float* C, float* tuv) {
  float t = 0, u = 0, v = 0;
  bool h = global_func::rayParallelogramIntersect(f3p(o), f3p(d), f3p(A), f3p(B), f3p(C), t, u, v);
  tuv[0] = t;
  tuv[1] = u;
  tuv[2] = v;
  return h ? 1 : 0;
}

void ref_angle2xyz(float theta, float phi, float* out) { put(out, global_func::angle2xyz(make_float2(theta, phi))); }

void ref_rotate_y(const float* o, const float* a, const float* b, float* out) {
  put(out, global_func::rotateY(f3p(o), f3p(a), f3p(b)));
}

// The table set_samplelights builds (scene_instance_process.cu:163-200):
// k and gamma by its two formula lines, then the reference's own
// parameters_generate and inter_larger_465_intensity.
void ref_buie_table(float csr, float* cdf_x, float* cdf_y, float* slope, float* params) {
  float k = 0.9f * logf(13.5f * csr) * powf(csr, -0.3f);
  float gamma = 2.2f * logf(0.52f * csr) * powf(csr, 0.43f) - 0.1f;
  float tail = samplelights::inter_larger_465_intensity(9.3f, k, gamma) -
               samplelights::inter_larger_465_intensity(4.65f, k, gamma);
  std::vector<float> hk(1024);
  float2* cdf = samplelights::parameters_generate(hk.data(), 1024, k, gamma, 4.65f);
  for (int i = 0; i <= 1024; ++i) {
    cdf_x[i] = cdf[i].x;
    cdf_y[i] = cdf[i].y;
  }
  for (int i = 0; i < 1024; ++i) slope[i] = hk[i];
  params[0] = k;
  params[1] = gamma;
  params[2] = cdf[1024].y;
  params[3] = cdf[1024].y + tail;
  params[4] = (gamma + 1) / expf(k);
  params[5] = powf(4.65, gamma + 1);
  delete[] cdf;
}

int ref_max_less_index(const float* cdf_x, const float* cdf_y, float value) {
  std::vector<float2> c(1025);
  for (int i = 0; i <= 1024; ++i) c[i] = make_float2(cdf_x[i], cdf_y[i]);
  return samplelights::max_less_index(c.data(), value, 1024);
}

// The reference's heap classes driven over one window in the order of the
// trimmed_mean kernel (image_smooth.cu:22-57).
float ref_heap_trimmed(const float* window, int cnt, float ratio) {
  std::vector<float> mx(cnt + 2), mn(cnt + 2);
  int k = cnt * ratio;
  Max_heap max_heap(k, mx.data());
  Min_heap min_heap(k, mn.data());
  float value = 0.0f;
  for (int i = 0; i < cnt; ++i) {
    float cur = window[i];
    value += cur;
    if (!max_heap.full()) {
      max_heap.insert(cur);
      min_heap.insert(cur);
    } else if (k > 0 && cur < max_heap.top()) {
      max_heap.delete_and_insert(cur);
    } else if (k > 0 && cur > min_heap.top()) {
      min_heap.delete_and_insert(cur);
    }
  }
  return (value - max_heap.sum() - min_heap.sum()) / float(cnt - 2 * k);
}

// RectangleHelio::CRotate with a given normal (heliostat.cpp:23-28) or aimed
// at `focus` for the sun direction (heliostat.cpp:16-21): 4 vertices + normal.
void ref_helio_vertices(const float* pos, const float* size, const float* normal_or_null, const float* focus,
                        const float* sun_dir, float* v4, float* n_out) {
  RectangleHelio h;
  h.pos_ = f3p(pos);
  h.size_ = f3p(size);
  h.row_col_ = make_int2(1, 1);
  h.gap_ = make_float2(0, 0);
  if (normal_or_null) h.CRotate(f3p(normal_or_null));
  else h.CRotate(f3p(focus), normalize(f3p(sun_dir)));
  for (int i = 0; i < 4; ++i) put(v4 + 3 * i, h.vertex_[i]);
  put(n_out, h.normal_);
}

// ---------------------------------------------------------------- device
struct RefScene {
  std::vector<Heliostat*> helios;
  RectGrid grid;
  RectangleReceiver recv;
};

static RefScene* make_ref_scene(int n, const float* pos, const float* size, const float* normal, const float* gpos,
                            const float* gsize, const float* ginter, const float* rpos, const float* rsize,
                            const float* rnorm, int rface, int geometry_info, float helio_pixel) {
  RefScene* s = new RefScene();
  for (int i = 0; i < n; ++i) {
    RectangleHelio* h = new RectangleHelio();
    h->pos_ = f3p(pos + 3 * i);
    h->size_ = f3p(size + 3 * i);
    h->row_col_ = make_int2(1, 1);
    h->gap_ = make_float2(0, 0);
    h->Cset_pixel_length(helio_pixel);
    h->CRotate(f3p(normal + 3 * i));
    s->helios.push_back(h);
  }
  s->grid.type_ = 0;
  s->grid.helio_type_ = 0;
  s->grid.start_helio_pos_ = 0;
  s->grid.num_helios_ = n;
  s->grid.pos_ = f3p(gpos);
  s->grid.size_ = f3p(gsize);
  s->grid.interval_ = f3p(ginter);
  s->grid.Cinit();
  s->grid.CGridHelioMatch(s->helios);
  s->recv.type_ = 0;
  s->recv.pos_ = f3p(rpos);
  s->recv.size_ = f3p(rsize);
  s->recv.normal_ = f3p(rnorm);
  s->recv.face_num_ = rface;
  s->recv.CInit(geometry_info);
  return s;
}

static void free_ref_scene(RefScene* s) {
  s->grid.CClear();
  s->recv.CClear();
  for (Heliostat* h : s->helios) delete h;
  delete s;
}

// CSR of RectGrid::CGridHelioMatch; cell_start [cells+1], entries [cap].
int ref_grid_match(int n, const float* pos, const float* size, const float* normal, const float* gpos,
                   const float* gsize, const float* ginter, int* dims_out, int* cell_start, int* entries, int cap) {
  float rp[3] = {0, 100, 0}, rs[3] = {1, 1, 0}, rn[3] = {0, 0, 1};
  RefScene* s = make_ref_scene(n, pos, size, normal, gpos, gsize, ginter, rp, rs, rn, 0, 10, 0.01f);
  int cells = s->grid.grid_num_.x * s->grid.grid_num_.y * s->grid.grid_num_.z;
  dims_out[0] = s->grid.grid_num_.x;
  dims_out[1] = s->grid.grid_num_.y;
  dims_out[2] = s->grid.grid_num_.z;
  int nm = (int)s->grid.num_grid_helio_match_;
  int ok = 0;
  if (cell_start && entries && nm <= cap) {
    cudaMemcpy(cell_start, s->grid.d_grid_helio_index_, sizeof(int) * (cells + 1), cudaMemcpyDeviceToHost);
    cudaMemcpy(entries, s->grid.d_grid_helio_match_, sizeof(int) * nm, cudaMemcpyDeviceToHost);
    ok = 1;
  }
  free_ref_scene(s);
  return ok ? nm : -nm;
}

// ImageSmoother::image_smooth on a host image (in place on a device copy).
int ref_image_smooth(const float* h_in, int w, int h, int radius, float ratio, float* h_out) {
  float* d = nullptr;
  if (cudaMalloc(&d, sizeof(float) * w * h) != cudaSuccess) return 1;
  cudaMemcpy(d, h_in, sizeof(float) * w * h, cudaMemcpyHostToDevice);
  ImageSmoother::image_smooth(d, radius, ratio, w, h);
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(h_out, d, sizeof(float) * w * h, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? 0 : 2;
}

// The reference's tracing pass over a field with caller-given sample tables
// (T = groups * lights unit vectors each) and per-point start offsets
// (concatenated over heliostats in the order of set_microhelio_centers).
// Per heliostat, as recthelio_ray_tracing (recthelio_tracing.cpp:46-80) but
// with the given offsets in place of set_microhelio_groups' cuRAND draws:
// set_microhelio_centers, set_helios_vertexes, ray_tracing (map_tracing).
// Writes the receiver image (res_y x res_x, raw |cos| sums) and the point
// count; returns 0 on success.  ms_out: device time of the ray_tracing calls.
int ref_trace_tables(int n, const float* pos, const float* size, const float* normal, const float* gpos,
                     const float* gsize, const float* ginter, const float* rpos, const float* rsize,
                     const float* rnorm, int rface, int geometry_info, float helio_pixel, const float* sun_dir,
                     int groups, int lights, const float* sun_local, const float* turb_local, const int* start,
                     long long points_cap, float* image, int* res_out, long long* points_out, float* ms_out) {
  RefScene* s = make_ref_scene(n, pos, size, normal, gpos, gsize, ginter, rpos, rsize, rnorm, rface, geometry_info,
                           helio_pixel);
  SunRay sun(normalize(f3p(sun_dir)), groups, lights, 1000.0f, 0.1f);
  size_t T = (size_t)groups * lights;
  cudaMalloc(&sun.d_samplelights_, sizeof(float3) * T);
  cudaMalloc(&sun.d_perturbation_, sizeof(float3) * T);
  cudaMemcpy(sun.d_samplelights_, sun_local, sizeof(float3) * T, cudaMemcpyHostToDevice);
  cudaMemcpy(sun.d_perturbation_, turb_local, sizeof(float3) * T, cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total_ms = 0;
  long long done = 0;
  int rc = 0;
  for (int i = 0; i < n && rc == 0; ++i) {
    RectangleHelio* rh = dynamic_cast<RectangleHelio*>(s->helios[i]);
    float3 *d_c = nullptr, *d_n = nullptr, *d_v = nullptr;
    int* d_g = nullptr;
    size_t m = 0;
    set_microhelio_centers(*rh, d_c, d_n, m);
    set_helios_vertexes(s->helios, 0, n, d_v);
    if (done + (long long)m > points_cap) {
      rc = 3;
    } else {
      cudaMalloc(&d_g, sizeof(int) * m);
      cudaMemcpy(d_g, start + done, sizeof(int) * m, cudaMemcpyHostToDevice);
      cudaEventRecord(e0);
      ray_tracing(sun, s->grid, s->recv, d_v, d_n, d_c, d_g, (int)m);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      total_ms += ms;
      done += (long long)m;
    }
    cudaFree(d_c);
    cudaFree(d_n);
    cudaFree(d_v);
    cudaFree(d_g);
  }
  res_out[0] = s->recv.resolution_.x;
  res_out[1] = s->recv.resolution_.y;
  if (rc == 0 && image)
    cudaMemcpy(image, s->recv.d_image_, sizeof(float) * s->recv.resolution_.x * s->recv.resolution_.y,
               cudaMemcpyDeviceToHost);
  *points_out = done;
  *ms_out = total_ms;
  if (cudaDeviceSynchronize() != cudaSuccess && rc == 0) rc = 2;
  sun.CClear();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  free_ref_scene(s);
  return rc;
}

// The reference's own pass over one sun position, timed: per heliostat of the
// field, as results_with_given_normal (Gtest.cu:21-35) does, regenerate the
// sun and perturbation tables with cuRAND (SceneProcessor::set_sunray_content,
// scene_instance_process.cu:6-11), then recthelio_ray_tracing's steps
// (recthelio_tracing.cpp:46-80: micro-points, all vertices, groups,
// ray_tracing = one map_tracing launch + cudaDeviceSynchronize, frees) with
// CUDA events around ray_tracing.  `reps` passes; per pass the host-clock
// time of the whole pass and the summed event time of its map_tracing
// launches.  The receiver image is replaced by one with a spare row and
// element after it, zeroed, so the one write the reference can make past its
// image (u == 1 gives row res_y, rectgrid_raytracing.cu:144; v == 1 in the
// last row gives index res) lands in memory this harness owns; *spill_out
// reports whether any did.  Writes the raw image of the last pass.
// Returns 0 on success.
int ref_run_field(int n, const float* pos, const float* size, const float* normal, const float* gpos,
                  const float* gsize, const float* ginter, const float* rpos, const float* rsize, const float* rnorm,
                  int rface, int geometry_info, float helio_pixel, const float* sun_dir, float dni, float csr,
                  float disturb_std, int groups, int lights, unsigned long long seed, int reps, float* image,
                  int* res_out, long long* rays_out, double* pass_ms, float* trace_ms, int* spill_out) {
  RefScene* s = make_ref_scene(n, pos, size, normal, gpos, gsize, ginter, rpos, rsize, rnorm, rface, geometry_info,
                               helio_pixel);
  const size_t res = (size_t)s->recv.resolution_.x * s->recv.resolution_.y;
  const size_t pad = (size_t)s->recv.resolution_.x + 1;
  float* padded = nullptr;
  if (cudaMalloc(&padded, sizeof(float) * (res + pad)) != cudaSuccess) {
    free_ref_scene(s);
    return 4;
  }
  cudaMemset(padded, 0, sizeof(float) * (res + pad));
  cudaFree(s->recv.d_image_);
  s->recv.d_image_ = padded;
  curandGenerator_t gen;
  curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT);
  curandSetPseudoRandomGeneratorSeed(gen, seed);
  RandomGenerator::gen = &gen;
  solarenergy::disturb_std = disturb_std;
  SunRay sun(normalize(f3p(sun_dir)), groups, lights, dni, csr);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  long long rays = 0;
  int rc = 0;
  for (int r = 0; r < reps && rc == 0; ++r) {
    float kms = 0;
    rays = 0;
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    s->recv.Cclean_image_content();
    for (int i = 0; i < n; ++i) {
      RectangleHelio* rh = dynamic_cast<RectangleHelio*>(s->helios[i]);
      SceneProcessor::set_sunray_content(sun);
      size_t m = 0;
      float3 *d_c = nullptr, *d_n = nullptr, *d_v = nullptr;
      int* d_g = nullptr;
      recthelio_ray_tracing_init(*rh, s->grid, s->helios, sun.num_sunshape_groups_ * sun.num_sunshape_lights_per_group_,
                                 m, d_c, d_n, d_v, d_g);
      cudaEventRecord(e0);
      ray_tracing(sun, s->grid, s->recv, d_v, d_n, d_c, d_g, (int)m);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      kms += ms;
      rays += (long long)m * sun.num_sunshape_lights_per_group_;
      cudaFree(d_c);
      cudaFree(d_n);
      cudaFree(d_v);
      cudaFree(d_g);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) rc = 2;
    auto t1 = std::chrono::steady_clock::now();
    pass_ms[r] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    trace_ms[r] = kms;
  }
  res_out[0] = s->recv.resolution_.x;
  res_out[1] = s->recv.resolution_.y;
  *rays_out = rays;
  std::vector<float> tail(pad);
  if (rc == 0 && image) cudaMemcpy(image, padded, sizeof(float) * res, cudaMemcpyDeviceToHost);
  cudaMemcpy(tail.data(), padded + res, sizeof(float) * pad, cudaMemcpyDeviceToHost);
  *spill_out = 0;
  for (float v : tail) *spill_out |= v != 0.0f;
  if (cudaDeviceSynchronize() != cudaSuccess && rc == 0) rc = 2;
  sun.CClear();
  curandDestroyGenerator(gen);
  RandomGenerator::gen = nullptr;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  free_ref_scene(s);
  return rc;
}

// Receiver corners after RectangleReceiver::CInit (receiver.cpp:24-118).
int ref_receiver_vertices(const float* rpos, const float* rsize, const float* rnorm, int rface, int geometry_info,
                          float* v4, int* res_out) {
  RectangleReceiver r;
  r.type_ = 0;
  r.pos_ = f3p(rpos);
  r.size_ = f3p(rsize);
  r.normal_ = f3p(rnorm);
  r.face_num_ = rface;
  r.CInit(geometry_info);
  for (int i = 0; i < 4; ++i) put(v4 + 3 * i, r.rect_vertex_[i]);
  res_out[0] = r.resolution_.x;
  res_out[1] = r.resolution_.y;
  r.CClear();
  return 0;
}

// The two text writers of image_save.cpp (flux map, intercept ratio); both
// append to `path`.
void ref_save_flux_txt(const char* path, int w, int h, float* data, int precision) {
  ImageSaver::savetxt(std::string(path), w, h, data, precision);
}
void ref_save_ratio_txt(const char* path, int w, int h, float* data, float total_energy) {
  ImageSaver::savetxt(std::string(path), w, h, data, total_energy);
}

}  // extern "C"
