// common.cuh — device/host helpers shared by the qmcrt kernels: small vector
// algebra in float and double (written for this library), the Philox4x32-10
// counter-based generator (Salmon et al., SC'11) and uniform conversions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define QMCRT_HD __host__ __device__ __forceinline__

namespace qm {

// ------------------------------------------------------------------ float3
QMCRT_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
QMCRT_HD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
QMCRT_HD float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
QMCRT_HD float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
QMCRT_HD float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
QMCRT_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
QMCRT_HD float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// ----------------------------------------------------------------- double3
struct d3 {
  double x, y, z;
};
QMCRT_HD d3 mk(double x, double y, double z) { return d3{x, y, z}; }
QMCRT_HD d3 operator+(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
QMCRT_HD d3 operator-(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
QMCRT_HD d3 operator*(double s, d3 a) { return mk(s * a.x, s * a.y, s * a.z); }
QMCRT_HD double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
QMCRT_HD d3 cross(d3 a, d3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
QMCRT_HD float3 to_f(d3 a) { return f3((float)a.x, (float)a.y, (float)a.z); }
QMCRT_HD d3 to_d(float3 a) { return mk(a.x, a.y, a.z); }

// Frame applied to a local vector: out = d.x*u + d.y*n + d.z*v, the matrix of
// local2world (global_function.cuh:47-49).
// Reciprocal and reciprocal square root in double: the hardware's 64-bit
// approximation (rcp.approx.ftz.f64, rsqrt.approx.ftz.f64: about 20 correct
// bits) refined by one Newton-Raphson step, y + y (1 - x y) for 1/x and
// y + (y / 2)(1 - x y^2) for 1/sqrt(x); a step squares the relative error, so
// the result is good to ~2^-40 = 1e-12 relative (checked against exact
// values by a GPU test), which moves a receiver coordinate by ~1e-10 of a
// pixel.  For normal, finite, nonzero x: the callers' determinants and
// squared lengths of near-unit vectors.
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return fma(y, fma(-x, y, 1.0), y);
}
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return fma(0.5 * y, fma(-x * y, y, 1.0), y);
}

// Additions to global memory without a returned value (red.global).  A batch
// item's map pointers are read from shared memory, where the compiler cannot
// see that they address global memory and would emit returning atomics.
__device__ __forceinline__ void red_add(uint32_t* p, uint32_t v) {
  asm volatile("{\n\t.reg .u64 g;\n\tcvta.to.global.u64 g, %0;\n\tred.global.add.u32 [g], %1;\n\t}"
               :: "l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_add(float* p, float v) {
  asm volatile("{\n\t.reg .u64 g;\n\tcvta.to.global.u64 g, %0;\n\tred.global.add.f32 [g], %1;\n\t}"
               :: "l"(p), "f"(v) : "memory");
}

// Doubles per heliostat in the per-sun frame array: the local2world axes
// u, n, v and the mirror centre c = pos + n * thickness / 2.
constexpr int kFrameStride = 12;

struct frame64 {
  d3 u, n, v;
};
QMCRT_HD d3 apply(const frame64& f, double x, double y, double z) {
  return mk(x * f.u.x + y * f.n.x + z * f.v.x, x * f.u.y + y * f.n.y + z * f.v.y,
            x * f.u.z + y * f.n.z + z * f.v.z);
}

// --------------------------------------------------------------- Philox
// Philox4x32 with 10 rounds; multipliers and Weyl increments from the
// published algorithm (Random123 paper, SC'11).
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;
QMCRT_HD uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
    uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += kPhiloxW0;
    k.y += kPhiloxW1;
  }
  return c;
}

// The key schedule of philox4x32_10 for `key`: rk[r] = key + r (W0, W1).
QMCRT_HD void philox_round_keys(uint2 key, uint2* rk) {
  for (int r = 0; r < 10; ++r) rk[r] = make_uint2(key.x + r * kPhiloxW0, key.y + r * kPhiloxW1);
}

// philox4x32_10 from precomputed round keys: a kernel that receives them as
// launch parameters reads each one from the constant bank as an operand
// instead of stepping the key in registers.
__device__ __forceinline__ uint4 philox4x32_10_rk(uint4 c, const uint2* rk) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ rk[r].x, lo1, hi0 ^ c.w ^ rk[r].y, lo0);
  }
  return c;
}

// Uniform in (0,1) from the top 24 bits: exact in float and double.
QMCRT_HD float u24f(uint32_t w) { return ((float)(w >> 8) + 0.5f) * (1.0f / 16777216.0f); }

// The ray sampler's uniform in (0,1): (k + 0.5) 2^-23 with k the low 23 bits
// of w, built from the bits: 1 + k 2^-23 as a float (one AND-OR of w), minus
// (1 - 2^-24), a float whose difference with it is exactly (k + 0.5) 2^-23, so
// one subtraction and no integer-to-float conversion on the XU pipe.
__device__ __forceinline__ float u23f(uint32_t w) {
  return __uint_as_float(0x3F800000u | (w & 0x7FFFFFu)) - 0x1.fffffep-1f;  // 1 - 2^-24
}

// Programmatic dependent launch (sm_90 and later): a kernel launched with
// programmatic stream serialization may start while the kernel before it in
// the stream finishes; pdl_wait() returns once that kernel has completed and
// its writes are visible, so it comes before any memory access.  A kernel
// launched without the attribute returns from it at once.  pdl_trigger()
// lets the next kernel start launching once every block of this one has
// passed it (it is implicit at a block's exit).
__device__ __forceinline__ void pdl_wait() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
__device__ __forceinline__ void pdl_trigger() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// Occluder candidates kept per heliostat and walk direction.
constexpr int kCandCap = 32;

constexpr uint32_t kTagTrace = 0x51A7u;
constexpr uint32_t kTagPoisson = 0x9015u;
constexpr uint32_t kPoissonKey0 = 0x5A17C0DEu;
constexpr uint32_t kPoissonKey1 = 0x0B5E55EDu;
constexpr float kEps = 1e-6f;  // global_constant.h:7

}  // namespace qm
