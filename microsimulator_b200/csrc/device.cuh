// Device-side helpers shared by the contact kernels.
//
// The whole library is compiled with --fmad=false and IEEE division and
// square root, so every float expression rounds after each operation as the
// reference's baseline-x86-64 build does.  The min/max/clamp helpers keep the
// exact semantics of std::min, std::max and std::clamp (which operand wins on
// ties, signed zeros and NaN), because the reference's results depend on them.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace msb {

// std::max(a, b): (a < b) ? b : a
template <typename T>
__host__ __device__ __forceinline__ T smax(T a, T b) {
  return (a < b) ? b : a;
}
// std::min(a, b): (b < a) ? b : a
template <typename T>
__host__ __device__ __forceinline__ T smin(T a, T b) {
  return (b < a) ? b : a;
}
// std::clamp(v, lo, hi)
template <typename T>
__host__ __device__ __forceinline__ T sclamp(T v, T lo, T hi) {
  return (v < lo) ? lo : ((hi < v) ? hi : v);
}

struct F3 {
  float x, y, z;
};

__host__ __device__ __forceinline__ F3 f3(float x, float y, float z) { return {x, y, z}; }
__host__ __device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
// ((ax*bx) + (ay*by)) + (az*bz), as types.hpp:46-48 of the reference.
__host__ __device__ __forceinline__ float dot(F3 a, F3 b) { return ((a.x * b.x) + (a.y * b.y)) + (a.z * b.z); }
__host__ __device__ __forceinline__ F3 cross(F3 a, F3 b) {
  return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)};
}
__device__ __forceinline__ float norm(F3 a) { return __fsqrt_rn(dot(a, a)); }
__device__ __forceinline__ bool finite3(F3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
// v * (1 / |v|).  Returns false (and leaves `out`) when |v| is not finite and
// positive, where the reference throws.
__device__ __forceinline__ bool normalized(F3 v, F3& out) {
  const float m = norm(v);
  if (!isfinite(m) || !(m > 0.0f)) return false;
  out = v * __fdiv_rn(1.0f, m);
  return true;
}
__device__ __forceinline__ F3 xyz(float4 v) { return {v.x, v.y, v.z}; }

// A capsule's FP64 box padded by half the margin on every side, as
// find_cell_contact_candidates forms it (cpp/core/contact_graph.cpp:17-34):
// centre -+ (|axis| * length / 2 + radius + margin / 2) per axis, into
// box[0..2] (low) and box[3..5] (high).  Every box test of the contact search
// goes through this one expression, so the boxes carry the same bits.
__device__ __forceinline__ void padded_box(float4 pos_len, float4 dir_rad, float margin, double box[6]) {
  const double half = double(pos_len.w) * 0.5;
  const double pad = double(dir_rad.w) + double(margin) * 0.5;
  const double c[3] = {double(pos_len.x), double(pos_len.y), double(pos_len.z)};
  const double d[3] = {double(dir_rad.x), double(dir_rad.y), double(dir_rad.z)};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double e = fabs(d[a]) * half + pad;
    box[a] = c[a] - e;
    box[3 + a] = c[a] + e;
  }
}

// The reference's box overlap test, touching included (contact_graph.cpp:37-41).
__device__ __forceinline__ bool boxes_overlap(const double* l, const double* r) {
  return l[3] >= r[0] && r[3] >= l[0] && l[4] >= r[1] && r[4] >= l[1] && l[5] >= r[2] && r[5] >= l[2];
}

__device__ __forceinline__ void raise_status(std::uint32_t* status, std::uint32_t code) {
  atomicCAS(status, 0u, code);
}

// Index checks of the checked build (MSB_DEVICE_CHECKS=1, libmsb200_checked.so):
// an index at or past its bound records kStatusIndex in *status and the
// caller skips the access.  In the ordinary build the check is compiled out.
#ifndef MSB_DEVICE_CHECKS
#define MSB_DEVICE_CHECKS 0
#endif
__device__ __forceinline__ bool index_ok(std::uint64_t index, std::uint64_t bound, std::uint32_t* status) {
  if constexpr (MSB_DEVICE_CHECKS != 0) {
    if (index >= bound) {
      if (status != nullptr) raise_status(status, kStatusIndex);
      return false;
    }
  }
  return true;
}

}  // namespace msb
