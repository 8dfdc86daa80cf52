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

// ---- maxima and counts gathered on one address
//
// Thousands of warps each issuing an atomic to the same word serialise on
// it (a jammed colony's millions of overlapping contacts raising one
// deepest-overlap word).  These helpers fold a thread's, a warp's and a
// block's values first, so each block issues one atomic per word.

// Non-negative floats order as their bits: a running maximum of the
// positive values among `value`s, as bits (0: none).
__device__ __forceinline__ std::uint32_t max_bits(std::uint32_t bits, float value) {
  return value > 0.0f ? ::max(bits, __float_as_uint(value)) : bits;
}

// atomicMax(target, bits) of every thread of the block, as one atomic per
// block.  Every thread of the block calls it (a block barrier).
__device__ __forceinline__ void block_max_into(std::uint32_t* target, std::uint32_t bits) {
  __shared__ std::uint32_t block_bits;
  if (threadIdx.x == 0) block_bits = 0u;
  __syncthreads();
  const std::uint32_t w = __reduce_max_sync(0xFFFFFFFFu, bits);
  if ((threadIdx.x & 31u) == 0u && w != 0u) atomicMax(&block_bits, w);
  __syncthreads();
  if (threadIdx.x == 0 && block_bits != 0u) atomicMax(target, block_bits);
}

// A contiguous range of items per warp (covering [0, count) over the grid),
// walked 32 at a time by the warp together: items next to each other in
// memory meet in one warp, so that per-key values of sorted keys can be
// folded before they are written.
struct WarpRange {
  std::uint32_t begin;
  std::uint32_t end;
};
__device__ __forceinline__ WarpRange warp_range(std::uint32_t count) {
  const std::uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const std::uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const std::uint64_t per = ((std::uint64_t(count) + warps - 1) / warps + 31) & ~std::uint64_t(31);
  const std::uint64_t b = std::uint64_t(warp) * per;
  return {std::uint32_t(b < count ? b : count), std::uint32_t(b + per < count ? b + per : count)};
}

// Per-key sums (Sum) or maxima of a warp's items whose keys mostly repeat
// from one item to the next, as the colonies of rows in first-id order do:
// lane 0 carries the total of the current key and adds it to targets[key]
// once the key changes (and at the end, carry_flush); 32 items with more
// than one key go to their targets lane by lane.  Called by the whole warp
// with lane 0 live.
struct KeyCarry {
  std::uint32_t key = 0xFFFFFFFFu;
  std::uint32_t value = 0u;
};
template <bool Sum>
__device__ __forceinline__ void carry_flush(std::uint32_t* targets, const KeyCarry& carry) {
  if (carry.key != 0xFFFFFFFFu && carry.value != 0u) {
    if constexpr (Sum) {
      atomicAdd(targets + carry.key, carry.value);
    } else {
      atomicMax(targets + carry.key, carry.value);
    }
  }
}
template <bool Sum>
__device__ __forceinline__ void carry_item(std::uint32_t* targets, KeyCarry& carry, bool live, std::uint32_t key,
                                           std::uint32_t value) {
  const std::uint32_t key0 = __shfl_sync(0xFFFFFFFFu, key, 0);
  if (__all_sync(0xFFFFFFFFu, !live || key == key0)) {
    const std::uint32_t v = live ? value : 0u;
    const std::uint32_t w = Sum ? __reduce_add_sync(0xFFFFFFFFu, v) : __reduce_max_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31u) == 0u) {
      if (carry.key != key0) {
        carry_flush<Sum>(targets, carry);
        carry = {key0, 0u};
      }
      carry.value = Sum ? carry.value + w : ::max(carry.value, w);
    }
  } else if (live && value != 0u) {
    if constexpr (Sum) {
      atomicAdd(targets + key, value);
    } else {
      atomicMax(targets + key, value);
    }
  }
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
