// Device arithmetic of the BB solve shared by the single-system solve
// (solve.cu) and the per-colony batched solve (batch.cu).
#pragma once

#include <cstdint>

#include "device.cuh"
#include "solve.h"
#include "../../include/msb200.h"

namespace msb {

__device__ __forceinline__ float growth_factor(std::uint32_t law, float sensitivity, float free_load,
                                               float stall_load, float load) {
  if (law == MSB_GROWTH_LAW_EXPONENTIAL) {
    // exp in FP64 rounded once to FP32.
    return float(exp(double(-sensitivity * smax(0.0f, load))));
  }
  if (law == MSB_GROWTH_LAW_LINEAR) {
    return sclamp(1.0f - (load - free_load) / (stall_load - free_load), 0.0f, 1.0f);
  }
  return 1.0f;
}

// apply_mobility (cpu_contact_dynamics.cpp:40-53) plus drift.  Without
// drift the additions are of +0.0f, which leaves every value's bits as they
// are, so the drift arrays are only read when the system has some.
template <class Desc>
__device__ __forceinline__ void respond(const Desc& d, std::uint32_t b, float4 ba, float4 bb, const float w[6],
                                        float load, float v[6], float& rate) {
  float4 da = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float4 db = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (d.has_drift) {
    da = d.bodies.drift_a[b];
    db = d.bodies.drift_b[b];
  }
  const F3 axis{ba.x, ba.y, ba.z};
  const F3 tq{w[3], w[4], w[5]};
  const float s = (bb.y - bb.x) * dot(axis, tq);
  const F3 ang = tq * bb.x + axis * s;
  v[0] = w[0] * ba.w;
  v[1] = w[1] * ba.w;
  v[2] = w[2] * ba.w;
  v[3] = ang.x;
  v[4] = ang.y;
  v[5] = ang.z;
  v[0] += da.x;
  v[1] += da.y;
  v[2] += da.z;
  v[3] += db.x;
  v[4] += db.y;
  v[5] += db.z;
  rate = bb.z > 0.0f ? bb.z * growth_factor(d.law, d.sensitivity, d.free_load, d.stall_load, load) : bb.z;
}
// The same with the body's record read here.
template <class Desc>
__device__ __forceinline__ void respond(const Desc& d, std::uint32_t b, const float w[6], float load, float v[6],
                                        float& rate) {
  respond(d, b, __ldcs(&d.bodies.a[b]), __ldcs(&d.bodies.b[b]), w, load, v, rate);
}

// wrench_dot(jacobian, velocity) - lever * rate: one side's term of a row's
// gap rate, as row_gap forms it (cpp/cpu/cpu_contact_dynamics.cpp:149-159).
__device__ __forceinline__ float side_term(float4 ea, float4 eb, const float v[6], float rate) {
  float r = 0.0f;
  r += ea.x * v[0];
  r += ea.y * v[1];
  r += ea.z * v[2];
  r += ea.w * v[3];
  r += eb.x * v[4];
  r += eb.y * v[5];
  return r - eb.z * rate;
}

__device__ __forceinline__ float row_residual(float m, float gap) {
  return m > 0.0f ? fabsf(gap) : smax(0.0f, -gap);
}

// next_contact_step_length (contact_solver.hpp:54-62).
__device__ __forceinline__ float next_step(float current, double ss, double sy, double yy, std::uint32_t iteration) {
  if (!(sy > 0.0) || !(yy > 0.0)) return current;
  const double next = (iteration % 2u) == 1u ? ss / sy : sy / yy;
  return isfinite(next) && next > 0.0 ? float(next) : current;
}

// contact_system_diagonal_bound (cpu_contact_dynamics.cpp:247-260).
__device__ __forceinline__ float diagonal(float4 ja, float4 jb, float4 ba, float4 bb) {
  const F3 axis{ba.x, ba.y, ba.z};
  const F3 tq{ja.w, jb.x, jb.y};
  const float s = (bb.y - bb.x) * dot(axis, tq);
  const F3 ang = tq * bb.x + axis * s;
  float r = 0.0f;
  r += ja.x * (ja.x * ba.w);
  r += ja.y * (ja.y * ba.w);
  r += ja.z * (ja.z * ba.w);
  r += ja.w * ang.x;
  r += jb.x * ang.y;
  r += jb.y * ang.z;
  return r;
}

}  // namespace msb
