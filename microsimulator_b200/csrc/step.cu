// Per-cell and per-row passes of the contact stepper
// (cpp/core/contact_dynamics.cpp:215-582 of the reference), in FP32 with the
// reference's operation order.

#include <cfloat>
#include <cstdint>

#include "device.cuh"
#include "kernels.h"
#include "step.h"
#include "../../include/msb200.h"

namespace msb {
namespace {

constexpr int kThreads = 256;
constexpr float kMaximumSubstepRotation = 0.5f;
constexpr float kMinimumLeverLength = 1.0e-6f;

__device__ __forceinline__ void atomic_max_nonnegative(std::uint32_t* bits, float value) {
  if (value > 0.0f) atomicMax(bits, __float_as_uint(value));
}

__global__ void pack_cells_kernel(std::uint32_t n, const float* px, const float* py, const float* pz,
                                  const float* dx, const float* dy, const float* dz, const float* len,
                                  const float* radius, GeometryBuffers out, std::uint32_t* status) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const F3 p{px[i], py[i], pz[i]};
    const F3 d{dx[i], dy[i], dz[i]};
    const float l = len[i];
    const float r = radius[i];
    const float m = norm(d);
    if (!finite3(p) || !finite3(d) || !isfinite(l) || !isfinite(r) || l < 0.0f || !(r > 0.0f) ||
        !(fabsf(m - 1.0f) <= 1.0e-5f)) {
      raise_status(status, kStatusGeometry);
    }
    out.pos_len[i] = make_float4(p.x, p.y, p.z, l);
    out.dir_rad[i] = make_float4(d.x, d.y, d.z, r);
  }
}

__global__ void unpack_cells_kernel(std::uint32_t n, GeometryBuffers in, float* px, float* py, float* pz, float* dx,
                                    float* dy, float* dz, float* len) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 pl = in.pos_len[i];
    const float4 dr = in.dir_rad[i];
    px[i] = pl.x;
    py[i] = pl.y;
    pz[i] = pl.z;
    len[i] = pl.w;
    dx[i] = dr.x;
    dy[i] = dr.y;
    dz[i] = dr.z;
  }
}

__global__ void make_bodies_kernel(std::uint32_t n, GeometryBuffers state, const float* __restrict__ growth,
                                   const std::uint8_t* __restrict__ fixed, GeometryBuffers rate_lengths,
                                   float colony_drag, BodyArrays bodies, Colonies colonies) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float drag = colonies.of_slot != nullptr ? colonies.drag[colonies.of_slot[s]] : colony_drag;
    const float4 pl = state.pos_len[s];
    const float4 dr = state.dir_rad[s];
    const float rate = growth[s] * rate_lengths.pos_len[s].w;
    float mt = 0.0f, ma = 0.0f, mtr = 0.0f;
    if (fixed == nullptr || fixed[s] == 0) {
      const float r = dr.w;
      const float total = pl.w + 2.0f * r;
      const float tr = drag * total;
      const float ax = 0.5f * tr * r * r;
      const float tv = tr * ((total * total) + 3.0f * r * r) / 12.0f;
      mt = 1.0f / tr;
      ma = 1.0f / ax;
      mtr = 1.0f / tv;
    }
    bodies.a[s] = make_float4(dr.x, dr.y, dr.z, mt);
    bodies.b[s] = make_float4(mtr, ma, rate, 0.0f);
    bodies.drift_a[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    bodies.drift_b[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
}

// length_lever (contact_dynamics.cpp:215-224).
__device__ __forceinline__ float length_lever(float4 pl, float4 dr, F3 centre, F3 outward) {
  const float length = pl.w;
  if (length <= kMinimumLeverLength) return 0.0f;
  const F3 axis = xyz(dr);
  const float coordinate = dot(axis, centre - xyz(pl)) / length;
  return smax(0.0f, sclamp(coordinate, -0.5f, 0.5f) * dot(axis, outward));
}

__device__ __forceinline__ float wrench_dot(float4 ja, float4 jb, float4 va, float4 vb) {
  float r = 0.0f;
  r += ja.x * va.x;
  r += ja.y * va.y;
  r += ja.z * va.z;
  r += ja.w * vb.x;
  r += jb.x * vb.y;
  r += jb.y * vb.z;
  return r;
}

__global__ void make_rows_kernel(const Touch* __restrict__ touches, std::uint32_t count, GeometryBuffers geometry,
                                 RowBuild prm, ResponseArrays response, int correct, RowArrays rows,
                                 std::uint32_t row_base, std::uint64_t* __restrict__ key_partner,
                                 float* __restrict__ multipliers, std::uint32_t* overlap_bits, Colonies colonies) {
  // Each warp takes a contiguous range of contacts, so that the deepest
  // overlap of each colony is folded per warp before it is written.
  const WarpRange range = warp_range(count);
  std::uint32_t deepest = 0u;
  KeyCarry carry;
  for (std::uint32_t base = range.begin; base < range.end; base += 32) {
    const std::uint32_t k = base + (threadIdx.x & 31u);
    const bool live = k < range.end;
    std::uint32_t colony = 0u;
    std::uint32_t depth = 0u;
    if (live) {
      const Touch t = touches[k];
      const bool wall = t.s2 == kInvalidSlot;
      colony = colonies.of_slot != nullptr ? colonies.of_slot[t.s1] : 0u;
      const float stiffness = colonies.of_slot != nullptr ? colonies.stiffness[colony] : prm.contact_stiffness;
      const float compliance = 1.0f / (wall ? prm.wall_stiffness : stiffness);
      float offset = smax(t.sep, -prm.recovery);
      const float c = t.sep < -prm.recovery ? compliance * prm.recovery / -t.sep : compliance;
      const F3 n{t.normal[0], t.normal[1], t.normal[2]};
      const F3 p{t.point[0], t.point[1], t.point[2]};
      const float4 pl1 = geometry.pos_len[t.s1];
      const float4 dr1 = geometry.dir_rad[t.s1];
      const F3 a1 = cross(p - xyz(pl1), n);
      const float l1 = length_lever(pl1, dr1, p - n * dr1.w, n);
      float4 ra = make_float4(-n.x, -n.y, -n.z, -a1.x);
      float4 rb = make_float4(-a1.y, -a1.z, l1, offset);
      float4 rc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      float4 rd = make_float4(0.0f, 0.0f, 0.0f, c);
      if (!wall) {
        const float4 pl2 = geometry.pos_len[t.s2];
        const float4 dr2 = geometry.dir_rad[t.s2];
        const F3 a2 = cross(p - xyz(pl2), n);
        const float l2 = length_lever(pl2, dr2, p + n * (t.sep + dr2.w), n * -1.0f);
        rc = make_float4(n.x, n.y, n.z, a2.x);
        rd = make_float4(a2.y, a2.z, l2, c);
      }
      if (correct) {
        // predicted_rate (contact_dynamics.cpp:286-301)
        float rate = wrench_dot(ra, rb, response.a[t.s1], response.b[t.s1]) - rb.z * response.a[t.s1].w;
        if (!wall) rate += wrench_dot(rc, rd, response.a[t.s2], response.b[t.s2]) - rd.z * response.a[t.s2].w;
        offset -= prm.dt * rate;
        rb.w = offset;
      }
      const std::uint32_t i = row_base + k;
      rows.a[i] = ra;
      rows.b[i] = rb;
      rows.c[i] = rc;
      rows.d[i] = rd;
      rows.slots[i] = make_uint2(t.s1, t.s2);
      key_partner[i] = wall ? (kWallTag | t.partner) : std::uint64_t(t.s2);
      multipliers[i] = 0.0f;
      depth = max_bits(0u, -t.sep);
      deepest = ::max(deepest, depth);
    }
    if (colonies.overlap_bits != nullptr) carry_item<false>(colonies.overlap_bits, carry, live, colony, depth);
  }
  if (colonies.overlap_bits != nullptr && (threadIdx.x & 31u) == 0u) carry_flush<false>(colonies.overlap_bits, carry);
  block_max_into(overlap_bits, deepest);
}

// ForceMemory::force with the occurrence rule of advance_substep
// (cpp/core/contact_dynamics.cpp:156-174,463-477): the force of the
// occurrence-th remembered row with the same key, or zero.  A remembered row
// counts only if its cells' ids match the current ones.
__global__ void warm_start_kernel(std::uint32_t rows, const uint2* __restrict__ slots, KeyedLists current,
                                  KeyedLists memory, MemoryCells cells, int has_memory,
                                  float* __restrict__ multipliers) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const uint2 sl = slots[i];
    const std::uint32_t first = sl.x;
    const std::uint64_t key = current.partner[i];
    std::uint32_t occurrence = 0;
    for (std::uint32_t k = current.offsets[first]; k < current.offsets[first + 1]; ++k) {
      const std::uint32_t r = current.rows[k];
      if (r >= i) break;
      occurrence += current.partner[r] == key ? 1u : 0u;
    }
    float force = 0.0f;
    if (has_memory && first < cells.cells) {
      const std::uint64_t first_id = cells.ids[first];
      const std::uint64_t partner_id = sl.y == kInvalidSlot ? key : cells.ids[sl.y];
      for (std::uint32_t k = memory.offsets[first]; k < memory.offsets[first + 1]; ++k) {
        const std::uint32_t r = memory.rows[k];
        if (memory.partner[r] == key && cells.first_ids[r] == first_id && cells.partner_ids[r] == partner_id) {
          if (occurrence == 0) {
            force = memory.multipliers[r];
            break;
          }
          --occurrence;
        }
      }
    }
    multipliers[i] = force;
  }
}

__global__ void memory_ids_kernel(std::uint32_t rows, const uint2* __restrict__ slots,
                                  const std::uint64_t* __restrict__ partner, const std::uint64_t* __restrict__ ids,
                                  std::uint64_t* __restrict__ first_ids, std::uint64_t* __restrict__ partner_ids) {
  for (std::uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const uint2 sl = slots[r];
    first_ids[r] = ids[sl.x];
    partner_ids[r] = sl.y == kInvalidSlot ? partner[r] : ids[sl.y];
  }
}

// rotate_axis_angle (cpp/core/mechanics_integration.cpp:9-20).
__device__ __forceinline__ bool rotate_axis_angle(F3 d, F3 rot, float max_rot, F3& out) {
  const float mag = norm(rot);
  if (mag <= 1.0e-12f || max_rot == 0.0f) {
    out = d;
    return true;
  }
  const float angle = smin(mag, max_rot);
  const F3 axis = rot * (1.0f / mag);
  const float c = cosf(angle);
  const float s = sinf(angle);
  return normalized(d * c + cross(axis, d) * s + axis * (dot(axis, d) * (1.0f - c)), out);
}

__global__ void move_kernel(std::uint32_t n, GeometryBuffers base, ResponseArrays response, float dt,
                            GeometryBuffers trial, std::uint32_t* rotation_bits, std::uint32_t* invalid,
                            std::uint32_t* status, std::uint32_t* displacement_bits) {
  std::uint32_t largest_rotation = 0u, largest_move = 0u;
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 va = response.a[s];
    const float4 vb = response.b[s];
    const F3 rot{vb.x * dt, vb.y * dt, vb.z * dt};
    if (!finite3(rot)) {
      atomicExch(invalid, 1u);
      continue;
    }
    const float angle = norm(rot);
    largest_rotation = max_bits(largest_rotation, angle);
    if (angle > kMaximumSubstepRotation) {
      atomicExch(invalid, 1u);
      continue;
    }
    const float4 pl = base.pos_len[s];
    const float4 dr = base.dir_rad[s];
    const F3 pos = xyz(pl) + F3{va.x, va.y, va.z} * dt;
    F3 dir;
    if (!rotate_axis_angle(xyz(dr), rot, kMaximumSubstepRotation, dir)) {
      raise_status(status, kStatusGeometry);
      atomicExch(invalid, 1u);
      continue;
    }
    const float len = pl.w + va.w * dt;
    if (!finite3(pos) || !finite3(dir) || !isfinite(len) || len < 0.0f) atomicExch(invalid, 1u);
    const float4 moved_pl = make_float4(pos.x, pos.y, pos.z, len);
    const float4 moved_dr = make_float4(dir.x, dir.y, dir.z, dr.w);
    trial.pos_len[s] = moved_pl;
    trial.dir_rad[s] = moved_dr;
    if (displacement_bits != nullptr) {
      // How far any face of the cell's unpadded box moved, rounded up: the
      // bound under which a re-check may reuse the substep's candidates.
      double from[6], to[6];
      padded_box(pl, dr, 0.0f, from);
      padded_box(moved_pl, moved_dr, 0.0f, to);
      double moved = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) moved = fmax(moved, fabs(to[k] - from[k]));
      const float bound = isfinite(moved) ? __double2float_ru(moved) : __int_as_float(0x7F800000);
      largest_move = max_bits(largest_move, bound);
    }
  }
  block_max_into(rotation_bits, largest_rotation);
  if (displacement_bits != nullptr) block_max_into(displacement_bits, largest_move);
}

__global__ void guess_response_kernel(std::uint32_t n, const float4* __restrict__ guess, BodyArrays bodies,
                                      float inverse_dt, ResponseArrays out) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 g = guess[s];
    const float rate = bodies.b[s].z;
    out.a[s] = make_float4(g.x * inverse_dt, g.y * inverse_dt, 0.0f, rate);
    out.b[s] = make_float4(0.0f, 0.0f, g.z * inverse_dt, 0.0f);
  }
}

// The wrench that moves body b by v (the inverse of apply_mobility,
// cpp/cpu/cpu_contact_dynamics.cpp:40-53); zero for a body that cannot move.
__device__ __forceinline__ void wrench_for(float4 ba, float4 bb, const float v[6], float w[6]) {
  const bool moves = ba.w > 0.0f && bb.x > 0.0f && bb.y > 0.0f;
  for (int k = 0; k < 6; ++k) w[k] = 0.0f;
  if (!moves) return;
  const F3 axis{ba.x, ba.y, ba.z};
  const F3 ang{v[3], v[4], v[5]};
  const float s = (1.0f / bb.y - 1.0f / bb.x) * dot(axis, ang);
  const F3 tq = ang * (1.0f / bb.x) + axis * s;
  w[0] = v[0] / ba.w;
  w[1] = v[1] / ba.w;
  w[2] = v[2] / ba.w;
  w[3] = tq.x;
  w[4] = tq.y;
  w[5] = tq.z;
}

__global__ void guess_forces_body_kernel(std::uint32_t n, IncidenceArrays inc, BodyArrays bodies,
                                         ResponseArrays current, ResponseArrays guess, const uint2* __restrict__ slots,
                                         float* __restrict__ delta) {
  for (std::uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
    const float4 ca = current.a[b], cb = current.b[b], ga = guess.a[b], gb = guess.b[b];
    const float dv[6] = {ga.x - ca.x, ga.y - ca.y, ga.z - ca.z, gb.x - cb.x, gb.y - cb.y, gb.z - cb.z};
    float w[6];
    wrench_for(bodies.a[b], bodies.b[b], dv, w);
    const std::uint32_t begin = inc.offsets[b], end = inc.offsets[b + 1];
    float uu = 0.0f;
    float r[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (std::uint32_t k = begin; k < end; ++k) {
      const float4 ea = inc.a[k], eb = inc.b[k];
      const float j[6] = {ea.x, ea.y, ea.z, ea.w, eb.x, eb.y};
      float u = 0.0f;
      for (int q = 0; q < 6; ++q) u += j[q] * w[q];
      uu += u * u;
      for (int q = 0; q < 6; ++q) r[q] += u * j[q];
    }
    float rr = 0.0f;
    for (int q = 0; q < 6; ++q) rr += r[q] * r[q];
    if (!(rr > 0.0f) || !(uu > 0.0f)) continue;
    const float alpha = uu / rr;
    for (std::uint32_t k = begin; k < end; ++k) {
      const float4 ea = inc.a[k], eb = inc.b[k];
      const float u = ea.x * w[0] + ea.y * w[1] + ea.z * w[2] + ea.w * w[3] + eb.x * w[4] + eb.y * w[5];
      const std::uint32_t row = __float_as_uint(eb.w) >> 1;  // side bits: row << 1 | side
      const float share = slots[row].y == kInvalidSlot ? 1.0f : 0.5f;
      // At most two additions onto zero per row: the sum does not depend on their order.
      atomicAdd(&delta[row], share * alpha * u);
    }
  }
}

__global__ void guess_forces_row_kernel(std::uint32_t rows, const float* __restrict__ delta,
                                        float* __restrict__ multipliers) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const float m = multipliers[i] + delta[i];
    multipliers[i] = isfinite(m) ? smax(0.0f, m) : multipliers[i];
  }
}

__global__ void largest_rotation_kernel(std::uint32_t n, ResponseArrays response, float dt,
                                        std::uint32_t* rotation_bits) {
  std::uint32_t largest = 0u;
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 vb = response.b[s];
    const float angle = norm(F3{vb.x * dt, vb.y * dt, vb.z * dt});
    largest = max_bits(largest, isfinite(angle) ? angle : __int_as_float(0x7F800000));
  }
  block_max_into(rotation_bits, largest);
}

__global__ void restore_kernel(std::uint32_t n, GeometryBuffers src, GeometryBuffers dst, std::uint32_t* status) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 pl = src.pos_len[s];
    const float4 dr = src.dir_rad[s];
    F3 d;
    if (!finite3(xyz(pl)) || !isfinite(pl.w) || pl.w < 0.0f || !normalized(xyz(dr), d)) {
      raise_status(status, kStatusGeometry);
      d = xyz(dr);
    }
    dst.pos_len[s] = pl;
    dst.dir_rad[s] = make_float4(d.x, d.y, d.z, dr.w);
  }
}

__global__ void recheck_kernel(const Touch* __restrict__ touches, std::uint32_t count, KeyedLists current,
                               const float* slack_ptr, float wall_stiffness, float contact_stiffness,
                               std::uint32_t* __restrict__ flags, std::uint32_t* overlap_bits, Colonies colonies) {
  // Contiguous ranges per warp, as in make_rows_kernel: the per-colony
  // deepest overlaps and flag counts are folded per warp.
  const WarpRange range = warp_range(count);
  std::uint32_t deepest = 0u;
  KeyCarry deepest_carry, flagged_carry;
  for (std::uint32_t base = range.begin; base < range.end; base += 32) {
    const std::uint32_t k = base + (threadIdx.x & 31u);
    const bool live = k < range.end;
    std::uint32_t colony = 0u;
    std::uint32_t depth = 0u;
    std::uint32_t flagged = 0u;
    if (live) {
      const Touch t = touches[k];
      depth = max_bits(0u, -t.sep);
      deepest = ::max(deepest, depth);
      colony = colonies.of_slot != nullptr ? colonies.of_slot[t.s1] : 0u;
      const float slack = colonies.slack != nullptr ? colonies.slack[colony] : *slack_ptr;
      if (colonies.stiffness != nullptr) contact_stiffness = colonies.stiffness[colony];
      const bool wall = t.s2 == kInvalidSlot;
      const std::uint64_t key = wall ? (kWallTag | t.partner) : std::uint64_t(t.s2);
      float force = 0.0f;
      for (std::uint32_t j = current.offsets[t.s1]; j < current.offsets[t.s1 + 1]; ++j) {
        const std::uint32_t r = current.rows[j];
        if (current.partner[r] == key) force += current.multipliers[r];
      }
      const float compliance = 1.0f / (wall ? wall_stiffness : contact_stiffness);
      const float allowed = slack + force * compliance;
      flagged = t.sep < -allowed ? 1u : 0u;
      flags[k] = flagged;
    }
    if (colonies.overlap_bits != nullptr) carry_item<false>(colonies.overlap_bits, deepest_carry, live, colony, depth);
    if (colonies.flagged != nullptr) carry_item<true>(colonies.flagged, flagged_carry, live, colony, flagged);
  }
  if ((threadIdx.x & 31u) == 0u) {
    if (colonies.overlap_bits != nullptr) carry_flush<false>(colonies.overlap_bits, deepest_carry);
    if (colonies.flagged != nullptr) carry_flush<true>(colonies.flagged, flagged_carry);
  }
  block_max_into(overlap_bits, deepest);
}

__global__ void gather_flagged_kernel(const Touch* __restrict__ touches, std::uint32_t count,
                                      const std::uint32_t* __restrict__ flags, const std::uint32_t* __restrict__ offsets,
                                      Touch* __restrict__ out) {
  for (std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    if (flags[k]) out[offsets[k]] = touches[k];
  }
}

__global__ void slack_kernel(const std::uint32_t* overlap_bits, float tolerance, float recovery, float* slack) {
  if (threadIdx.x == 0) {
    const float starting = __uint_as_float(*overlap_bits);
    *slack = tolerance + smax(0.0f, starting - recovery);
  }
}

__global__ void colony_slack_kernel(std::uint32_t colonies, const std::uint32_t* overlap_bits,
                                    const float* tolerance, float recovery, float* slack) {
  for (std::uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < colonies; c += gridDim.x * blockDim.x) {
    const float starting = __uint_as_float(overlap_bits[c]);
    slack[c] = tolerance[c] + smax(0.0f, starting - recovery);
  }
}

__global__ void colony_refine_kernel(std::uint32_t colonies, const std::uint32_t* __restrict__ flagged,
                                     std::uint32_t* __restrict__ active) {
  for (std::uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < colonies; c += gridDim.x * blockDim.x) {
    active[c] = (active[c] != 0u && flagged[c] != 0u) ? 1u : 0u;
  }
}

__global__ void colony_reset_overlap_kernel(std::uint32_t colonies, const std::uint32_t* __restrict__ active,
                                            std::uint32_t* __restrict__ overlap_bits) {
  for (std::uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < colonies; c += gridDim.x * blockDim.x) {
    if (active[c] != 0u) overlap_bits[c] = 0u;
  }
}

__global__ void colony_of_slot_kernel(std::uint32_t colonies, const std::uint32_t* __restrict__ offsets,
                                      std::uint32_t n, std::uint32_t* __restrict__ of_slot) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    // The last colony whose first slot is at or before s.
    std::uint32_t lo = 0, hi = colonies;
    while (hi - lo > 1) {
      const std::uint32_t mid = (lo + hi) / 2;
      if (offsets[mid] <= s) {
        lo = mid;
      } else {
        hi = mid;
      }
    }
    of_slot[s] = lo;
  }
}

__global__ void growth_bound_kernel(std::uint32_t n, GeometryBuffers state, const float* __restrict__ growth, float dt,
                                    std::uint32_t* bits) {
  float local = 0.0f;
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float g = fabsf(growth[s]) * state.pos_len[s].w * 0.5f * dt / state.dir_rad[s].w;
    local = smax(local, g);
  }
  for (int o = 16; o > 0; o >>= 1) local = smax(local, __shfl_down_sync(0xFFFFFFFFu, local, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonnegative(bits, local);
}

__global__ void outputs_kernel(std::uint32_t n, ResponseArrays response, GeometryBuffers base, GeometryBuffers initial,
                               float* velocities, float* loads, float* increments) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    if (velocities != nullptr) {
      const float4 va = response.a[s];
      velocities[3 * std::uint64_t(s)] = va.x;
      velocities[3 * std::uint64_t(s) + 1] = va.y;
      velocities[3 * std::uint64_t(s) + 2] = va.z;
    }
    if (loads != nullptr) loads[s] = response.b[s].w;
    if (increments != nullptr) increments[s] = base.pos_len[s].w - initial.pos_len[s].w;
  }
}

__global__ void copy_loads_kernel(std::uint32_t n, ResponseArrays response, float* loads) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    loads[s] = response.b[s].w;
  }
}

__global__ void rows_from_records_kernel(const msb_contact_row* __restrict__ in, std::uint32_t count, RowArrays rows) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const msb_contact_row r = in[i];
    rows.a[i] = make_float4(r.first_jacobian[0], r.first_jacobian[1], r.first_jacobian[2], r.first_jacobian[3]);
    rows.b[i] = make_float4(r.first_jacobian[4], r.first_jacobian[5], r.first_length_lever, r.offset);
    rows.c[i] = make_float4(r.second_jacobian[0], r.second_jacobian[1], r.second_jacobian[2], r.second_jacobian[3]);
    rows.d[i] = make_float4(r.second_jacobian[4], r.second_jacobian[5], r.second_length_lever, r.compliance);
    rows.slots[i] = make_uint2(r.first_slot, r.second_slot);
  }
}

__global__ void bodies_from_records_kernel(const msb_contact_body* __restrict__ in, std::uint32_t count,
                                           BodyArrays bodies) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const msb_contact_body b = in[i];
    bodies.a[i] = make_float4(b.axis.x, b.axis.y, b.axis.z, b.translational_mobility);
    bodies.b[i] = make_float4(b.transverse_mobility, b.axial_mobility, b.length_rate, 0.0f);
    bodies.drift_a[i] = make_float4(b.drift[0], b.drift[1], b.drift[2], 0.0f);
    bodies.drift_b[i] = make_float4(b.drift[3], b.drift[4], b.drift[5], 0.0f);
  }
}

__global__ void response_layout_kernel(std::uint32_t n, ResponseArrays response, float* velocities, float* loads,
                                       float* rates) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 va = response.a[s];
    const float4 vb = response.b[s];
    if (velocities != nullptr) {
      float* v = velocities + 6 * std::uint64_t(s);
      v[0] = va.x;
      v[1] = va.y;
      v[2] = va.z;
      v[3] = vb.x;
      v[4] = vb.y;
      v[5] = vb.z;
    }
    if (loads != nullptr) loads[s] = vb.w;
    if (rates != nullptr) rates[s] = va.w;
  }
}

}  // namespace

void launch_pack_cells(std::uint32_t n, const float* px, const float* py, const float* pz, const float* dx,
                       const float* dy, const float* dz, const float* len, const float* radius, GeometryBuffers out,
                       std::uint32_t* status, cudaStream_t stream) {
  if (n == 0) return;
  pack_cells_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, px, py, pz, dx, dy, dz, len, radius, out,
                                                                     status);
  count_launch();
}

void launch_unpack_cells(std::uint32_t n, GeometryBuffers in, float* px, float* py, float* pz, float* dx, float* dy,
                         float* dz, float* len, cudaStream_t stream) {
  if (n == 0) return;
  unpack_cells_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, in, px, py, pz, dx, dy, dz, len);
  count_launch();
}

void launch_make_bodies(std::uint32_t n, GeometryBuffers state, const float* growth_rates, const std::uint8_t* fixed,
                        GeometryBuffers rate_lengths, float drag, BodyArrays bodies, cudaStream_t stream,
                        Colonies colonies) {
  if (n == 0) return;
  make_bodies_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, state, growth_rates, fixed, rate_lengths,
                                                                      drag, bodies, colonies);
  count_launch();
}

void launch_make_rows(const Touch* touches, std::uint32_t count, GeometryBuffers geometry, RowBuild prm,
                      const ResponseArrays* response, RowArrays rows, std::uint32_t row_base,
                      std::uint64_t* key_partner, float* multipliers, std::uint32_t* overlap_bits,
                      cudaStream_t stream, Colonies colonies) {
  if (count == 0) return;
  const ResponseArrays none{nullptr, nullptr};
  make_rows_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(
      touches, count, geometry, prm, response != nullptr ? *response : none, response != nullptr ? 1 : 0, rows,
      row_base, key_partner, multipliers, overlap_bits, colonies);
  count_launch();
}

void launch_warm_start(std::uint32_t rows, const uint2* slots, KeyedLists current, const KeyedLists* memory,
                       MemoryCells cells, float* multipliers, cudaStream_t stream) {
  if (rows == 0) return;
  const KeyedLists none{nullptr, nullptr, nullptr, nullptr};
  warm_start_kernel<<<grid_for(rows, kThreads), kThreads, 0, stream>>>(
      rows, slots, current, memory != nullptr ? *memory : none, cells, memory != nullptr ? 1 : 0, multipliers);
  count_launch();
}

void launch_memory_ids(std::uint32_t rows, const uint2* slots, const std::uint64_t* partner, const std::uint64_t* ids,
                       std::uint64_t* first_ids, std::uint64_t* partner_ids, cudaStream_t stream) {
  if (rows == 0) return;
  memory_ids_kernel<<<grid_for(rows, kThreads), kThreads, 0, stream>>>(rows, slots, partner, ids, first_ids,
                                                                        partner_ids);
  count_launch();
}

void launch_move(std::uint32_t n, GeometryBuffers base, ResponseArrays response, float dt, GeometryBuffers trial,
                 std::uint32_t* rotation_bits, std::uint32_t* invalid, std::uint32_t* status, cudaStream_t stream,
                 std::uint32_t* displacement_bits) {
  if (n == 0) return;
  move_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, base, response, dt, trial, rotation_bits, invalid,
                                                               status, displacement_bits);
  count_launch();
}

void launch_guess_response(std::uint32_t n, const float4* guess, BodyArrays bodies, float step_dt,
                           ResponseArrays out, cudaStream_t stream) {
  if (n == 0) return;
  guess_response_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, guess, bodies, 1.0f / step_dt, out);
  count_launch();
}

void launch_guess_forces(std::uint32_t n, std::uint32_t rows, IncidenceArrays incidence, BodyArrays bodies,
                         ResponseArrays current, ResponseArrays guess, const uint2* slots, float* delta,
                         float* multipliers, cudaStream_t stream) {
  if (n == 0 || rows == 0) return;
  cudaMemsetAsync(delta, 0, rows * sizeof(float), stream);
  guess_forces_body_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, incidence, bodies, current, guess,
                                                                          slots, delta);
  count_launch();
  guess_forces_row_kernel<<<grid_for(rows, kThreads), kThreads, 0, stream>>>(rows, delta, multipliers);
  count_launch();
}

void launch_largest_rotation(std::uint32_t n, ResponseArrays response, float dt, std::uint32_t* rotation_bits,
                             cudaStream_t stream) {
  if (n == 0) return;
  largest_rotation_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, response, dt, rotation_bits);
  count_launch();
}

void launch_restore(std::uint32_t n, GeometryBuffers src, GeometryBuffers dst, std::uint32_t* status,
                    cudaStream_t stream) {
  if (n == 0) return;
  restore_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, src, dst, status);
  count_launch();
}

void launch_recheck(const Touch* touches, std::uint32_t count, KeyedLists current, const float* slack,
                    float wall_stiffness, float contact_stiffness, std::uint32_t* flags, std::uint32_t* overlap_bits,
                    cudaStream_t stream, Colonies colonies) {
  if (count == 0) return;
  recheck_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(touches, count, current, slack, wall_stiffness,
                                                                      contact_stiffness, flags, overlap_bits, colonies);
  count_launch();
}

void launch_gather_flagged(const Touch* touches, std::uint32_t count, const std::uint32_t* flags,
                           const std::uint32_t* offsets, Touch* out, cudaStream_t stream) {
  if (count == 0) return;
  gather_flagged_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(touches, count, flags, offsets, out);
  count_launch();
}

void launch_slack(const std::uint32_t* overlap_bits, float tolerance, float recovery, float* slack,
                  cudaStream_t stream) {
  slack_kernel<<<1, 32, 0, stream>>>(overlap_bits, tolerance, recovery, slack);
  count_launch();
}

void launch_colony_slack(std::uint32_t colonies, const std::uint32_t* overlap_bits, const float* tolerance,
                         float recovery, float* slack, cudaStream_t stream) {
  if (colonies == 0) return;
  colony_slack_kernel<<<grid_for(colonies, kThreads), kThreads, 0, stream>>>(colonies, overlap_bits, tolerance,
                                                                             recovery, slack);
  count_launch();
}

void launch_colony_refine(std::uint32_t colonies, const std::uint32_t* flagged, std::uint32_t* active,
                          cudaStream_t stream) {
  if (colonies == 0) return;
  colony_refine_kernel<<<grid_for(colonies, kThreads), kThreads, 0, stream>>>(colonies, flagged, active);
  count_launch();
}

void launch_colony_reset_overlap(std::uint32_t colonies, const std::uint32_t* active, std::uint32_t* overlap_bits,
                                 cudaStream_t stream) {
  if (colonies == 0) return;
  colony_reset_overlap_kernel<<<grid_for(colonies, kThreads), kThreads, 0, stream>>>(colonies, active, overlap_bits);
  count_launch();
}

void launch_colony_of_slot(std::uint32_t colonies, const std::uint32_t* offsets, std::uint32_t n,
                           std::uint32_t* of_slot, cudaStream_t stream) {
  if (n == 0 || colonies == 0) return;
  colony_of_slot_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(colonies, offsets, n, of_slot);
  count_launch();
}

void launch_growth_bound(std::uint32_t n, GeometryBuffers state, const float* growth_rates, float dt,
                         std::uint32_t* bits, cudaStream_t stream) {
  if (n == 0) return;
  growth_bound_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, state, growth_rates, dt, bits);
  count_launch();
}

void launch_outputs(std::uint32_t n, ResponseArrays response, GeometryBuffers base, GeometryBuffers initial,
                    float* velocities, float* loads, float* increments, cudaStream_t stream) {
  if (n == 0) return;
  outputs_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, response, base, initial, velocities, loads,
                                                                  increments);
  count_launch();
}

void launch_copy_loads(std::uint32_t n, ResponseArrays response, float* loads, cudaStream_t stream) {
  if (n == 0) return;
  copy_loads_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, response, loads);
  count_launch();
}

void launch_rows_from_records(const void* records, std::uint32_t count, RowArrays rows, cudaStream_t stream) {
  if (count == 0) return;
  rows_from_records_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(
      static_cast<const msb_contact_row*>(records), count, rows);
  count_launch();
}

void launch_bodies_from_records(const void* records, std::uint32_t count, BodyArrays bodies, cudaStream_t stream) {
  if (count == 0) return;
  bodies_from_records_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(
      static_cast<const msb_contact_body*>(records), count, bodies);
  count_launch();
}

void launch_response_to_host_layout(std::uint32_t n, ResponseArrays response, float* velocities, float* loads,
                                    float* rates, cudaStream_t stream) {
  if (n == 0) return;
  response_layout_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, response, velocities, loads, rates);
  count_launch();
}

}  // namespace msb
