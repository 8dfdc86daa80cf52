// Flow drift of the cells inside the contact stepper: per body, the velocity
// and angular velocity that a fluid velocity field gives it over a substep,
// as Simulation::flow_drift_rates (cpp/core/simulation.cpp:159-186) computes
// them for detail::advance_contact_dynamics (cpp/core/contact_dynamics.cpp:426-431):
//
//   - SignalGrid::sample_velocity (cpp/core/signals.cpp:923-955) over the
//     interpolation stencil of signal_grid_stencil (signals.cpp:98-127,
//     357-420), clamped to the lattice; with obstacles, solid sites weigh
//     nothing and only the face-connected fluid component of the heaviest
//     site counts, renormalised;
//   - Simulation::flow_derivative (simulation.cpp:133-157): central
//     differences of the sampled velocity along each axis of more than one
//     site, and the equivalent-spheroid Jeffery rate of the axis;
//   - the midpoint rule of flow_drift_rates.
//
// Every float operation is the reference's, in its order (the library is
// built without contracted multiply-adds).
#include "flow.h"

#include <cmath>

#include "device.cuh"

namespace msb {
namespace {

constexpr int kThreads = 256;

struct Axis {
  std::uint32_t index[2];
  float weight[2];
  std::uint32_t count;
};

// interpolation_axis with GridSampleBound::clamped.
__device__ __forceinline__ Axis axis_weights(float position, float origin, float spacing, std::uint32_t dimension) {
  Axis a{{0u, 0u}, {1.0f, 0.0f}, 1u};
  if (dimension == 1) return a;
  double coordinate = (double(position) - double(origin)) / double(spacing);
  const double upper = double(dimension - 1);
  coordinate = sclamp(coordinate, 0.0, upper);
  const std::uint32_t lower = std::uint32_t(floor(coordinate));
  if (lower == dimension - 1) {
    a.index[0] = a.index[1] = lower;
    return a;
  }
  const float fraction = float(coordinate - double(lower));
  a.index[0] = lower;
  a.index[1] = lower + 1;
  a.weight[0] = 1.0f - fraction;
  a.weight[1] = fraction;
  a.count = 2;
  return a;
}

__device__ __forceinline__ std::size_t site_of(const FlowField& f, std::uint32_t x, std::uint32_t y, std::uint32_t z) {
  return std::size_t(x) * f.shape_y * f.shape_z + std::size_t(y) * f.shape_z + z;
}

// SignalGrid::sample_velocity(position, clamped).  A site's velocity is the
// mean of its two faces along each axis, w * 0.5f * (face0 + face1) per
// axis; the face sums come precomputed per site (the same float additions),
// so one float4 load replaces six scalar ones.
__device__ F3 sample_velocity(const FlowField& f, F3 p) {
  const Axis ax = axis_weights(p.x, f.origin.x, f.spacing.x, f.shape_x);
  const Axis ay = axis_weights(p.y, f.origin.y, f.spacing.y, f.shape_y);
  const Axis az = axis_weights(p.z, f.origin.z, f.spacing.z, f.shape_z);
  if (f.obstacles == nullptr) {
    // The stencil in the reference's order (x, then y, then z); entries
    // beyond an axis's count have weight 0 and are skipped, as are zero
    // weights.
    F3 r{0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const float w = ax.weight[i] * ay.weight[j] * az.weight[k];
          if (w == 0.0f) continue;
          const float4 s = f.sites[site_of(f, ax.index[i], ay.index[j], az.index[k])];
          r.x += w * 0.5f * s.x;
          r.y += w * 0.5f * s.y;
          r.z += w * 0.5f * s.z;
        }
      }
    }
    return r;
  }
  std::uint32_t cx[8], cy[8], cz[8];
  float weight[8];
  std::uint32_t count = 0;
  for (std::uint32_t i = 0; i < ax.count; ++i) {
    for (std::uint32_t j = 0; j < ay.count; ++j) {
      for (std::uint32_t k = 0; k < az.count; ++k) {
        cx[count] = ax.index[i];
        cy[count] = ay.index[j];
        cz[count] = az.index[k];
        weight[count] = ax.weight[i] * ay.weight[j] * az.weight[k];
        ++count;
      }
    }
  }
  if (f.obstacles != nullptr) {
    std::uint32_t seed = count;
    for (std::uint32_t i = 0; i < count; ++i) {
      if (f.obstacles[site_of(f, cx[i], cy[i], cz[i])] != 0) weight[i] = 0.0f;
      if (weight[i] > 0.0f && (seed == count || weight[i] > weight[seed])) seed = i;
    }
    if (seed == count) return F3{0.0f, 0.0f, 0.0f};  // all solid: no drift
    bool connected[8] = {false, false, false, false, false, false, false, false};
    connected[seed] = true;
    for (bool grew = true; grew;) {
      grew = false;
      for (std::uint32_t i = 0; i < count; ++i) {
        if (weight[i] <= 0.0f || connected[i]) continue;
        for (std::uint32_t j = 0; j < count; ++j) {
          const unsigned distance = unsigned(abs(int(cx[i]) - int(cx[j]))) + unsigned(abs(int(cy[i]) - int(cy[j]))) +
                                    unsigned(abs(int(cz[i]) - int(cz[j])));
          if (connected[j] && distance == 1) {
            connected[i] = true;
            grew = true;
            break;
          }
        }
      }
    }
    float total = 0.0f;
    for (std::uint32_t i = 0; i < count; ++i) {
      if (!connected[i]) weight[i] = 0.0f;
      total += weight[i];
    }
    for (std::uint32_t i = 0; i < count; ++i) weight[i] /= total;
  }
  F3 r{0.0f, 0.0f, 0.0f};
  for (std::uint32_t i = 0; i < count; ++i) {
    const float w = weight[i];
    if (w == 0.0f) continue;
    const float4 s = f.sites[site_of(f, cx[i], cy[i], cz[i])];
    r.x += w * 0.5f * s.x;
    r.y += w * 0.5f * s.y;
    r.z += w * 0.5f * s.z;
  }
  return r;
}

__global__ void flow_sites_kernel(FlowField f, float4* __restrict__ sites) {
  const std::uint64_t count = std::uint64_t(f.shape_x) * f.shape_y * f.shape_z;
  for (std::uint64_t s = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; s < count;
       s += std::uint64_t(gridDim.x) * blockDim.x) {
    const std::uint32_t z = std::uint32_t(s % f.shape_z);
    const std::uint32_t y = std::uint32_t((s / f.shape_z) % f.shape_y);
    const std::uint32_t x = std::uint32_t(s / (std::uint64_t(f.shape_z) * f.shape_y));
    const std::size_t xf0 = std::size_t(x) * f.shape_y * f.shape_z + std::size_t(y) * f.shape_z + z;
    const std::size_t xf1 = std::size_t(x + 1) * f.shape_y * f.shape_z + std::size_t(y) * f.shape_z + z;
    const std::size_t yf0 = std::size_t(x) * (f.shape_y + 1) * f.shape_z + std::size_t(y) * f.shape_z + z;
    const std::size_t yf1 = std::size_t(x) * (f.shape_y + 1) * f.shape_z + std::size_t(y + 1) * f.shape_z + z;
    const std::size_t zf0 = std::size_t(x) * f.shape_y * (f.shape_z + 1) + std::size_t(y) * (f.shape_z + 1) + z;
    const std::size_t zf1 = zf0 + 1;
    sites[s] = make_float4(f.x_faces[xf0] + f.x_faces[xf1], f.y_faces[yf0] + f.y_faces[yf1],
                           f.z_faces[zf0] + f.z_faces[zf1], 0.0f);
  }
}

// Simulation::flow_derivative(point, axis, lambda, rotates = true).
__device__ void flow_derivative(const FlowField& f, F3 point, F3 axis, float lambda, F3& velocity, F3& orientation) {
  const float h[3] = {f.spacing.x, f.spacing.y, f.spacing.z};
  const std::uint32_t dims[3] = {f.shape_x, f.shape_y, f.shape_z};
  F3 gradient[3] = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}};
  for (int k = 0; k < 3; ++k) {
    if (dims[k] == 1) continue;
    F3 offset{0.0f, 0.0f, 0.0f};
    if (k == 0) offset.x = h[k] * 0.5f;
    if (k == 1) offset.y = h[k] * 0.5f;
    if (k == 2) offset.z = h[k] * 0.5f;
    gradient[k] = (sample_velocity(f, point + offset) - sample_velocity(f, point - offset)) * (1.0f / h[k]);
  }
  const F3 ap = gradient[0] * axis.x + gradient[1] * axis.y + gradient[2] * axis.z;
  const F3 atp{dot(gradient[0], axis), dot(gradient[1], axis), dot(gradient[2], axis)};
  const F3 strain = (ap + atp) * 0.5f;
  const F3 spin = (ap - atp) * 0.5f;
  orientation = spin + (strain - axis * dot(axis, strain)) * lambda;
  velocity = sample_velocity(f, point);
}

// Simulation::flow_drift_rates(dt) for one body.
__device__ void drift_rates(const FlowField& f, float4 pl, float4 dr, float dt, F3& linear, F3& angular,
                            bool& valid) {
  const F3 position = xyz(pl);
  const F3 direction = xyz(dr);
  const float radius = dr.w;
  const float aspect = (pl.w + 2.0f * radius) / (2.0f * radius);
  const float lambda = (aspect * aspect - 1.0f) / (aspect * aspect + 1.0f);
  F3 velocity, orientation;
  flow_derivative(f, position, direction, lambda, velocity, orientation);
  const F3 midpoint = position + velocity * (dt * 0.5f);
  F3 mid_direction;
  valid = normalized(direction + orientation * (dt * 0.5f), mid_direction);
  if (!valid) return;
  F3 mid_velocity, mid_orientation;
  flow_derivative(f, midpoint, mid_direction, lambda, mid_velocity, mid_orientation);
  linear = mid_velocity;
  angular = cross(direction, mid_orientation);
}

__global__ void flow_drift_kernel(std::uint32_t n, GeometryBuffers state, const std::uint8_t* __restrict__ fixed,
                                  FlowField field, float dt, BodyArrays bodies, std::uint32_t* status) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    F3 linear{0.0f, 0.0f, 0.0f}, angular{0.0f, 0.0f, 0.0f};
    if (fixed == nullptr || fixed[s] == 0) {
      bool valid = true;
      drift_rates(field, state.pos_len[s], state.dir_rad[s], dt, linear, angular, valid);
      if (!valid || !finite3(linear) || !finite3(angular)) {
        raise_status(status, kStatusGeometry);
        linear = angular = F3{0.0f, 0.0f, 0.0f};
      }
    }
    bodies.drift_a[s] = make_float4(linear.x, linear.y, linear.z, 0.0f);
    bodies.drift_b[s] = make_float4(angular.x, angular.y, angular.z, 0.0f);
  }
}

// The largest drift speed at the start of a step (rates over dt = 0).
__global__ void flow_speed_kernel(std::uint32_t n, GeometryBuffers state, const std::uint8_t* __restrict__ fixed,
                                  FlowField field, std::uint32_t* speed_bits, std::uint32_t* status) {
  float largest = 0.0f;
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    if (fixed != nullptr && fixed[s] != 0) continue;
    F3 linear{0.0f, 0.0f, 0.0f}, angular{0.0f, 0.0f, 0.0f};
    bool valid = true;
    drift_rates(field, state.pos_len[s], state.dir_rad[s], 0.0f, linear, angular, valid);
    if (!valid) {
      raise_status(status, kStatusGeometry);
      continue;
    }
    largest = smax(largest, norm(linear));
  }
  for (int o = 16; o > 0; o >>= 1) largest = smax(largest, __shfl_down_sync(0xFFFFFFFFu, largest, o));
  if ((threadIdx.x & 31) == 0) {
    if (isfinite(largest)) {
      atomicMax(speed_bits, __float_as_uint(largest));
    } else {
      atomicMax(speed_bits, 0x7F800000u);
    }
  }
}

}  // namespace

void launch_flow_sites(const FlowField& field, float4* sites, cudaStream_t stream) {
  const std::uint64_t count = std::uint64_t(field.shape_x) * field.shape_y * field.shape_z;
  if (count == 0) return;
  flow_sites_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(field, sites);
  count_launch();
}

void launch_flow_drift(std::uint32_t n, GeometryBuffers state, const std::uint8_t* fixed, const FlowField& field,
                       float dt, BodyArrays bodies, std::uint32_t* status, cudaStream_t stream) {
  if (n == 0) return;
  flow_drift_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, state, fixed, field, dt, bodies, status);
  count_launch();
}

void launch_flow_speed(std::uint32_t n, GeometryBuffers state, const std::uint8_t* fixed, const FlowField& field,
                       std::uint32_t* speed_bits, std::uint32_t* status, cudaStream_t stream) {
  if (n == 0) return;
  flow_speed_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, state, fixed, field, speed_bits, status);
  count_launch();
}

}  // namespace msb
