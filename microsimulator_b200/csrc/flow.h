// Flow drift of the cells inside the contact stepper (flow.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"
#include "solve.h"
#include "step.h"

namespace msb {

// A velocity field on a lattice of sites (device pointers): face velocities
// x-major as the reference's signal grid stores them, optional solid mask,
// and per site the sums of its two faces along each axis (launch_flow_sites).
struct FlowField {
  std::uint32_t shape_x, shape_y, shape_z;
  float3 origin;
  float3 spacing;
  const float* x_faces;
  const float* y_faces;
  const float* z_faces;
  const std::uint8_t* obstacles;  // null: no obstacles
  const float4* sites;            // (x0 + x1, y0 + y1, z0 + z1, 0) per site
};

// The per-site face sums of `field` into `sites` (one float4 per site).
void launch_flow_sites(const FlowField& field, float4* sites, cudaStream_t stream);

// Writes each body's drift (drift_a: velocity, drift_b: angular velocity)
// for a substep of length dt from the geometry in `state`; fixed cells get
// none.  kStatusGeometry on a non-finite rate.
void launch_flow_drift(std::uint32_t n, GeometryBuffers state, const std::uint8_t* fixed, const FlowField& field,
                       float dt, BodyArrays bodies, std::uint32_t* status, cudaStream_t stream);
// The largest drift speed (float bits, atomic max into *speed_bits, which the
// caller zeroes) of the rates at dt = 0, for the substep plan.
void launch_flow_speed(std::uint32_t n, GeometryBuffers state, const std::uint8_t* fixed, const FlowField& field,
                       std::uint32_t* speed_bits, std::uint32_t* status, cudaStream_t stream);

}  // namespace msb
