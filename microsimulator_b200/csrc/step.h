// Per-cell and per-row passes of the contact stepper on the device.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"
#include "solve.h"

namespace msb {

// Geometry buffers of one set of cells (see kernels.h for the layout).
struct GeometryBuffers {
  float4* pos_len;
  float4* dir_rad;
};

constexpr std::uint64_t kWallTag = 1ull << 63;

// A batch of independent colonies stepped together: the colony of each cell
// slot and each colony's drag and contact stiffness, and each colony's
// deepest overlap (bits of a non-negative float) and overlap slack.  All
// null for a single system, whose scalar parameters apply.
struct Colonies {
  const std::uint32_t* of_slot;
  const float* drag;
  const float* stiffness;
  std::uint32_t* overlap_bits;
  const float* slack;
  std::uint32_t* flagged;  // per colony: touches the overlap test flagged
};
// Between refinement rounds of a batch: colonies whose overlap test flagged
// nothing leave the search (active = 0) and keep their overlap record;
// the others reset their record for the next test.
void launch_colony_refine(std::uint32_t colonies, const std::uint32_t* flagged, std::uint32_t* active,
                          cudaStream_t stream);
void launch_colony_reset_overlap(std::uint32_t colonies, const std::uint32_t* active, std::uint32_t* overlap_bits,
                                 cudaStream_t stream);

// Packs SoA cell arrays (device pointers) into float4 geometry, checking
// what WorldState::validate checks.  status: kStatusGeometry on bad input.
void launch_pack_cells(std::uint32_t n, const float* px, const float* py, const float* pz, const float* dx,
                       const float* dy, const float* dz, const float* len, const float* radius,
                       GeometryBuffers out, std::uint32_t* status, cudaStream_t stream);
void launch_unpack_cells(std::uint32_t n, GeometryBuffers in, float* px, float* py, float* pz, float* dx, float* dy,
                         float* dz, float* len, cudaStream_t stream);

// make_bodies (contact_dynamics.cpp:257-284).
// Elongation rates use the lengths of `rate_lengths` (the step's initial geometry).
void launch_make_bodies(std::uint32_t n, GeometryBuffers state, const float* growth_rates, const std::uint8_t* fixed,
                        GeometryBuffers rate_lengths, float drag, BodyArrays bodies, cudaStream_t stream,
                        Colonies colonies = {});

// make_row over `count` touches into rows [row_base, row_base + count), with
// their keys; the deepest overlap goes to *overlap_bits.  With `response`,
// each row's offset is moved by -dt * predicted rate (refinement rows).
struct RowBuild {
  float wall_stiffness;
  float contact_stiffness;
  float recovery;
  float dt;
};
void launch_make_rows(const Touch* touches, std::uint32_t count, GeometryBuffers geometry, RowBuild prm,
                      const ResponseArrays* response, RowArrays rows, std::uint32_t row_base,
                      std::uint64_t* key_partner, float* multipliers, std::uint32_t* overlap_bits,
                      cudaStream_t stream, Colonies colonies = {});

// Initial multipliers from the previous substep's forces (ForceMemory).
struct KeyedLists {
  const std::uint32_t* offsets;
  const std::uint32_t* rows;
  const std::uint64_t* partner;
  const float* multipliers;
};
// The cells a remembered row belongs to, so that forces carried from one
// step to the next never reach a slot that now holds another cell (a
// divided parent's slot holds its first daughter).
struct MemoryCells {
  const std::uint64_t* first_ids;    // per remembered row: its first cell's id
  const std::uint64_t* partner_ids;  // per remembered row: its second cell's id, or its wall key
  const std::uint64_t* ids;          // the current ids, by slot
  std::uint32_t cells;               // cells when the memory was made; later slots are new
};
void launch_warm_start(std::uint32_t rows, const uint2* slots, KeyedLists current, const KeyedLists* memory,
                       MemoryCells cells, float* multipliers, cudaStream_t stream);
// Records the cell ids of remembered rows (see MemoryCells).
void launch_memory_ids(std::uint32_t rows, const uint2* slots, const std::uint64_t* partner,
                       const std::uint64_t* ids, std::uint64_t* first_ids, std::uint64_t* partner_ids,
                       cudaStream_t stream);

// moved (contact_dynamics.cpp:311-356): trial geometry, largest rotation
// (bits) and a validity flag (0 = valid).
// With displacement_bits, also the largest distance any face of a cell's
// unpadded FP64 box moved (float bits, rounded up).
void launch_move(std::uint32_t n, GeometryBuffers base, ResponseArrays response, float dt, GeometryBuffers trial,
                 std::uint32_t* rotation_bits, std::uint32_t* invalid, std::uint32_t* status, cudaStream_t stream,
                 std::uint32_t* displacement_bits = nullptr);
// A response from a per-cell motion guess: guess[s] = (dx, dy, dtheta, _),
// the displacement in the xy-plane and the turn about z over `step_dt`;
// the elongation rate is each body's nominal rate.
void launch_guess_response(std::uint32_t n, const float4* guess, BodyArrays bodies, float step_dt,
                           ResponseArrays out, cudaStream_t stream);
// Moves start multipliers toward the forces a motion guess asks of each
// body.  Per body b: the wrench w = M^-1 (guessed - current response) that
// the guess lacks, and the least-squares step along its rows' jacobians
// (delta_k = alpha j_k.w, alpha = sum (j_k.w)^2 / |sum (j_k.w) j_k|^2); a
// row takes the mean of its bodies' steps (a wall row its one body's), and
// multipliers become max(0, multipliers + delta).  `delta` is scratch of
// `rows` floats.
void launch_guess_forces(std::uint32_t n, std::uint32_t rows, IncidenceArrays incidence, BodyArrays bodies,
                         ResponseArrays current, ResponseArrays guess, const uint2* slots, float* delta,
                         float* multipliers, cudaStream_t stream);
// Largest angle of a response (infinity when one is not finite).
void launch_largest_rotation(std::uint32_t n, ResponseArrays response, float dt, std::uint32_t* rotation_bits,
                             cudaStream_t stream);
// WorldState::set_cell_geometry over all cells: dst = src with normalized directions.
void launch_restore(std::uint32_t n, GeometryBuffers src, GeometryBuffers dst, std::uint32_t* status,
                    cudaStream_t stream);
// The overlap test after a move (contact_dynamics.cpp:520-548): flags the
// touches deeper than the slack plus what their own force presses in.
void launch_recheck(const Touch* touches, std::uint32_t count, KeyedLists current, const float* slack,
                    float wall_stiffness, float contact_stiffness, std::uint32_t* flags, std::uint32_t* overlap_bits,
                    cudaStream_t stream, Colonies colonies = {});
void launch_gather_flagged(const Touch* touches, std::uint32_t count, const std::uint32_t* flags,
                           const std::uint32_t* offsets, Touch* out, cudaStream_t stream);
// The substep slack: tolerance + max(0, deepest - recovery).
void launch_slack(const std::uint32_t* overlap_bits, float tolerance, float recovery, float* slack,
                  cudaStream_t stream);
// The slack of each colony of a batch from its deepest overlap and tolerance.
void launch_colony_slack(std::uint32_t colonies, const std::uint32_t* overlap_bits, const float* tolerance,
                         float recovery, float* slack, cudaStream_t stream);
// colony_of_slot[s] for cells laid out colony after colony (offsets: colonies + 1).
void launch_colony_of_slot(std::uint32_t colonies, const std::uint32_t* offsets, std::uint32_t n,
                           std::uint32_t* of_slot, cudaStream_t stream);
// Largest growth per step, in radii (contact_dynamics.cpp:700-706).
void launch_growth_bound(std::uint32_t n, GeometryBuffers state, const float* growth_rates, float dt,
                         std::uint32_t* bits, cudaStream_t stream);
// Step outputs.
void launch_outputs(std::uint32_t n, ResponseArrays response, GeometryBuffers base, GeometryBuffers initial,
                    float* velocities, float* loads, float* increments, cudaStream_t stream);
void launch_copy_loads(std::uint32_t n, ResponseArrays response, float* loads, cudaStream_t stream);
// ContactRow / ContactBody records to arrays.
void launch_rows_from_records(const void* records, std::uint32_t count, RowArrays rows, cudaStream_t stream);
void launch_bodies_from_records(const void* records, std::uint32_t count, BodyArrays bodies, cudaStream_t stream);
void launch_response_to_host_layout(std::uint32_t n, ResponseArrays response, float* velocities, float* loads,
                                    float* rates, cudaStream_t stream);

}  // namespace msb
