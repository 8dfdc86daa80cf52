// The batched contact solve: many independent colonies, each relaxed by its
// own Barzilai-Borwein projected gradient (its own step length, residual,
// tolerance and iteration count), in one persistent launch of thread-block
// clusters.  A cluster takes the next colony from a work queue (largest
// colonies first), runs that colony's whole solve with cluster barriers
// between the body and row passes and a rank-ordered reduction of the BB
// products through distributed shared memory, then takes the next.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "solve.h"

namespace msb {

struct ColonyState {
  float step;
  float residual;
  float bound;
  std::uint32_t iterations;
  std::uint32_t status;  // msb_solve_status, or 3 for a colony without a positive diagonal
};

struct BatchDesc {
  RowArrays rows;
  BodyArrays bodies;
  IncidenceArrays incidence;
  ResponseArrays response;
  float* multipliers;
  float* gaps;
  float2* iterate;  // (multiplier, gap) of each row inside a solve
  const std::uint32_t* colony_rows;   // row indices grouped by colony, row order within one
  const std::uint32_t* row_offsets;   // colonies + 1
  const std::uint32_t* cell_offsets;  // colonies + 1: a colony's bodies are a slot range
  const std::uint32_t* order;         // colonies in the order the queue hands them out
  // Colonies to solve (null: all).  A colony left out keeps its multipliers
  // and response from its last solve and reports 0 iterations: the stepper
  // leaves out colonies whose rows are unchanged since a converged solve.
  const std::uint32_t* active;
  const float* tolerance;             // per colony
  ColonyState* state;                 // per colony
  std::uint32_t* next;                // the queue's counter, zero at launch
  std::uint32_t colonies;
  float dt;
  std::uint32_t law;
  float sensitivity;
  float free_load;
  float stall_load;
  std::uint32_t max_iterations;
  std::uint32_t has_drift;
};

// A launch shape of the batched solve: CTAs per cluster and threads per CTA.
struct BatchShape {
  int cluster;  // 1, 2, 4, 8 or 16 (16: a non-portable cluster size)
  int threads;  // 256 or 512
  bool lean;    // 64-register form (one gather in flight per thread, more resident warps)
};

// Clusters of `shape` that fit on the device at once (0 if none).
int batch_resident_clusters(BatchShape shape);
// Launches the batched solve with `clusters` persistent clusters; returns a
// CUDA error code.  desc.next must be zero.
int launch_batch_solve(const BatchDesc& desc, BatchShape shape, int clusters, cudaStream_t stream);
// Keys (colony of each row's first slot) and row indices for grouping rows by colony.
void launch_colony_row_keys(const uint2* slots, std::uint32_t rows, const std::uint32_t* of_slot,
                            std::uint32_t* keys, std::uint32_t* values, std::uint32_t* counts, cudaStream_t stream);

}  // namespace msb
