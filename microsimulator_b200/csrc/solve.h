// The device-resident Barzilai-Borwein projected-gradient contact solve.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace msb {

// Rows as structure of arrays (72 bytes per row):
//   a = first jacobian 0..3          b = first jacobian 4, 5, first lever, offset
//   c = second jacobian 0..3         d = second jacobian 4, 5, second lever, compliance
//   slots = (first slot, second slot or kInvalidSlot)
struct RowArrays {
  float4* a;
  float4* b;
  float4* c;
  float4* d;
  uint2* slots;
};

// Bodies (48 bytes per body):
//   a = axis x, y, z, translational mobility
//   b = transverse mobility, axial mobility, nominal elongation rate, 0
//   drift_a / drift_b = drift velocity and angular velocity (w unused)
struct BodyArrays {
  float4* a;
  float4* b;
  float4* drift_a;
  float4* drift_b;
};

// What a set of multipliers does to each body (32 bytes per body):
//   a = velocity x, y, z, loaded elongation rate
//   b = angular velocity x, y, z, axial load
struct ResponseArrays {
  float4* a;
  float4* b;
};

// Per body, its rows in row order (CSR): entry a = jacobian 0..3,
// entry b = jacobian 4, 5, lever, side (bits: row << 1 | 0 for the row's
// first slot, 1 for its second).
// Per row, for the BB passes (null where no BB pass runs on them):
//   constants = (offset, compliance), written with the incidence;
//   sides     = each side's term of the gap rate, jacobian . velocity -
//               lever * elongation rate, indexed by the entries' side bits
//               and written by the body pass.  A constraint row's second
//               side holds -0.0f, which adds nothing: x + -0.0f == x.
struct IncidenceArrays {
  std::uint32_t* offsets;
  float4* a;
  float4* b;
  float2* constants;
  float2* sides;
};

// Everything one solve reads and writes, in device memory at a fixed address
// so that the captured solve graph can be replayed for any system.
struct SolveDesc {
  RowArrays rows;
  BodyArrays bodies;
  IncidenceArrays incidence;
  ResponseArrays response;
  float* multipliers;
  float* gaps;
  // (multiplier, gap) of every row while a solve runs: the body pass
  // gathers both with one load.  The bound pass fills it from `multipliers`;
  // launch_unpack_iterate writes the solution back.
  float2* iterate;
  double* partials;  // 5 doubles per block of the row pass
  std::uint32_t row_count;
  std::uint32_t body_count;
  float dt;
  std::uint32_t law;
  float sensitivity;
  float free_load;
  float stall_load;
  float tolerance;
  std::uint32_t max_iterations;
  std::uint32_t has_drift;  // 0: every drift is zero and the drift arrays are not read
  // solver state
  float step;
  float residual;
  float bound;
  std::uint32_t iterations;
  std::uint32_t status;  // msb_solve_status
  std::uint32_t mode;    // 0: evaluate the initial multipliers; 1: iterate
  std::uint32_t ticket;
  std::uint32_t proceed;
  unsigned long long handle;  // cudaGraphConditionalHandle of the WHILE node
  std::uint32_t bound_ticket;
  std::uint32_t bound_bits;
  // grid barrier of the fused solve (relax_kernel)
  std::uint32_t barrier_count;
  std::uint32_t barrier_generation;
  std::uint32_t barrier_abort;  // a barrier wait ran out of time: every block stops
  std::uint32_t check_status;   // checked build: the first index check that failed (0: none)
};

// Builds the incidence of `rows` over `bodies` bodies.  Scratch: `keys` and
// `values` hold 2 * rows words each, `counts` bodies + 1 words, `temp`
// sort_temp_words(2 * rows) words.
void build_incidence(RowArrays rows, std::uint32_t row_count, std::uint32_t body_count, IncidenceArrays incidence,
                     std::uint32_t* keys, std::uint32_t* values, std::uint32_t* counts, std::uint32_t* temp,
                     cudaStream_t stream, std::uint32_t* status = nullptr);

// Stable lists of each first slot's rows (ForceMemory's KeyedRows).
void build_keyed(const uint2* slots, std::uint32_t row_count, std::uint32_t body_count, std::uint32_t* offsets,
                 std::uint32_t* rows_out, std::uint32_t* keys, std::uint32_t* counts, std::uint32_t* temp,
                 cudaStream_t stream);

// A solve graph for a fixed grid size: bound -> initial gaps -> WHILE
// (not converged) { body pass; row pass }.
class SolveGraph {
 public:
  SolveGraph() = default;
  SolveGraph(const SolveGraph&) = delete;
  SolveGraph& operator=(const SolveGraph&) = delete;
  ~SolveGraph();
  // Returns a CUDA error code.
  int create(SolveDesc* desc, int blocks, cudaStream_t stream);
  int launch(cudaStream_t stream);
  int blocks() const { return blocks_; }
  // Kernel launches of the WHILE node for a solve of `iterations`
  // iterations (whole evaluations of its unrolled body).
  static int loop_launches(std::uint32_t iterations);

 private:
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  int blocks_ = 0;
  SolveDesc* desc_ = nullptr;
  unsigned long long handle_ = 0;
};

// The fused solve: bound, initial gaps and every projected iteration in ONE
// cooperative launch of `blocks` co-resident blocks, with two bounded grid
// barriers per iteration (the last block to reach the second combines the
// BB products and decides).  The whole descriptor, state included, must be
// reset before the launch; `problem` is its host copy, passed by value as a
// kernel parameter.  Returns a CUDA error code.
int launch_relax(const SolveDesc& problem, SolveDesc* desc, int blocks, cudaStream_t stream);
// Blocks of relax_kernel that fit on the device at once.
int relax_resident_blocks();
// How long a barrier wait may take before the solve stops with
// barrier_abort set.
constexpr unsigned long long kBarrierTimeoutNs = 5'000'000'000ull;

// Evaluates the response of desc->multipliers once (no solve), as
// evaluate_contact_response does; also the gaps when `with_gaps`.  A solve
// writes no response itself: this evaluation of its final multipliers
// follows it.
void launch_evaluate(SolveDesc* desc, int blocks, bool with_gaps, cudaStream_t stream);
// The multipliers and gaps a solve reached (desc->iterate) into
// desc->multipliers and desc->gaps.
void launch_unpack_iterate(SolveDesc* desc, int blocks, cudaStream_t stream);

// One more projected iteration of the last solved system (body pass then
// row pass), for timing; `between` is recorded between the two passes.
void launch_iteration(SolveDesc* desc, int blocks, cudaEvent_t between, cudaStream_t stream);

constexpr int kSolveThreads = 256;
// Blocks of a BB pass at most: the per-block partials hold this many.
constexpr int kMaxPassBlocks = 1184;

}  // namespace msb
