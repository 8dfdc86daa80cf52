// The warm-start network: per-cell features of the 16 nearest neighbours and
// a 81 -> 128 -> 128 -> 128 -> 3 GELU MLP with BF16 weights and activations
// and FP32 accumulation on the fifth-generation tensor cores (tcgen05.mma
// with TMEM accumulators, mlp_tc.cu), in inference and in training.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "kernels.h"

namespace msb::mlp {

constexpr int kNeighbours = 16;
constexpr int kFeatures = 5 * kNeighbours + 1;  // 81
constexpr int kInput = 96;                      // features padded to a multiple of 16
constexpr int kHidden = 128;
constexpr int kOutputs = 3;
constexpr int kOutputPad = 8;  // one n8 tile
// Flat parameter layout, weights row-major (out, in):
//   W0 128 x 96 | W1 128 x 128 | W2 128 x 128 | W3 8 x 128 | b0 128 | b1 128 | b2 128 | b3 8
constexpr std::uint32_t kW0 = 0;
constexpr std::uint32_t kW1 = kW0 + kHidden * kInput;
constexpr std::uint32_t kW2 = kW1 + kHidden * kHidden;
constexpr std::uint32_t kW3 = kW2 + kHidden * kHidden;
constexpr std::uint32_t kWeights = kW3 + kOutputPad * kHidden;  // 45056
constexpr std::uint32_t kB0 = 0;
constexpr std::uint32_t kB1 = kB0 + kHidden;
constexpr std::uint32_t kB2 = kB1 + kHidden;
constexpr std::uint32_t kB3 = kB2 + kHidden;
constexpr std::uint32_t kBiases = kB3 + kOutputPad;  // 392
constexpr std::uint32_t kParameters = kWeights + kBiases;
// Scales of the features: centre offsets over kPositionScale, lengths over kLengthScale.
constexpr float kPositionScale = 5.0f;
constexpr float kLengthScale = 3.0f;
// Bin side of the neighbour grid (um); the 3 x 3 bins around a cell are searched.
constexpr float kBinSide = 6.0f;

// Bytes of the split-K partial sums tc_gemm may use.
constexpr std::uint64_t kGemmPartialBytes = std::uint64_t(32) * 128 * 128 * 4;

// Bytes of the activations the forward pass keeps for the backward pass:
// H1..H3 (bf16) and Z1..Z3 (fp32), n x 128 each.
inline std::uint64_t activation_bytes(std::uint64_t n) { return n * kHidden * (3 * 2 + 3 * 4); }
// Bytes of the backward pass's scratch (its GEMMs' split-K partials last).
inline std::uint64_t backward_scratch_bytes(std::uint64_t n) {
  return n * kHidden * (4 + 4 + 2) + n * 16 * 2 + 256 + kGemmPartialBytes + 256;
}

// The activations a training forward pass keeps, in activation_bytes(n):
// H1..H3 (bf16) then Z1..Z3 (fp32), n x 128 each.
struct Activations {
  __nv_bfloat16* h[3];
  float* z[3];
};
Activations activations_at(void* base, std::uint32_t n);

// C (m x n, fp32) = A (m x k) * B (k x n) with bf16 operands addressed
// through element strides, so that one kernel serves every transpose of the
// backward pass.  n <= 128.
struct Gemm {
  std::uint32_t m, n, k;
  const std::uint16_t* a;
  std::int64_t sam, sak;
  const std::uint16_t* b;
  std::int64_t sbk, sbn;
  float* c;
  std::int64_t scm, scn;
};
// The GEMM on tcgen05 (mlp_tc.cu): 128-row tiles of C accumulated in TMEM,
// a long k split over up to 32 CTAs whose partial sums (in `partials`,
// kGemmPartialBytes) are added in a fixed order.  *error (if not null)
// becomes kStatusIterations when a wait for the tensor cores gave up.
// Returns a CUDA error code.
int tc_gemm(const Gemm& p, float* partials, std::uint32_t* error, cudaStream_t stream);

struct Grid {
  float x0, y0, inverse_side;
  std::uint32_t nx, ny;
  const std::uint32_t* offsets;  // nx * ny + 1
  const std::uint32_t* slots;    // cells sorted by bin
  const float2* centres;         // their centres (x, y), in the same order
};

// Bounds of the cell centres: out[0..3] = min x, min y, max x, max y (as
// ordered uint bits of floats, see kernels).  out must hold 4 words set to
// the identity by the caller (launch_centre_bounds does it).
void launch_centre_bounds(std::uint32_t n, const float4* pos_len, std::uint32_t* out, cudaStream_t stream);
// Bin keys of each cell and per-bin counts (counts zeroed by the caller).
void launch_bin_keys(std::uint32_t n, const float4* pos_len, Grid grid, std::uint32_t* keys, std::uint32_t* values,
                     std::uint32_t* counts, cudaStream_t stream);
// The bin-sorted copy of the centres (grid.centres) from grid.slots.
void launch_sorted_centres(std::uint32_t n, const float4* pos_len, const std::uint32_t* slots, float2* centres,
                           cudaStream_t stream);
// Features of every cell, n x kInput bf16 (as uint16 bits), zero padded.
void launch_features(std::uint32_t n, const float4* pos_len, const float4* dir_rad, Grid grid,
                     std::uint16_t* features, cudaStream_t stream);
// The network over n rows of features on the tcgen05 tensor cores with TMEM
// accumulators (mlp_tc.cu): outputs n x 3 fp32.  With `activations`
// (activation_bytes(n)), also keeps H1..H3 and Z1..Z3 for the backward
// pass.  *error (if not null) becomes kStatusIterations when a wait for the
// tensor cores gave up.  Returns a CUDA error code.
int launch_forward_tc(const std::uint16_t* weights, const float* biases, const std::uint16_t* features,
                      std::uint32_t n, float* outputs, void* activations, std::uint32_t* error,
                      cudaStream_t stream);
// Gradients of the parameters (fp32, flat layout) for output gradients
// `output_grad` (n x 3) from the activations of launch_forward_tc, with the
// GEMMs on tcgen05.  Returns a CUDA error code.
int launch_backward(const std::uint16_t* weights, const std::uint16_t* features, std::uint32_t n,
                    const void* activations, const float* output_grad, float* grads, void* scratch,
                    std::uint32_t* error, cudaStream_t stream);
// One Adam step over the flat fp32 parameters; writes the bf16 weights and
// fp32 biases the kernels read.
void launch_adam(float* params, const float* grads, float* m, float* v, std::uint32_t step, float lr, float beta1,
                 float beta2, float epsilon, std::uint16_t* weights, float* biases, cudaStream_t stream);
// Network outputs (normalized body-frame displacement: along the axis,
// across it, turn) to motion guesses (dx, dy, dtheta, 0) in the plane.
void launch_outputs_to_guess(std::uint32_t n, const float* outputs, const float* scale, const float4* dir_rad,
                             float4* guess, cudaStream_t stream);

}  // namespace msb::mlp
