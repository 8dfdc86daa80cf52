// The warm-start network around its tensor-core kernels (mlp_tc.cu): the
// neighbour features, the backward pass's elementwise steps and its GEMMs
// (on tcgen05 through tc_gemm), and Adam.
#include "mlp.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "device.cuh"

namespace msb::mlp {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ std::uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const std::uint32_t*>(&v);
}

// The derivative of GELU in its exact error-function form.
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Floats as unsigned words that order like the floats.
__device__ __forceinline__ std::uint32_t ordered(float f) {
  const std::uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) != 0 ? ~b : (b | 0x80000000u);
}

__global__ void centre_bounds_kernel(std::uint32_t n, const float4* __restrict__ pos_len, std::uint32_t* out) {
  float lo_x = INFINITY, lo_y = INFINITY, hi_x = -INFINITY, hi_y = -INFINITY;
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 p = pos_len[s];
    lo_x = fminf(lo_x, p.x);
    lo_y = fminf(lo_y, p.y);
    hi_x = fmaxf(hi_x, p.x);
    hi_y = fmaxf(hi_y, p.y);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo_x = fminf(lo_x, __shfl_down_sync(0xFFFFFFFFu, lo_x, o));
    lo_y = fminf(lo_y, __shfl_down_sync(0xFFFFFFFFu, lo_y, o));
    hi_x = fmaxf(hi_x, __shfl_down_sync(0xFFFFFFFFu, hi_x, o));
    hi_y = fmaxf(hi_y, __shfl_down_sync(0xFFFFFFFFu, hi_y, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&out[0], ordered(lo_x));
    atomicMin(&out[1], ordered(lo_y));
    atomicMax(&out[2], ordered(hi_x));
    atomicMax(&out[3], ordered(hi_y));
  }
}

__device__ __forceinline__ std::uint32_t bin_of(const Grid& g, float x, float y, std::uint32_t& bx,
                                                std::uint32_t& by) {
  const float fx = (x - g.x0) * g.inverse_side;
  const float fy = (y - g.y0) * g.inverse_side;
  bx = std::uint32_t(fminf(fmaxf(fx, 0.0f), float(g.nx - 1)));
  by = std::uint32_t(fminf(fmaxf(fy, 0.0f), float(g.ny - 1)));
  return by * g.nx + bx;
}

__global__ void sorted_centres_kernel(std::uint32_t n, const float4* __restrict__ pos_len,
                                      const std::uint32_t* __restrict__ slots, float2* __restrict__ centres) {
  for (std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float4 p = pos_len[slots[k]];
    centres[k] = make_float2(p.x, p.y);
  }
}

__global__ void bin_keys_kernel(std::uint32_t n, const float4* __restrict__ pos_len, Grid grid,
                                std::uint32_t* __restrict__ keys, std::uint32_t* __restrict__ values,
                                std::uint32_t* __restrict__ counts) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 p = pos_len[s];
    std::uint32_t bx, by;
    const std::uint32_t bin = bin_of(grid, p.x, p.y, bx, by);
    keys[s] = bin;
    values[s] = s;
    atomicAdd(&counts[bin], 1u);
  }
}

// One thread per cell: the 16 nearest centres among the 3 x 3 bins around
// the cell, in (squared distance, slot) order, kept sorted in registers.
__global__ void __launch_bounds__(kThreads) features_kernel(std::uint32_t n, const float4* __restrict__ pos_len,
                                                             const float4* __restrict__ dir_rad, Grid grid,
                                                             std::uint16_t* __restrict__ features) {
  // Cells in bin order, so that a warp's cells search the same bins.
  for (std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const std::uint32_t s = grid.slots[k];
    const float4 p = pos_len[s];
    const float4 d = dir_rad[s];
    float ax = d.x, ay = d.y;
    const float an = sqrtf(ax * ax + ay * ay);
    if (an > 0.0f) {
      ax /= an;
      ay /= an;
    } else {
      ax = 1.0f;
      ay = 0.0f;
    }
    float best_d[kNeighbours];
    std::uint32_t best_s[kNeighbours];
#pragma unroll
    for (int q = 0; q < kNeighbours; ++q) {
      best_d[q] = INFINITY;
      best_s[q] = kInvalidSlot;
    }
    std::uint32_t bx, by;
    bin_of(grid, p.x, p.y, bx, by);
    for (int oy = -1; oy <= 1; ++oy) {
      const int y = int(by) + oy;
      if (y < 0 || y >= int(grid.ny)) continue;
      for (int ox = -1; ox <= 1; ++ox) {
        const int x = int(bx) + ox;
        if (x < 0 || x >= int(grid.nx)) continue;
        const std::uint32_t bin = std::uint32_t(y) * grid.nx + std::uint32_t(x);
        for (std::uint32_t m = grid.offsets[bin]; m < grid.offsets[bin + 1]; ++m) {
          const std::uint32_t o = grid.slots[m];
          if (o == s) continue;
          const float2 q = grid.centres[m];
          const float dx = q.x - p.x, dy = q.y - p.y;
          const float d2 = dx * dx + dy * dy;
          if (d2 > best_d[kNeighbours - 1] || (d2 == best_d[kNeighbours - 1] && o > best_s[kNeighbours - 1])) continue;
          best_d[kNeighbours - 1] = d2;
          best_s[kNeighbours - 1] = o;
#pragma unroll
          for (int q2 = kNeighbours - 1; q2 > 0; --q2) {
            const bool before = best_d[q2] < best_d[q2 - 1] || (best_d[q2] == best_d[q2 - 1] && best_s[q2] < best_s[q2 - 1]);
            if (before) {
              const float td = best_d[q2];
              best_d[q2] = best_d[q2 - 1];
              best_d[q2 - 1] = td;
              const std::uint32_t ts = best_s[q2];
              best_s[q2] = best_s[q2 - 1];
              best_s[q2 - 1] = ts;
            }
          }
        }
      }
    }
    std::uint32_t* out = reinterpret_cast<std::uint32_t*>(features + std::size_t(s) * kInput);
    // Five features per neighbour, written as bf16 pairs: the centre offset
    // in the cell's frame (along, across), the neighbour's orientation
    // relative to the cell's (cos, sin, axis signs aligned) and its length.
    float f[kFeatures + 1];
#pragma unroll
    for (int q = 0; q < kNeighbours; ++q) {
      float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f, v3 = 0.0f, v4 = 0.0f;
      if (best_s[q] != kInvalidSlot) {
        const float4 o = pos_len[best_s[q]];
        const float4 od = dir_rad[best_s[q]];
        const float dx = o.x - p.x, dy = o.y - p.y;
        v0 = (dx * ax + dy * ay) / kPositionScale;
        v1 = (dy * ax - dx * ay) / kPositionScale;
        float bxn = od.x, byn = od.y;
        const float bn = sqrtf(bxn * bxn + byn * byn);
        if (bn > 0.0f) {
          bxn /= bn;
          byn /= bn;
        }
        float c = ax * bxn + ay * byn;
        float sn = ax * byn - ay * bxn;
        if (c < 0.0f) {
          c = -c;
          sn = -sn;
        }
        v2 = c;
        v3 = sn;
        v4 = o.w / kLengthScale;
      }
      f[5 * q + 0] = v0;
      f[5 * q + 1] = v1;
      f[5 * q + 2] = v2;
      f[5 * q + 3] = v3;
      f[5 * q + 4] = v4;
    }
    f[kFeatures - 1] = p.w / kLengthScale;
    f[kFeatures] = 0.0f;
#pragma unroll
    for (int k = 0; k < (kFeatures + 1) / 2; ++k) out[k] = pack_bf16(f[2 * k], f[2 * k + 1]);
#pragma unroll
    for (int k = (kFeatures + 1) / 2; k < kInput / 2; ++k) out[k] = 0u;
  }
}

__global__ void output_grad_kernel(std::uint32_t n, const float* __restrict__ dy, std::uint16_t* __restrict__ out) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n * kOutputPad;
       i += gridDim.x * blockDim.x) {
    const std::uint32_t r = i / kOutputPad, c = i % kOutputPad;
    const float v = c < kOutputs ? dy[std::size_t(r) * kOutputs + c] : 0.0f;
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    out[i] = *reinterpret_cast<const std::uint16_t*>(&b);
  }
}

// dZ = dH * gelu'(Z), in fp32 (for the bias sums) and bf16 (for the GEMMs).
__global__ void gelu_backward_kernel(std::uint64_t count, const float* __restrict__ dh, const float* __restrict__ z,
                                     float* __restrict__ dz, std::uint16_t* __restrict__ dz_bf16) {
  for (std::uint64_t i = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; i < count;
       i += std::uint64_t(gridDim.x) * blockDim.x) {
    const float v = dh[i] * gelu_grad(z[i]);
    dz[i] = v;
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    dz_bf16[i] = *reinterpret_cast<const std::uint16_t*>(&b);
  }
}

// Column sums of an n x cols fp32 matrix (row stride `stride`), in row order.
__global__ void column_sums_kernel(std::uint32_t n, std::uint32_t cols, std::uint32_t stride,
                                   const float* __restrict__ x, float* __restrict__ out) {
  const std::uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (std::uint32_t r = 0; r < n; ++r) s += x[std::size_t(r) * stride + c];
  out[c] = s;
}

__global__ void adam_kernel(float* __restrict__ params, const float* __restrict__ grads, float* __restrict__ m,
                            float* __restrict__ v, float lr, float beta1, float beta2, float epsilon,
                            float correction1, float correction2, std::uint16_t* __restrict__ weights,
                            float* __restrict__ biases) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kParameters; i += gridDim.x * blockDim.x) {
    const float gr = grads[i];
    const float mi = beta1 * m[i] + (1.0f - beta1) * gr;
    const float vi = beta2 * v[i] + (1.0f - beta2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    const float p = params[i] - lr * (mi / correction1) / (sqrtf(vi / correction2) + epsilon);
    params[i] = p;
    if (i < kWeights) {
      const __nv_bfloat16 b = __float2bfloat16_rn(p);
      weights[i] = *reinterpret_cast<const std::uint16_t*>(&b);
    } else {
      biases[i - kWeights] = p;
    }
  }
}

__global__ void outputs_to_guess_kernel(std::uint32_t n, const float* __restrict__ outputs, float sx, float sy,
                                        float st, const float4* __restrict__ dir_rad, float4* __restrict__ guess) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 d = dir_rad[s];
    float ax = d.x, ay = d.y;
    const float an = sqrtf(ax * ax + ay * ay);
    if (an > 0.0f) {
      ax /= an;
      ay /= an;
    } else {
      ax = 1.0f;
      ay = 0.0f;
    }
    const float along = outputs[3 * std::size_t(s)] * sx;
    const float across = outputs[3 * std::size_t(s) + 1] * sy;
    const float turn = outputs[3 * std::size_t(s) + 2] * st;
    float4 out = make_float4(along * ax - across * ay, along * ay + across * ax, turn, 0.0f);
    if (!isfinite(out.x) || !isfinite(out.y) || !isfinite(out.z)) out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    guess[s] = out;
  }
}

}  // namespace

void launch_centre_bounds(std::uint32_t n, const float4* pos_len, std::uint32_t* out, cudaStream_t stream) {
  cudaMemsetAsync(out, 0xFF, 2 * sizeof(std::uint32_t), stream);  // minima start at the largest word
  cudaMemsetAsync(out + 2, 0, 2 * sizeof(std::uint32_t), stream);   // maxima at the smallest
  if (n == 0) return;
  centre_bounds_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, pos_len, out);
  count_launch();
}

void launch_bin_keys(std::uint32_t n, const float4* pos_len, Grid grid, std::uint32_t* keys, std::uint32_t* values,
                     std::uint32_t* counts, cudaStream_t stream) {
  if (n == 0) return;
  bin_keys_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, pos_len, grid, keys, values, counts);
  count_launch();
}

void launch_sorted_centres(std::uint32_t n, const float4* pos_len, const std::uint32_t* slots, float2* centres,
                           cudaStream_t stream) {
  if (n == 0) return;
  sorted_centres_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, pos_len, slots, centres);
  count_launch();
}

void launch_features(std::uint32_t n, const float4* pos_len, const float4* dir_rad, Grid grid,
                     std::uint16_t* features, cudaStream_t stream) {
  if (n == 0) return;
  features_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, pos_len, dir_rad, grid, features);
  count_launch();
}

Activations activations_at(void* base, std::uint32_t n) {
  Activations a{};
  auto* p = static_cast<unsigned char*>(base);
  for (int l = 0; l < 3; ++l) {
    a.h[l] = reinterpret_cast<__nv_bfloat16*>(p);
    p += std::size_t(n) * kHidden * 2;
  }
  for (int l = 0; l < 3; ++l) {
    a.z[l] = reinterpret_cast<float*>(p);
    p += std::size_t(n) * kHidden * 4;
  }
  return a;
}

int launch_backward(const std::uint16_t* weights, const std::uint16_t* features, std::uint32_t n,
                    const void* activations, const float* output_grad, float* grads, void* scratch,
                    std::uint32_t* error, cudaStream_t stream) {
  if (n == 0) {
    return int(cudaMemsetAsync(grads, 0, kParameters * sizeof(float), stream));
  }
  const Activations act = activations_at(const_cast<void*>(activations), n);
  auto* p = static_cast<unsigned char*>(scratch);
  float* dh = reinterpret_cast<float*>(p);
  p += std::size_t(n) * kHidden * 4;
  float* dz = reinterpret_cast<float*>(p);
  p += std::size_t(n) * kHidden * 4;
  auto* dzb = reinterpret_cast<std::uint16_t*>(p);
  p += std::size_t(n) * kHidden * 2;
  auto* dyb = reinterpret_cast<std::uint16_t*>(p);
  p += std::size_t(n) * 16 * 2;
  // The GEMMs' split-K partials, 256-byte aligned.
  auto* partials = reinterpret_cast<float*>((reinterpret_cast<std::uintptr_t>(p) + 255) & ~std::uintptr_t(255));

  output_grad_kernel<<<grid_for(std::uint64_t(n) * kOutputPad, kThreads), kThreads, 0, stream>>>(n, output_grad, dyb);
  count_launch();
  float* gw = grads;
  float* gb = grads + kWeights;
  cudaMemsetAsync(gb + kB3, 0, kOutputPad * sizeof(float), stream);
  column_sums_kernel<<<1, 32, 0, stream>>>(n, kOutputs, kOutputs, output_grad, gb + kB3);
  count_launch();
  const auto* h3 = reinterpret_cast<const std::uint16_t*>(act.h[2]);
  int status = 0;
  const auto gemm = [&](const Gemm& g) {
    if (status == 0) status = tc_gemm(g, partials, error, stream);
  };
  // dW3 (8 x 128) = dY^T H3;  dH3 (n x 128) = dY W3.
  gemm({kOutputPad, kHidden, n, dyb, 1, kOutputPad, h3, kHidden, 1, gw + kW3, kHidden, 1});
  gemm({n, kHidden, kOutputPad, dyb, kOutputPad, 1, weights + kW3, kHidden, 1, dh, kHidden, 1});
  const std::uint32_t bias_at[3] = {kB0, kB1, kB2};
  const std::uint32_t weight_at[3] = {kW0, kW1, kW2};
  for (int l = 2; l >= 0; --l) {
    const std::uint64_t count = std::uint64_t(n) * kHidden;
    gelu_backward_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(count, dh, act.z[l], dz, dzb);
    count_launch();
    column_sums_kernel<<<1, kHidden, 0, stream>>>(n, kHidden, kHidden, dz, gb + bias_at[l]);
    count_launch();
    const std::uint16_t* input = l == 0 ? features : reinterpret_cast<const std::uint16_t*>(act.h[l - 1]);
    const std::uint32_t width = l == 0 ? kInput : kHidden;
    // dW_l (128 x width) = dZ^T H_{l-1}.
    gemm({kHidden, width, n, dzb, 1, kHidden, input, width, 1, gw + weight_at[l], width, 1});
    // dH_{l-1} (n x 128) = dZ W_l.
    if (l > 0) gemm({n, kHidden, kHidden, dzb, kHidden, 1, weights + weight_at[l], kHidden, 1, dh, kHidden, 1});
  }
  return status;
}

void launch_adam(float* params, const float* grads, float* m, float* v, std::uint32_t step, float lr, float beta1,
                 float beta2, float epsilon, std::uint16_t* weights, float* biases, cudaStream_t stream) {
  const float c1 = 1.0f - float(std::pow(double(beta1), double(step)));
  const float c2 = 1.0f - float(std::pow(double(beta2), double(step)));
  adam_kernel<<<grid_for(kParameters, kThreads), kThreads, 0, stream>>>(params, grads, m, v, lr, beta1, beta2,
                                                                        epsilon, c1, c2, weights, biases);
  count_launch();
}

void launch_outputs_to_guess(std::uint32_t n, const float* outputs, const float* scale, const float4* dir_rad,
                             float4* guess, cudaStream_t stream) {
  if (n == 0) return;
  outputs_to_guess_kernel<<<grid_for(n, kThreads), kThreads, 0, stream>>>(n, outputs, scale[0], scale[1], scale[2],
                                                                          dir_rad, guess);
  count_launch();
}

}  // namespace msb::mlp
