// The warm-start network on the tensor cores: neighbour features, a fused
// forward pass that keeps each 16-cell tile's activations in registers
// between layers, the backward GEMMs and Adam.
//
// Tensor-core form: mma.sync.m16n8k16 with bf16 A and B and fp32
// accumulators.  The accumulator fragment of one layer (rows g and g + 8,
// columns 2t and 2t + 1 of each n8 tile) is, after bias and GELU and a
// rounding to bf16, exactly the A fragment of the next layer (two n8 tiles
// make one k16 step), so the forward pass reads each cell's features once
// and writes only its three outputs.
#include "mlp.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "device.cuh"

namespace msb::mlp {
namespace {

constexpr int kThreads = 256;
constexpr int kForwardWarps = 4;
constexpr int kStrideIn = kInput + 8;   // bf16 elements per W0 row in shared memory
constexpr int kStrideH = kHidden + 8;   // per W1..W3 row
constexpr int kSmemW0 = kHidden * kStrideIn;
constexpr int kSmemW1 = kHidden * kStrideH;
constexpr int kSmemW3 = kOutputPad * kStrideH;
constexpr std::size_t kForwardSmem =
    (std::size_t(kSmemW0) + 2 * kSmemW1 + kSmemW3) * 2 + std::size_t(kBiases) * 4;

struct Activations {
  __nv_bfloat16* h[3];  // H1..H3, n x 128
  float* z[3];          // Z1..Z3, n x 128
};

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

__device__ __forceinline__ void mma_bf16(float (&d)[4], const std::uint32_t (&a)[4], std::uint32_t b0,
                                         std::uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ std::uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const std::uint32_t*>(&v);
}

__device__ __forceinline__ std::uint32_t load_pair(const std::uint16_t* p) {
  return *reinterpret_cast<const std::uint32_t*>(p);
}

// GELU with the exact error-function form.
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
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

template <int KT>
__device__ __forceinline__ void dense(const std::uint16_t* w, int stride, const std::uint32_t (&a)[8][4],
                                      float (&acc)[16][4], int g, int t) {
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
    const std::uint16_t* row = w + (nt * 8 + g) * stride + 2 * t;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) mma_bf16(acc[nt], a[kt], load_pair(row + kt * 16), load_pair(row + kt * 16 + 8));
  }
}

// Bias, GELU, optional store of Z and H, and the next layer's A fragments.
__device__ __forceinline__ void activate(float (&acc)[16][4], const float* bias, std::uint32_t (&a)[8][4],
                                         __nv_bfloat16* h_out, float* z_out, std::uint32_t lo, std::uint32_t hi,
                                         std::uint32_t n, int t) {
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    const int c = nt * 8 + 2 * t;
    const float z00 = acc[nt][0] + bias[c], z01 = acc[nt][1] + bias[c + 1];
    const float z10 = acc[nt][2] + bias[c], z11 = acc[nt][3] + bias[c + 1];
    const std::uint32_t h0 = pack_bf16(gelu(z00), gelu(z01));
    const std::uint32_t h1 = pack_bf16(gelu(z10), gelu(z11));
    if (z_out != nullptr) {
      if (lo < n) {
        *reinterpret_cast<float2*>(z_out + std::size_t(lo) * kHidden + c) = make_float2(z00, z01);
        *reinterpret_cast<std::uint32_t*>(h_out + std::size_t(lo) * kHidden + c) = h0;
      }
      if (hi < n) {
        *reinterpret_cast<float2*>(z_out + std::size_t(hi) * kHidden + c) = make_float2(z10, z11);
        *reinterpret_cast<std::uint32_t*>(h_out + std::size_t(hi) * kHidden + c) = h1;
      }
    }
    const int kt = nt >> 1;
    if ((nt & 1) == 0) {
      a[kt][0] = h0;
      a[kt][1] = h1;
    } else {
      a[kt][2] = h0;
      a[kt][3] = h1;
    }
  }
}

__global__ void __launch_bounds__(32 * kForwardWarps) forward_kernel(const std::uint16_t* __restrict__ weights,
                                                                     const float* __restrict__ biases,
                                                                     const std::uint16_t* __restrict__ x,
                                                                     std::uint32_t n, float* __restrict__ y,
                                                                     Activations act, int keep) {
  extern __shared__ __align__(16) unsigned char smem[];
  std::uint16_t* w0 = reinterpret_cast<std::uint16_t*>(smem);
  std::uint16_t* w1 = w0 + kSmemW0;
  std::uint16_t* w2 = w1 + kSmemW1;
  std::uint16_t* w3 = w2 + kSmemW1;
  float* bias = reinterpret_cast<float*>(w3 + kSmemW3);
  for (int i = threadIdx.x; i < kHidden * kInput; i += blockDim.x) {
    w0[(i / kInput) * kStrideIn + i % kInput] = weights[kW0 + i];
  }
  for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x) {
    w1[(i / kHidden) * kStrideH + i % kHidden] = weights[kW1 + i];
    w2[(i / kHidden) * kStrideH + i % kHidden] = weights[kW2 + i];
  }
  for (int i = threadIdx.x; i < kOutputPad * kHidden; i += blockDim.x) {
    w3[(i / kHidden) * kStrideH + i % kHidden] = weights[kW3 + i];
  }
  for (int i = threadIdx.x; i < int(kBiases); i += blockDim.x) bias[i] = biases[i];
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const std::uint32_t tiles = (n + 15) / 16;
  for (std::uint32_t tile = blockIdx.x * kForwardWarps + warp; tile < tiles; tile += gridDim.x * kForwardWarps) {
    const std::uint32_t lo = tile * 16 + g, hi = lo + 8;
    std::uint32_t a[8][4];
#pragma unroll
    for (int kt = 0; kt < kInput / 16; ++kt) {
      const std::uint16_t* rl = x + std::size_t(lo) * kInput + kt * 16 + 2 * t;
      const std::uint16_t* rh = x + std::size_t(hi) * kInput + kt * 16 + 2 * t;
      a[kt][0] = lo < n ? load_pair(rl) : 0u;
      a[kt][1] = hi < n ? load_pair(rh) : 0u;
      a[kt][2] = lo < n ? load_pair(rl + 8) : 0u;
      a[kt][3] = hi < n ? load_pair(rh + 8) : 0u;
    }
#pragma unroll
    for (int kt = kInput / 16; kt < 8; ++kt) a[kt][0] = a[kt][1] = a[kt][2] = a[kt][3] = 0u;
    float acc[16][4];
    dense<kInput / 16>(w0, kStrideIn, a, acc, g, t);
    activate(acc, bias + kB0, a, keep ? act.h[0] : nullptr, keep ? act.z[0] : nullptr, lo, hi, n, t);
    dense<8>(w1, kStrideH, a, acc, g, t);
    activate(acc, bias + kB1, a, keep ? act.h[1] : nullptr, keep ? act.z[1] : nullptr, lo, hi, n, t);
    dense<8>(w2, kStrideH, a, acc, g, t);
    activate(acc, bias + kB2, a, keep ? act.h[2] : nullptr, keep ? act.z[2] : nullptr, lo, hi, n, t);
    float out[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const std::uint16_t* row = w3 + g * kStrideH + 2 * t;
#pragma unroll
    for (int kt = 0; kt < 8; ++kt) mma_bf16(out, a[kt], load_pair(row + kt * 16), load_pair(row + kt * 16 + 8));
    const int c = 2 * t;
    if (c < kOutputs) {
      if (lo < n) y[std::size_t(lo) * kOutputs + c] = out[0] + bias[kB3 + c];
      if (hi < n) y[std::size_t(hi) * kOutputs + c] = out[2] + bias[kB3 + c];
    }
    if (c + 1 < kOutputs) {
      if (lo < n) y[std::size_t(lo) * kOutputs + c + 1] = out[1] + bias[kB3 + c + 1];
      if (hi < n) y[std::size_t(hi) * kOutputs + c + 1] = out[3] + bias[kB3 + c + 1];
    }
  }
}

// C (M x N, fp32) = A (M x K) * B (K x N), bf16 operands addressed through
// element strides so that one kernel serves every transpose of the backward
// pass.  64 x 64 block tiles, k-tiles of 32 staged in shared memory, four
// warps of 32 x 32 (2 m16 x 4 n8 mma tiles each).
struct Gemm {
  std::uint32_t m, n, k;
  const std::uint16_t* a;
  std::int64_t sam, sak;
  const std::uint16_t* b;
  std::int64_t sbk, sbn;
  float* c;
  std::int64_t scm, scn;
};

__global__ void __launch_bounds__(128) gemm_kernel(Gemm p) {
  __shared__ __align__(16) std::uint16_t as[64][40];  // [m][k]
  __shared__ __align__(16) std::uint16_t bs[64][40];  // [n][k]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 1, wn = warp & 1;
  const std::uint32_t m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  float acc[2][4][4] = {};
  for (std::uint32_t k0 = 0; k0 < p.k; k0 += 32) {
    for (int i = threadIdx.x; i < 64 * 32; i += blockDim.x) {
      const int r = i >> 5, kk = i & 31;
      const std::uint32_t mm = m0 + r, nn = n0 + r, k = k0 + kk;
      as[r][kk] = (mm < p.m && k < p.k) ? p.a[std::int64_t(mm) * p.sam + std::int64_t(k) * p.sak] : std::uint16_t(0);
      bs[r][kk] = (nn < p.n && k < p.k) ? p.b[std::int64_t(k) * p.sbk + std::int64_t(nn) * p.sbn] : std::uint16_t(0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 32; kk += 16) {
      std::uint32_t af[2][4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        const int r = wm * 32 + mi * 16 + g;
        af[mi][0] = load_pair(&as[r][kk + 2 * t]);
        af[mi][1] = load_pair(&as[r + 8][kk + 2 * t]);
        af[mi][2] = load_pair(&as[r][kk + 2 * t + 8]);
        af[mi][3] = load_pair(&as[r + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int c = wn * 32 + ni * 8 + g;
        const std::uint32_t b0 = load_pair(&bs[c][kk + 2 * t]);
        const std::uint32_t b1 = load_pair(&bs[c][kk + 2 * t + 8]);
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) mma_bf16(acc[mi][ni], af[mi], b0, b1);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 2; ++mi) {
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const std::uint32_t row = m0 + wm * 32 + mi * 16 + g + (r >= 2 ? 8 : 0);
        const std::uint32_t col = n0 + wn * 32 + ni * 8 + 2 * t + (r & 1);
        if (row < p.m && col < p.n) p.c[std::int64_t(row) * p.scm + std::int64_t(col) * p.scn] = acc[mi][ni][r];
      }
    }
  }
}

void gemm(const Gemm& p, cudaStream_t stream) {
  if (p.m == 0 || p.n == 0) return;
  const dim3 grid((p.n + 63) / 64, (p.m + 63) / 64);
  gemm_kernel<<<grid, 128, 0, stream>>>(p);
  count_launch();
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

void launch_forward(const std::uint16_t* weights, const float* biases, const std::uint16_t* features,
                    std::uint32_t n, float* outputs, void* activations, cudaStream_t stream) {
  if (n == 0) return;
  cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kForwardSmem));
  const Activations act = activations != nullptr ? activations_at(activations, n) : Activations{};
  const std::uint32_t tiles = (n + 15) / 16;
  int device = 0, sms = kSmCount;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const std::uint32_t wanted = (tiles + kForwardWarps - 1) / kForwardWarps;
  const std::uint32_t blocks = std::max(1u, std::min<std::uint32_t>(wanted, 2u * std::uint32_t(sms)));
  forward_kernel<<<blocks, 32 * kForwardWarps, kForwardSmem, stream>>>(weights, biases, features, n, outputs, act,
                                                                         activations != nullptr ? 1 : 0);
  count_launch();
}

void launch_backward(const std::uint16_t* weights, const std::uint16_t* features, std::uint32_t n,
                     const void* activations, const float* output_grad, float* grads, void* scratch,
                     cudaStream_t stream) {
  if (n == 0) {
    cudaMemsetAsync(grads, 0, kParameters * sizeof(float), stream);
    return;
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

  output_grad_kernel<<<grid_for(std::uint64_t(n) * kOutputPad, kThreads), kThreads, 0, stream>>>(n, output_grad, dyb);
  count_launch();
  float* gw = grads;
  float* gb = grads + kWeights;
  cudaMemsetAsync(gb + kB3, 0, kOutputPad * sizeof(float), stream);
  column_sums_kernel<<<1, 32, 0, stream>>>(n, kOutputs, kOutputs, output_grad, gb + kB3);
  count_launch();
  const auto* h3 = reinterpret_cast<const std::uint16_t*>(act.h[2]);
  // dW3 (8 x 128) = dY^T H3;  dH3 (n x 128) = dY W3.
  gemm({kOutputPad, kHidden, n, dyb, 1, kOutputPad, h3, kHidden, 1, gw + kW3, kHidden, 1}, stream);
  gemm({n, kHidden, kOutputPad, dyb, kOutputPad, 1, weights + kW3, kHidden, 1, dh, kHidden, 1}, stream);
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
    gemm({kHidden, width, n, dzb, 1, kHidden, input, width, 1, gw + weight_at[l], width, 1}, stream);
    // dH_{l-1} (n x 128) = dZ W_l.
    if (l > 0) gemm({n, kHidden, kHidden, dzb, kHidden, 1, weights + weight_at[l], kHidden, 1, dh, kHidden, 1}, stream);
  }
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
