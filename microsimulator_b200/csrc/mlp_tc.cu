// The warm-start network on the fifth-generation tensor cores: tcgen05.mma
// with both operands in shared memory and the fp32 accumulator in tensor
// memory (TMEM), for the forward pass (inference, and training with its
// activations kept) and for the backward pass's GEMMs.
//
// One CTA of 512 threads per SM works through 128-cell tiles.  Per layer:
// thread 0 issues the layer's K/16 MMAs (M = 128 cells, N = 128 outputs, or 16
// for the output layer) and commits them to an mbarrier; then each of the 16
// warps reads a 32-lane x 32-column block of the accumulator (warp w: lanes
// of quarter w % 4, one per cell, columns 32 * (w / 4) on) with tcgen05.ld,
// adds the bias, applies GELU, rounds to bf16 and writes it into the
// shared-memory operand of the next layer.  Weights stay in shared memory for
// the whole launch.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices, rows of a core matrix 16 bytes apart, row
// groups 128 bytes apart (the descriptor's stride byte offset) and 8-element
// K blocks R/8 * 128 bytes apart (its leading byte offset) for R rows.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "device.cuh"
#include "mlp.h"

namespace msb::mlp {
namespace {

constexpr int kTile = 128;
constexpr int kTcThreads = 512;
constexpr std::uint32_t kTmemColumns = 128;
constexpr std::uint32_t kOutputRows = 16;  // the output layer's N (8 weight rows, zero padded)
// Bytes of each shared-memory operand.
constexpr std::uint32_t kBytesW0 = kHidden * kInput * 2;             // 24 KB
constexpr std::uint32_t kBytesW1 = kHidden * kHidden * 2;            // 32 KB
constexpr std::uint32_t kBytesW3 = kOutputRows * kHidden * 2;        // 4 KB
constexpr std::uint32_t kBytesA = kTile * kHidden * 2;               // 32 KB
constexpr std::uint32_t kOffW0 = 0;
constexpr std::uint32_t kOffW1 = kOffW0 + kBytesW0;
constexpr std::uint32_t kOffW2 = kOffW1 + kBytesW1;
constexpr std::uint32_t kOffW3 = kOffW2 + kBytesW1;
constexpr std::uint32_t kOffA = kOffW3 + kBytesW3;
constexpr std::uint32_t kOffBias = kOffA + kBytesA;
constexpr std::uint32_t kOffBarrier = kOffBias + kBiases * 4;         // 8-byte aligned
constexpr std::uint32_t kOffTmem = kOffBarrier + 8;
constexpr std::size_t kTcSmem = kOffTmem + 8;
static_assert(kOffBarrier % 8 == 0, "mbarrier alignment");
static_assert(kTcSmem <= 227 * 1024, "shared memory");
// An mbarrier wait gives up after this many polls and reports an error.
constexpr std::uint32_t kWaitPolls = 1u << 26;

// Byte offset of element (row, k) in a K-major no-swizzle operand of `rows` rows.
__host__ __device__ constexpr std::uint32_t core_offset(std::uint32_t rows, std::uint32_t row, std::uint32_t k) {
  return (k / 8) * (rows / 8) * 128 + (row / 8) * 128 + (row % 8) * 16 + (k % 8) * 2;
}

// Shared-memory matrix descriptor: start address, leading byte offset (K
// blocks), stride byte offset (row groups), descriptor version 1, no swizzle.
__device__ __forceinline__ std::uint64_t smem_descriptor(std::uint32_t address, std::uint32_t lbo,
                                                         std::uint32_t sbo) {
  std::uint64_t d = 0;
  d |= std::uint64_t((address >> 4) & 0x3FFFu);
  d |= std::uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= std::uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= std::uint64_t(1) << 46;
  return d;
}

// Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr std::uint32_t instr_descriptor(std::uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma(std::uint32_t tmem, std::uint64_t a, std::uint64_t b, std::uint32_t idesc,
                                    std::uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(std::uint32_t barrier) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(barrier)
               : "memory");
}

__device__ __forceinline__ bool try_wait(std::uint32_t barrier, std::uint32_t phase) {
  std::uint32_t done;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(done)
      : "r"(barrier), "r"(phase)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void load32(std::uint32_t address, float (&v)[32]) {
  std::uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(address));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ std::uint32_t pack(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const std::uint32_t*>(&v);
}

// Copies a row-major (rows x k) bf16 matrix from global memory into the
// operand layout, zero rows from `valid` on.
__device__ void stage_weights(unsigned char* smem, const std::uint16_t* w, std::uint32_t rows, std::uint32_t valid,
                              std::uint32_t k) {
  const std::uint32_t chunks = rows * (k / 8);
  for (std::uint32_t c = threadIdx.x; c < chunks; c += blockDim.x) {
    const std::uint32_t row = c / (k / 8), kb = c % (k / 8);
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (row < valid) v = *reinterpret_cast<const uint4*>(w + std::size_t(row) * k + kb * 8);
    *reinterpret_cast<uint4*>(smem + core_offset(rows, row, kb * 8)) = v;
  }
}

__global__ void __launch_bounds__(kTcThreads, 1) forward_tc_kernel(const std::uint16_t* __restrict__ weights,
                                                              const float* __restrict__ biases,
                                                              const std::uint16_t* __restrict__ x, std::uint32_t n,
                                                              float* __restrict__ y, Activations act, int keep,
                                                              std::uint32_t* error) {
  extern __shared__ __align__(128) unsigned char smem[];
  const std::uint32_t base = static_cast<std::uint32_t>(__cvta_generic_to_shared(smem));
  const std::uint32_t barrier = base + kOffBarrier;
  float* bias = reinterpret_cast<float*>(smem + kOffBias);
  std::uint32_t* tmem_slot = reinterpret_cast<std::uint32_t*>(smem + kOffTmem);
  __shared__ int ok;

  stage_weights(smem + kOffW0, weights + kW0, kHidden, kHidden, kInput);
  stage_weights(smem + kOffW1, weights + kW1, kHidden, kHidden, kHidden);
  stage_weights(smem + kOffW2, weights + kW2, kHidden, kHidden, kHidden);
  stage_weights(smem + kOffW3, weights + kW3, kOutputRows, kOutputPad, kHidden);
  for (std::uint32_t i = threadIdx.x; i < kBiases; i += blockDim.x) bias[i] = biases[i];
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(barrier), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    ok = 1;
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + kOffTmem),
                 "r"(kTmemColumns)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const std::uint32_t tmem = *tmem_slot;
  const std::uint32_t warp = threadIdx.x >> 5;
  const std::uint32_t quarter = warp % 4, chunk = warp / 4;
  const std::uint32_t lane_base = tmem + ((quarter * 32u) << 16);
  const std::uint32_t row = quarter * 32 + (threadIdx.x & 31);  // this thread's cell in a tile = its TMEM lane
  std::uint32_t phase = 0;
  unsigned char* a = smem + kOffA;

  const std::uint32_t tiles = (n + kTile - 1) / kTile;
  for (std::uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    // The tile's features into the A operand (K = 96), zero rows past n.
    const std::uint32_t cell = tile * kTile + row;
    for (std::uint32_t e = threadIdx.x; e < std::uint32_t(kTile) * (kInput / 8); e += blockDim.x) {
      const std::uint32_t r = e / (kInput / 8), kb = e % (kInput / 8);
      const std::uint32_t c = tile * kTile + r;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (c < n) v = *reinterpret_cast<const uint4*>(x + std::size_t(c) * kInput + kb * 8);
      *reinterpret_cast<uint4*>(a + core_offset(kTile, r, kb * 8)) = v;
    }
    for (int layer = 0; layer < 4; ++layer) {
      const std::uint32_t k = layer == 0 ? kInput : kHidden;
      const std::uint32_t rows_b = layer == 3 ? kOutputRows : kHidden;
      const std::uint32_t w_off = layer == 0 ? kOffW0 : (layer == 1 ? kOffW1 : (layer == 2 ? kOffW2 : kOffW3));
      fence_async_smem();  // the operand rows written above, for the tensor cores
      fence_before();
      __syncthreads();
      if (threadIdx.x == 0) {
        fence_after();
        const std::uint32_t idesc = instr_descriptor(rows_b);
        for (std::uint32_t s = 0; s < k / 16; ++s) {
          const std::uint64_t ad = smem_descriptor(base + kOffA + 2 * s * (kTile / 8) * 128, (kTile / 8) * 128, 128);
          const std::uint64_t bd = smem_descriptor(base + w_off + 2 * s * (rows_b / 8) * 128, (rows_b / 8) * 128, 128);
          mma(tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
        }
        commit(barrier);
        std::uint32_t polls = 0;
        while (!try_wait(barrier, phase)) {
          if (++polls > kWaitPolls) {
            ok = 0;
            if (error != nullptr) atomicExch(error, std::uint32_t(kStatusIterations));
            break;
          }
        }
      }
      phase ^= 1u;
      __syncthreads();
      if (!ok) break;
      fence_after();
      if (layer < 3) {
        const float* b = bias + (layer == 0 ? kB0 : (layer == 1 ? kB1 : kB2));
        {
          const std::uint32_t c = chunk;
          float v[32];
          load32(lane_base + c * 32, v);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const std::uint32_t k0 = c * 32 + q * 8;
            float z[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) z[j] = v[q * 8 + j] + b[k0 + j];
            uint4 out;
            out.x = pack(gelu(z[0]), gelu(z[1]));
            out.y = pack(gelu(z[2]), gelu(z[3]));
            out.z = pack(gelu(z[4]), gelu(z[5]));
            out.w = pack(gelu(z[6]), gelu(z[7]));
            *reinterpret_cast<uint4*>(a + core_offset(kTile, row, k0)) = out;
            if (keep && cell < n) {
              // Training: this layer's pre-activations and activations for the backward pass.
              float* zr = act.z[layer] + std::size_t(cell) * kHidden + k0;
              *reinterpret_cast<float4*>(zr) = make_float4(z[0], z[1], z[2], z[3]);
              *reinterpret_cast<float4*>(zr + 4) = make_float4(z[4], z[5], z[6], z[7]);
              *reinterpret_cast<uint4*>(act.h[layer] + std::size_t(cell) * kHidden + k0) = out;
            }
          }
        }
      } else if (chunk == 0) {
        float v[32];
        load32(lane_base, v);
        if (cell < n) {
#pragma unroll
          for (int j = 0; j < kOutputs; ++j) y[std::size_t(cell) * kOutputs + j] = v[j] + bias[kB3 + j];
        }
      }
    }
    if (!ok) break;
  }
  fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemColumns) : "memory");
  }
}

// ------------------------------------------------------------- the GEMM
//
// C (m x n) = A (m x k) B (k x n), bf16 operands through element strides.
// A CTA computes a 128-row tile of C (rows past m zero) over its share of k
// (grid z splits k): per 64-wide k chunk its 128 threads stage the A chunk
// (128 x 64) and the B chunk (n rounded up to 16, x 64) in the canonical
// K-major layout, thread 0 issues four tcgen05.mma (K = 16 each) into the
// TMEM accumulator and commits them to an mbarrier, and the chunk after
// waits for them.  The four warps then read their 32 lanes of the
// accumulator with tcgen05.ld and store C (or the split's partial sums).

constexpr int kGemmThreads = 128;
constexpr std::uint32_t kGemmChunk = 64;
constexpr std::uint32_t kGemmMaxSplits = 32;
constexpr std::uint32_t kGemmBytesA = 128 * kGemmChunk * 2;  // 16 KB
constexpr std::uint32_t kGemmBytesB = 128 * kGemmChunk * 2;  // 16 KB (n <= 128)
constexpr std::uint32_t kGemmOffB = kGemmBytesA;
constexpr std::uint32_t kGemmOffBarrier = kGemmOffB + kGemmBytesB;
constexpr std::uint32_t kGemmOffTmem = kGemmOffBarrier + 8;
// More shared memory than the operands need, so that at most four CTAs
// share an SM: four 128-column accumulators fill its 512 TMEM columns.
constexpr std::size_t kGemmSmem = 56 * 1024;
static_assert(kGemmOffTmem + 8 <= kGemmSmem, "gemm shared memory");

__global__ void __launch_bounds__(kGemmThreads) gemm_tc_kernel(Gemm p, std::uint32_t chunk_split, float* partials,
                                                              std::uint32_t* error) {
  extern __shared__ __align__(128) unsigned char smem[];
  const std::uint32_t base = static_cast<std::uint32_t>(__cvta_generic_to_shared(smem));
  const std::uint32_t barrier = base + kGemmOffBarrier;
  std::uint32_t* tmem_slot = reinterpret_cast<std::uint32_t*>(smem + kGemmOffTmem);
  __shared__ int ok;
  const std::uint32_t nt = (p.n + 15) / 16 * 16;  // the MMA's N
  const std::uint32_t m0 = blockIdx.y * 128;
  const std::uint32_t k_begin = blockIdx.z * chunk_split * kGemmChunk;
  const std::uint32_t k_end = smin<std::uint32_t>(p.k, k_begin + chunk_split * kGemmChunk);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(barrier), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    ok = 1;
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + kGemmOffTmem),
                 "r"(kTmemColumns)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const std::uint32_t tmem = *tmem_slot;
  unsigned char* sa = smem;
  unsigned char* sb = smem + kGemmOffB;
  std::uint32_t phase = 0;
  std::uint32_t issued = 0;
  for (std::uint32_t k0 = k_begin; k0 < k_end; k0 += kGemmChunk) {
    // Stage the chunk: A (128 x 64) and B (nt x 64), zero outside the matrices.
    for (std::uint32_t e = threadIdx.x; e < 128 * kGemmChunk; e += kGemmThreads) {
      const std::uint32_t r = e / kGemmChunk, kk = e % kGemmChunk;
      const std::uint32_t mm = m0 + r, k = k0 + kk;
      const std::uint16_t va = (mm < p.m && k < k_end) ? p.a[std::int64_t(mm) * p.sam + std::int64_t(k) * p.sak] : 0;
      *reinterpret_cast<std::uint16_t*>(sa + core_offset(128, r, kk)) = va;
      if (r < nt) {
        const std::uint16_t vb = (r < p.n && k < k_end) ? p.b[std::int64_t(k) * p.sbk + std::int64_t(r) * p.sbn] : 0;
        *reinterpret_cast<std::uint16_t*>(sb + core_offset(nt, r, kk)) = vb;
      }
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_after();
      const std::uint32_t idesc = instr_descriptor(nt);
      for (std::uint32_t s = 0; s < kGemmChunk / 16; ++s) {
        const std::uint64_t ad = smem_descriptor(base + 2 * s * (128 / 8) * 128, (128 / 8) * 128, 128);
        const std::uint64_t bd = smem_descriptor(base + kGemmOffB + 2 * s * (nt / 8) * 128, (nt / 8) * 128, 128);
        mma(tmem, ad, bd, idesc, (issued > 0 || s > 0) ? 1u : 0u);
      }
      commit(barrier);
      std::uint32_t polls = 0;
      while (!try_wait(barrier, phase)) {
        if (++polls > kWaitPolls) {
          ok = 0;
          if (error != nullptr) atomicExch(error, std::uint32_t(kStatusIterations));
          break;
        }
      }
    }
    phase ^= 1u;
    ++issued;
    __syncthreads();
    if (!ok) break;
  }
  fence_after();
  // Epilogue: warp w holds rows 32w..32w+31 of the tile, one per lane.
  const std::uint32_t warp = threadIdx.x >> 5;
  const std::uint32_t row = m0 + warp * 32 + (threadIdx.x & 31);
  if (ok) {
    for (std::uint32_t c0 = 0; c0 < nt; c0 += 32) {
      float v[32];
      if (issued > 0) {
        load32(tmem + ((warp * 32u) << 16) + c0, v);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = 0.0f;  // an empty share of k
      }
      if (row < p.m) {
        for (std::uint32_t j = 0; j < 32 && c0 + j < p.n; ++j) {
          const std::uint32_t col = c0 + j;
          if (partials != nullptr) {
            partials[(std::size_t(blockIdx.z) * p.m + row) * p.n + col] = v[j];
          } else {
            p.c[std::int64_t(row) * p.scm + std::int64_t(col) * p.scn] = v[j];
          }
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemColumns) : "memory");
  }
}

// C = the sum of the splits' partial sums, in split order.
__global__ void gemm_reduce_kernel(Gemm p, std::uint32_t splits, const float* __restrict__ partials) {
  const std::uint64_t total = std::uint64_t(p.m) * p.n;
  for (std::uint64_t i = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; i < total;
       i += std::uint64_t(gridDim.x) * blockDim.x) {
    float sum = 0.0f;
    for (std::uint32_t z = 0; z < splits; ++z) sum += partials[z * total + i];
    const std::uint32_t row = std::uint32_t(i / p.n), col = std::uint32_t(i % p.n);
    p.c[std::int64_t(row) * p.scm + std::int64_t(col) * p.scn] = sum;
  }
}

}  // namespace

int tc_gemm(const Gemm& p, float* partials, std::uint32_t* error, cudaStream_t stream) {
  if (p.m == 0 || p.n == 0) return 0;
  if (p.n > 128) return int(cudaErrorInvalidValue);
  cudaError_t e = cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGemmSmem));
  if (e != cudaSuccess) return int(e);
  const std::uint32_t tiles = (p.m + 127) / 128;
  const std::uint32_t chunks = std::max<std::uint32_t>(1, (p.k + kGemmChunk - 1) / kGemmChunk);
  // A long k over several CTAs when the tiles alone leave SMs idle.
  std::uint32_t splits = 1;
  if (tiles < 64 && partials != nullptr && std::uint64_t(p.m) * p.n * kGemmMaxSplits * 4 <= kGemmPartialBytes) {
    splits = std::min(std::min(kGemmMaxSplits, chunks), std::max<std::uint32_t>(1, 128 / tiles));
  }
  const std::uint32_t per_split = (chunks + splits - 1) / splits;
  splits = (chunks + per_split - 1) / per_split;
  const dim3 grid(1, tiles, splits);
  gemm_tc_kernel<<<grid, kGemmThreads, kGemmSmem, stream>>>(p, per_split, splits > 1 ? partials : nullptr, error);
  count_launch();
  if (splits > 1) {
    gemm_reduce_kernel<<<grid_for(std::uint64_t(p.m) * p.n, 256), 256, 0, stream>>>(p, splits, partials);
    count_launch();
  }
  return int(cudaGetLastError());
}

int launch_forward_tc(const std::uint16_t* weights, const float* biases, const std::uint16_t* features,
                      std::uint32_t n, float* outputs, void* activations, std::uint32_t* error,
                      cudaStream_t stream) {
  if (n == 0) return 0;
  cudaError_t e = cudaFuncSetAttribute(forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTcSmem));
  if (e != cudaSuccess) return int(e);
  int device = 0, sms = kSmCount;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const std::uint32_t tiles = (n + kTile - 1) / kTile;
  const std::uint32_t blocks = std::max(1u, std::min<std::uint32_t>(tiles, std::uint32_t(sms)));
  const Activations act = activations != nullptr ? activations_at(activations, n) : Activations{};
  forward_tc_kernel<<<blocks, kTcThreads, kTcSmem, stream>>>(weights, biases, features, n, outputs, act,
                                                             activations != nullptr ? 1 : 0, error);
  count_launch();
  return int(cudaGetLastError());
}

}  // namespace msb::mlp
