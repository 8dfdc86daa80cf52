// Scan, stable radix sort and small reductions: the building blocks of the
// device cell list, the row incidence and the keyed row lists.
//
// Both primitives are deterministic: the scan sums in a fixed tree, and the
// LSD radix sort is stable (ties keep input order), which is what lets the
// incidence lists keep each body's rows in row order, as the reference's
// make_incidence does (cpp/cpu/cpu_contact_dynamics.cpp:78-106).

#include <cstdint>

#include "device.cuh"
#include "kernels.h"

namespace msb {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ std::uint32_t block_exclusive_sum(std::uint32_t value, std::uint32_t* total) {
  __shared__ std::uint32_t warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  std::uint32_t inclusive = value;
#pragma unroll
  for (int offset = 1; offset < 32; offset <<= 1) {
    const std::uint32_t up = __shfl_up_sync(0xFFFFFFFFu, inclusive, offset);
    if (lane >= offset) inclusive += up;
  }
  if (lane == 31) warp_sums[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    std::uint32_t w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int offset = 1; offset < 32; offset <<= 1) {
      const std::uint32_t up = __shfl_up_sync(0xFFFFFFFFu, w, offset);
      if (lane >= offset) w += up;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = w;
  }
  __syncthreads();
  const std::uint32_t warp_prefix = warp == 0 ? 0 : warp_sums[warp - 1];
  if (total != nullptr) *total = warp_sums[kScanThreads / 32 - 1];
  __syncthreads();
  return warp_prefix + inclusive - value;
}

__global__ void scan_tile_sums(const std::uint32_t* __restrict__ in, std::uint64_t n,
                               std::uint32_t* __restrict__ sums) {
  const std::uint64_t base = std::uint64_t(blockIdx.x) * kScanTile + std::uint64_t(threadIdx.x) * kScanItems;
  std::uint32_t local = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const std::uint64_t i = base + k;
    if (i < n) local += in[i];
  }
  std::uint32_t total;
  block_exclusive_sum(local, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void scan_tiles(const std::uint32_t* __restrict__ in, std::uint64_t n,
                           const std::uint32_t* __restrict__ tile_offsets, std::uint32_t* __restrict__ out) {
  const std::uint64_t base = std::uint64_t(blockIdx.x) * kScanTile + std::uint64_t(threadIdx.x) * kScanItems;
  std::uint32_t values[kScanItems];
  std::uint32_t local = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const std::uint64_t i = base + k;
    values[k] = i < n ? in[i] : 0;
    local += values[k];
  }
  std::uint32_t running = block_exclusive_sum(local, nullptr);
  if (tile_offsets != nullptr) running += tile_offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const std::uint64_t i = base + k;
    if (i < n) out[i] = running;
    running += values[k];
  }
}

// ---- stable LSD radix sort, 8-bit digits ---------------------------------

constexpr int kSortWarps = 8;
constexpr int kSortRounds = 8;
constexpr int kSortTile = kSortWarps * 32 * kSortRounds;  // 2048 items per block

__global__ void radix_histogram(const std::uint32_t* __restrict__ keys, std::uint64_t n, int shift,
                                std::uint64_t tiles, std::uint32_t* __restrict__ histogram) {
  __shared__ std::uint32_t counts[256];
  counts[threadIdx.x] = 0;
  __syncthreads();
  const std::uint64_t base = std::uint64_t(blockIdx.x) * kSortTile;
  for (int k = threadIdx.x; k < kSortTile; k += blockDim.x) {
    const std::uint64_t i = base + k;
    if (i < n) atomicAdd(&counts[(keys[i] >> shift) & 0xFFu], 1u);
  }
  __syncthreads();
  histogram[std::uint64_t(threadIdx.x) * tiles + blockIdx.x] = counts[threadIdx.x];
}

__global__ void radix_scatter(const std::uint32_t* __restrict__ keys_in,
                              const std::uint32_t* __restrict__ values_in, std::uint64_t n, int shift,
                              std::uint64_t tiles, const std::uint32_t* __restrict__ offsets,
                              std::uint32_t* __restrict__ keys_out, std::uint32_t* __restrict__ values_out) {
  __shared__ std::uint32_t counts[kSortWarps][256];
  __shared__ std::uint32_t tile_offset[256];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < kSortWarps * 256; k += blockDim.x) counts[k / 256][k % 256] = 0;
  tile_offset[threadIdx.x] = offsets[std::uint64_t(threadIdx.x) * tiles + blockIdx.x];
  __syncthreads();
  const std::uint64_t warp_base = std::uint64_t(blockIdx.x) * kSortTile + std::uint64_t(warp) * 32 * kSortRounds;
  std::uint32_t key[kSortRounds], value[kSortRounds], rank[kSortRounds];
  const std::uint32_t lower_lanes = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const std::uint64_t i = warp_base + std::uint64_t(r) * 32 + lane;
    const bool valid = i < n;
    key[r] = valid ? keys_in[i] : 0u;
    value[r] = valid ? values_in[i] : 0u;
    // Lanes past the end take a class of their own so they match nobody.
    const std::uint32_t digit = valid ? ((key[r] >> shift) & 0xFFu) : (256u + lane);
    const std::uint32_t peers = __match_any_sync(0xFFFFFFFFu, digit);
    const std::uint32_t before = __popc(peers & lower_lanes);
    std::uint32_t base = 0;
    if (valid) base = counts[warp][digit];
    __syncwarp();
    if (valid && before == 0) counts[warp][digit] = base + __popc(peers);
    __syncwarp();
    rank[r] = base + before;
  }
  __syncthreads();
  {
    // Exclusive prefix of each digit's count over the warps of the tile.
    const int digit = threadIdx.x;
    std::uint32_t running = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const std::uint32_t c = counts[w][digit];
      counts[w][digit] = running;
      running += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const std::uint64_t i = warp_base + std::uint64_t(r) * 32 + lane;
    if (i < n) {
      const std::uint32_t digit = (key[r] >> shift) & 0xFFu;
      const std::uint32_t at = tile_offset[digit] + counts[warp][digit] + rank[r];
      keys_out[at] = key[r];
      values_out[at] = value[r];
    }
  }
}

__global__ void fill_iota(std::uint32_t* out, std::uint64_t n) {
  for (std::uint64_t i = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += std::uint64_t(gridDim.x) * blockDim.x) {
    out[i] = std::uint32_t(i);
  }
}

}  // namespace

std::uint64_t scan_temp_words(std::uint64_t n) {
  std::uint64_t words = 0;
  std::uint64_t level = n;
  while (level > kScanTile) {
    level = (level + kScanTile - 1) / kScanTile;
    words += 2 * level + 32;
  }
  return words + 64;
}

// Exclusive scan of `n` words; `out` may alias `in`.  `temp` holds
// scan_temp_words(n) words.
void exclusive_scan(const std::uint32_t* in, std::uint32_t* out, std::uint64_t n, std::uint32_t* temp,
                    cudaStream_t stream) {
  if (n == 0) return;
  const std::uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    scan_tiles<<<1, kScanThreads, 0, stream>>>(in, n, nullptr, out);
    count_launch();
    return;
  }
  std::uint32_t* sums = temp;
  std::uint32_t* offsets = temp + tiles + 16;
  std::uint32_t* rest = offsets + tiles + 16;
  scan_tile_sums<<<unsigned(tiles), kScanThreads, 0, stream>>>(in, n, sums);
  count_launch();
  exclusive_scan(sums, offsets, tiles, rest, stream);
  scan_tiles<<<unsigned(tiles), kScanThreads, 0, stream>>>(in, n, offsets, out);
  count_launch();
}

std::uint64_t sort_temp_words(std::uint64_t n) {
  const std::uint64_t tiles = (n + kSortTile - 1) / kSortTile;
  return 2 * n + 2 * 256 * tiles + scan_temp_words(256 * tiles) + 64;
}

// Stable sort of (key, value) pairs by the low `key_bits` bits of the key.
// The result is left in keys/values.  `temp` holds sort_temp_words(n) words.
void radix_sort_pairs(std::uint32_t* keys, std::uint32_t* values, std::uint64_t n, int key_bits,
                      std::uint32_t* temp, cudaStream_t stream) {
  if (n <= 1 || key_bits <= 0) return;
  const std::uint64_t tiles = (n + kSortTile - 1) / kSortTile;
  std::uint32_t* alt_keys = temp;
  std::uint32_t* alt_values = temp + n;
  std::uint32_t* histogram = temp + 2 * n;
  std::uint32_t* offsets = histogram + 256 * tiles;
  std::uint32_t* scan_temp = offsets + 256 * tiles;
  std::uint32_t* src_k = keys;
  std::uint32_t* src_v = values;
  std::uint32_t* dst_k = alt_keys;
  std::uint32_t* dst_v = alt_values;
  int passes = 0;
  for (int shift = 0; shift < key_bits; shift += 8) {
    radix_histogram<<<unsigned(tiles), 256, 0, stream>>>(src_k, n, shift, tiles, histogram);
    count_launch();
    exclusive_scan(histogram, offsets, 256 * tiles, scan_temp, stream);
    radix_scatter<<<unsigned(tiles), 256, 0, stream>>>(src_k, src_v, n, shift, tiles, offsets, dst_k, dst_v);
    count_launch();
    std::swap(src_k, dst_k);
    std::swap(src_v, dst_v);
    ++passes;
  }
  if (passes % 2 == 1) {
    cudaMemcpyAsync(keys, src_k, n * sizeof(std::uint32_t), cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(values, src_v, n * sizeof(std::uint32_t), cudaMemcpyDeviceToDevice, stream);
  }
}

void iota(std::uint32_t* out, std::uint64_t n, cudaStream_t stream) {
  if (n == 0) return;
  fill_iota<<<grid_for(n, 256), 256, 0, stream>>>(out, n);
  count_launch();
}

}  // namespace msb
