// Contact detection on the device: the uniform-grid cell list, the
// candidate sweep, the capsule narrow phase and the wall contacts.
//
// Results match the reference CPU backend bit for bit:
//  * Candidates are the pairs (lower id, higher id) whose FP64 padded boxes
//    overlap, touching included (cpp/core/contact_graph.cpp:17-41,254-300).
//    The grid is only an index: any grid whose boxes are at least as wide as
//    the widest padded capsule box finds exactly those pairs.
//  * The narrow phase repeats the reference's FP32 operations in order
//    (cpp/cpu/cpu_contacts.cpp:54-212); the library is built with
//    --fmad=false, so no multiply-add is contracted.
//  * Output order is (first id, second id, ordinal) for pairs, and
//    (cell id, constraint id, location) for walls, reached by writing each
//    cell's contacts at its rank in id order.

#include <cfloat>
#include <cstdint>

#include "device.cuh"
#include "kernels.h"
#include "../../include/msb200.h"

namespace msb {
namespace {

constexpr int kThreads = 256;

// ------------------------------------------------------------ cell boxes

__global__ void cell_bounds_kernel(GeometryView g, float margin, double* __restrict__ bounds,
                                   double* __restrict__ partials) {
  double low[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
  double high[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  double width[3] = {0.0, 0.0, 0.0};
  double finite = 1.0;
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.count; i += gridDim.x * blockDim.x) {
    double box[6];
    padded_box(g.pos_len[i], g.dir_rad[i], margin, box);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double lo = box[a];
      const double hi = box[3 + a];
      bounds[6 * std::uint64_t(i) + a] = lo;
      bounds[6 * std::uint64_t(i) + 3 + a] = hi;
      if (!isfinite(lo) || !isfinite(hi)) finite = 0.0;
      low[a] = fmin(low[a], lo);
      high[a] = fmax(high[a], hi);
      width[a] = fmax(width[a], hi - lo);
    }
  }
  // Block reduction of the ten values (min, max and a finite flag).
  __shared__ double shared[10][kThreads / 32];
  double v[10] = {low[0], low[1], low[2], high[0], high[1], high[2], width[0], width[1], width[2], finite};
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_down_sync(0xFFFFFFFFu, v[k], o);
      v[k] = (k < 3 || k == 9) ? fmin(v[k], other) : fmax(v[k], other);
    }
    if (lane == 0) shared[k][warp] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 10) {
    const int k = threadIdx.x;
    double r = shared[k][0];
    for (int w = 1; w < kThreads / 32; ++w) r = (k < 3 || k == 9) ? fmin(r, shared[k][w]) : fmax(r, shared[k][w]);
    partials[10 * blockIdx.x + k] = r;
  }
}

__global__ void grid_setup_kernel(const double* __restrict__ partials, std::uint32_t partial_count,
                                  std::uint32_t cells, std::uint64_t bucket_capacity, GridParams* grid,
                                  double box_scale, std::uint32_t colonies) {
  // Block reduction of the per-block partials (minima, maxima, finite flag).
  __shared__ double shared[10][kThreads / 32];
  double v[10];
  for (int k = 0; k < 10; ++k) v[k] = (k < 3 || k == 9) ? DBL_MAX : -DBL_MAX;
  v[6] = v[7] = v[8] = 0.0;
  for (std::uint32_t p = threadIdx.x; p < partial_count; p += blockDim.x) {
    for (int k = 0; k < 10; ++k) {
      const double x = partials[10 * p + k];
      v[k] = (k < 3 || k == 9) ? fmin(v[k], x) : fmax(v[k], x);
    }
  }
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int k = 0; k < 10; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_down_sync(0xFFFFFFFFu, v[k], o);
      v[k] = (k < 3 || k == 9) ? fmin(v[k], other) : fmax(v[k], other);
    }
    if (lane == 0) shared[k][warp] = v[k];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int k = 0; k < 10; ++k) {
    v[k] = shared[k][0];
    for (int w = 1; w < kThreads / 32; ++w) v[k] = (k < 3 || k == 9) ? fmin(v[k], shared[k][w]) : fmax(v[k], shared[k][w]);
  }
  GridParams out{};
  out.status = v[9] > 0.5 ? 0u : 1u;
  const double limit = 8.0 * double(cells) + 4096.0;
  bool dense = true;
  double boxes = 1.0;
  for (int a = 0; a < 3; ++a) {
    // Boxes 0.1% wider than the widest padded capsule keep rounding from
    // putting overlapping capsules two boxes apart.
    const double box_width = smax(v[6 + a] * 1.001 * box_scale, DBL_MIN);
    const double extent = floor((v[3 + a] - v[a]) / box_width) + 1.0;
    out.low[a] = v[a];
    out.inv_width[a] = 1.0 / box_width;
    if (!(extent <= limit)) {
      dense = false;
      out.dims[a] = 0xFFFFFFFFFFFFull;
    } else {
      out.dims[a] = std::uint64_t(extent);
      boxes *= extent;
    }
  }
  if (!(boxes <= limit)) dense = false;
  if (colonies > 0) {
    // A batch: each colony gets its own range of z boxes, two boxes apart
    // from the next colony's, in a hashed table.
    const double extent = floor((v[5] - v[2]) * out.inv_width[2]) + 1.0;
    const double stride = extent + 2.0;
    if (!(stride * double(colonies) < 9.0e15)) out.status = 1u;
    out.colony_stride = std::uint32_t(smin(stride, 4.0e9));
    dense = false;
  }
  if (dense) {
    out.hashed = 0;
    out.buckets = std::uint32_t(boxes);
  } else {
    std::uint64_t table = 1;
    while (table < 2ull * cells) table <<= 1;
    out.hashed = 1;
    out.buckets = std::uint32_t(table);
    for (int a = 0; a < 3; ++a) {
      const double extent = floor((v[3 + a] - v[a]) * out.inv_width[a]) + 1.0;
      out.dims[a] = extent < 9.0e15 ? std::uint64_t(extent) : 9000000000000000ull;
    }
    if (colonies > 0) out.dims[2] = std::uint64_t(out.colony_stride) * colonies;
  }
  if (out.buckets + 1ull > bucket_capacity) out.status = 2u;
  *grid = out;
}

__device__ __forceinline__ void box_of(const double* b, const GridParams& grid, std::int64_t at[3],
                                       std::uint32_t colony) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double centre = 0.5 * (b[a] + b[3 + a]);
    const double position = smax(0.0, (centre - grid.low[a]) * grid.inv_width[a]);
    const bool stacked = a == 2 && grid.colony_stride > 0;
    const double top = stacked ? double(grid.colony_stride - 3) : double(grid.dims[a] - 1);
    at[a] = std::int64_t(smin(top, floor(position)));
    if (stacked) at[a] += std::int64_t(colony) * std::int64_t(grid.colony_stride);
  }
}

__device__ __forceinline__ std::uint32_t bucket_of(const GridParams& grid, std::int64_t x, std::int64_t y,
                                                   std::int64_t z) {
  if (grid.hashed == 0) {
    return std::uint32_t((std::uint64_t(x) * grid.dims[1] + std::uint64_t(y)) * grid.dims[2] + std::uint64_t(z));
  }
  std::uint64_t h = std::uint64_t(x) * 0x9E3779B97F4A7C15ull;
  h ^= std::uint64_t(y) * 0xC2B2AE3D27D4EB4Full + (h >> 29);
  h ^= std::uint64_t(z) * 0x165667B19E3779F9ull + (h >> 31);
  h ^= h >> 33;
  return std::uint32_t(h & std::uint64_t(grid.buckets - 1));
}

__global__ void bin_cells_kernel(GeometryView g, const double* __restrict__ bounds, const GridParams* grid_ptr,
                                 std::uint32_t* __restrict__ cell_bucket, std::int64_t* __restrict__ coords,
                                 std::uint32_t* __restrict__ counts) {
  const GridParams grid = *grid_ptr;
  if (grid.status != 0) return;
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.count; i += gridDim.x * blockDim.x) {
    std::int64_t at[3];
    box_of(bounds + 6 * std::uint64_t(i), grid, at, g.colony != nullptr ? g.colony[i] : 0u);
    const std::uint32_t b = bucket_of(grid, at[0], at[1], at[2]);
    cell_bucket[i] = b;
    if (grid.hashed) {
      coords[3 * std::uint64_t(i)] = at[0];
      coords[3 * std::uint64_t(i) + 1] = at[1];
      coords[3 * std::uint64_t(i) + 2] = at[2];
    }
    atomicAdd(&counts[b], 1u);
  }
}

// Places each cell at its bucket's next position, with its box rounded
// outward to FP32 (a box that overlaps in FP64 overlaps in these), its slot
// in lo.w and its id: the sweep then reads a bucket's cells contiguously.
__global__ void scatter_cells_kernel(GeometryView g, const double* __restrict__ bounds,
                                     const std::uint32_t* __restrict__ cell_bucket,
                                     const std::uint32_t* __restrict__ starts, std::uint32_t* __restrict__ fill,
                                     float4* __restrict__ sorted_lo, float4* __restrict__ sorted_hi,
                                     std::uint64_t* __restrict__ sorted_id) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.count; i += gridDim.x * blockDim.x) {
    const std::uint32_t b = cell_bucket[i];
    const std::uint32_t at = starts[b] + atomicAdd(&fill[b], 1u);
    const double* box = bounds + 6 * std::uint64_t(i);
    sorted_lo[at] = make_float4(__double2float_rd(box[0]), __double2float_rd(box[1]), __double2float_rd(box[2]),
                                __uint_as_float(i));
    sorted_hi[at] = make_float4(__double2float_ru(box[3]), __double2float_ru(box[4]), __double2float_ru(box[5]), 0.0f);
    sorted_id[at] = g.ids[i];
  }
}

constexpr int kLocalPartners = 32;
static_assert(kLocalPartners == int(kSlabPartners), "slab rows hold the locally kept partners");

// One thread per cell, cells taken in bucket order so that a warp's cells
// share their neighbour buckets in cache: the partners of higher id among
// the cells of the 27 (or fewer) grid boxes around it whose padded boxes
// overlap its own.  The FP32 outward-rounded boxes cull; the reference's
// FP64 box test decides (cpp/core/contact_graph.cpp:37-41).
// Eight resident 128-thread blocks per SM cap the sweep at 64 registers:
// the kept partners spill a little, and the extra resident warps hide more of
// the candidate loads' latency (measured: search 6.2 -> 5.0 ms per 1M step).
#ifndef MSB_BROAD_MIN_BLOCKS
#define MSB_BROAD_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(128, MSB_BROAD_MIN_BLOCKS) broad_phase_kernel(GeometryView g, const double* __restrict__ bounds, const GridParams* grid_ptr,
                                   const std::uint32_t* __restrict__ starts, const float4* __restrict__ sorted_lo,
                                   const float4* __restrict__ sorted_hi, const std::uint64_t* __restrict__ sorted_id,
                                   const std::int64_t* __restrict__ coords, const std::uint32_t* __restrict__ rank,
                                   std::uint32_t* __restrict__ counts, const std::uint32_t* __restrict__ offsets,
                                   uint2* __restrict__ pairs, std::uint32_t* __restrict__ slab,
                                   std::uint32_t* status) {
  const GridParams grid = *grid_ptr;
  if (grid.status != 0) return;
  const bool fill = pairs != nullptr;
  // With a slab and no pairs, one pass counts and keeps up to kLocalPartners
  // sorted partners per cell in its slab row; the fill pass then only runs
  // for the cells with more.
  const bool keep = slab != nullptr && !fill;
  for (std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < g.count; k += gridDim.x * blockDim.x) {
    const float4 my_lo = sorted_lo[k];
    const float4 my_hi = sorted_hi[k];
    const std::uint32_t a = __float_as_uint(my_lo.w);
    if (fill && slab != nullptr && counts[rank[a]] <= std::uint32_t(kLocalPartners)) continue;
    const std::uint32_t colony = g.colony != nullptr ? g.colony[a] : 0u;
    if (g.colony_active != nullptr && g.colony_active[colony] == 0u) {
      if (!fill) counts[rank[a]] = 0;  // a settled colony of a batch: no partners this round
      continue;
    }
    const std::uint64_t id = sorted_id[k];
    double box[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) box[q] = bounds[6 * std::uint64_t(a) + q];
    std::int64_t at[3];
    box_of(box, grid, at, colony);
    std::int64_t first[3], last[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      first[q] = at[q] == 0 ? 0 : at[q] - 1;
      last[q] = smin(std::int64_t(grid.dims[q]) - 1, at[q] + 1);
    }
    if (grid.colony_stride > 0) {
      // Only the colony's own z boxes hold its cells.
      const std::int64_t own = std::int64_t(colony) * std::int64_t(grid.colony_stride);
      first[2] = smax(first[2], own);
      last[2] = smin(last[2], own + std::int64_t(grid.colony_stride) - 3);
    }
    const std::uint32_t base = fill ? offsets[rank[a]] : 0;
    std::uint32_t found = 0;
    std::uint64_t local_id[kLocalPartners];
    std::uint32_t local_slot[kLocalPartners];
    for (std::int64_t x = first[0]; x <= last[0]; ++x) {
      for (std::int64_t y = first[1]; y <= last[1]; ++y) {
        for (std::int64_t z = first[2]; z <= last[2]; ++z) {
          const std::uint32_t b = bucket_of(grid, x, y, z);
          const std::uint32_t end = starts[b + 1];
          for (std::uint32_t m = starts[b]; m < end; ++m) {
            const std::uint64_t other = sorted_id[m];
            if (!(other > id)) continue;
            const float4 lo = sorted_lo[m];
            const float4 hi = sorted_hi[m];
            if (!(my_hi.x >= lo.x && hi.x >= my_lo.x && my_hi.y >= lo.y && hi.y >= my_lo.y && my_hi.z >= lo.z &&
                  hi.z >= my_lo.z)) {
              continue;
            }
            const std::uint32_t j = __float_as_uint(lo.w);
            if (grid.hashed) {
              const std::int64_t* c = coords + 3 * std::uint64_t(j);
              if (c[0] != x || c[1] != y || c[2] != z) continue;
            }
            if (!boxes_overlap(box, bounds + 6 * std::uint64_t(j))) continue;
            if (keep) {
              if (found < kLocalPartners) {
                local_id[found] = other;
                local_slot[found] = j;
              }
            } else if (fill) {
              if (found < kLocalPartners) {
                local_id[found] = other;
                local_slot[found] = j;
              } else {
                pairs[base + found] = make_uint2(a, j);
              }
            }
            ++found;
          }
        }
      }
    }
    if (keep) {
      counts[rank[a]] = found;
      if (found > std::uint32_t(kLocalPartners)) atomicAdd(&counts[g.count], 1u);  // cells for the fill pass
      if (found <= kLocalPartners) {
        for (std::uint32_t i = 1; i < found; ++i) {
          const std::uint64_t kid = local_id[i];
          const std::uint32_t ks = local_slot[i];
          std::uint32_t j = i;
          while (j > 0 && local_id[j - 1] > kid) {
            local_id[j] = local_id[j - 1];
            local_slot[j] = local_slot[j - 1];
            --j;
          }
          local_id[j] = kid;
          local_slot[j] = ks;
        }
        std::uint32_t* row = slab + std::uint64_t(rank[a]) * kLocalPartners;
        for (std::uint32_t i = 0; i < found; ++i) row[i] = local_slot[i];
      }
      continue;
    }
    if (!fill) {
      counts[rank[a]] = found;
      continue;
    }
    if (found <= kLocalPartners) {
      // Insertion sort by partner id in registers, then write.
      for (std::uint32_t i = 1; i < found; ++i) {
        const std::uint64_t kid = local_id[i];
        const std::uint32_t ks = local_slot[i];
        std::uint32_t j = i;
        while (j > 0 && local_id[j - 1] > kid) {
          local_id[j] = local_id[j - 1];
          local_slot[j] = local_slot[j - 1];
          --j;
        }
        local_id[j] = kid;
        local_slot[j] = ks;
      }
      for (std::uint32_t i = 0; i < found; ++i) pairs[base + i] = make_uint2(a, local_slot[i]);
    } else {
      for (std::uint32_t i = 0; i < kLocalPartners; ++i) pairs[base + i] = make_uint2(a, local_slot[i]);
      // Many partners: insertion sort of the segment in global memory.
      for (std::uint32_t i = 1; i < found; ++i) {
        const uint2 key = pairs[base + i];
        const std::uint64_t kid = g.ids[key.y];
        std::uint32_t j = i;
        while (j > 0 && g.ids[pairs[base + j - 1].y] > kid) {
          pairs[base + j] = pairs[base + j - 1];
          --j;
        }
        pairs[base + j] = key;
      }
    }
    if (counts != nullptr && counts[rank[a]] != found) raise_status(status, kStatusCapacity);
  }
}

// The slab rows of cells with at most kLocalPartners partners, copied into
// their places in the pair list: thread per (cell rank, partner).
__global__ void compact_slab_kernel(std::uint32_t n, const std::uint32_t* __restrict__ counts,
                                    const std::uint32_t* __restrict__ offsets, const std::uint32_t* __restrict__ order,
                                    const std::uint32_t* __restrict__ slab, uint2* __restrict__ pairs) {
  const std::uint64_t total = std::uint64_t(n) * kLocalPartners;
  for (std::uint64_t t = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; t < total;
       t += std::uint64_t(gridDim.x) * blockDim.x) {
    const std::uint32_t r = std::uint32_t(t / kLocalPartners);
    const std::uint32_t i = std::uint32_t(t % kLocalPartners);
    const std::uint32_t count = counts[r];
    if (count > std::uint32_t(kLocalPartners) || i >= count) continue;
    pairs[offsets[r] + i] = make_uint2(order[r], slab[t]);
  }
}

// ---------------------------------------------------------- partial re-search
//
// An overlap re-check whose substep's kept candidates (padded by a margin P
// at the substep's base geometry) may no longer cover every pair, because
// some cells moved more than P / 2 since: the pairs of two cells that each
// moved less are still covered, and the pairs of the others ("fast" cells)
// are searched again on a grid of the current geometry.  Those not already
// kept (usually none: the kept list's padding covers most of a fast cell's
// move) are merged into the kept list in (first id, second id) order.

// Cells whose unpadded box moved by more than the kept candidates allow
// between `from` and `to` (a face moved by `bound`, rounded up as the move
// kernel rounds it, with 2 * bound > allowance), appended to `list` in any
// order; *count their number.  Cells of a batch's settled colonies are left
// out, as their pairs are in every search of the round.
__global__ void fast_cells_kernel(GeometryView from, GeometryView to, double allowance, std::uint32_t* __restrict__ fast,
                                  std::uint32_t* __restrict__ list, std::uint32_t* count) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < to.count; s += gridDim.x * blockDim.x) {
    double a[6], b[6];
    padded_box(from.pos_len[s], from.dir_rad[s], 0.0f, a);
    padded_box(to.pos_len[s], to.dir_rad[s], 0.0f, b);
    double moved = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) moved = fmax(moved, fabs(b[k] - a[k]));
    const float bound = isfinite(moved) ? __double2float_ru(moved) : __int_as_float(0x7F800000);
    bool f = !(2.0 * double(bound) <= allowance);
    if (f && to.colony_active != nullptr && to.colony_active[to.colony[s]] == 0u) f = false;
    fast[s] = f ? 1u : 0u;
    if (f) list[atomicAdd(count, 1u)] = s;
  }
}

// (ids[first], ids[second]) of pair p is below that of pair q.
__device__ __forceinline__ bool pair_before(const std::uint64_t* ids, uint2 p, uint2 q) {
  const std::uint64_t a = ids[p.x], b = ids[q.x];
  return a < b || (a == b && ids[p.y] < ids[q.y]);
}

// The first of `count` pairs sorted by (first id, second id) that is not
// before pair p.
__device__ __forceinline__ std::uint32_t lower_bound_pair(const uint2* sorted, std::uint32_t count,
                                                          const std::uint64_t* ids, uint2 p) {
  std::uint32_t lo = 0, hi = count;
  while (lo < hi) {
    const std::uint32_t mid = lo + (hi - lo) / 2;
    if (pair_before(ids, sorted[mid], p)) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

// The partners of each listed fast cell on the grid of the current
// geometry (boxes at margin 0): every cell whose FP64 box overlaps its own,
// except another fast cell of lower id (whose own query lists that pair) and
// the pairs the kept list holds (a cell's kept pairs as first cell are
// kept[kept_offsets[rank[cell]] ...], the broad phase's list order).  Count
// pass (pairs null): counts[i]; fill pass: the pairs at offsets[i], each as
// (lower-id slot, higher-id slot).  The listed cells' number is read from
// *fast_count.
__global__ void fast_partners_kernel(GeometryView g, const double* __restrict__ bounds, const GridParams* grid_ptr,
                                     const std::uint32_t* __restrict__ starts, const float4* __restrict__ sorted_lo,
                                     const float4* __restrict__ sorted_hi, const std::uint64_t* __restrict__ sorted_id,
                                     const std::int64_t* __restrict__ coords, const std::uint32_t* __restrict__ fast,
                                     const std::uint32_t* __restrict__ list, const std::uint32_t* fast_count_ptr,
                                     std::uint32_t cap, const uint2* __restrict__ kept,
                                     const std::uint32_t* __restrict__ kept_offsets,
                                     const std::uint32_t* __restrict__ rank, std::uint32_t* __restrict__ counts,
                                     const std::uint32_t* __restrict__ offsets,
                                     uint2* __restrict__ pairs) {
  const GridParams grid = *grid_ptr;
  const std::uint32_t fast_count = *fast_count_ptr < cap ? *fast_count_ptr : cap;
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
    if (grid.status != 0 || i >= fast_count) {
      if (pairs == nullptr) counts[i] = 0;
      continue;
    }
    const std::uint32_t f = list[i];
    const std::uint32_t colony = g.colony != nullptr ? g.colony[f] : 0u;
    double box[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) box[q] = bounds[6 * std::uint64_t(f) + q];
    const float4 my_lo = make_float4(__double2float_rd(box[0]), __double2float_rd(box[1]), __double2float_rd(box[2]), 0.0f);
    const float4 my_hi = make_float4(__double2float_ru(box[3]), __double2float_ru(box[4]), __double2float_ru(box[5]), 0.0f);
    const std::uint64_t id = g.ids[f];
    std::int64_t at[3];
    box_of(box, grid, at, colony);
    std::int64_t first[3], last[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      first[q] = at[q] == 0 ? 0 : at[q] - 1;
      last[q] = smin(std::int64_t(grid.dims[q]) - 1, at[q] + 1);
    }
    if (grid.colony_stride > 0) {
      const std::int64_t own = std::int64_t(colony) * std::int64_t(grid.colony_stride);
      first[2] = smax(first[2], own);
      last[2] = smin(last[2], own + std::int64_t(grid.colony_stride) - 3);
    }
    const std::uint32_t base = pairs != nullptr ? offsets[i] : 0u;
    std::uint32_t found = 0;
    for (std::int64_t x = first[0]; x <= last[0]; ++x) {
      for (std::int64_t y = first[1]; y <= last[1]; ++y) {
        for (std::int64_t z = first[2]; z <= last[2]; ++z) {
          const std::uint32_t b = bucket_of(grid, x, y, z);
          const std::uint32_t end = starts[b + 1];
          for (std::uint32_t m = starts[b]; m < end; ++m) {
            const float4 lo = sorted_lo[m];
            const std::uint32_t j = __float_as_uint(lo.w);
            if (j == f) continue;
            const std::uint64_t other = sorted_id[m];
            if (fast[j] != 0u && other < id) continue;
            const float4 hi = sorted_hi[m];
            if (!(my_hi.x >= lo.x && hi.x >= my_lo.x && my_hi.y >= lo.y && hi.y >= my_lo.y && my_hi.z >= lo.z &&
                  hi.z >= my_lo.z)) {
              continue;
            }
            if (grid.hashed) {
              const std::int64_t* c = coords + 3 * std::uint64_t(j);
              if (c[0] != x || c[1] != y || c[2] != z) continue;
            }
            if (!boxes_overlap(box, bounds + 6 * std::uint64_t(j))) continue;
            const uint2 pair = id < other ? make_uint2(f, j) : make_uint2(j, f);
            const std::uint32_t r = rank[pair.x];
            bool held = false;
            for (std::uint32_t k = kept_offsets[r]; k < kept_offsets[r + 1] && !held; ++k) held = kept[k].y == pair.y;
            if (held) continue;
            if (pairs != nullptr) pairs[base + found] = pair;
            ++found;
          }
        }
      }
    }
    if (pairs == nullptr) counts[i] = found;
  }
}

// The fast pairs in (first id, second id) order: each pair's place is the
// number of pairs before it (all pairs are distinct).
__global__ void sort_fast_pairs_kernel(const uint2* __restrict__ in, std::uint32_t m, const std::uint64_t* __restrict__ ids,
                                       uint2* __restrict__ out) {
  for (std::uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
    const uint2 mine = in[p];
    std::uint32_t place = 0;
    for (std::uint32_t q = 0; q < m; ++q) place += pair_before(ids, in[q], mine) ? 1u : 0u;
    out[place] = mine;
  }
}

// Each sorted new pair j at its place in the merged list, j + (kept pairs
// before it), found by bisection of the kept list; shift[kept pairs before
// it] counts it for the kept pairs' places.
__global__ void place_fast_pairs_kernel(const uint2* __restrict__ sorted_fast, std::uint32_t m,
                                        const uint2* __restrict__ kept, std::uint32_t kept_count,
                                        const std::uint64_t* __restrict__ ids, uint2* __restrict__ merged,
                                        std::uint32_t* __restrict__ shift) {
  for (std::uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    const uint2 p = sorted_fast[j];
    const std::uint32_t before = lower_bound_pair(kept, kept_count, ids, p);
    merged[j + before] = p;
    atomicAdd(&shift[before], 1u);
  }
}

// Each kept pair k at its place: k plus the new pairs before it
// (shift_scan[k + 1], an exclusive scan of shift).
__global__ void place_kept_pairs_kernel(const uint2* __restrict__ kept, std::uint32_t kept_count,
                                        const std::uint32_t* __restrict__ shift_scan, uint2* __restrict__ merged) {
  for (std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < kept_count; k += gridDim.x * blockDim.x) {
    merged[k + shift_scan[k + 1]] = kept[k];
  }
}

// ---------------------------------------------------------- narrow phase

struct Capsule {
  F3 c;
  F3 a;
  float len;
  float r;
};

struct PointPair {
  F3 first, second;
};

__device__ __forceinline__ Capsule capsule_at(GeometryView g, std::uint32_t i) {
  const float4 pl = g.pos_len[i];
  const float4 dr = g.dir_rad[i];
  return {xyz(pl), xyz(dr), pl.w, dr.w};
}

// cpu_contacts.cpp:54-108
__device__ PointPair closest_points(const Capsule& p, const Capsule& q, float eps) {
  const float ph = p.len * 0.5f;
  const float qh = q.len * 0.5f;
  const F3 p0 = p.c - (p.a * ph);
  const F3 p1 = p.c + (p.a * ph);
  const F3 q0 = q.c - (q.a * qh);
  const F3 q1 = q.c + (q.a * qh);
  const F3 d1 = p1 - p0;
  const F3 d2 = q1 - q0;
  const F3 r = p0 - q0;
  const float a = dot(d1, d1);
  const float e = dot(d2, d2);
  const float f = dot(d2, r);
  float s = 0.0f, t = 0.0f;
  const float eps2 = eps * eps;
  if (a <= eps2 && e <= eps2) return {p0, q0};
  if (a <= eps2) {
    t = sclamp(f / e, 0.0f, 1.0f);
  } else {
    const float c = dot(d1, r);
    if (e <= eps2) {
      s = sclamp(-c / a, 0.0f, 1.0f);
    } else {
      const float b = dot(d1, d2);
      const float denom = (a * e) - (b * b);
      const float tol = FLT_EPSILON * a * e;
      if (denom > tol) s = sclamp(((b * f) - (c * e)) / denom, 0.0f, 1.0f);
      t = (b * s + f) / e;
      if (t < 0.0f) {
        t = 0.0f;
        s = sclamp(-c / a, 0.0f, 1.0f);
      } else if (t > 1.0f) {
        t = 1.0f;
        s = sclamp((b - c) / a, 0.0f, 1.0f);
      }
    }
  }
  return {p0 + (d1 * s), q0 + (d2 * t)};
}

// cpu_contacts.cpp:110-140
__device__ int contact_points(const Capsule& p, const Capsule& q, float sine_threshold, float eps,
                              PointPair out[2]) {
  const float ad = sclamp(dot(p.a, q.a), -1.0f, 1.0f);
  const float sine = __fsqrt_rn(smax(0.0f, 1.0f - (ad * ad)));
  if (sine > sine_threshold || p.len <= eps || q.len <= eps) {
    out[0] = closest_points(p, q, eps);
    return 1;
  }
  const float ph = p.len * 0.5f;
  const float qh = q.len * 0.5f;
  const float cc = dot(q.c - p.c, p.a);
  const float proj = qh * fabsf(ad);
  const float begin = smax(-ph, cc - proj);
  const float end = smin(ph, cc + proj);
  if (end - begin <= eps) {
    out[0] = closest_points(p, q, eps);
    return 1;
  }
  const float params[2] = {begin, end};
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const F3 on_p = p.c + (p.a * params[k]);
    const float t = sclamp(dot(on_p - q.c, q.a), -qh, qh);
    out[k] = {on_p, q.c + (q.a * t)};
  }
  return 2;
}

// cpu_contacts.cpp:142-166.  Inputs are validated unit axes, so every branch
// normalizes a non-zero vector.
__device__ F3 deterministic_normal(const Capsule& p, const Capsule& q, const PointPair& pts, float eps) {
  F3 out{1.0f, 0.0f, 0.0f};
  const F3 delta = pts.second - pts.first;
  if (norm(delta) > eps) {
    normalized(delta, out);
    return out;
  }
  const F3 ax = cross(p.a, q.a);
  if (norm(ax) > eps) {
    normalized(ax, out);
    return out;
  }
  const F3 cd = q.c - p.c;
  const F3 tr = cd - (p.a * dot(cd, p.a));
  if (norm(tr) > eps) {
    normalized(tr, out);
    return out;
  }
  const F3 basis[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  int best = 0;
  for (int k = 1; k < 3; ++k) {
    if (fabsf(dot(p.a, basis[k])) < fabsf(dot(p.a, basis[best]))) best = k;
  }
  normalized(cross(p.a, basis[best]), out);
  return out;
}

__global__ void narrow_phase_kernel(GeometryView g, const uint2* __restrict__ pairs, std::uint64_t pair_count,
                                    ContactSearchParams prm, std::uint32_t* __restrict__ counts,
                                    const std::uint32_t* __restrict__ offsets, Touch* __restrict__ touches,
                                    std::uint32_t* status) {
  for (std::uint64_t k = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; k < pair_count;
       k += std::uint64_t(gridDim.x) * blockDim.x) {
    // The fill pass skips the pairs that the count pass found without a
    // touch (most of a padded candidate list): no geometry loads for them.
    if (touches != nullptr && offsets[k + 1] == offsets[k]) continue;
    const uint2 pair = pairs[k];
    if (!index_ok(pair.x, g.count, status) || !index_ok(pair.y, g.count, status)) {
      if (counts != nullptr) counts[k] = 0;
      continue;
    }
    if (g.colony_active != nullptr && g.colony_active[g.colony[pair.x]] == 0u) {
      // A settled colony of a batch takes no part in this round, as in the
      // broad phase.
      if (counts != nullptr) counts[k] = 0;
      continue;
    }
    if (prm.box_margin >= 0.0f) {
      // Candidates from a wider search (or from another geometry): only
      // the pairs whose boxes at box_margin overlap here are the
      // reference's candidates.
      double first[6], second[6];
      padded_box(g.pos_len[pair.x], g.dir_rad[pair.x], prm.box_margin, first);
      padded_box(g.pos_len[pair.y], g.dir_rad[pair.y], prm.box_margin, second);
      if (!boxes_overlap(first, second)) {
        if (counts != nullptr) counts[k] = 0;
        continue;
      }
    }
    const Capsule p = capsule_at(g, pair.x);
    const Capsule q = capsule_at(g, pair.y);
    PointPair pts[2];
    const int n = contact_points(p, q, prm.sine_threshold, prm.epsilon, pts);
    const float weight = n == 2 ? 0.7071067811865475f : 1.0f;
    std::uint32_t written = 0;
    const std::uint32_t base = touches != nullptr ? offsets[k] : 0;
    for (int o = 0; o < n; ++o) {
      const float sep = norm(pts[o].second - pts[o].first) - (p.r + q.r);
      if (sep >= prm.margin) continue;
      if (touches != nullptr) {
        const F3 nrm = deterministic_normal(p, q, pts[o], prm.epsilon);
        const F3 point = pts[o].first + (nrm * p.r);
        Touch t;
        t.s1 = pair.x;
        t.s2 = pair.y;
        t.partner = pair.y;
        t.point[0] = point.x;
        t.point[1] = point.y;
        t.point[2] = point.z;
        t.normal[0] = nrm.x;
        t.normal[1] = nrm.y;
        t.normal[2] = nrm.z;
        t.sep = sep;
        t.weight = weight;
        t.tag = std::uint32_t(o);
        t.kind = 0;
        t.pad[0] = t.pad[1] = 0;
        touches[base + written] = t;
      }
      ++written;
    }
    if (touches == nullptr) counts[k] = written;
  }
}

// --------------------------------------------------------- wall contacts
// cpp/cpu/cpu_constraints.cpp:24-612

struct Surface {
  float distance;
  F3 outward;
};

struct WallEmitter {
  Touch* out;
  std::uint32_t count;
  std::uint32_t slot;
  __device__ void emit(const DeviceConstraint& c, std::uint32_t location, F3 point, F3 normal, float sep,
                       float weight) {
    if (out != nullptr) {
      Touch t;
      t.s1 = slot;
      t.s2 = kInvalidSlot;
      t.partner = c.id;
      t.point[0] = point.x;
      t.point[1] = point.y;
      t.point[2] = point.z;
      t.normal[0] = normal.x;
      t.normal[1] = normal.y;
      t.normal[2] = normal.z;
      t.sep = sep;
      t.weight = weight;
      t.tag = location;
      t.kind = c.kind;
      t.pad[0] = t.pad[1] = 0;
      out[count] = t;
    }
    ++count;
  }
};

__device__ __forceinline__ F3 ca(const DeviceConstraint& c) { return {c.a[0], c.a[1], c.a[2]}; }
__device__ __forceinline__ F3 cb(const DeviceConstraint& c) { return {c.b[0], c.b[1], c.b[2]}; }

__device__ bool segment_hits_box(F3 s, F3 e, F3 lo, F3 hi) {
  const F3 d = e - s;
  const float ss[3] = {s.x, s.y, s.z}, dd[3] = {d.x, d.y, d.z}, ll[3] = {lo.x, lo.y, lo.z},
              uu[3] = {hi.x, hi.y, hi.z};
  float entry = 0.0f, exit = 1.0f;
  for (int a = 0; a < 3; ++a) {
    if (dd[a] == 0.0f) {
      if (ss[a] < ll[a] || ss[a] > uu[a]) return false;
      continue;
    }
    float f = (ll[a] - ss[a]) / dd[a];
    float h = (uu[a] - ss[a]) / dd[a];
    if (f > h) {
      const float t = f;
      f = h;
      h = t;
    }
    entry = smax(entry, f);
    exit = smin(exit, h);
    if (entry > exit) return false;
  }
  return true;
}

__device__ Surface box_surface(F3 p, const DeviceConstraint& box, float eps) {
  const F3 d = p - ca(box);
  const F3 cl{sclamp(d.x, -box.b[0], box.b[0]), sclamp(d.y, -box.b[1], box.b[1]), sclamp(d.z, -box.b[2], box.b[2])};
  const F3 o = d - cl;
  const float od = norm(o);
  if (od > eps) return {od, o * (1.0f / od)};
  const float clear[3] = {box.b[0] - fabsf(d.x), box.b[1] - fabsf(d.y), box.b[2] - fabsf(d.z)};
  int ax = 0;
  for (int k = 1; k < 3; ++k) {
    if (clear[k] < clear[ax]) ax = k;
  }
  const float off[3] = {d.x, d.y, d.z};
  const float sign = fabsf(off[ax]) <= eps || off[ax] >= 0.0f ? 1.0f : -1.0f;
  F3 out{0.0f, 0.0f, 0.0f};
  if (ax == 0) out.x = sign;
  else if (ax == 1) out.y = sign;
  else out.z = sign;
  return {-clear[ax], out};
}

__device__ Surface cylinder_surface(F3 p, const DeviceConstraint& cy, float eps) {
  const F3 d{p.x - cy.a[0], p.y - cy.a[1], 0.0f};
  const float rd = norm(d);
  const F3 radial = rd > eps ? d * (1.0f / rd) : F3{1.0f, 0.0f, 0.0f};
  const float zo = p.z - cy.a[2];
  const float zs = zo >= 0.0f ? 1.0f : -1.0f;
  const F3 axial{0.0f, 0.0f, zs};
  const float re = rd - cy.radius;
  const float ae = fabsf(zo) - cy.half_height;
  if (re > 0.0f && ae > 0.0f) {
    const float dist = __fsqrt_rn((re * re) + (ae * ae));
    return {dist, (radial * re + axial * ae) * (1.0f / dist)};
  }
  if (re > 0.0f) return {re, radial};
  if (ae > 0.0f) return {ae, axial};
  if (-re <= -ae) return {re, radial};
  return {ae, axial};
}

struct Minimum {
  F3 point;
  Surface surface;
};

template <typename F>
__device__ Minimum minimize_on_segment(F3 s, F3 e, const F& at) {
  const F3 d = e - s;
  float lo = 0.0f, hi = 1.0f;
  for (int it = 0; it < 40; ++it) {
    const float u = lo + (hi - lo) / 3.0f;
    const float v = hi - (hi - lo) / 3.0f;
    const Surface fu = at(s + d * u);
    const Surface fv = at(s + d * v);
    if (fu.distance < fv.distance) {
      hi = v;
    } else if (fv.distance < fu.distance) {
      lo = u;
    } else {
      lo = u;
      hi = v;
    }
  }
  Minimum best{s, at(s)};
  const float probes[5] = {1.0f, 0.5f, lo, (lo + hi) * 0.5f, hi};
  for (int k = 0; k < 5; ++k) {
    const F3 p = s + d * probes[k];
    const Surface f = at(p);
    if (f.distance < best.surface.distance) best = {p, f};
  }
  return best;
}

__device__ void outside_rows(WallEmitter& em, const DeviceConstraint& c, float r, const F3 ends[2],
                             const Surface surf[2], const Minimum& m, float margin, float eps) {
  if (m.surface.distance - r >= margin) return;
  const float nearest = smin(surf[0].distance, surf[1].distance);
  const bool at_end = nearest - m.surface.distance <= eps;
  std::uint32_t loc[2];
  F3 pts[2];
  Surface fs[2];
  int count = 0;
  for (int k = 0; at_end && k < 2; ++k) {
    if (surf[k].distance - r < margin) {
      loc[count] = std::uint32_t(k);
      pts[count] = ends[k];
      fs[count] = surf[k];
      ++count;
    }
  }
  if (count == 0) {
    loc[0] = MSB_ROD_INTERIOR;
    pts[0] = m.point;
    fs[0] = m.surface;
    count = 1;
  }
  const float weight = c.coefficient * (count == 2 ? 0.7071067811865475f : 1.0f);
  for (int k = 0; k < count; ++k) {
    const F3 n = fs[k].outward * -1.0f;
    em.emit(c, loc[k], pts[k] + n * r, n, fs[k].distance - r, weight);
  }
}

__device__ void inside_rows(WallEmitter& em, const DeviceConstraint& c, float r, const F3 ends[2],
                            const Surface surf[2], float margin) {
  float sep[2];
  bool active[2];
  for (int k = 0; k < 2; ++k) {
    sep[k] = -surf[k].distance - r;
    active[k] = sep[k] < margin;
  }
  const unsigned n_active = unsigned(active[0]) + unsigned(active[1]);
  const float weight = c.coefficient * (n_active == 2 ? 0.7071067811865475f : 1.0f);
  for (int k = 0; k < 2; ++k) {
    if (!active[k]) continue;
    em.emit(c, std::uint32_t(k), ends[k] + surf[k].outward * r, surf[k].outward, sep[k], weight);
  }
}

__device__ void constraint_rows(WallEmitter& em, const DeviceConstraint& c, const Capsule& cap, float margin,
                                float eps, bool every_face) {
  const float h = cap.len * 0.5f;
  const F3 ends[2] = {cap.c - cap.a * h, cap.c + cap.a * h};
  const float r = cap.r;
  switch (c.kind) {
    case MSB_CONSTRAINT_PLANE: {
      float sep[2];
      bool active[2];
      for (int k = 0; k < 2; ++k) {
        sep[k] = dot(ends[k] - ca(c), cb(c)) - r;
        active[k] = sep[k] < margin;
      }
      const unsigned n_active = unsigned(active[0]) + unsigned(active[1]);
      const float weight = c.coefficient * (n_active == 2 ? 0.7071067811865475f : 1.0f);
      const F3 n = cb(c) * -1.0f;
      for (int k = 0; k < 2; ++k) {
        if (active[k]) em.emit(c, std::uint32_t(k), ends[k] + n * r, n, sep[k], weight);
      }
      return;
    }
    case MSB_CONSTRAINT_SPHERE: {
      Surface surf[2];
      for (int k = 0; k < 2; ++k) {
        const F3 cd = ends[k] - ca(c);
        const float dist = norm(cd);
        const F3 radial = dist > eps ? cd * (1.0f / dist) : F3{1.0f, 0.0f, 0.0f};
        surf[k] = {dist - c.radius, radial};
      }
      if (c.region == MSB_REGION_OUTSIDE) {
        const F3 st = ends[0];
        const F3 d = ends[1] - st;
        const float lsq = dot(d, d);
        const float t = lsq > eps * eps ? sclamp(-dot(st - ca(c), d) / lsq, 0.0f, 1.0f) : 0.0f;
        const F3 p = st + d * t;
        const F3 cd = p - ca(c);
        const float dist = norm(cd);
        const F3 radial = dist > eps ? cd * (1.0f / dist) : F3{1.0f, 0.0f, 0.0f};
        outside_rows(em, c, r, ends, surf, Minimum{p, {dist - c.radius, radial}}, margin, eps);
        return;
      }
      inside_rows(em, c, r, ends, surf, margin);
      return;
    }
    case MSB_CONSTRAINT_BOX: {
      if (every_face && c.region == MSB_REGION_INSIDE) {
        for (int k = 0; k < 2; ++k) {
          const F3 d = ends[k] - ca(c);
          const float off[3] = {d.x, d.y, d.z};
          for (int ax = 0; ax < 3; ++ax) {
            for (int s = 0; s < 2; ++s) {
              const float sign = s == 0 ? -1.0f : 1.0f;
              const float sep = c.b[ax] - sign * off[ax] - r;
              if (sep >= margin) continue;
              F3 n{0.0f, 0.0f, 0.0f};
              if (ax == 0) n.x = sign;
              else if (ax == 1) n.y = sign;
              else n.z = sign;
              em.emit(c, std::uint32_t(k), ends[k] + n * r, n, sep, c.coefficient);
            }
          }
        }
        return;
      }
      Surface surf[2];
      for (int k = 0; k < 2; ++k) surf[k] = box_surface(ends[k], c, eps);
      if (c.region == MSB_REGION_OUTSIDE) {
        const float reach = r + margin;
        const F3 lo{c.a[0] - c.b[0] - reach, c.a[1] - c.b[1] - reach, c.a[2] - c.b[2] - reach};
        const F3 hi{c.a[0] + c.b[0] + reach, c.a[1] + c.b[1] + reach, c.a[2] + c.b[2] + reach};
        if (!segment_hits_box(ends[0], ends[1], lo, hi)) return;
        const Minimum m = minimize_on_segment(ends[0], ends[1], [&](F3 p) { return box_surface(p, c, eps); });
        outside_rows(em, c, r, ends, surf, m, margin, eps);
        return;
      }
      inside_rows(em, c, r, ends, surf, margin);
      return;
    }
    case MSB_CONSTRAINT_CYLINDER: {
      if (every_face && c.region == MSB_REGION_INSIDE) {
        for (int k = 0; k < 2; ++k) {
          const F3 rdel{ends[k].x - c.a[0], ends[k].y - c.a[1], 0.0f};
          const float rd = norm(rdel);
          const F3 radial = rd > eps ? rdel * (1.0f / rd) : F3{1.0f, 0.0f, 0.0f};
          const float sep = c.radius - rd - r;
          if (sep < margin) em.emit(c, std::uint32_t(k), ends[k] + radial * r, radial, sep, c.coefficient);
          const float zo = ends[k].z - c.a[2];
          for (int s = 0; s < 2; ++s) {
            const float sign = s == 0 ? -1.0f : 1.0f;
            const F3 n{0.0f, 0.0f, sign};
            const float zsep = c.half_height - sign * zo - r;
            if (zsep < margin) em.emit(c, std::uint32_t(k), ends[k] + n * r, n, zsep, c.coefficient);
          }
        }
        return;
      }
      Surface surf[2];
      for (int k = 0; k < 2; ++k) surf[k] = cylinder_surface(ends[k], c, eps);
      if (c.region == MSB_REGION_OUTSIDE) {
        const float reach = r + margin;
        const F3 lo{c.a[0] - c.radius - reach, c.a[1] - c.radius - reach, c.a[2] - c.half_height - reach};
        const F3 hi{c.a[0] + c.radius + reach, c.a[1] + c.radius + reach, c.a[2] + c.half_height + reach};
        if (!segment_hits_box(ends[0], ends[1], lo, hi)) return;
        const F3 st = ends[0];
        const F3 d = ends[1] - st;
        auto at = [&](F3 p) { return cylinder_surface(p, c, eps); };
        Minimum m = minimize_on_segment(st, ends[1], at);
        auto consider = [&](float t) {
          const F3 p = st + d * sclamp(t, 0.0f, 1.0f);
          const Surface f = at(p);
          if (f.distance <= m.surface.distance) m = {p, f};
        };
        if (fabsf(d.z) > eps) consider((c.a[2] - st.z) / d.z);
        const float rl = d.x * d.x + d.y * d.y;
        if (rl > eps * eps) consider(-((st.x - c.a[0]) * d.x + (st.y - c.a[1]) * d.y) / rl);
        outside_rows(em, c, r, ends, surf, m, margin, eps);
        return;
      }
      inside_rows(em, c, r, ends, surf, margin);
      return;
    }
  }
}

__global__ void wall_contacts_kernel(GeometryView g, const DeviceConstraint* __restrict__ constraints,
                                     std::uint32_t constraint_count, float margin, float eps,
                                     std::uint32_t every_face, const std::uint32_t* __restrict__ rank,
                                     std::uint32_t* __restrict__ counts, const std::uint32_t* __restrict__ offsets,
                                     Touch* __restrict__ touches) {
  for (std::uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < g.count; s += gridDim.x * blockDim.x) {
    const Capsule cap = capsule_at(g, s);
    WallEmitter em{touches != nullptr ? touches + offsets[rank[s]] : nullptr, 0, s};
    for (std::uint32_t k = 0; k < constraint_count; ++k) {
      constraint_rows(em, constraints[k], cap, margin, eps, every_face != 0);
    }
    if (touches == nullptr) counts[rank[s]] = em.count;
  }
}

// ------------------------------------------------------ output records

__global__ void to_cell_contacts_kernel(const Touch* __restrict__ t, std::uint64_t count,
                                        const std::uint64_t* __restrict__ ids, msb_cell_contact* __restrict__ out) {
  for (std::uint64_t k = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; k < count;
       k += std::uint64_t(gridDim.x) * blockDim.x) {
    const Touch x = t[k];
    msb_cell_contact c;
    c.first_id = ids[x.s1];
    c.second_id = ids[x.s2];
    c.first_slot = x.s1;
    c.second_slot = x.s2;
    c.ordinal = x.tag;
    c.point_on_first = {x.point[0], x.point[1], x.point[2]};
    c.normal = {x.normal[0], x.normal[1], x.normal[2]};
    c.signed_separation = x.sep;
    c.weight = x.weight;
    c.reserved = 0;
    out[k] = c;
  }
}

__global__ void to_external_contacts_kernel(const Touch* __restrict__ t, std::uint64_t count,
                                            const std::uint64_t* __restrict__ ids,
                                            msb_external_contact* __restrict__ out) {
  for (std::uint64_t k = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; k < count;
       k += std::uint64_t(gridDim.x) * blockDim.x) {
    const Touch x = t[k];
    msb_external_contact c;
    c.cell_id = ids[x.s1];
    c.constraint_id = x.partner;
    c.cell_slot = x.s1;
    c.constraint_kind = x.kind;
    c.location = x.tag;
    c.point_on_cell = {x.point[0], x.point[1], x.point[2]};
    c.normal = {x.normal[0], x.normal[1], x.normal[2]};
    c.signed_separation = x.sep;
    c.weight = x.weight;
    c.reserved = 0;
    out[k] = c;
  }
}

// ------------------------------------------------------------ id order

__global__ void id_words_kernel(const std::uint64_t* __restrict__ ids, std::uint32_t cells, int shift,
                                const std::uint32_t* __restrict__ order, std::uint32_t* __restrict__ keys) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += gridDim.x * blockDim.x) {
    const std::uint32_t slot = order != nullptr ? order[i] : i;
    keys[i] = std::uint32_t(ids[slot] >> shift);
  }
}

__global__ void invert_kernel(const std::uint32_t* __restrict__ order, std::uint32_t cells,
                              std::uint32_t* __restrict__ rank) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += gridDim.x * blockDim.x) {
    rank[order[i]] = i;
  }
}

__global__ void unique_ids_kernel(const std::uint64_t* __restrict__ ids, const std::uint32_t* __restrict__ order,
                                  std::uint32_t cells, std::uint32_t* status) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += gridDim.x * blockDim.x) {
    const std::uint64_t id = ids[order[i]];
    if (id == 0 || (i > 0 && ids[order[i - 1]] == id)) raise_status(status, kStatusIndex);
  }
}

__global__ void max_u64_kernel(const std::uint64_t* __restrict__ values, std::uint32_t count,
                               unsigned long long* result) {
  unsigned long long local = 0;
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    local = values[i] > local ? values[i] : local;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_down_sync(0xFFFFFFFFu, local, o);
    local = other > local ? other : local;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(result, local);
}

}  // namespace

std::uint64_t grid_bucket_capacity(std::uint32_t cells) {
  std::uint64_t table = 1;
  while (table < 2ull * cells) table <<= 1;
  const std::uint64_t dense = 8ull * cells + 4096ull;
  return (dense > table ? dense : table) + 1;
}

std::uint32_t bound_partials(std::uint32_t cells) { return std::uint32_t(grid_for(cells, kThreads, 4)); }

void launch_cell_bounds(GeometryView g, float margin, double* bounds, double* partials, cudaStream_t stream) {
  cell_bounds_kernel<<<bound_partials(g.count), kThreads, 0, stream>>>(g, margin, bounds, partials);
  count_launch();
}

void launch_grid_setup(const double* partials, std::uint32_t partial_count, std::uint32_t cells,
                       std::uint64_t bucket_capacity, GridParams* grid, cudaStream_t stream, float box_scale,
                       std::uint32_t colonies) {
  grid_setup_kernel<<<1, kThreads, 0, stream>>>(partials, partial_count, cells, bucket_capacity, grid,
                                                double(box_scale), colonies);
  count_launch();
}

void launch_bin_cells(GeometryView g, const double* bounds, const GridParams* grid, std::uint32_t* cell_bucket,
                      std::int64_t* cell_coords, std::uint32_t* bucket_counts, cudaStream_t stream) {
  bin_cells_kernel<<<grid_for(g.count, kThreads), kThreads, 0, stream>>>(g, bounds, grid, cell_bucket, cell_coords,
                                                                          bucket_counts);
  count_launch();
}

void launch_scatter_cells(GeometryView g, const double* bounds, const std::uint32_t* cell_bucket,
                          const std::uint32_t* bucket_starts, std::uint32_t* bucket_fill, float4* sorted_lo,
                          float4* sorted_hi, std::uint64_t* sorted_id, cudaStream_t stream) {
  scatter_cells_kernel<<<grid_for(g.count, kThreads), kThreads, 0, stream>>>(g, bounds, cell_bucket, bucket_starts,
                                                                              bucket_fill, sorted_lo, sorted_hi,
                                                                              sorted_id);
  count_launch();
}

void launch_broad_phase(GeometryView g, const double* bounds, const GridParams* grid,
                        const std::uint32_t* bucket_starts, const float4* sorted_lo, const float4* sorted_hi,
                        const std::uint64_t* sorted_id, const std::int64_t* cell_coords, const std::uint32_t* rank,
                        std::uint32_t* counts, const std::uint32_t* offsets, uint2* pairs, std::uint32_t* status,
                        cudaStream_t stream, std::uint32_t* slab) {
  broad_phase_kernel<<<grid_for(g.count, 128, 16), 128, 0, stream>>>(g, bounds, grid, bucket_starts, sorted_lo,
                                                                      sorted_hi, sorted_id, cell_coords, rank, counts,
                                                                      offsets, pairs, slab, status);
  count_launch();
}

void launch_compact_slab(std::uint32_t n, const std::uint32_t* counts, const std::uint32_t* offsets,
                         const std::uint32_t* order, const std::uint32_t* slab, uint2* pairs, cudaStream_t stream) {
  if (n == 0) return;
  const std::uint64_t total = std::uint64_t(n) * kLocalPartners;
  compact_slab_kernel<<<grid_for(total, 256), 256, 0, stream>>>(n, counts, offsets, order, slab, pairs);
  count_launch();
}

void launch_narrow_phase(GeometryView g, const uint2* pairs, std::uint64_t pair_count, ContactSearchParams p,
                         std::uint32_t* counts, const std::uint32_t* offsets, Touch* touches, cudaStream_t stream,
                         std::uint32_t* status) {
  if (pair_count == 0) return;
  narrow_phase_kernel<<<grid_for(pair_count, kThreads, 16), kThreads, 0, stream>>>(g, pairs, pair_count, p, counts,
                                                                                    offsets, touches, status);
  count_launch();
}

void launch_wall_contacts(GeometryView g, const DeviceConstraint* constraints, std::uint32_t constraint_count,
                          float margin, float epsilon, std::uint32_t every_face, const std::uint32_t* rank,
                          std::uint32_t* counts, const std::uint32_t* offsets, Touch* touches, cudaStream_t stream) {
  wall_contacts_kernel<<<grid_for(g.count, 128, 16), 128, 0, stream>>>(g, constraints, constraint_count, margin,
                                                                        epsilon, every_face, rank, counts, offsets,
                                                                        touches);
  count_launch();
}

void launch_touches_to_cell_contacts(const Touch* touches, std::uint64_t count, const std::uint64_t* ids, void* out,
                                     cudaStream_t stream) {
  if (count == 0) return;
  to_cell_contacts_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(
      touches, count, ids, static_cast<msb_cell_contact*>(out));
  count_launch();
}

void launch_touches_to_external_contacts(const Touch* touches, std::uint64_t count, const std::uint64_t* ids,
                                         void* out, cudaStream_t stream) {
  if (count == 0) return;
  to_external_contacts_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(
      touches, count, ids, static_cast<msb_external_contact*>(out));
  count_launch();
}

void launch_id_low_words(const std::uint64_t* ids, std::uint32_t cells, int shift, const std::uint32_t* order,
                         std::uint32_t* keys, cudaStream_t stream) {
  id_words_kernel<<<grid_for(cells, kThreads), kThreads, 0, stream>>>(ids, cells, shift, order, keys);
  count_launch();
}

void launch_invert_permutation(const std::uint32_t* order, std::uint32_t cells, std::uint32_t* rank,
                               cudaStream_t stream) {
  invert_kernel<<<grid_for(cells, kThreads), kThreads, 0, stream>>>(order, cells, rank);
  count_launch();
}

void launch_check_unique_ids(const std::uint64_t* ids, const std::uint32_t* order, std::uint32_t cells,
                             std::uint32_t* status, cudaStream_t stream) {
  unique_ids_kernel<<<grid_for(cells, kThreads), kThreads, 0, stream>>>(ids, order, cells, status);
  count_launch();
}

void launch_max_u64(const std::uint64_t* values, std::uint32_t count, std::uint64_t* result, cudaStream_t stream) {
  max_u64_kernel<<<grid_for(count, kThreads), kThreads, 0, stream>>>(values, count,
                                                                      reinterpret_cast<unsigned long long*>(result));
  count_launch();
}


void launch_fast_cells(GeometryView from, GeometryView to, double allowance, std::uint32_t* fast, std::uint32_t* list,
                       std::uint32_t* count, cudaStream_t stream) {
  if (to.count == 0) return;
  fast_cells_kernel<<<grid_for(to.count, kThreads), kThreads, 0, stream>>>(from, to, allowance, fast, list, count);
  count_launch();
}

void launch_fast_partners(GeometryView g, const double* bounds, const GridParams* grid,
                          const std::uint32_t* bucket_starts, const float4* sorted_lo, const float4* sorted_hi,
                          const std::uint64_t* sorted_id, const std::int64_t* cell_coords, const std::uint32_t* fast,
                          const std::uint32_t* list, const std::uint32_t* fast_count, std::uint32_t cap,
                          const uint2* kept, const std::uint32_t* kept_offsets, const std::uint32_t* rank,
                          std::uint32_t* counts, const std::uint32_t* offsets, uint2* pairs, cudaStream_t stream) {
  if (cap == 0) return;
  fast_partners_kernel<<<grid_for(cap, 128, 16), 128, 0, stream>>>(g, bounds, grid, bucket_starts, sorted_lo, sorted_hi,
                                                                   sorted_id, cell_coords, fast, list, fast_count, cap,
                                                                   kept, kept_offsets, rank, counts, offsets, pairs);
  count_launch();
}

void launch_merge_fast_pairs(const uint2* fast_pairs, std::uint32_t fast_pair_count, uint2* sorted_fast,
                             const uint2* kept, std::uint32_t kept_count, const std::uint64_t* ids,
                             std::uint32_t* shift, std::uint32_t* shift_scan, std::uint32_t* temp, uint2* merged,
                             cudaStream_t stream) {
  // Every place of the merged list is written below; zeroed first so that
  // no place can ever hold anything but a valid slot pair.
  cudaMemsetAsync(merged, 0, (std::uint64_t(kept_count) + fast_pair_count) * sizeof(uint2), stream);
  cudaMemsetAsync(shift, 0, (kept_count + 1ull) * sizeof(std::uint32_t), stream);
  if (fast_pair_count > 0) {
    sort_fast_pairs_kernel<<<grid_for(fast_pair_count, 128), 128, 0, stream>>>(fast_pairs, fast_pair_count, ids,
                                                                             sorted_fast);
    place_fast_pairs_kernel<<<grid_for(fast_pair_count, 128), 128, 0, stream>>>(sorted_fast, fast_pair_count, kept,
                                                                              kept_count, ids, merged, shift);
    count_launch(2);
  }
  exclusive_scan(shift, shift_scan, kept_count + 1ull, temp, stream);
  place_kept_pairs_kernel<<<grid_for(kept_count, kThreads), kThreads, 0, stream>>>(kept, kept_count, shift_scan, merged);
  count_launch();
}

}  // namespace msb
