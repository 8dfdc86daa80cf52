// The batched contact solve (see batch.h).  The arithmetic of each pass is
// the single-system solve's (solve_math.cuh): a colony relaxed here follows
// the same iteration as it would alone, up to the order of the FP64 sums of
// the BB products, which here are reduced per CTA in a fixed tree and then
// across the cluster's CTAs in rank order.
#include "batch.h"

#include <cooperative_groups.h>

#include "device.cuh"
#include "kernels.h"
#include "solve_math.cuh"

namespace cg = cooperative_groups;

namespace msb {
namespace {

// Response of the colony's bodies to its (projected, with project)
// multipliers; each thread keeps kBatch entries' gathers in flight.  Inside
// the iterations each row's multiplier and gap come as one float2 (the
// iterate), one gather instead of two: the 256-colony sweep's solve phase
// measured 40.6-41.1 -> 39.1 ms per step, the same iterations and bits.
template <int kBatch>
__device__ void colony_body_pass(const BatchDesc& d, std::uint32_t b0, std::uint32_t b1, std::uint32_t tid,
                                 std::uint32_t stride, bool project, float alpha) {
  const float* g = d.multipliers;
  for (std::uint32_t b = b0 + tid; b < b1; b += stride) {
    float w[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    float load = 0.0f;
    const std::uint32_t begin = d.incidence.offsets[b];
    const std::uint32_t end = d.incidence.offsets[b + 1];
    for (std::uint32_t k0 = begin; k0 < end; k0 += kBatch) {
      float4 ea[kBatch], eb[kBatch];
      float gv[kBatch], pv[kBatch];
#pragma unroll
      for (int t = 0; t < kBatch; ++t) {
        if (k0 + t < end) {
          ea[t] = __ldcs(&d.incidence.a[k0 + t]);
          eb[t] = __ldcs(&d.incidence.b[k0 + t]);
        }
      }
#pragma unroll
      for (int t = 0; t < kBatch; ++t) {
        if (k0 + t < end) {
          const std::uint32_t row = __float_as_uint(eb[t].w) >> 1;  // side bits: row << 1 | side
          if (project) {
            const float2 q = __ldcg(&d.iterate[row]);  // (multiplier, gap) in one gather
            gv[t] = q.x;
            pv[t] = q.y;
          } else {
            gv[t] = __ldcg(&g[row]);
            pv[t] = 0.0f;
          }
        }
      }
#pragma unroll
      for (int t = 0; t < kBatch; ++t) {
        if (k0 + t < end) {
          const float m = project ? smax(0.0f, gv[t] - alpha * pv[t]) : gv[t];
          if (m == 0.0f) continue;
          w[0] += m * ea[t].x;
          w[1] += m * ea[t].y;
          w[2] += m * ea[t].z;
          w[3] += m * ea[t].w;
          w[4] += m * eb[t].x;
          w[5] += m * eb[t].y;
          load += eb[t].z * m;
        }
      }
    }
    float v[6];
    float rate;
    respond(d, b, w, load, v, rate);
    __stcg(&d.response.a[b], make_float4(v[0], v[1], v[2], rate));
    __stcg(&d.response.b[b], make_float4(v[3], v[4], v[5], load));
  }
}

struct Sums {
  double ss, sy, yy;
  float residual;
  bool finite;
};

// Gaps of the colony's rows (and, with project, one projected step with its
// BB products), written with the rows' multipliers into the iterate; the
// initial pass reads the multipliers array, the projected ones the iterate.
__device__ Sums colony_row_pass(const BatchDesc& d, std::uint32_t r0, std::uint32_t r1, std::uint32_t tid,
                                std::uint32_t stride, bool project, float alpha) {
  Sums s{0.0, 0.0, 0.0, 0.0f, true};
  const float dt = d.dt;
  for (std::uint32_t j = r0 + tid; j < r1; j += stride) {
    const std::uint32_t i = d.colony_rows[j];
    float gi, gpi = 0.0f;
    if (project) {
      const float2 q = __ldcg(&d.iterate[i]);
      gi = q.x;
      gpi = q.y;
    } else {
      gi = __ldcg(&d.multipliers[i]);
    }
    const uint2 sl = __ldcs(&d.rows.slots[i]);
    const float4 ra = __ldcs(&d.rows.a[i]);
    const float4 rb = __ldcs(&d.rows.b[i]);
    const float4 rd = __ldcs(&d.rows.d[i]);
    const float4 va = __ldcg(&d.response.a[sl.x]);
    const float4 vb = __ldcg(&d.response.b[sl.x]);
    const float m = project ? smax(0.0f, gi - alpha * gpi) : gi;
    const float v1[6] = {va.x, va.y, va.z, vb.x, vb.y, vb.z};
    float rate = side_term(ra, rb, v1, va.w);
    if (sl.y != kInvalidSlot) {
      const float4 rc = __ldcs(&d.rows.c[i]);
      const float4 wa = __ldcg(&d.response.a[sl.y]);
      const float4 wb = __ldcg(&d.response.b[sl.y]);
      const float v2[6] = {wa.x, wa.y, wa.z, wb.x, wb.y, wb.z};
      rate += side_term(rc, rd, v2, wa.w);
    }
    const float gn = rb.w + dt * rate + rd.w * m;
    s.residual = smax(s.residual, row_residual(m, gn));
    s.finite = s.finite && isfinite(gn);
    if (project) {
      const double moved = double(m) - double(gi);
      const double change = double(gn) - double(gpi);
      s.ss += moved * moved;
      s.sy += moved * change;
      s.yy += change * change;
    }
    __stcg(&d.iterate[i], make_float2(m, gn));
  }
  return s;
}

// Block reduction in a fixed tree of 5 values: sums (0..2), max (3), min (4).
template <int Threads>
__device__ void block_reduce(double (&v)[5], double (&red)[5][Threads / 32], double* out) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_down_sync(0xFFFFFFFFu, v[k], o);
      v[k] = k < 3 ? v[k] + other : (k == 3 ? fmax(v[k], other) : fmin(v[k], other));
    }
    if (lane == 0) red[k][warp] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    const int k = threadIdx.x;
    double r = red[k][0];
    for (int w = 1; w < Threads / 32; ++w) r = k < 3 ? r + red[k][w] : (k == 3 ? fmax(r, red[k][w]) : fmin(r, red[k][w]));
    out[k] = r;
  }
}

// Two forms, picked by the autotuner: Lean = false keeps 4 incidence
// entries' gathers in flight per thread (128 registers); Lean = true one
// (64 registers), for twice the resident warps.
template <int Threads, bool Lean>
__global__ void __launch_bounds__(Threads, Lean ? 1024 / Threads : 1) batch_solve_kernel(BatchDesc d) {
  constexpr int kBatch = Lean ? 1 : 4;
  cg::cluster_group cluster = cg::this_cluster();
  const std::uint32_t rank = cluster.block_rank();
  const std::uint32_t size = cluster.num_blocks();
  __shared__ double red[5][Threads / 32];
  __shared__ double part[6];  // this CTA's reduced values (5) and its diagonal bound
  __shared__ std::uint32_t claimed;
  __shared__ float bound_part;
  const std::uint32_t tid = rank * Threads + threadIdx.x;
  const std::uint32_t stride = size * Threads;

  for (;;) {
    if (rank == 0 && threadIdx.x == 0) claimed = atomicAdd(d.next, 1u);
    cluster.sync();
    const std::uint32_t slot = *cluster.map_shared_rank(&claimed, 0);
    // Every CTA has read rank 0's claim before rank 0 exits (its shared
    // memory must outlive every remote read) or claims again.
    cluster.sync();
    if (slot >= d.colonies) break;
    const std::uint32_t colony = d.order[slot];
    if (d.active != nullptr && d.active[colony] == 0u) {
      if (rank == 0 && threadIdx.x == 0) d.state[colony].iterations = 0;
      continue;
    }
    const std::uint32_t r0 = d.row_offsets[colony], r1 = d.row_offsets[colony + 1];
    const std::uint32_t b0 = d.cell_offsets[colony], b1 = d.cell_offsets[colony + 1];
    const float tolerance = d.tolerance[colony];

    // contact_system_diagonal_bound over the colony's rows.
    float bound = 0.0f;
    for (std::uint32_t j = r0 + tid; j < r1; j += stride) {
      const std::uint32_t i = d.colony_rows[j];
      const uint2 s = d.rows.slots[i];
      const float4 rd = d.rows.d[i];
      float entry = diagonal(d.rows.a[i], d.rows.b[i], d.bodies.a[s.x], d.bodies.b[s.x]);
      if (s.y != kInvalidSlot) entry += diagonal(d.rows.c[i], rd, d.bodies.a[s.y], d.bodies.b[s.y]);
      bound = smax(bound, d.dt * entry + rd.w);
    }
    for (int o = 16; o > 0; o >>= 1) bound = smax(bound, __shfl_down_sync(0xFFFFFFFFu, bound, o));
    if (threadIdx.x == 0) bound_part = 0.0f;
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && bound > 0.0f) atomicMax(reinterpret_cast<unsigned*>(&bound_part), __float_as_uint(bound));

    // Mode 0: the response and gaps of the initial multipliers.
    colony_body_pass<kBatch>(d, b0, b1, tid, stride, false, 0.0f);
    __threadfence();
    cluster.sync();
    Sums s = colony_row_pass(d, r0, r1, tid, stride, false, 0.0f);
    double v[5] = {0.0, 0.0, 0.0, double(s.residual), s.finite ? 1.0 : 0.0};
    block_reduce<Threads>(v, red, part);
    if (threadIdx.x == 0) part[5] = double(bound_part);
    __threadfence();
    cluster.sync();

    // Every CTA's thread 0 reads all ranks' partials in rank order and takes
    // the same decision (the same reads in the same order), so no CTA waits
    // for another's decision: two cluster barriers per iteration.
    __shared__ float step_s;
    __shared__ std::uint32_t proceed_s;
    float step = 0.0f, residual = 0.0f, colony_bound = 0.0f;
    std::uint32_t iterations = 0, status = MSB_SOLVE_ITERATION_LIMIT;
    if (threadIdx.x == 0) {
      double total_residual = 0.0, finite = 1.0, b = 0.0;
      for (std::uint32_t r = 0; r < size; ++r) {
        const double* p = cluster.map_shared_rank(part, r);
        total_residual = fmax(total_residual, p[3]);
        finite = fmin(finite, p[4]);
        b = fmax(b, p[5]);
      }
      colony_bound = float(b);
      residual = finite > 0.5 ? float(total_residual) : __int_as_float(0x7FC00000);
      std::uint32_t proceed = 0;
      if (!isfinite(colony_bound) || !(colony_bound > 0.0f)) {
        status = r1 > r0 ? 3u : std::uint32_t(MSB_SOLVE_CONVERGED);
        if (r1 == r0) residual = 0.0f;
      } else if (!isfinite(residual)) {
        status = MSB_SOLVE_BREAKDOWN;
      } else if (residual <= tolerance) {
        status = MSB_SOLVE_CONVERGED;
      } else {
        status = MSB_SOLVE_ITERATION_LIMIT;
        step = 1.0f / colony_bound;
        proceed = d.max_iterations > 0 ? 1u : 0u;
      }
      step_s = step;
      proceed_s = proceed;
    }
    __syncthreads();

    while (proceed_s != 0) {
      const float alpha = step_s;
      colony_body_pass<kBatch>(d, b0, b1, tid, stride, true, alpha);
      __threadfence();
      cluster.sync();
      s = colony_row_pass(d, r0, r1, tid, stride, true, alpha);
      double w[5] = {s.ss, s.sy, s.yy, double(s.residual), s.finite ? 1.0 : 0.0};
      block_reduce<Threads>(w, red, part);
      __threadfence();
      cluster.sync();
      if (threadIdx.x == 0) {
        double t[5] = {0.0, 0.0, 0.0, 0.0, 1.0};
        for (std::uint32_t r = 0; r < size; ++r) {
          const double* p = cluster.map_shared_rank(part, r);
          t[0] += p[0];
          t[1] += p[1];
          t[2] += p[2];
          t[3] = fmax(t[3], p[3]);
          t[4] = fmin(t[4], p[4]);
        }
        iterations += 1;
        residual = t[4] > 0.5 ? float(t[3]) : __int_as_float(0x7FC00000);
        std::uint32_t proceed = 0;
        if (!isfinite(residual)) {
          status = MSB_SOLVE_BREAKDOWN;
        } else if (!(residual > tolerance)) {
          status = MSB_SOLVE_CONVERGED;
        } else {
          step = next_step(step, t[0], t[1], t[2], iterations);
          status = MSB_SOLVE_ITERATION_LIMIT;
          proceed = iterations < d.max_iterations ? 1u : 0u;
        }
        step_s = step;
        proceed_s = proceed;
      }
      __syncthreads();
    }
    // Each thread's rows of the last row pass back into the multiplier and
    // gap arrays.
    for (std::uint32_t j = r0 + tid; j < r1; j += stride) {
      const std::uint32_t i = d.colony_rows[j];
      const float2 q = __ldcg(&d.iterate[i]);
      d.multipliers[i] = q.x;
      d.gaps[i] = q.y;
    }
    if (rank == 0 && threadIdx.x == 0) d.state[colony] = {step, residual, colony_bound, iterations, status};
    // The next claim's two barriers order every remote read of this colony's
    // partials before any CTA writes them again or exits.
  }
}

template <int Threads, bool Lean>
void allow_wide_clusters();

template <int Threads, bool Lean>
cudaError_t launch_shape(const BatchDesc& desc, int cluster, int clusters, cudaStream_t stream) {
  if (cluster > 8) allow_wide_clusters<Threads, Lean>();
  cudaLaunchConfig_t config{};
  config.gridDim = dim3(unsigned(cluster * clusters));
  config.blockDim = dim3(Threads);
  config.dynamicSmemBytes = 0;
  config.stream = stream;
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeClusterDimension;
  attribute[0].val.clusterDim.x = unsigned(cluster);
  attribute[0].val.clusterDim.y = 1;
  attribute[0].val.clusterDim.z = 1;
  config.attrs = attribute;
  config.numAttrs = 1;
  return cudaLaunchKernelEx(&config, batch_solve_kernel<Threads, Lean>, desc);
}

// Clusters of 16 CTAs are beyond the portable size of 8 and must be allowed
// per kernel first.
template <int Threads, bool Lean>
void allow_wide_clusters() {
  cudaFuncSetAttribute(batch_solve_kernel<Threads, Lean>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

template <int Threads, bool Lean>
int resident_clusters(int cluster) {
  if (cluster > 8) allow_wide_clusters<Threads, Lean>();
  cudaLaunchConfig_t config{};
  config.gridDim = dim3(unsigned(cluster));
  config.blockDim = dim3(Threads);
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeClusterDimension;
  attribute[0].val.clusterDim.x = unsigned(cluster);
  attribute[0].val.clusterDim.y = 1;
  attribute[0].val.clusterDim.z = 1;
  config.attrs = attribute;
  config.numAttrs = 1;
  int count = 0;
  if (cudaOccupancyMaxActiveClusters(&count, batch_solve_kernel<Threads, Lean>, &config) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return count;
}

__global__ void colony_row_keys_kernel(const uint2* __restrict__ slots, std::uint32_t rows,
                                       const std::uint32_t* __restrict__ of_slot, std::uint32_t* __restrict__ keys,
                                       std::uint32_t* __restrict__ values, std::uint32_t* __restrict__ counts) {
  // Contiguous ranges per warp: rows in first-id order mostly share their
  // colony with their neighbours, so the counts are folded per warp.
  const WarpRange range = warp_range(rows);
  KeyCarry carry;
  for (std::uint32_t base = range.begin; base < range.end; base += 32) {
    const std::uint32_t i = base + (threadIdx.x & 31u);
    const bool live = i < range.end;
    std::uint32_t colony = 0u;
    if (live) {
      colony = of_slot[slots[i].x];
      keys[i] = colony;
      values[i] = i;
    }
    carry_item<true>(counts, carry, live, colony, 1u);
  }
  if ((threadIdx.x & 31u) == 0u) carry_flush<true>(counts, carry);
}

}  // namespace

int batch_resident_clusters(BatchShape shape) {
  if (shape.lean) {
    return shape.threads == 512 ? resident_clusters<512, true>(shape.cluster)
                                : resident_clusters<256, true>(shape.cluster);
  }
  return shape.threads == 512 ? resident_clusters<512, false>(shape.cluster)
                              : resident_clusters<256, false>(shape.cluster);
}

int launch_batch_solve(const BatchDesc& desc, BatchShape shape, int clusters, cudaStream_t stream) {
  if (clusters <= 0 || desc.colonies == 0) return int(cudaSuccess);
  cudaError_t e;
  if (shape.lean) {
    e = shape.threads == 512 ? launch_shape<512, true>(desc, shape.cluster, clusters, stream)
                             : launch_shape<256, true>(desc, shape.cluster, clusters, stream);
  } else {
    e = shape.threads == 512 ? launch_shape<512, false>(desc, shape.cluster, clusters, stream)
                             : launch_shape<256, false>(desc, shape.cluster, clusters, stream);
  }
  count_launch();
  return int(e);
}

void launch_colony_row_keys(const uint2* slots, std::uint32_t rows, const std::uint32_t* of_slot,
                            std::uint32_t* keys, std::uint32_t* values, std::uint32_t* counts, cudaStream_t stream) {
  if (rows == 0) return;
  colony_row_keys_kernel<<<grid_for(rows, 256), 256, 0, stream>>>(slots, rows, of_slot, keys, values, counts);
  count_launch();
}

}  // namespace msb
