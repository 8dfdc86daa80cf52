// Barzilai-Borwein projected gradient on the contact multipliers, resident on
// the device (cpp/core/contact_solver.hpp:44-120,
// cpp/cpu/cpu_contact_dynamics.cpp:40-338 of the reference).
//
// One iteration is two passes:
//   body pass  one thread per body sums its rows' projected multipliers
//              times their jacobians in row order (the reference's
//              incidence order, so a body's force and torque carry the same
//              bits), applies the mobility and the growth-load law, and
//              stores each of its rows' side terms of the gap rate;
//   row pass   one thread per row adds its two side terms into the new gap
//              and forms the FP64 BB products and the complementarity
//              residual; the last block to finish
//              combines the per-block partials in block order (so the result
//              does not depend on scheduling), sets the next step length and
//              the convergence flag, and writes the flag into the WHILE node
//              of the CUDA graph that repeats the two passes.
// The host launches the graph once per solve and reads the report once.  The
// WHILE body holds MSB_WHILE_UNROLL (body, row) pairs; a pair whose solve
// has already converged returns at once, so the result is that of one pair
// per evaluation.

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "device.cuh"
#include "kernels.h"
#include "solve.h"
#include "solve_math.cuh"
#include "../../include/msb200.h"

namespace msb {
namespace {

// Tuning constants of the BB passes: entries whose gathers one body-pass
// thread keeps in flight together, and the minimum resident blocks per SM
// the compiler must fit (which caps registers).
// (1M capsules, solve phase: 3 entries 20.5 ms, 4 entries 20.9 ms, 5
// entries spill at 64 registers, 27.4 ms.)
#ifndef MSB_BODY_BATCH
#define MSB_BODY_BATCH 3
#endif
#ifndef MSB_BODY_MIN_BLOCKS
#define MSB_BODY_MIN_BLOCKS 4
#endif
#ifndef MSB_ROW_MIN_BLOCKS
#define MSB_ROW_MIN_BLOCKS 1
#endif
// (body pass, row pass) pairs per WHILE-node body of the solve graph; a pair
// after the one that converged returns at once.  Fewer evaluations of the
// WHILE node: per BB iteration, 1 -> 8 pairs measured 116 -> 112 us at 1M
// capsules, 24.6 -> 21.0 us at 100k, 19.7 -> 16.0 us at 20k.
#ifndef MSB_WHILE_UNROLL
#define MSB_WHILE_UNROLL 8
#endif
#ifndef MSB_RELAX_MIN_BLOCKS
#define MSB_RELAX_MIN_BLOCKS 3
#endif
// Back-off of a barrier wait between polls (0: poll without sleeping).
#ifndef MSB_BARRIER_SLEEP_NS
#define MSB_BARRIER_SLEEP_NS 64
#endif
constexpr int kBatch = MSB_BODY_BATCH;


// One thread per body sums its rows' multipliers times their jacobians in
// entry order, which is row order: the products and the order of the sums
// are those of the reference's evaluate (cpp/cpu/cpu_contact_dynamics.cpp:116-146),
// so a body's force, torque and load carry the reference's bits.  The entries
// are read kBatch at a time and their multiplier gathers issued together, so
// that each thread keeps several independent loads in flight.
// The thread then forms, for each of its entries, that side's term of the
// row's gap rate (jacobian . velocity - lever * elongation rate, as row_gap
// forms it, cpp/cpu/cpu_contact_dynamics.cpp:149-159) and stores it in the
// row's side slot.  The row pass then adds a row's two terms instead of
// reading its jacobians again and gathering both bodies' responses.
// mode 0 and 2 evaluate the multipliers as they are, mode 1 their
// projection; mode 2 (an evaluation, not a solve) also writes the response.
// `Tag` only names a second instance of the same code for the timing hook,
// so that a profiler can select its launches apart from the solve graph's.
// Loads of data that other blocks write during a fused solve go through L2
// (ld.global.cg): L1 is not coherent across SMs within one launch.
// Two things shorten each thread's chain of dependent loads: the next body's
// entry range and this body's record are loaded before this body's entries,
// and the first batch of a body with more than one batch is kept in shared
// memory (one slot per thread, 24 KB a block) for the side terms, so that
// only the entries between it and the last batch are read again.  At 1M
// capsules this took the body pass from 83 to 78 us, the same bits; a
// stash of two batches (48 KB a block) was slower, 88 us, the L1 left to the
// gathers being smaller.
template <bool Coherent>
__device__ __forceinline__ float shared_load(const float* p) {
  if constexpr (Coherent) {
    return __ldcg(p);
  } else {
    return *p;
  }
}
template <bool Coherent>
__device__ __forceinline__ float2 shared_load(const float2* p) {
  if constexpr (Coherent) {
    return __ldcg(p);
  } else {
    return *p;
  }
}

// The body pass over bodies block, block + blocks, ... of the grid.
template <bool Coherent>
__device__ __forceinline__ void body_pass(const SolveDesc& d, std::uint32_t mode, float alpha, std::uint32_t block,
                                          std::uint32_t blocks, std::uint32_t* check) {
  const float* __restrict__ g = d.multipliers;
  const float2* __restrict__ iterate = d.iterate;
  const std::uint32_t* __restrict__ offsets = d.incidence.offsets;
  const float4* __restrict__ entry_a = d.incidence.a;
  const float4* __restrict__ entry_b = d.incidence.b;
  float* __restrict__ sides = reinterpret_cast<float*>(d.incidence.sides);
  constexpr int kStash = kBatch;  // entries kept per thread, a multiple of kBatch
  __shared__ float4 stash_a[kStash][kSolveThreads], stash_b[kStash][kSolveThreads];
  const std::uint32_t stride = blocks * blockDim.x;
  std::uint32_t next_begin = 0, next_end = 0;
  if (block * blockDim.x + threadIdx.x < d.body_count) {
    next_begin = offsets[block * blockDim.x + threadIdx.x];
    next_end = offsets[block * blockDim.x + threadIdx.x + 1];
  }
  for (std::uint32_t b = block * blockDim.x + threadIdx.x; b < d.body_count; b += stride) {
    float w[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    float load = 0.0f;
    const std::uint32_t begin = next_begin;
    std::uint32_t end = next_end;
    const float4 body_a = __ldcs(&d.bodies.a[b]);
    const float4 body_b = __ldcs(&d.bodies.b[b]);
    if (b + stride < d.body_count) {
      next_begin = offsets[b + stride];
      next_end = offsets[b + stride + 1];
    }
    if (!index_ok(end, std::uint64_t(2) * d.row_count + 1, check) || !index_ok(begin, std::uint64_t(end) + 1, check)) {
      end = begin;  // offsets out of range or not monotone: no entries
    }
    // The batch of entries read last stays in registers for the side terms.
    float4 ea[kBatch], eb[kBatch];
    std::uint32_t last = begin;
    for (std::uint32_t k0 = begin; k0 < end; k0 += kBatch) {
      last = k0;
      float gv[kBatch], pv[kBatch];
#pragma unroll
      for (int t = 0; t < kBatch; ++t) {
        if (k0 + t < end) {
          ea[t] = entry_a[k0 + t];
          eb[t] = entry_b[k0 + t];
        }
      }
      if (k0 + kBatch < end && k0 - begin < kStash) {
#pragma unroll
        for (int t = 0; t < kBatch; ++t) {
          stash_a[k0 - begin + t][threadIdx.x] = ea[t];
          stash_b[k0 - begin + t][threadIdx.x] = eb[t];
        }
      }
#pragma unroll
      for (int t = 0; t < kBatch; ++t) {
        if (k0 + t < end) {
          const std::uint32_t row = __float_as_uint(eb[t].w) >> 1;
          const bool ok = index_ok(row, d.row_count, check);
          if (mode == 2) {
            gv[t] = ok ? g[row] : 0.0f;
            pv[t] = 0.0f;
          } else {
            // One gather brings the row's multiplier and gap.
            const float2 q = ok ? shared_load<Coherent>(&iterate[row]) : make_float2(0.0f, 0.0f);
            gv[t] = q.x;
            pv[t] = mode == 1 ? q.y : 0.0f;
          }
        }
      }
#pragma unroll
      for (int t = 0; t < kBatch; ++t) {
        if (k0 + t < end) {
          const float m = mode == 1 ? smax(0.0f, gv[t] - alpha * pv[t]) : gv[t];
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
    respond(d, b, body_a, body_b, w, load, v, rate);
    if (mode == 2) {
      // An evaluation: the response is the result.  Inside a solve only
      // the side terms are needed; the solve ends with an evaluation of
      // its final multipliers.
      d.response.a[b] = make_float4(v[0], v[1], v[2], rate);
      d.response.b[b] = make_float4(v[3], v[4], v[5], load);
    }
    // Each entry's side term of its row's rate: the entries before the last
    // batch read again (a body with more than kBatch entries), then the
    // last batch from registers.
    const std::uint64_t side_count = std::uint64_t(2) * d.row_count;
    for (std::uint32_t k = begin; k < last; ++k) {
      float4 a0, b0;
      if (k - begin < kStash) {
        a0 = stash_a[k - begin][threadIdx.x];
        b0 = stash_b[k - begin][threadIdx.x];
      } else {
        a0 = __ldcs(&entry_a[k]);
        b0 = __ldcs(&entry_b[k]);
      }
      const std::uint32_t s0 = __float_as_uint(b0.w);
      if (index_ok(s0, side_count, check)) sides[s0] = side_term(a0, b0, v, rate);
    }
#pragma unroll
    for (int t = 0; t < kBatch; ++t) {
      if (last + t < end) {
        const std::uint32_t side = __float_as_uint(eb[t].w);
        if (index_ok(side, side_count, check)) sides[side] = side_term(ea[t], eb[t], v, rate);
      }
    }
  }
}

template <int Tag>
__global__ void __launch_bounds__(kSolveThreads, MSB_BODY_MIN_BLOCKS) body_pass_kernel(SolveDesc* desc, int fixed_mode) {
  const SolveDesc& d = *desc;
  const std::uint32_t mode = fixed_mode >= 0 ? std::uint32_t(fixed_mode) : d.mode;
  if (fixed_mode < 0 && mode == 1 && d.proceed == 0u) return;  // an unrolled pair after convergence
  body_pass<false>(d, mode, d.step, blockIdx.x, gridDim.x, &desc->check_status);
}

// The row pass over rows block, block + blocks, ... of the grid; unless
// mode is 2, the block's BB products, residual and finiteness into
// d.partials[5 * block ...], reduced in a fixed tree.
template <bool Coherent>
__device__ __forceinline__ void row_pass(const SolveDesc& d, std::uint32_t mode, float alpha, std::uint32_t block,
                                         std::uint32_t blocks, std::uint32_t* check) {
  const float dt = d.dt;
  const float* __restrict__ g = d.multipliers;
  float* __restrict__ gap = d.gaps;
  float2* __restrict__ iterate = d.iterate;
  const float2* __restrict__ sides = d.incidence.sides;
  const float2* __restrict__ constants = d.incidence.constants;
  double ss = 0.0, sy = 0.0, yy = 0.0;
  float residual = 0.0f;
  bool finite = true;
  (void)check;
  // row_gap (cpp/cpu/cpu_contact_dynamics.cpp:149-159): offset + dt * (first
  // side's term + second side's term) + compliance * multiplier.  The body
  // pass formed each side's term; a constraint row's second is -0.0f, and
  // x + -0.0f == x, so the sum is the reference's bit for bit.
  const bool project = mode == 1;
  for (std::uint32_t i = block * blockDim.x + threadIdx.x; i < d.row_count; i += blocks * blockDim.x) {
    // mode 2 (an evaluation) reads the multipliers; a solve its iterate.
    const float2 q = mode == 2 ? make_float2(g[i], 0.0f) : shared_load<Coherent>(&iterate[i]);
    const float gi = q.x;
    const float gpi = project ? q.y : 0.0f;
    const float2 side = shared_load<Coherent>(&sides[i]);
    const float2 k = __ldcs(&constants[i]);
    const float m = project ? smax(0.0f, gi - alpha * gpi) : gi;
    const float rate = side.x + side.y;
    const float gn = k.x + dt * rate + k.y * m;
    residual = smax(residual, row_residual(m, gn));
    finite = finite && isfinite(gn);
    if (project) {
      const double moved = double(m) - double(gi);
      const double change = double(gn) - double(gpi);
      ss += moved * moved;
      sy += moved * change;
      yy += change * change;
    }
    if (mode == 2) {
      gap[i] = gn;
    } else {
      iterate[i] = make_float2(m, gn);
    }
  }
  if (mode == 2) return;

  // Block reduction in a fixed tree.
  __shared__ double red[5][kSolveThreads / 32];
  double v[5] = {ss, sy, yy, double(residual), finite ? 1.0 : 0.0};
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
    for (int w = 1; w < kSolveThreads / 32; ++w) {
      r = k < 3 ? r + red[k][w] : (k == 3 ? fmax(r, red[k][w]) : fmin(r, red[k][w]));
    }
    d.partials[5 * block + k] = r;
  }
  __syncthreads();
}

// One block combines the partials of `blocks` blocks in block order (so the
// result does not depend on scheduling), sets the next step length, the
// status and whether to go on (d.proceed), as one iteration of
// iterate_contact_steps does (cpp/core/contact_solver.hpp:66-82); mode 0
// judges the initial multipliers.  Returns d.proceed (thread 0).
__device__ __forceinline__ std::uint32_t decide(SolveDesc& d, std::uint32_t mode, std::uint32_t blocks) {
  __shared__ double red[5][kSolveThreads / 32];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  double t[5] = {0.0, 0.0, 0.0, 0.0, 1.0};
  for (std::uint32_t p = threadIdx.x; p < blocks; p += blockDim.x) {
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const double x = __ldcg(&d.partials[5 * p + k]);
      t[k] = k < 3 ? t[k] + x : (k == 3 ? fmax(t[k], x) : fmin(t[k], x));
    }
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_down_sync(0xFFFFFFFFu, t[k], o);
      t[k] = k < 3 ? t[k] + other : (k == 3 ? fmax(t[k], other) : fmin(t[k], other));
    }
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 5; ++k) red[k][warp] = t[k];
  }
  __syncthreads();
  if (threadIdx.x != 0) return 0;
  double total[5];
  for (int k = 0; k < 5; ++k) {
    total[k] = red[k][0];
    for (int w = 1; w < kSolveThreads / 32; ++w) {
      total[k] = k < 3 ? total[k] + red[k][w] : (k == 3 ? fmax(total[k], red[k][w]) : fmin(total[k], red[k][w]));
    }
  }
  d.ticket = 0;
  const float reported = total[4] > 0.5 ? float(total[3]) : __int_as_float(0x7FC00000);
  d.residual = reported;
  std::uint32_t proceed = 0;
  if (mode == 0) {
    const float bound = __uint_as_float(__ldcg(&d.bound_bits));
    d.bound = bound;
    d.iterations = 0;
    if (!isfinite(bound) || !(bound > 0.0f)) {
      d.status = 3;  // no positive diagonal: an invalid system
    } else if (!isfinite(reported)) {
      d.status = MSB_SOLVE_BREAKDOWN;
    } else if (reported <= d.tolerance) {
      d.status = MSB_SOLVE_CONVERGED;
    } else {
      d.status = MSB_SOLVE_ITERATION_LIMIT;
      d.step = 1.0f / bound;
      proceed = d.max_iterations > 0 ? 1u : 0u;
    }
    d.mode = 1;
  } else {
    const std::uint32_t iteration = d.iterations + 1;
    d.iterations = iteration;
    if (!isfinite(reported)) {
      d.status = MSB_SOLVE_BREAKDOWN;
    } else if (!(reported > d.tolerance)) {
      d.status = MSB_SOLVE_CONVERGED;
    } else {
      d.step = next_step(d.step, total[0], total[1], total[2], iteration);
      d.status = MSB_SOLVE_ITERATION_LIMIT;
      proceed = iteration < d.max_iterations ? 1u : 0u;
    }
  }
  d.proceed = proceed;
  return proceed;
}

// mode 0: gaps of the initial multipliers and the first residual (sets the
// graph condition); mode 1: one projected step (sets the condition);
// mode 2: gaps only.  The last block to finish decides.
template <int Tag>
__global__ void __launch_bounds__(kSolveThreads, MSB_ROW_MIN_BLOCKS) row_pass_kernel(SolveDesc* desc, int fixed_mode, int set_condition) {
  SolveDesc& d = *desc;
  const std::uint32_t mode = fixed_mode >= 0 ? std::uint32_t(fixed_mode) : d.mode;
  if (fixed_mode < 0 && mode == 1 && d.proceed == 0u) return;  // an unrolled pair after convergence
  row_pass<false>(d, mode, d.step, blockIdx.x, gridDim.x, &desc->check_status);
  if (mode == 2) return;
  __threadfence();
  __shared__ bool last;
  if (threadIdx.x == 0) last = atomicAdd(&d.ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const std::uint32_t proceed = decide(d, mode, gridDim.x);
  if (threadIdx.x == 0 && set_condition) cudaGraphSetConditional(cudaGraphConditionalHandle(d.handle), proceed);
}

// contact_system_diagonal_bound (cpp/cpu/cpu_contact_dynamics.cpp:247-260):
// the largest dt * J M J^T + c over rows, as an atomic max of float bits.
__device__ __forceinline__ void bound_pass(const SolveDesc& d, std::uint32_t* bound_bits, std::uint32_t block,
                                           std::uint32_t blocks) {
  float bound = 0.0f;
  for (std::uint32_t i = block * blockDim.x + threadIdx.x; i < d.row_count; i += blocks * blockDim.x) {
    d.iterate[i] = make_float2(d.multipliers[i], 0.0f);
    const uint2 s = d.rows.slots[i];
    const float4 ra = d.rows.a[i];
    const float4 rb = d.rows.b[i];
    float entry = diagonal(ra, rb, d.bodies.a[s.x], d.bodies.b[s.x]);
    const float4 rd = d.rows.d[i];
    if (s.y != kInvalidSlot) entry += diagonal(d.rows.c[i], rd, d.bodies.a[s.y], d.bodies.b[s.y]);
    bound = smax(bound, d.dt * entry + rd.w);
  }
  for (int o = 16; o > 0; o >>= 1) bound = smax(bound, __shfl_down_sync(0xFFFFFFFFu, bound, o));
  if ((threadIdx.x & 31) == 0 && bound > 0.0f) atomicMax(bound_bits, __float_as_uint(bound));
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A grid barrier over `blocks` co-resident blocks.  Thread 0 of each block
// arrives on a counter; the last to arrive (with `decide_mode` >= 0) first
// combines the row pass's partials and decides with its whole block, then
// resets the counter and advances the generation that the others wait on.
// A wait longer than kBarrierTimeoutNs sets barrier_abort, which every
// waiting block sees.  Returns false once the solve is aborted.
__device__ __forceinline__ bool grid_barrier(SolveDesc& d, std::uint32_t blocks, int decide_mode) {
  __shared__ std::uint32_t generation;
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    generation = atomicAdd(&d.barrier_generation, 0u);
    __threadfence();
    last = atomicAdd(&d.barrier_count, 1u) + 1u == blocks;
  }
  __syncthreads();
  if (last) {
    __threadfence();
    if (decide_mode >= 0) decide(d, std::uint32_t(decide_mode), blocks);
    __syncthreads();
    if (threadIdx.x == 0) {
      d.barrier_count = 0;
      __threadfence();
      atomicAdd(&d.barrier_generation, 1u);
    }
  } else if (threadIdx.x == 0) {
    const unsigned long long start = global_ns();
    const volatile std::uint32_t* gen = &d.barrier_generation;
    const volatile std::uint32_t* abort = &d.barrier_abort;
    while (*gen == generation && *abort == 0u) {
      if (global_ns() - start > kBarrierTimeoutNs) {
        atomicExch(&d.barrier_abort, 1u);
        break;
      }
      if (MSB_BARRIER_SLEEP_NS > 0) __nanosleep(MSB_BARRIER_SLEEP_NS);
    }
    __threadfence();
  }
  __syncthreads();
  return *static_cast<const volatile std::uint32_t*>(&d.barrier_abort) == 0u;
}

// The fused solve: bound -> initial gaps and residual -> while not done
// { body pass; barrier; row pass; barrier and decision }.  The problem (the
// arrays and constants) comes as a grid-constant parameter, read from the
// constant bank; the solver state lives in *state (the same descriptor in
// device memory).
__global__ void __launch_bounds__(kSolveThreads, MSB_RELAX_MIN_BLOCKS)
    relax_kernel(const __grid_constant__ SolveDesc problem, SolveDesc* state) {
  const std::uint32_t blocks = gridDim.x;
  bound_pass(problem, &state->bound_bits, blockIdx.x, blocks);
  if (!grid_barrier(*state, blocks, -1)) return;
  const volatile SolveDesc* shared = state;
  // mode 0 evaluates the initial multipliers, mode 1 iterates.
  std::uint32_t mode = 0;
  float alpha = 0.0f;
  for (;;) {
    body_pass<true>(problem, mode, alpha, blockIdx.x, blocks, &state->check_status);
    if (!grid_barrier(*state, blocks, -1)) return;
    row_pass<true>(problem, mode, alpha, blockIdx.x, blocks, &state->check_status);
    if (!grid_barrier(*state, blocks, int(mode))) return;
    if (shared->proceed == 0u) return;
    mode = 1;
    alpha = shared->step;
  }
}

__global__ void __launch_bounds__(kSolveThreads) bound_kernel(SolveDesc* desc) {
  SolveDesc& d = *desc;
  float bound = 0.0f;
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < d.row_count; i += gridDim.x * blockDim.x) {
    d.iterate[i] = make_float2(d.multipliers[i], 0.0f);  // the solve's starting multipliers
    const uint2 s = d.rows.slots[i];
    const float4 ra = d.rows.a[i];
    const float4 rb = d.rows.b[i];
    float entry = diagonal(ra, rb, d.bodies.a[s.x], d.bodies.b[s.x]);
    const float4 rd = d.rows.d[i];
    if (s.y != kInvalidSlot) entry += diagonal(d.rows.c[i], rd, d.bodies.a[s.y], d.bodies.b[s.y]);
    bound = smax(bound, d.dt * entry + rd.w);
  }
  for (int o = 16; o > 0; o >>= 1) bound = smax(bound, __shfl_down_sync(0xFFFFFFFFu, bound, o));
  // Non-negative floats order as their bit patterns.
  if ((threadIdx.x & 31) == 0 && bound > 0.0f) atomicMax(&d.bound_bits, __float_as_uint(bound));
}

__global__ void unpack_iterate_kernel(const SolveDesc* desc) {
  const SolveDesc& d = *desc;
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < d.row_count; i += gridDim.x * blockDim.x) {
    const float2 q = d.iterate[i];
    d.multipliers[i] = q.x;
    d.gaps[i] = q.y;
  }
}

__global__ void solve_reset_kernel(SolveDesc* desc) {
  if (threadIdx.x == 0) {
    desc->mode = 0;
    desc->ticket = 0;
    desc->iterations = 0;
    desc->bound_bits = 0;
    desc->status = MSB_SOLVE_CONVERGED;
    desc->proceed = 0;
    desc->check_status = 0;
  }
}

// ------------------------------------------------------------- incidence

// Entries per body: one for a row's first slot, one for its second (a
// constraint row has none).  With `constants`, also each row's (offset,
// compliance) and -0.0f as a constraint row's second side term.
__global__ void incidence_counts_kernel(RowArrays r, std::uint32_t rows, std::uint32_t* __restrict__ counts,
                                        float2* __restrict__ constants, float2* __restrict__ sides) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const uint2 s = r.slots[i];
    atomicAdd(&counts[s.x], 1u);
    if (s.y != kInvalidSlot) atomicAdd(&counts[s.y], 1u);
    if (constants != nullptr) {
      constants[i] = make_float2(r.b[i].w, r.d[i].w);
      if (s.y == kInvalidSlot) reinterpret_cast<float*>(sides)[2 * std::uint64_t(i) + 1] = -0.0f;
    }
  }
}

// Each entry (row << 1 | side) to a free place in its body's range, in any
// order (the counts run back to zero).
__global__ void incidence_scatter_kernel(const uint2* __restrict__ slots, std::uint32_t rows,
                                         const std::uint32_t* __restrict__ offsets,
                                         std::uint32_t* __restrict__ counts, std::uint32_t* __restrict__ values) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const uint2 s = slots[i];
    values[offsets[s.x] + atomicSub(&counts[s.x], 1u) - 1u] = i << 1;
    if (s.y != kInvalidSlot) values[offsets[s.y] + atomicSub(&counts[s.y], 1u) - 1u] = (i << 1) | 1u;
  }
}

template <int N>
__device__ __forceinline__ void bitonic_sort_u32(std::uint32_t (&v)[N]) {
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const std::uint32_t a = v[i], b = v[l];
          const bool swap = (i & k) == 0 ? (a > b) : (a < b);
          v[i] = swap ? b : a;
          v[l] = swap ? a : b;
        }
      }
    }
  }
}

constexpr std::uint32_t kRegisterEntries = 16;
constexpr std::uint32_t kLocalEntries = 64;

__device__ __noinline__ void sort_local(std::uint32_t* __restrict__ values, std::uint32_t begin, std::uint32_t k) {
  std::uint32_t v[kLocalEntries];
  for (std::uint32_t j = 0; j < k; ++j) v[j] = values[begin + j];
  for (std::uint32_t i = 1; i < k; ++i) {
    const std::uint32_t x = v[i];
    std::uint32_t j = i;
    while (j > 0 && v[j - 1] > x) {
      v[j] = v[j - 1];
      --j;
    }
    v[j] = x;
  }
  for (std::uint32_t j = 0; j < k; ++j) values[begin + j] = v[j];
}

__device__ __noinline__ void sort_global(std::uint32_t* __restrict__ values, std::uint32_t begin, std::uint32_t k) {
  for (std::uint32_t i = 1; i < k; ++i) {
    const std::uint32_t x = values[begin + i];
    std::uint32_t j = i;
    while (j > 0 && values[begin + j - 1] > x) {
      values[begin + j] = values[begin + j - 1];
      --j;
    }
    values[begin + j] = x;
  }
}

// One thread per body: its entries sorted by row (row << 1 | side orders as
// the row), the order of make_incidence (cpp/cpu/cpu_contact_dynamics.cpp:78-106).
__global__ void incidence_order_kernel(const std::uint32_t* __restrict__ offsets, std::uint32_t bodies,
                                       std::uint32_t* __restrict__ values) {
  for (std::uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < bodies; b += gridDim.x * blockDim.x) {
    const std::uint32_t begin = offsets[b];
    const std::uint32_t k = offsets[b + 1] - begin;
    if (k <= 1) continue;
    if (k <= kRegisterEntries) {
      std::uint32_t v[kRegisterEntries];
#pragma unroll
      for (std::uint32_t j = 0; j < kRegisterEntries; ++j) v[j] = j < k ? values[begin + j] : 0xFFFFFFFFu;
      bitonic_sort_u32(v);
#pragma unroll
      for (std::uint32_t j = 0; j < kRegisterEntries; ++j) {
        if (j < k) values[begin + j] = v[j];
      }
    } else if (k <= kLocalEntries) {
      sort_local(values, begin, k);
    } else {
      sort_global(values, begin, k);
    }
  }
}

// The jacobian, lever and side bits (row << 1 | side) of every entry
// (`total` entries: the last body's end offset).
__global__ void incidence_gather_kernel(RowArrays r, const std::uint32_t* __restrict__ values,
                                        const std::uint32_t* __restrict__ total, std::uint32_t rows,
                                        float4* __restrict__ out_a, float4* __restrict__ out_b,
                                        std::uint32_t* status) {
  const std::uint32_t entries = *total;
  for (std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < entries; k += gridDim.x * blockDim.x) {
    const std::uint32_t v = values[k];
    const std::uint32_t row = v >> 1;
    if (!index_ok(row, rows, status)) continue;
    if (v & 1u) {
      const float4 c = r.c[row];
      const float4 d = r.d[row];
      out_a[k] = c;
      out_b[k] = make_float4(d.x, d.y, d.z, __uint_as_float(v));
    } else {
      const float4 a = r.a[row];
      const float4 b = r.b[row];
      out_a[k] = a;
      out_b[k] = make_float4(b.x, b.y, b.z, __uint_as_float(v));
    }
  }
}

__global__ void keyed_counts_kernel(const uint2* __restrict__ slots, std::uint32_t rows,
                                    std::uint32_t* __restrict__ counts) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    atomicAdd(&counts[slots[i].x], 1u);
  }
}

// Each row to a free place in its first slot's list (the counts run back to zero).
__global__ void keyed_scatter_kernel(const uint2* __restrict__ slots, std::uint32_t rows,
                                     const std::uint32_t* __restrict__ offsets, std::uint32_t* __restrict__ counts,
                                     std::uint32_t* __restrict__ rows_out) {
  for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const std::uint32_t s = slots[i].x;
    rows_out[offsets[s] + atomicSub(&counts[s], 1u) - 1u] = i;
  }
}

}  // namespace

namespace {

void incidence_pass(RowArrays rows, std::uint32_t row_count, std::uint32_t body_count, IncidenceArrays incidence,
                    std::uint32_t* values, std::uint32_t* counts, std::uint32_t* temp, cudaStream_t stream,
                    std::uint32_t* status) {
  // Counts per body, their scan, the entries scattered into their bodies'
  // ranges, each range sorted by row, then the jacobians gathered.
  cudaMemsetAsync(counts, 0, (body_count + 1) * sizeof(std::uint32_t), stream);
  if (row_count > 0) {
    incidence_counts_kernel<<<grid_for(row_count, 256), 256, 0, stream>>>(rows, row_count, counts,
                                                                         incidence.constants, incidence.sides);
    count_launch();
  }
  exclusive_scan(counts, incidence.offsets, body_count + 1, temp, stream);
  if (row_count == 0) return;
  incidence_scatter_kernel<<<grid_for(row_count, 256), 256, 0, stream>>>(rows.slots, row_count, incidence.offsets,
                                                                          counts, values);
  count_launch();
  incidence_order_kernel<<<grid_for(body_count, 256), 256, 0, stream>>>(incidence.offsets, body_count, values);
  count_launch();
  incidence_gather_kernel<<<grid_for(2ull * row_count, 256), 256, 0, stream>>>(
      rows, values, incidence.offsets + body_count, row_count, incidence.a, incidence.b, status);
  count_launch();
}

}  // namespace

void build_incidence(RowArrays rows, std::uint32_t row_count, std::uint32_t body_count, IncidenceArrays incidence,
                     std::uint32_t* keys, std::uint32_t* values, std::uint32_t* counts, std::uint32_t* temp,
                     cudaStream_t stream, std::uint32_t* status) {
  (void)keys;
  incidence_pass(rows, row_count, body_count, incidence, values, counts, temp, stream, status);
}

void build_keyed(const uint2* slots, std::uint32_t row_count, std::uint32_t body_count, std::uint32_t* offsets,
                 std::uint32_t* rows_out, std::uint32_t* keys, std::uint32_t* counts, std::uint32_t* temp,
                 cudaStream_t stream) {
  // Counts per first slot, their scan, the rows scattered into their lists,
  // each list sorted by row (a stable grouping, as KeyedRows keeps).
  (void)keys;
  cudaMemsetAsync(counts, 0, (body_count + 1) * sizeof(std::uint32_t), stream);
  if (row_count > 0) {
    keyed_counts_kernel<<<grid_for(row_count, 256), 256, 0, stream>>>(slots, row_count, counts);
    count_launch();
  }
  exclusive_scan(counts, offsets, body_count + 1, temp, stream);
  if (row_count == 0) return;
  keyed_scatter_kernel<<<grid_for(row_count, 256), 256, 0, stream>>>(slots, row_count, offsets, counts, rows_out);
  count_launch();
  incidence_order_kernel<<<grid_for(body_count, 256), 256, 0, stream>>>(offsets, body_count, rows_out);
  count_launch();
}

// One resident wave of row-pass blocks, at most kMaxPassBlocks (the
// descriptor's partials hold that many).
static int row_pass_blocks() {
  int device = 0, sms = kSmCount, active = 1;
  if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&active, row_pass_kernel<0>, kSolveThreads, 0);
  return std::max(1, std::min(int(kMaxPassBlocks), sms * std::max(1, active)));
}

SolveGraph::~SolveGraph() {
  if (exec_ != nullptr) cudaGraphExecDestroy(exec_);
  if (graph_ != nullptr) cudaGraphDestroy(graph_);
}

int SolveGraph::create(SolveDesc* desc, int blocks, cudaStream_t stream) {
  // At most one resident wave: a grid-stride pass whose blocks do not all
  // fit at once leaves a partly empty second wave.
  int device = 0, sms = kSmCount, body_active = 1, row_active = 1;
  if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&body_active, body_pass_kernel<0>, kSolveThreads, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&row_active, row_pass_kernel<0>, kSolveThreads, 0);
  const int wave = sms * std::max(1, std::min(body_active, row_active));
  // The row pass fills its own resident wave (5 blocks per SM at 46
  // registers against the body pass's 4): 22.3 against 23.0 us at 1M
  // capsules.  Its block partials fit the descriptor's 1,184.
  const int row_blocks = row_pass_blocks();
  blocks = std::max(1, std::min(blocks, wave));
  blocks_ = blocks;
  desc_ = desc;
  cudaError_t err = cudaGraphCreate(&graph_, 0);
  if (err != cudaSuccess) return err;
  cudaGraphConditionalHandle handle;
  err = cudaGraphConditionalHandleCreate(&handle, graph_, 0, cudaGraphCondAssignDefault);
  if (err != cudaSuccess) return err;
  handle_ = handle;

  auto kernel_node = [&](cudaGraph_t graph, cudaGraphNode_t* node, const cudaGraphNode_t* deps, size_t ndeps,
                         void* func, void** args, int grid, int threads = kSolveThreads) {
    cudaKernelNodeParams p{};
    p.func = func;
    p.gridDim = dim3(grid);
    p.blockDim = dim3(threads);
    p.sharedMemBytes = 0;
    p.kernelParams = args;
    p.extra = nullptr;
    return cudaGraphAddKernelNode(node, graph, deps, ndeps, &p);
  };

  SolveDesc* d = desc;
  int mode_auto = -1;
  int with_condition = 1;
  void* reset_args[] = {&d};
  void* bound_args[] = {&d};
  void* body_args[] = {&d, &mode_auto};
  void* row_args[] = {&d, &mode_auto, &with_condition};
  cudaGraphNode_t reset, bound, body0, row0, loop;
  if ((err = kernel_node(graph_, &reset, nullptr, 0, (void*)solve_reset_kernel, reset_args, 1, 32)) != cudaSuccess) return err;
  if ((err = kernel_node(graph_, &bound, &reset, 1, (void*)bound_kernel, bound_args, blocks)) != cudaSuccess) return err;
  if ((err = kernel_node(graph_, &body0, &bound, 1, (void*)body_pass_kernel<0>, body_args, blocks)) != cudaSuccess) return err;
  if ((err = kernel_node(graph_, &row0, &body0, 1, (void*)row_pass_kernel<0>, row_args, row_blocks)) != cudaSuccess) return err;

  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if ((err = cudaGraphAddNode(&loop, graph_, &row0, 1, &cp)) != cudaSuccess) return err;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaGraphNode_t previous = nullptr;
  for (int pair = 0; pair < MSB_WHILE_UNROLL; ++pair) {
    cudaGraphNode_t body1, row1;
    if ((err = kernel_node(body, &body1, previous != nullptr ? &previous : nullptr, previous != nullptr ? 1 : 0,
                           (void*)body_pass_kernel<0>, body_args, blocks)) != cudaSuccess) {
      return err;
    }
    if ((err = kernel_node(body, &row1, &body1, 1, (void*)row_pass_kernel<0>, row_args, row_blocks)) != cudaSuccess) return err;
    previous = row1;
  }
  err = cudaGraphInstantiate(&exec_, graph_, 0);
  count_launch(0);
  return err;
}

int SolveGraph::loop_launches(std::uint32_t iterations) {
  const std::uint32_t evaluations = (iterations + MSB_WHILE_UNROLL - 1) / MSB_WHILE_UNROLL;
  return int(evaluations * 2 * MSB_WHILE_UNROLL);
}

int SolveGraph::launch(cudaStream_t stream) {
  // Each graph has its own WHILE-node handle; the row pass reads it here.
  cudaError_t err = cudaMemcpyAsync(&desc_->handle, &handle_, sizeof(handle_), cudaMemcpyHostToDevice, stream);
  if (err != cudaSuccess) return err;
  count_launch(4);
  return cudaGraphLaunch(exec_, stream);
}

int relax_resident_blocks() {
  int device = 0, sms = kSmCount, per_sm = 0;
  if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, relax_kernel, kSolveThreads, 0) != cudaSuccess) return 0;
  return sms * per_sm;
}

int launch_relax(const SolveDesc& problem, SolveDesc* desc, int blocks, cudaStream_t stream) {
  SolveDesc copy = problem;
  void* args[] = {&copy, &desc};
  count_launch();
  return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(relax_kernel), dim3(blocks), dim3(kSolveThreads), args,
                                     0, stream);
}

void launch_iteration(SolveDesc* desc, int blocks, cudaEvent_t between, cudaStream_t stream) {
  body_pass_kernel<1><<<blocks, kSolveThreads, 0, stream>>>(desc, 1);
  if (between != nullptr) cudaEventRecord(between, stream);
  row_pass_kernel<1><<<row_pass_blocks(), kSolveThreads, 0, stream>>>(desc, 1, 0);
  count_launch(2);
}

void launch_unpack_iterate(SolveDesc* desc, int blocks, cudaStream_t stream) {
  unpack_iterate_kernel<<<blocks, kSolveThreads, 0, stream>>>(desc);
  count_launch();
}

void launch_evaluate(SolveDesc* desc, int blocks, bool with_gaps, cudaStream_t stream) {
  body_pass_kernel<0><<<blocks, kSolveThreads, 0, stream>>>(desc, 2);
  count_launch();
  if (with_gaps) {
    row_pass_kernel<0><<<blocks, kSolveThreads, 0, stream>>>(desc, 2, 0);
    count_launch();
  }
}

}  // namespace msb
