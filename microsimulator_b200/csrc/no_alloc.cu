// An allocation-free variant of the contact solve, for callers that cannot
// allocate device memory: code under an allocator policy that forbids new
// device allocations once it has started (a pool sized at start-up, or a
// memory budget fixed by a host framework), and real-time loops that must not
// pause for the driver's allocator.  It is not for stream capture or host
// callbacks: it copies from pageable host arrays and synchronises `stream`
// before it returns, which neither context allows.
//
// Every buffer the solve needs lives in one file-scope device array of
// kScratchBytes (8 MiB), so systems are limited to kMaxRows rows and
// kMaxBodies bodies; larger systems are rejected with MSB_ERR_CAPACITY.
// Every GPU that loads this library holds the array until the process exits.
// All calls share it and it keeps the last call's contents: the counters
// that must start at zero are cleared on every call, and calls that overlap
// on the GPU (from two threads, or on two streams without ordering) race on
// it.  The first call on a device looks up the array's device address with
// that device current.
//
// The solve is the same Barzilai-Borwein projected gradient as the main
// path, with the same per-body and per-row arithmetic (solve_math.cuh): the
// incidence is built by the main path's counting scatter and per-body sort
// by row on the static scratch, and one thread block runs the whole
// iteration loop (body pass, row pass, a fixed-tree block reduction of the
// BB products, the step length update) without returning to the host.

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "device.cuh"
#include "kernels.h"
#include "solve.h"
#include "solve_math.cuh"
#include "step.h"
#include "../../include/msb200.h"

namespace msb {
namespace {

constexpr std::uint32_t kMaxRows = 16384;
constexpr std::uint32_t kMaxBodies = 8192;
constexpr std::size_t kScratchBytes = std::size_t(8) << 20;
constexpr int kBlock = 512;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct SmallState {
  float step;
  float residual;
  float bound;
  std::uint32_t iterations;
  std::uint32_t status;
};

struct SmallSolve {
  RowArrays rows;
  BodyArrays bodies;
  IncidenceArrays incidence;
  ResponseArrays response;
  float* multipliers;
  float* gaps;
  SmallState* state;
  std::uint32_t row_count;
  std::uint32_t body_count;
  float dt;
  std::uint32_t law;
  float sensitivity;
  float free_load;
  float stall_load;
  float tolerance;
  std::uint32_t max_iterations;
  bool has_drift;  // read by respond(): the drift arrays hold something
};

// Per body: the wrench of its rows' multipliers in row order, then the
// mobility, drift and loaded elongation rate (respond, as the main path).
__device__ void small_body_pass(const SmallSolve& s, bool project, float alpha) {
  for (std::uint32_t b = threadIdx.x; b < s.body_count; b += blockDim.x) {
    float w[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    float load = 0.0f;
    for (std::uint32_t k = s.incidence.offsets[b]; k < s.incidence.offsets[b + 1]; ++k) {
      const float4 ea = s.incidence.a[k];
      const float4 eb = s.incidence.b[k];
      const std::uint32_t row = __float_as_uint(eb.w) >> 1;  // side bits: row << 1 | side
      const float g = s.multipliers[row];
      const float m = project ? smax(0.0f, g - alpha * s.gaps[row]) : g;
      if (m == 0.0f) continue;
      w[0] += m * ea.x;
      w[1] += m * ea.y;
      w[2] += m * ea.z;
      w[3] += m * ea.w;
      w[4] += m * eb.x;
      w[5] += m * eb.y;
      load += eb.z * m;
    }
    float v[6];
    float rate;
    respond(s, b, w, load, v, rate);
    s.response.a[b] = make_float4(v[0], v[1], v[2], rate);
    s.response.b[b] = make_float4(v[3], v[4], v[5], load);
  }
}

// One side's term of a row's gap rate from a body's stored response.
__device__ __forceinline__ float small_side(float4 ja, float4 jb, float4 ra, float4 rb) {
  const float v[6] = {ra.x, ra.y, ra.z, rb.x, rb.y, rb.z};
  return side_term(ja, jb, v, ra.w);
}

// row_gap (cpu_contact_dynamics.cpp:149-159) of row i with multiplier m.
__device__ __forceinline__ float small_gap(const SmallSolve& s, std::uint32_t i, float m) {
  const uint2 sl = s.rows.slots[i];
  const float4 rb = s.rows.b[i];
  const float4 rd = s.rows.d[i];
  float rate = small_side(s.rows.a[i], rb, s.response.a[sl.x], s.response.b[sl.x]);
  if (sl.y != kInvalidSlot) rate += small_side(s.rows.c[i], rd, s.response.a[sl.y], s.response.b[sl.y]);
  return rb.w + s.dt * rate + rd.w * m;
}

// Fixed-tree block reduction of five values (three sums, a max, a min).
__device__ void small_reduce(double v[5], double (*shared)[kBlock / 32]) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_down_sync(0xFFFFFFFFu, v[k], o);
      v[k] = k < 3 ? v[k] + other : (k == 3 ? fmax(v[k], other) : fmin(v[k], other));
    }
    if (lane == 0) shared[k][warp] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < 5; ++k) {
      double r = shared[k][0];
      for (int w2 = 1; w2 < kBlock / 32; ++w2) {
        r = k < 3 ? r + shared[k][w2] : (k == 3 ? fmax(r, shared[k][w2]) : fmin(r, shared[k][w2]));
      }
      v[k] = r;
    }
  }
}

// The whole solve in one block: contact_solver.hpp:86-120 with the
// projected step of cpu_contact_dynamics.cpp:411-445 of the reference.
__global__ void __launch_bounds__(kBlock) small_solve_kernel(SmallSolve s) {
  __shared__ double shared[5][kBlock / 32];
  __shared__ float alpha_shared;
  __shared__ int proceed_shared;

  // The first step length is one over the largest diagonal entry.
  float bound = 0.0f;
  for (std::uint32_t i = threadIdx.x; i < s.row_count; i += blockDim.x) {
    const uint2 sl = s.rows.slots[i];
    float entry = diagonal(s.rows.a[i], s.rows.b[i], s.bodies.a[sl.x], s.bodies.b[sl.x]);
    const float4 rd = s.rows.d[i];
    if (sl.y != kInvalidSlot) entry += diagonal(s.rows.c[i], rd, s.bodies.a[sl.y], s.bodies.b[sl.y]);
    bound = smax(bound, s.dt * entry + rd.w);
  }
  {
    double v[5] = {0.0, 0.0, 0.0, double(bound), 1.0};
    small_reduce(v, shared);
    if (threadIdx.x == 0) {
      const float b = float(v[3]);
      s.state->bound = b;
      s.state->iterations = 0;
      proceed_shared = isfinite(b) && b > 0.0f ? 1 : 0;
      if (!proceed_shared) s.state->status = 3;  // no positive diagonal
      alpha_shared = 1.0f / b;
    }
    __syncthreads();
    if (!proceed_shared) return;
  }

  // Gaps of the initial multipliers.
  small_body_pass(s, false, 0.0f);
  __syncthreads();
  {
    float residual = 0.0f;
    bool finite = true;
    for (std::uint32_t i = threadIdx.x; i < s.row_count; i += blockDim.x) {
      const float m = s.multipliers[i];
      const float gap = small_gap(s, i, m);
      s.gaps[i] = gap;
      residual = smax(residual, row_residual(m, gap));
      finite = finite && isfinite(gap);
    }
    double v[5] = {0.0, 0.0, 0.0, double(residual), finite ? 1.0 : 0.0};
    small_reduce(v, shared);
    if (threadIdx.x == 0) {
      const float reported = v[4] > 0.5 ? float(v[3]) : __int_as_float(0x7FC00000);
      s.state->residual = reported;
      if (!isfinite(reported)) {
        s.state->status = MSB_SOLVE_BREAKDOWN;
        proceed_shared = 0;
      } else if (reported <= s.tolerance) {
        s.state->status = MSB_SOLVE_CONVERGED;
        proceed_shared = 0;
      } else {
        s.state->status = MSB_SOLVE_ITERATION_LIMIT;
        proceed_shared = s.max_iterations > 0 ? 1 : 0;
      }
    }
    __syncthreads();
  }

  for (std::uint32_t iteration = 1; proceed_shared; ++iteration) {
    const float alpha = alpha_shared;
    small_body_pass(s, true, alpha);
    __syncthreads();
    double ss = 0.0, sy = 0.0, yy = 0.0;
    float residual = 0.0f;
    bool finite = true;
    for (std::uint32_t i = threadIdx.x; i < s.row_count; i += blockDim.x) {
      const float gi = s.multipliers[i];
      const float gpi = s.gaps[i];
      const float m = smax(0.0f, gi - alpha * gpi);
      const float gn = small_gap(s, i, m);
      const double moved = double(m) - double(gi);
      const double change = double(gn) - double(gpi);
      ss += moved * moved;
      sy += moved * change;
      yy += change * change;
      residual = smax(residual, row_residual(m, gn));
      finite = finite && isfinite(gn);
      s.multipliers[i] = m;
      s.gaps[i] = gn;
    }
    double v[5] = {ss, sy, yy, double(residual), finite ? 1.0 : 0.0};
    small_reduce(v, shared);
    if (threadIdx.x == 0) {
      const float reported = v[4] > 0.5 ? float(v[3]) : __int_as_float(0x7FC00000);
      s.state->residual = reported;
      s.state->iterations = iteration;
      int proceed = 0;
      if (!isfinite(reported)) {
        s.state->status = MSB_SOLVE_BREAKDOWN;
      } else if (!(reported > s.tolerance)) {
        s.state->status = MSB_SOLVE_CONVERGED;
      } else {
        s.state->status = MSB_SOLVE_ITERATION_LIMIT;
        alpha_shared = next_step(alpha_shared, v[0], v[1], v[2], iteration);
        proceed = iteration < s.max_iterations ? 1 : 0;
      }
      proceed_shared = proceed;
    }
    __syncthreads();
  }
}

// A bump allocator over the static scratch, 256-byte aligned pieces.
struct Carver {
  unsigned char* base;
  std::size_t used = 0;
  template <typename T>
  T* take(std::size_t count) {
    used = (used + 255) & ~std::size_t(255);
    T* p = reinterpret_cast<T*>(base + used);
    used += count * sizeof(T);
    return p;
  }
};

std::mutex setup_mutex;
void* scratch_address[kMaxDevices] = {};

bool finite_body(const msb_contact_body& b) {
  bool ok = std::isfinite(b.axis.x) && std::isfinite(b.axis.y) && std::isfinite(b.axis.z) &&
            std::isfinite(b.translational_mobility) && std::isfinite(b.transverse_mobility) &&
            std::isfinite(b.axial_mobility) && std::isfinite(b.length_rate) && b.translational_mobility >= 0.0f &&
            b.transverse_mobility >= 0.0f && b.axial_mobility >= 0.0f;
  for (float v : b.drift) ok = ok && std::isfinite(v);
  return ok;
}

bool valid_row(const msb_contact_row& r, std::uint64_t bodies) {
  if (r.first_slot >= bodies || (r.second_slot != kInvalidSlot && r.second_slot >= bodies)) return false;
  bool ok = std::isfinite(r.offset) && std::isfinite(r.compliance) && r.compliance >= 0.0f &&
            std::isfinite(r.first_length_lever) && std::isfinite(r.second_length_lever) &&
            r.first_length_lever >= 0.0f && r.second_length_lever >= 0.0f;
  for (int k = 0; k < 6; ++k) ok = ok && std::isfinite(r.first_jacobian[k]) && std::isfinite(r.second_jacobian[k]);
  return ok;
}

}  // namespace
}  // namespace msb

using namespace msb;

extern "C" int msb_solve_contact_forces_no_alloc(const msb_contact_system* system, const float* initial_multipliers,
                                                 const msb_contact_solve_parameters* parameters, float* multipliers,
                                                 msb_contact_solve_report* report, void* stream_handle) {
  // Argument checks of solve_contact_system_cpu and validate_contact_system
  // (cpp/cpu/cpu_contact_dynamics.cpp:384-397, cpp/core/contact_dynamics.cpp:640-672).
  if (system == nullptr || parameters == nullptr || report == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  if (system->row_count > kMaxRows || system->body_count > kMaxBodies) return MSB_ERR_CAPACITY;
  const auto rows = std::uint32_t(system->row_count);
  const auto bodies = std::uint32_t(system->body_count);
  if ((rows > 0 && (system->rows == nullptr || initial_multipliers == nullptr || multipliers == nullptr)) ||
      (bodies > 0 && system->bodies == nullptr)) {
    return MSB_ERR_INVALID_ARGUMENT;
  }
  const auto& g = system->growth;
  if (!std::isfinite(system->dt) || system->dt <= 0.0f || g.law > MSB_GROWTH_LAW_LINEAR ||
      !std::isfinite(g.sensitivity) || g.sensitivity < 0.0f || !std::isfinite(g.free_load) ||
      !std::isfinite(g.stall_load) || g.free_load < 0.0f || g.stall_load <= g.free_load ||
      !std::isfinite(parameters->tolerance) || parameters->tolerance <= 0.0f) {
    return MSB_ERR_INVALID_ARGUMENT;
  }
  for (std::uint32_t b = 0; b < bodies; ++b) {
    if (!finite_body(system->bodies[b])) return MSB_ERR_INVALID_ARGUMENT;
  }
  for (std::uint32_t r = 0; r < rows; ++r) {
    if (!valid_row(system->rows[r], bodies)) return MSB_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(initial_multipliers[r]) || initial_multipliers[r] < 0.0f) return MSB_ERR_INVALID_ARGUMENT;
  }
  if (rows == 0) {
    *report = {MSB_SOLVE_CONVERGED, 0, 0.0f};
    return MSB_OK;
  }

  // Set-up, once per device with that device current: the device address
  // of the static scratch.
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return MSB_ERR_CUDA;
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(setup_mutex);
    if (scratch_address[device] == nullptr) {
      void* address = nullptr;
      if (cudaGetSymbolAddress(&address, g_scratch) != cudaSuccess) return MSB_ERR_CUDA;
      scratch_address[device] = address;
    }
    base = scratch_address[device];
  }
  auto stream = static_cast<cudaStream_t>(stream_handle);

  Carver carve{static_cast<unsigned char*>(base)};
  SmallSolve s{};
  s.rows = {carve.take<float4>(rows), carve.take<float4>(rows), carve.take<float4>(rows), carve.take<float4>(rows),
            carve.take<uint2>(rows)};
  s.bodies = {carve.take<float4>(bodies), carve.take<float4>(bodies), carve.take<float4>(bodies),
              carve.take<float4>(bodies)};
  const std::size_t record_bytes = std::max<std::size_t>(std::size_t(rows) * sizeof(msb_contact_row),
                                                         std::size_t(bodies) * sizeof(msb_contact_body));
  unsigned char* records = carve.take<unsigned char>(record_bytes);
  s.multipliers = carve.take<float>(rows);
  s.gaps = carve.take<float>(rows);
  s.incidence = {carve.take<std::uint32_t>(bodies + 1ull), carve.take<float4>(2ull * rows),
                 carve.take<float4>(2ull * rows), nullptr, nullptr};  // its own passes need no side terms
  // The incidence build needs per-entry values, per-body counts and the
  // scan's scratch; it takes no sort keys.
  std::uint32_t* values = carve.take<std::uint32_t>(2ull * rows);
  std::uint32_t* counts = carve.take<std::uint32_t>(bodies + 1ull);
  std::uint32_t* temp = carve.take<std::uint32_t>(scan_temp_words(bodies + 1ull) + 64);
  s.response = {carve.take<float4>(std::max<std::uint32_t>(bodies, 1)), carve.take<float4>(std::max<std::uint32_t>(bodies, 1))};
  s.state = carve.take<SmallState>(1);
  if (carve.used > kScratchBytes) return MSB_ERR_CAPACITY;
  s.row_count = rows;
  s.body_count = bodies;
  s.dt = system->dt;
  s.law = g.law;
  s.sensitivity = g.sensitivity;
  s.free_load = g.free_load;
  s.stall_load = g.stall_load;
  s.tolerance = parameters->tolerance;
  s.max_iterations = parameters->max_iterations;
  s.has_drift = false;
  for (std::uint32_t b = 0; b < bodies && !s.has_drift; ++b) {
    for (float v : system->bodies[b].drift) s.has_drift = s.has_drift || v != 0.0f || std::signbit(v);
  }

  if (bodies > 0) {
    if (cudaMemcpyAsync(records, system->bodies, bodies * sizeof(msb_contact_body), cudaMemcpyHostToDevice, stream) !=
        cudaSuccess) {
      return MSB_ERR_CUDA;
    }
    launch_bodies_from_records(records, bodies, s.bodies, stream);
  }
  if (cudaMemcpyAsync(records + 0, system->rows, rows * sizeof(msb_contact_row), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(s.multipliers, initial_multipliers, rows * sizeof(float), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess) {
    return MSB_ERR_CUDA;
  }
  launch_rows_from_records(records, rows, s.rows, stream);
  build_incidence(s.rows, rows, bodies, s.incidence, nullptr, values, counts, temp, stream);
  small_solve_kernel<<<1, kBlock, 0, stream>>>(s);
  count_launch();
  // On a CUDA error `multipliers` may already hold part of the device copy
  // and *report is left as it was.
  SmallState state{};
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&state, s.state, sizeof(state), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(multipliers, s.multipliers, rows * sizeof(float), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    return MSB_ERR_CUDA;
  }
  if (state.status == 3) return MSB_ERR_INVALID_ARGUMENT;
  *report = {state.status, state.iterations, state.residual};
  return MSB_OK;
}
