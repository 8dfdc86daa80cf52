// Host engine of the B200 contact backend (C++23).
//
// A context owns one non-blocking stream, device buffers that grow by powers
// of two (as the reference's CudaBuffer does, cpp/cuda/cuda_backend.cu:40-88)
// and the captured solve graphs.  Every per-cell, per-row and per-contact
// pass runs on the device; the host keeps the substep controller of
// detail::advance_contact_dynamics (cpp/core/contact_dynamics.cpp:676-782)
// and reads a few scalars at its decision points.  The C-ABI entry points at
// the end (declared in include/msb200.h) map exceptions to status codes.

#include <algorithm>
#include <array>
#include <atomic>
#include <bit>
#include <condition_variable>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <span>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/msb200.h"
#include "batch.h"
#include "flow.h"
#include "graph.h"
#include "kernels.h"
#include "solve.h"
#include "step.h"
#include "mlp.h"

namespace msb {

namespace {
std::atomic<std::uint64_t> launches{0};
}

void count_launch(int n) { launches.fetch_add(std::uint64_t(n), std::memory_order_relaxed); }

namespace {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct DeviceCheckError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct CapacityError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check(cudaError_t err, const char* what) {
  if (err != cudaSuccess) {
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(err));
  }
}

template <typename T>
struct DBuf {
  T* p = nullptr;
  std::size_t cap = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(std::exchange(o.p, nullptr)), cap(std::exchange(o.cap, 0)) {}
  DBuf& operator=(DBuf&& o) noexcept {
    std::swap(p, o.p);
    std::swap(cap, o.cap);
    return *this;
  }
  ~DBuf() { release(); }
  void release() {
    if (p != nullptr) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  // Capacity for n elements: twice n, rounded up to a power of two, so that
  // a colony growing by divisions reallocates rarely (a reallocation frees
  // the old buffer, which waits for the device, and a step that regrows many
  // buffers at once measured 9-40 ms slower at 1.4M capsules).
  static std::size_t capacity_for(std::size_t n) { return std::bit_ceil(std::max<std::size_t>(2 * n, 64)); }
  // Grows to at least n elements; contents are not kept.
  T* ensure(std::size_t n) {
    if (n > cap) {
      release();
      const std::size_t c = capacity_for(n);
      check(cudaMalloc(&p, c * sizeof(T)), "cudaMalloc");
      cap = c;
    }
    return p;
  }
  // Grows to at least n elements keeping the first `keep`.
  T* grow(std::size_t n, std::size_t keep, cudaStream_t stream) {
    if (n <= cap) return p;
    const std::size_t c = capacity_for(n);
    T* q = nullptr;
    check(cudaMalloc(&q, c * sizeof(T)), "cudaMalloc");
    if (keep > 0) check(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, stream), "grow copy");
    check(cudaStreamSynchronize(stream), "grow");
    release();
    p = q;
    cap = c;
    return p;
  }
};

struct Geometry {
  DBuf<float4> pos_len;
  DBuf<float4> dir_rad;
  GeometryBuffers view() { return {pos_len.p, dir_rad.p}; }
  void ensure(std::size_t n) {
    pos_len.ensure(n);
    dir_rad.ensure(n);
  }
};

// The rows of one substep with their keys, multipliers and keyed lists.
struct RowStore {
  DBuf<float4> a, b, c, d;
  DBuf<uint2> slots;
  DBuf<std::uint64_t> partner;
  DBuf<float> multipliers;
  DBuf<float> gaps;
  DBuf<float2> iterate;  // (multiplier, gap) inside a solve
  DBuf<std::uint32_t> keyed_offsets;
  DBuf<std::uint32_t> keyed_rows;
  std::uint32_t count = 0;

  RowArrays arrays() { return {a.p, b.p, c.p, d.p, slots.p}; }
  void ensure(std::size_t n) {
    a.ensure(n);
    b.ensure(n);
    c.ensure(n);
    d.ensure(n);
    slots.ensure(n);
    partner.ensure(n);
    multipliers.ensure(n);
    gaps.ensure(n);
    iterate.ensure(n);
  }
  void grow(std::size_t n, cudaStream_t s) {
    a.grow(n, count, s);
    b.grow(n, count, s);
    c.grow(n, count, s);
    d.grow(n, count, s);
    slots.grow(n, count, s);
    partner.grow(n, count, s);
    multipliers.grow(n, count, s);
    gaps.grow(n, count, s);
    iterate.ensure(n);  // filled by each solve
  }
  KeyedLists keyed() const { return {keyed_offsets.p, keyed_rows.p, partner.p, multipliers.p}; }
};

// Small scalars read back at the controller's decision points.
enum Scalar : int {
  kStatus = 0,
  kOverlapBits = 1,
  kRotationBits = 2,
  kInvalid = 3,
  kGrowthBits = 4,
  kDisplacementBits = 5,
  kFastCount = 6,
  kScalarCount = 16
};

struct SolveOutcome {
  std::uint32_t status = MSB_SOLVE_CONVERGED;
  std::uint32_t iterations = 0;
  float residual = 0.0f;
};

constexpr std::uint32_t kRotationProbeIterations = 128;
constexpr float kSolveToleranceFraction = 0.25f;
constexpr float kLoadResolutionFraction = 0.1f;
constexpr std::uint32_t kEasyRefinements = 2;
constexpr std::uint32_t kMaxColonies = 1u << 20;
// Warm-start flags (msb_set_warm_start).
constexpr std::uint32_t kWarmCarry = 1;       // the previous step's final forces
constexpr std::uint32_t kWarmGuess = 2;    // forces that a motion guess asks of each body
constexpr std::uint32_t kWarmLearned = 4;  // the warm-start network makes the motion guess
constexpr std::uint32_t kWarmFlags = kWarmCarry | kWarmGuess | kWarmLearned;
// Systems up to this many rows (or bodies) take the fused relaxation when the
// form is automatic; larger ones the graph.  Measured on B200 the graph is
// faster at every size (per iteration: 116 against 149 us at 1M capsules,
// 24 against 28 us at 100k, 19 against 22 us at 20k), so automatic is the
// graph.
constexpr std::uint32_t kFusedRelaxationItems = 0;
// The substep's first search pads its candidate boxes by this much more
// than the candidate margin, so that its candidates serve the overlap
// re-checks while no box face has moved more than half the padded margin.
// Measured at 1.35M capsules over 10 steps, search phase per step: 0.05 um
// 4.92 ms (more re-checks fall back to a full search), 0.1 um 3.76, 0.15 um
// 3.19, 0.2 um 3.29 (more candidates to narrow).
constexpr float kRecheckReach = 0.15f;
// The same for a batch, whose re-checks fall back to a full search when any
// cell of any colony moved further: the 256-colony sweep (3.0M capsules,
// area fraction 0.7, colonies growing from loose starts) measured 61-62 ms
// per step at 0.15 um, 50-51 ms at 0.4 um and 52-53 ms at 1.0 um.
constexpr float kBatchRecheckReach = 0.4f;
// Active colonies at most for the batched solve's wide clusters (solve_batch).
constexpr std::uint32_t kFewColonies = 96;
constexpr float kMaximumSubstepRotation = 0.5f;
constexpr float kPlannedSubstepRotation = 0.8f * kMaximumSubstepRotation;

bool positive(float v) { return std::isfinite(v) && v > 0.0f; }

void validate_contact_parameters(const msb_contact_parameters& p) {
  if (!std::isfinite(p.activation_margin) || p.activation_margin < 0.0f) {
    throw std::invalid_argument("contact activation margin must be finite and non-negative");
  }
  if (!std::isfinite(p.parallel_sine_threshold) || p.parallel_sine_threshold < 0.0f ||
      p.parallel_sine_threshold > 1.0f) {
    throw std::invalid_argument("contact parallel threshold must be between zero and one");
  }
  if (!positive(p.degeneracy_epsilon)) {
    throw std::invalid_argument("contact degeneracy epsilon must be finite and positive");
  }
}

void validate_constraint_parameters(const msb_constraint_contact_parameters& p) {
  if (!std::isfinite(p.activation_margin) || p.activation_margin < 0.0f) {
    throw std::invalid_argument("constraint activation margin must be finite and non-negative");
  }
  if (!positive(p.degeneracy_epsilon)) {
    throw std::invalid_argument("constraint degeneracy epsilon must be finite and positive");
  }
}

void validate_growth(const msb_growth_load_response& g) {
  if (g.law > MSB_GROWTH_LAW_LINEAR) throw std::invalid_argument("growth load law is invalid");
  if (!std::isfinite(g.sensitivity) || g.sensitivity < 0.0f) {
    throw std::invalid_argument("growth load sensitivity must be finite and non-negative");
  }
  if (!std::isfinite(g.free_load) || !std::isfinite(g.stall_load) || g.free_load < 0.0f ||
      g.stall_load <= g.free_load) {
    throw std::invalid_argument("growth stall load must be finite and exceed a finite, non-negative free load");
  }
}

void validate_dynamics(const msb_contact_dynamics_parameters& p) {
  if (!positive(p.drag)) throw std::invalid_argument("contact dynamics drag must be finite and positive");
  if (!positive(p.contact_stiffness) || !positive(p.wall_stiffness)) {
    throw std::invalid_argument("contact and wall stiffness must be finite and positive");
  }
  if (!positive(p.overlap_tolerance)) {
    throw std::invalid_argument("contact overlap tolerance must be finite and positive");
  }
  if (!std::isfinite(p.candidate_margin) || p.candidate_margin < 0.0f) {
    throw std::invalid_argument("contact candidate margin must be finite and non-negative");
  }
  if (!positive(p.max_overlap_recovery)) {
    throw std::invalid_argument("contact overlap recovery must be finite and positive");
  }
  if (!positive(p.max_growth_fraction)) {
    throw std::invalid_argument("contact growth fraction must be finite and positive");
  }
  if (p.max_iterations == 0) throw std::invalid_argument("contact dynamics iteration limit must be positive");
  validate_growth(p.growth);
}

float effective_overlap_tolerance(const msb_contact_dynamics_parameters& p) {
  float load_scale = 0.0f;
  if (p.growth.law == MSB_GROWTH_LAW_LINEAR) {
    load_scale = p.growth.stall_load - p.growth.free_load;
  } else if (p.growth.law == MSB_GROWTH_LAW_EXPONENTIAL && p.growth.sensitivity > 0.0f) {
    load_scale = 1.0f / p.growth.sensitivity;
  }
  if (load_scale <= 0.0f) return p.overlap_tolerance;
  return std::min(p.overlap_tolerance, kLoadResolutionFraction * load_scale / p.contact_stiffness);
}

bool finite_row(const msb_contact_row& r) {
  bool ok = std::isfinite(r.offset) && std::isfinite(r.compliance) && r.compliance >= 0.0f &&
            std::isfinite(r.first_length_lever) && std::isfinite(r.second_length_lever) &&
            r.first_length_lever >= 0.0f && r.second_length_lever >= 0.0f;
  for (int k = 0; k < 6; ++k) ok = ok && std::isfinite(r.first_jacobian[k]) && std::isfinite(r.second_jacobian[k]);
  return ok;
}

// validate_contact_system (contact_dynamics.cpp:640-672) on the host records.
void validate_system(const msb_contact_system& s) {
  if (!std::isfinite(s.dt) || s.dt <= 0.0f) {
    throw std::invalid_argument("contact system time step must be finite and positive");
  }
  validate_growth(s.growth);
  if (s.body_count > 0xFFFFFFF0ull || s.row_count > 0x7FFFFFF0ull) {
    throw std::overflow_error("contact system has too many rows or bodies");
  }
  for (std::uint64_t i = 0; i < s.body_count; ++i) {
    const auto& b = s.bodies[i];
    bool ok = std::isfinite(b.axis.x) && std::isfinite(b.axis.y) && std::isfinite(b.axis.z) &&
              std::isfinite(b.translational_mobility) && std::isfinite(b.transverse_mobility) &&
              std::isfinite(b.axial_mobility) && std::isfinite(b.length_rate) && b.translational_mobility >= 0.0f &&
              b.transverse_mobility >= 0.0f && b.axial_mobility >= 0.0f;
    for (float v : b.drift) ok = ok && std::isfinite(v);
    if (!ok) throw std::invalid_argument("contact body is invalid");
  }
  for (std::uint64_t i = 0; i < s.row_count; ++i) {
    const auto& r = s.rows[i];
    if (r.first_slot >= s.body_count || (r.second_slot != kInvalidSlot && r.second_slot >= s.body_count)) {
      throw std::invalid_argument("contact row slot is out of range");
    }
    if (!finite_row(r)) throw std::invalid_argument("contact row is invalid");
  }
}

void require_multipliers(const float* m, std::uint64_t n) {
  for (std::uint64_t i = 0; i < n; ++i) {
    if (!std::isfinite(m[i]) || m[i] < 0.0f) {
      throw std::invalid_argument("contact multipliers must be finite and non-negative");
    }
  }
}

}  // namespace
}  // namespace msb

namespace msb {

// Copies between a caller's pageable host arrays and pinned staging memory,
// split over a few threads: the device side of a host-buffer call is then
// one DMA per array at full PCIe speed, and the host side runs in parallel
// (pageable cudaMemcpy goes through the driver's single bounce buffer).
class HostCopies {
 public:
  // A host copy of `bytes` from src to dst.  With `ready`, the copy first
  // waits for that event (a download's DMA into src).  With `device`, the
  // copy is followed by a DMA of dst to device on `stream` (an upload's
  // chunk starts on its way as soon as it is staged).
  struct Job {
    void* dst;
    const void* src;
    std::size_t bytes;
    cudaEvent_t ready = nullptr;
    void* device = nullptr;
    cudaStream_t stream = nullptr;
  };

  HostCopies() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned helpers = std::min(15u, hw > 1 ? hw - 1 : 0u);
    for (unsigned t = 0; t < helpers; ++t) threads_.emplace_back([this] { serve(); });
  }
  HostCopies(const HostCopies&) = delete;
  HostCopies& operator=(const HostCopies&) = delete;
  ~HostCopies() {
    {
      std::lock_guard<std::mutex> lock(mutex_);
      stop_ = true;
    }
    wake_.notify_all();
    for (auto& t : threads_) t.join();
  }

  // Runs every job (split into chunks) on the pool and this thread; returns
  // when all are done (and every upload DMA is queued).  Returns the first
  // CUDA error a chunk met.
  cudaError_t run(const std::vector<Job>& jobs) {
    chunks_.clear();
    error_.store(cudaSuccess);
    constexpr std::size_t kChunk = std::size_t(1) << 21;
    for (const auto& j : jobs) {
      for (std::size_t at = 0; at < j.bytes; at += kChunk) {
        const std::size_t len = std::min(kChunk, j.bytes - at);
        chunks_.push_back({static_cast<char*>(j.dst) + at, static_cast<const char*>(j.src) + at, len, j.ready,
                           j.device != nullptr ? static_cast<char*>(j.device) + at : nullptr, j.stream});
      }
    }
    if (chunks_.empty()) return cudaSuccess;
    {
      std::lock_guard<std::mutex> lock(mutex_);
      next_.store(0);
      busy_ = threads_.size();
      ++generation_;
    }
    wake_.notify_all();
    work();
    std::unique_lock<std::mutex> lock(mutex_);
    done_.wait(lock, [this] { return busy_ == 0; });
    return error_.load();
  }

 private:
  void fail(cudaError_t e) {
    cudaError_t expected = cudaSuccess;
    if (e != cudaSuccess) error_.compare_exchange_strong(expected, e);
  }
  void work() {
    for (;;) {
      const std::size_t k = next_.fetch_add(1);
      if (k >= chunks_.size()) return;
      const Job& j = chunks_[k];
      if (j.ready != nullptr) fail(cudaEventSynchronize(j.ready));
      std::memcpy(j.dst, j.src, j.bytes);
      if (j.device != nullptr) fail(cudaMemcpyAsync(j.device, j.dst, j.bytes, cudaMemcpyHostToDevice, j.stream));
    }
  }
  void serve() {
    std::uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lock(mutex_);
        wake_.wait(lock, [&] { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
      }
      work();
      {
        std::lock_guard<std::mutex> lock(mutex_);
        if (--busy_ == 0) done_.notify_all();
      }
    }
  }

  std::vector<std::thread> threads_;
  std::vector<Job> chunks_;
  std::atomic<std::size_t> next_{0};
  std::atomic<cudaError_t> error_{cudaSuccess};
  std::mutex mutex_;
  std::condition_variable wake_, done_;
  std::size_t busy_ = 0;
  std::uint64_t generation_ = 0;
  bool stop_ = false;
};

// Pinned host memory grown on demand.
struct PinnedBuffer {
  unsigned char* p = nullptr;
  std::size_t cap = 0;
  PinnedBuffer() = default;
  PinnedBuffer(const PinnedBuffer&) = delete;
  PinnedBuffer& operator=(const PinnedBuffer&) = delete;
  ~PinnedBuffer() { release(); }
  void release() {
    if (p != nullptr) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
  unsigned char* ensure(std::size_t bytes) {
    if (bytes > cap) {
      release();
      const std::size_t c = std::bit_ceil(std::max<std::size_t>(bytes + bytes / 4, 1 << 20));
      if (cudaMallocHost(reinterpret_cast<void**>(&p), c) != cudaSuccess) {
        p = nullptr;
        throw std::runtime_error("cudaMallocHost failed for staging memory");
      }
      cap = c;
    }
    return p;
  }
};

}  // namespace msb

struct msb_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  std::string device_name;
  std::uint64_t launches_at_create = 0;

  // cells
  std::uint32_t n = 0;
  msb::DBuf<std::uint64_t> ids;
  msb::DBuf<float> growth;
  msb::DBuf<std::uint8_t> fixed;
  std::array<msb::DBuf<float>, 8> staging;  // px, py, pz, dx, dy, dz, len, radius
  msb::Geometry state, base, initial, trial;
  msb::DBuf<std::uint32_t> order, rank;

  // scratch for scans and sorts
  msb::DBuf<std::uint32_t> temp, sort_keys, sort_values, counts;

  // contact search
  msb::DBuf<double> bounds, bound_partials;
  msb::DBuf<msb::GridParams> grid;
  msb::DBuf<std::uint32_t> cell_bucket, bucket_counts, bucket_starts, bucket_fill;
  msb::DBuf<float4> sorted_lo, sorted_hi;
  msb::DBuf<std::uint64_t> sorted_id;
  msb::DBuf<std::int64_t> coords;
  msb::DBuf<std::uint32_t> cand_counts, cand_offsets, pair_counts, pair_offsets, wall_counts, wall_offsets;
  msb::DBuf<uint2> pairs;
  msb::DBuf<std::uint32_t> slab;  // the broad phase's kept partners, kSlabPartners per cell
  // The candidate pairs of the current substep's first search (boxes padded
  // by kept_margin at the substep's base geometry), which the overlap
  // re-checks of its refinement rounds reuse while the cells have moved less
  // than half of kept_margin (flag_overlaps).
  msb::DBuf<uint2> kept_pairs;
  msb::DBuf<std::uint32_t> kept_offsets;
  // Partial re-search (find_touches_partial): fast-cell flags and list, their
  // new partners and the merge's shifts.
  msb::DBuf<std::uint32_t> fast_flags, fast_list, fast_counts, fast_offsets, shift, shift_scan;
  msb::DBuf<uint2> fast_pairs, fast_sorted;
  // Overlap re-checks of the last step by kind: a full search, the kept
  // candidates, the kept candidates with a partial re-search.  search_reuse:
  // 0 all kinds, 1 no partial re-search, 2 full searches only.
  std::uint32_t searches[3] = {0, 0, 0};
  std::uint32_t search_reuse = 0;
  std::uint32_t kept_count = 0;
  float kept_margin = 0.0f;
  bool kept_valid = false;
  float displacement = 0.0f;  // the last move's largest box-face displacement
  msb::DBuf<msb::Touch> touches, found, flagged;
  msb::DBuf<std::uint32_t> flags, flag_offsets;
  msb::DBuf<msb::DeviceConstraint> constraints;
  std::uint32_t constraint_count = 0;

  // the contact system
  msb::RowStore rows, memory;
  bool has_memory = false;
  // Warm-start flags (msb_set_warm_start) and the cells of the memory.
  std::uint32_t warm_start_mode = 0;
  std::uint32_t memory_cells = 0;
  msb::DBuf<std::uint64_t> memory_first_ids, memory_partner_ids;
  // A per-cell motion guess for the next step (msb_set_motion_guess).
  msb::DBuf<float4> guess, guess_a, guess_b;
  msb::DBuf<float> guess_delta;
  // The warm-start network (msb_set_warm_start_network) and its buffers.
  msb::DBuf<std::uint16_t> net_weights;
  msb::DBuf<float> net_biases;
  float net_scale[3] = {1.0f, 1.0f, 1.0f};
  bool has_network = false;
  msb::DBuf<std::uint16_t> features;
  msb::DBuf<float> net_outputs;
  msb::DBuf<std::uint32_t> knn_keys, knn_values, knn_counts, knn_offsets, knn_bounds;
  msb::DBuf<float2> knn_centres;
  bool has_guess = false;
  std::uint32_t guess_cells = 0;
  float guess_dt = 0.0f;
  bool has_drift = false;  // a loaded system with some drift other than +0.0f
  // The flow field of msb_set_flow_field, for steps with flow drift.
  bool has_flow = false;
  msb::FlowField flow{};
  msb::DBuf<float> flow_x, flow_y, flow_z;
  msb::DBuf<std::uint8_t> flow_obstacles;
  msb::DBuf<float4> flow_sites;  // per site the sums of its two faces along each axis
  float flow_travel_limit = 0.0f;
  msb::DBuf<float4> body_a, body_b, drift_a, drift_b;
  msb::DBuf<std::uint32_t> inc_offsets;
  msb::DBuf<float4> inc_a, inc_b, resp_a, resp_b, accepted_a, accepted_b;
  msb::DBuf<float2> inc_constants, inc_sides;  // per row: (offset, compliance), the two side terms
  msb::DBuf<float> slack;

  // A batch of independent colonies (msb_advance_contact_dynamics_batch);
  // colonies == 0 for a single system.
  std::uint32_t colonies = 0;
  std::vector<std::uint32_t> host_colony_offsets;
  msb::DBuf<std::uint32_t> colony_offsets, colony_of_slot, colony_order, colony_overlap, colony_rows,
      colony_row_counts, colony_row_offsets, batch_next, colony_active, colony_flagged;
  msb::DBuf<float> colony_drag, colony_stiffness, colony_tolerance, colony_solve_tolerance, colony_slack,
      batch_saved;
  msb::DBuf<msb::ColonyState> colony_state;
  std::vector<msb::ColonyState> host_colony_state;
  std::vector<std::uint64_t> colony_iterations;
  std::vector<std::uint32_t> colony_status;
  std::vector<float> colony_max_overlap;
  std::vector<std::uint32_t> colony_rows_at_accept;
  msb::BatchShape batch_shape{4, 256, false};
  int batch_clusters = 0;
  bool batch_tuned = false;
  std::vector<std::uint32_t> host_colony_active;
  float box_scale = 1.0f;        // the contact search's box scale for the current call
  float batch_box_scale = 1.0f;  // the autotuner's choice for batches
  bool tune_search = true;

  // solve
  int last_blocks = 0;
  msb::SolveDesc* desc = nullptr;
  msb::DBuf<double> partials;
  std::vector<std::unique_ptr<msb::SolveGraph>> graphs;
  std::uint32_t relaxation = 0;  // msb_set_relaxation: 0 automatic, 1 graph, 2 fused
  int relax_blocks = -1;         // co-resident blocks of the fused solve (-1: not asked yet)

  // scalars
  msb::DBuf<std::uint32_t> scalars;
  std::uint32_t* host_scalars = nullptr;
  msb::SolveDesc* host_desc = nullptr;

  // host-buffer calls: pinned staging both ways and the host-side copy pool
  std::unique_ptr<msb::HostCopies> copies;
  msb::PinnedBuffer upload, download;
  std::vector<msb::HostCopies::Job> pending;  // download copies, each waiting for its DMA's event
  std::vector<cudaEvent_t> download_events;

  // phase timing of the last step: events at phase boundaries
  std::vector<cudaEvent_t> phase_events;
  bool nvtx_open = false;  // an NVTX range of the current phase is open
  std::vector<int> phase_marks;
  std::vector<msb_solve_record> solve_log;  // the solves of the last step, in order
  std::array<double, 8> phase_ms{};

  // outputs staging for host calls
  msb::DBuf<float> out_velocities, out_loads, out_increments;
  msb::DBuf<std::uint8_t> records;

  // contact graph index: a copy of host contacts, scratch, staging of the
  // index for host calls, and the validation words
  msb::DBuf<std::uint8_t> graph_contacts;
  msb::DBuf<std::uint32_t> graph_scratch;
  msb::DBuf<std::uint64_t> graph_incidence_offsets, graph_incidence, graph_neighbor_offsets, graph_neighbors;
  msb::DBuf<unsigned long long> graph_words;
};

namespace msb {
namespace {

using Ctx = msb_context;

// Phases of a step, in the order msb_last_step_phases reports them.
enum Phase : int {
  kPhaseLoad = 0,       // upload, validation, id order
  kPhaseSearch = 1,     // cell list, broad and narrow phase, wall contacts
  kPhaseRows = 2,       // bodies, rows, keys, warm start, refinement rows
  kPhaseIncidence = 3,  // per-body incidence of the rows
  kPhaseSolve = 4,      // the BB solves
  kPhaseMove = 5,       // move, restore, overlap re-check
  kPhaseOutput = 6,     // outputs and download
  kPhaseGuess = 7,      // neighbour features and the warm-start network
  kPhaseEnd = 8
};

constexpr const char* kPhaseNames[] = {"msb load", "msb search", "msb rows",   "msb incidence",
                                       "msb solve", "msb move",   "msb output", "msb guess"};

// Records an event on the stream where `phase` begins (the previous phase
// ends), and opens an NVTX range of the phase's name for profilers (closed
// at the next mark).
void mark(Ctx& c, int phase) {
  if (c.nvtx_open) nvtxRangePop();
  c.nvtx_open = phase != kPhaseEnd;
  if (c.nvtx_open) nvtxRangePushA(kPhaseNames[phase]);
  if (c.phase_marks.size() == c.phase_events.size()) {
    cudaEvent_t e;
    check(cudaEventCreate(&e), "event");
    c.phase_events.push_back(e);
  }
  check(cudaEventRecord(c.phase_events[c.phase_marks.size()], c.stream), "event");
  c.phase_marks.push_back(phase);
}

void collect_phases(Ctx& c) {
  c.phase_ms.fill(0.0);
  if (c.phase_marks.empty()) return;
  check(cudaEventSynchronize(c.phase_events[c.phase_marks.size() - 1]), "event");
  for (std::size_t k = 0; k + 1 < c.phase_marks.size(); ++k) {
    float ms = 0.0f;
    check(cudaEventElapsedTime(&ms, c.phase_events[k], c.phase_events[k + 1]), "event");
    c.phase_ms[c.phase_marks[k]] += ms;
  }
  c.phase_marks.clear();
}

void sync(Ctx& c) { check(cudaStreamSynchronize(c.stream), "stream"); }

// Clears the scalar words except the status word, which keeps the first
// failure until read_scalars reports it.
void reset_scalars(Ctx& c) {
  check(cudaMemsetAsync(c.scalars.p + 1, 0, (kScalarCount - 1) * 4, c.stream), "memset");
}

void reset_status(Ctx& c) { check(cudaMemsetAsync(c.scalars.p, 0, kScalarCount * 4, c.stream), "memset"); }

void read_scalars(Ctx& c) {
  check(cudaMemcpyAsync(c.host_scalars, c.scalars.p, kScalarCount * 4, cudaMemcpyDeviceToHost, c.stream), "read");
  sync(c);
  if (c.host_scalars[kStatus] != kStatusOk) {
    const auto code = c.host_scalars[kStatus];
    if (code == kStatusGeometry) throw std::invalid_argument("cell geometry is invalid (non-finite, negative or unnormalized)");
    if (code == kStatusIndex) throw std::invalid_argument("cell identifiers must be non-zero and unique");

    throw DeviceCheckError("a device-side check failed (code " + std::to_string(code) + ")");
  }
}

float bits_to_float(std::uint32_t bits) {
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

std::uint32_t read_u32(Ctx& c, const std::uint32_t* device_ptr) {
  std::uint32_t v = 0;
  check(cudaMemcpyAsync(c.host_scalars + kScalarCount, device_ptr, 4, cudaMemcpyDeviceToHost, c.stream), "read");
  sync(c);
  v = c.host_scalars[kScalarCount];
  return v;
}

GeometryView view_of(Ctx& c, Geometry& g) {
  return {g.pos_len.p, g.dir_rad.p, c.ids.p, c.n, c.colonies > 0 ? c.colony_of_slot.p : nullptr,
          c.colonies > 0 ? c.colony_active.p : nullptr};
}

// ---- cells ---------------------------------------------------------------

Colonies colonies_of(Ctx& c) {
  if (c.colonies == 0) return {};
  return {c.colony_of_slot.p,   c.colony_drag.p,  c.colony_stiffness.p,
          c.colony_overlap.p,   c.colony_slack.p, c.colony_flagged.p};
}

msb::HostCopies& host_copies(Ctx& c) {
  if (!c.copies) c.copies = std::make_unique<msb::HostCopies>();
  return *c.copies;
}

// Whether `p` is page-locked host memory the device can reach by DMA
// (cudaHostAlloc / cudaHostRegister / a pinned torch tensor): such caller
// arrays are copied directly, without the staging buffers.
bool pinned_host(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// A device-to-host copy into the caller's `dst`: directly when `dst` is
// pinned, else through the pinned download buffer (the DMA is queued now,
// the host copy waits in c.pending for the stream's next sync,
// flush_downloads).  `at` is the running offset in the download buffer.
void stage_download(Ctx& c, void* dst, const void* device_src, std::size_t bytes, std::size_t& at) {
  if (pinned_host(dst)) {
    check(cudaMemcpyAsync(dst, device_src, bytes, cudaMemcpyDeviceToHost, c.stream), "copy back");
    return;
  }
  unsigned char* slot = c.download.p + at;
  check(cudaMemcpyAsync(slot, device_src, bytes, cudaMemcpyDeviceToHost, c.stream), "copy back");
  // The host copy of this array may start once its own DMA is done.
  const std::size_t k = c.pending.size();
  if (k == c.download_events.size()) {
    cudaEvent_t e;
    check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    c.download_events.push_back(e);
  }
  check(cudaEventRecord(c.download_events[k], c.stream), "event");
  c.pending.push_back({dst, slot, bytes, c.download_events[k]});
  at += (bytes + 255) & ~std::size_t(255);
}

void flush_downloads(Ctx& c) {
  if (c.pending.empty()) return;
  const cudaError_t err = host_copies(c).run(c.pending);
  c.pending.clear();
  check(err, "copy back");
}

void load_cells(Ctx& c, const msb_cell_arrays& cells, bool device_pointers) {
  if (cells.count >= 0xFFFFFFF0ull) throw std::overflow_error("cell count exceeds the slot index space");
  if (cells.count > 0 && (cells.ids == nullptr || cells.position_x == nullptr || cells.position_y == nullptr ||
                          cells.position_z == nullptr || cells.direction_x == nullptr ||
                          cells.direction_y == nullptr || cells.direction_z == nullptr || cells.lengths == nullptr ||
                          cells.radii == nullptr)) {
    throw std::invalid_argument("cell arrays must not be null");
  }
  c.n = std::uint32_t(cells.count);
  const std::size_t n = c.n;
  if (n == 0) return;
  c.ids.ensure(n);
  c.growth.ensure(n);
  c.fixed.ensure(n);
  const float* src[8] = {cells.position_x,  cells.position_y,  cells.position_z, cells.direction_x,
                         cells.direction_y, cells.direction_z, cells.lengths,    cells.radii};
  std::vector<msb::HostCopies::Job> uploads;  // (device destination, caller's source, bytes)
  uploads.push_back({c.ids.p, cells.ids, n * 8});
  for (int k = 0; k < 8; ++k) {
    c.staging[k].ensure(n);
    uploads.push_back({c.staging[k].p, src[k], n * 4});
  }
  if (cells.growth_rates != nullptr) {
    uploads.push_back({c.growth.p, cells.growth_rates, n * 4});
  } else {
    check(cudaMemsetAsync(c.growth.p, 0, n * 4, c.stream), "memset");
  }
  if (cells.fixed != nullptr) {
    uploads.push_back({c.fixed.p, cells.fixed, n});
  } else {
    check(cudaMemsetAsync(c.fixed.p, 0, n, c.stream), "memset");
  }
  if (device_pointers) {
    for (const auto& u : uploads) {
      check(cudaMemcpyAsync(u.dst, u.src, u.bytes, cudaMemcpyDeviceToDevice, c.stream), "copy cells");
    }
  } else {
    // Pinned caller arrays go straight to the device; the others through
    // pinned staging: the host side in parallel, each 2 MiB chunk's DMA
    // queued as soon as it is staged.
    std::vector<msb::HostCopies::Job> pageable;
    std::size_t total = 0;
    for (const auto& u : uploads) {
      if (pinned_host(u.src)) {
        check(cudaMemcpyAsync(u.dst, u.src, u.bytes, cudaMemcpyHostToDevice, c.stream), "copy cells");
      } else {
        pageable.push_back(u);
        total += (u.bytes + 255) & ~std::size_t(255);
      }
    }
    if (!pageable.empty()) {
      unsigned char* base = c.upload.ensure(total);
      std::vector<msb::HostCopies::Job> host;
      std::size_t at = 0;
      for (const auto& u : pageable) {
        host.push_back({base + at, u.src, u.bytes, nullptr, u.dst, c.stream});
        at += (u.bytes + 255) & ~std::size_t(255);
      }
      check(host_copies(c).run(host), "copy cells");
    }
  }
  c.state.ensure(n);
  reset_status(c);
  launch_pack_cells(c.n, c.staging[0].p, c.staging[1].p, c.staging[2].p, c.staging[3].p, c.staging[4].p,
                    c.staging[5].p, c.staging[6].p, c.staging[7].p, c.state.view(), c.scalars.p + kStatus, c.stream);

  // Id order: LSD radix sort of the ids (low word, then high word if used).
  c.order.ensure(n);
  c.rank.ensure(n);
  c.sort_keys.ensure(n);
  c.temp.ensure(sort_temp_words(n) + scan_temp_words(4 * n + 8192) + 64);
  launch_max_u64(c.ids.p, c.n, reinterpret_cast<std::uint64_t*>(c.scalars.p + 8), c.stream);
  read_scalars(c);
  std::uint64_t max_id = 0;
  std::memcpy(&max_id, c.host_scalars + 8, 8);
  const int bits = max_id == 0 ? 1 : 64 - std::countl_zero(max_id);
  iota(c.order.p, n, c.stream);
  launch_id_low_words(c.ids.p, c.n, 0, nullptr, c.sort_keys.p, c.stream);
  radix_sort_pairs(c.sort_keys.p, c.order.p, n, std::min(bits, 32), c.temp.p, c.stream);
  if (bits > 32) {
    launch_id_low_words(c.ids.p, c.n, 32, c.order.p, c.sort_keys.p, c.stream);
    radix_sort_pairs(c.sort_keys.p, c.order.p, n, bits - 32, c.temp.p, c.stream);
  }
  launch_invert_permutation(c.order.p, c.n, c.rank.p, c.stream);
  launch_check_unique_ids(c.ids.p, c.order.p, c.n, c.scalars.p + kStatus, c.stream);
  read_scalars(c);
}

// A constraint record as ConstraintSet holds it: the checks of
// validate_plane / _sphere / _box / _cylinder (cpp/core/constraints.cpp:17-80),
// which a set built by add_plane etc. meets (a plane's inward normal is
// stored normalized, constraints.cpp:169-186).
void validate_constraint(const msb_constraint& k) {
  const auto finite3 = [](const msb_vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
  if (!std::isfinite(k.coefficient) || k.coefficient <= 0.0f) {
    throw std::invalid_argument("constraint coefficient must be finite and positive");
  }
  const bool region_ok = k.allowed_region == MSB_REGION_OUTSIDE || k.allowed_region == MSB_REGION_INSIDE;
  switch (k.kind) {
    case MSB_CONSTRAINT_PLANE: {
      if (!finite3(k.a) || !finite3(k.b)) throw std::invalid_argument("plane contains an invalid field");
      // norm() of types.hpp in FP32: sqrt((x*x + y*y) + z*z).
      const float length = std::sqrt((k.b.x * k.b.x + k.b.y * k.b.y) + k.b.z * k.b.z);
      if (std::fabs(length - 1.0f) > 1.0e-5f) throw std::invalid_argument("plane inward normal is not normalized");
      return;
    }
    case MSB_CONSTRAINT_SPHERE:
      if (!finite3(k.a) || !std::isfinite(k.radius) || k.radius <= 0.0f) {
        throw std::invalid_argument("sphere contains invalid geometry");
      }
      break;
    case MSB_CONSTRAINT_BOX:
      if (!finite3(k.a) || !std::isfinite(k.b.x) || !(k.b.x > 0.0f) || !std::isfinite(k.b.y) || !(k.b.y > 0.0f) ||
          !std::isfinite(k.b.z) || !(k.b.z > 0.0f)) {
        throw std::invalid_argument("box contains invalid geometry");
      }
      break;
    default:
      if (!finite3(k.a) || !std::isfinite(k.radius) || k.radius <= 0.0f || !std::isfinite(k.half_height) ||
          k.half_height <= 0.0f) {
        throw std::invalid_argument("cylinder contains invalid geometry");
      }
      break;
  }
  if (!region_ok) throw std::invalid_argument("constraint uses an unknown allowed region");
}

void load_constraints(Ctx& c, const msb_constraint* constraints, std::uint64_t count) {
  if (count > 0 && constraints == nullptr) throw std::invalid_argument("constraint array must not be null");
  std::vector<DeviceConstraint> sorted(count);
  for (std::uint64_t i = 0; i < count; ++i) {
    const auto& k = constraints[i];
    if (k.kind > MSB_CONSTRAINT_CYLINDER) throw std::invalid_argument("constraint kind is invalid");
    if (k.id == 0) throw std::invalid_argument("constraint identifier is invalid");
    validate_constraint(k);
    static_assert(sizeof(DeviceConstraint) == sizeof(msb_constraint));
    std::memcpy(&sorted[i], &k, sizeof(k));
  }
  // Within a cell, the reference emits planes, spheres, boxes and cylinders in
  // insertion order and then sorts stably by constraint id; ids are unique,
  // so sorting the constraints by id gives the same order.
  std::stable_sort(sorted.begin(), sorted.end(), [](const auto& l, const auto& r) { return l.id < r.id; });
  for (std::size_t i = 1; i < sorted.size(); ++i) {
    if (sorted[i].id == sorted[i - 1].id) throw std::invalid_argument("constraint identifiers must be unique");
  }
  c.constraint_count = std::uint32_t(count);
  if (count > 0) {
    c.constraints.ensure(count);
    check(cudaMemcpyAsync(c.constraints.p, sorted.data(), count * sizeof(DeviceConstraint), cudaMemcpyHostToDevice,
                          c.stream),
          "copy constraints");
    sync(c);
  }
}

// ---- contact search ------------------------------------------------------

// Touches at prm.margin among the candidate pairs in c.pairs[0, pair_count):
// a count pass, its scan and a fill pass into out[0, count); returns count.
std::uint32_t narrow_touches(Ctx& c, const GeometryView& g, ContactSearchParams prm, const uint2* pairs,
                             std::uint32_t pair_count, DBuf<Touch>& out) {
  if (pair_count == 0) return 0;
  c.pair_counts.ensure(pair_count + 1ull);
  c.pair_offsets.ensure(pair_count + 1ull);
  c.temp.ensure(scan_temp_words(pair_count + 1ull) + 64);
  check(cudaMemsetAsync(c.pair_counts.p + pair_count, 0, 4, c.stream), "memset");
  launch_narrow_phase(g, pairs, pair_count, prm, c.pair_counts.p, nullptr, nullptr, c.stream, c.scalars.p + kStatus);
  exclusive_scan(c.pair_counts.p, c.pair_offsets.p, pair_count + 1ull, c.temp.p, c.stream);
  // The touch total and the status words in one round trip.
  check(cudaMemcpyAsync(c.host_scalars + kScalarCount + 5, c.pair_offsets.p + pair_count, 4, cudaMemcpyDeviceToHost,
                        c.stream),
        "read");
  read_scalars(c);
  const std::uint32_t touch_count = c.host_scalars[kScalarCount + 5];
  if (touch_count == 0) return 0;
  out.ensure(touch_count + 1ull);
  launch_narrow_phase(g, pairs, pair_count, prm, nullptr, c.pair_offsets.p, out.p, c.stream, c.scalars.p + kStatus);
  return touch_count;
}

// The grid of `g` with boxes padded by `margin`: the cells' FP64 boxes, the
// grid parameters, and the cells sorted by bucket with their FP32 boxes.
void build_grid(Ctx& c, const GeometryView& g, float margin) {
  const std::uint32_t n = c.n;
  const std::uint32_t partials = bound_partials(n);
  c.bounds.ensure(6ull * n);
  c.bound_partials.ensure(10ull * partials);
  c.grid.ensure(1);
  launch_cell_bounds(g, margin, c.bounds.p, c.bound_partials.p, c.stream);
  const std::uint64_t capacity = grid_bucket_capacity(n);
  launch_grid_setup(c.bound_partials.p, partials, n, capacity, c.grid.p, c.stream, c.box_scale, c.colonies);
  c.cell_bucket.ensure(n);
  c.coords.ensure(3ull * n);
  c.bucket_counts.ensure(capacity);
  c.bucket_starts.ensure(capacity);
  c.bucket_fill.ensure(capacity);
  c.sorted_lo.ensure(n);
  c.sorted_hi.ensure(n);
  c.sorted_id.ensure(n);
  c.temp.ensure(scan_temp_words(capacity) + sort_temp_words(n) + 64);
  check(cudaMemsetAsync(c.bucket_counts.p, 0, capacity * 4, c.stream), "memset");
  check(cudaMemsetAsync(c.bucket_fill.p, 0, capacity * 4, c.stream), "memset");
  launch_bin_cells(g, c.bounds.p, c.grid.p, c.cell_bucket.p, c.coords.p, c.bucket_counts.p, c.stream);
  exclusive_scan(c.bucket_counts.p, c.bucket_starts.p, capacity, c.temp.p, c.stream);
  launch_scatter_cells(g, c.bounds.p, c.cell_bucket.p, c.bucket_starts.p, c.bucket_fill.p, c.sorted_lo.p, c.sorted_hi.p,
                       c.sorted_id.p, c.stream);
}

// Cell-pair touches of `geometry` at prm.margin into out[0, count); returns
// count.  The broad phase pads the boxes by `candidate_margin` >= prm.margin;
// with a wider one the narrow phase first applies the box test at
// prm.margin, so the touches are those of a search at prm.margin.  With
// `keep` the candidate pairs stay in c.kept_pairs.
std::uint32_t find_pairs(Ctx& c, Geometry& geometry, ContactSearchParams prm, DBuf<Touch>& out,
                         float candidate_margin = -1.0f, bool keep = false) {
  candidate_margin = std::max(candidate_margin, prm.margin);
  const std::uint32_t n = c.n;
  if (keep) {
    c.kept_valid = true;
    c.kept_count = 0;
    c.kept_margin = candidate_margin;
  }
  if (n < 2) return 0;
  const GeometryView g = view_of(c, geometry);
  build_grid(c, g, candidate_margin);
  c.cand_counts.ensure(n + 1ull);
  c.cand_offsets.ensure(n + 1ull);
  c.slab.ensure(std::size_t(n) * kSlabPartners);
  check(cudaMemsetAsync(c.cand_counts.p + n, 0, 4, c.stream), "memset");
  reset_scalars(c);
  // One enumeration: counts, and the partners of cells with at most
  // kSlabPartners of them in the slab (cand_counts[n] counts the others).
  launch_broad_phase(g, c.bounds.p, c.grid.p, c.bucket_starts.p, c.sorted_lo.p, c.sorted_hi.p, c.sorted_id.p,
                     c.coords.p, c.rank.p, c.cand_counts.p, nullptr, nullptr, c.scalars.p + kStatus, c.stream,
                     c.slab.p);
  exclusive_scan(c.cand_counts.p, c.cand_offsets.p, n + 1ull, c.temp.p, c.stream);
  // grid status, the candidate total and the cells with many partners
  GridParams grid{};
  check(cudaMemcpyAsync(&c.host_scalars[kScalarCount + 2], c.cand_offsets.p + n, 4, cudaMemcpyDeviceToHost, c.stream),
        "read");
  check(cudaMemcpyAsync(&c.host_scalars[kScalarCount + 3], c.cand_counts.p + n, 4, cudaMemcpyDeviceToHost, c.stream),
        "read");
  check(cudaMemcpyAsync(&grid, c.grid.p, sizeof(GridParams), cudaMemcpyDeviceToHost, c.stream), "read grid");
  read_scalars(c);
  if (grid.status == 1) throw std::invalid_argument("cell geometry is not finite");
  if (grid.status != 0) throw DeviceCheckError("grid bucket capacity exceeded");
  const std::uint32_t pair_count = c.host_scalars[kScalarCount + 2];
  const std::uint32_t crowded = c.host_scalars[kScalarCount + 3];
  if (pair_count == 0) return 0;
  c.pairs.ensure(pair_count);
  launch_compact_slab(n, c.cand_counts.p, c.cand_offsets.p, c.order.p, c.slab.p, c.pairs.p, c.stream);
  if (crowded > 0) {
    launch_broad_phase(g, c.bounds.p, c.grid.p, c.bucket_starts.p, c.sorted_lo.p, c.sorted_hi.p, c.sorted_id.p,
                       c.coords.p, c.rank.p, c.cand_counts.p, c.cand_offsets.p, c.pairs.p, c.scalars.p + kStatus,
                       c.stream, c.slab.p);
  }
  if (candidate_margin > prm.margin) prm.box_margin = prm.margin;
  const std::uint32_t touch_count = narrow_touches(c, g, prm, c.pairs.p, pair_count, out);
  if (keep) {
    std::swap(c.pairs, c.kept_pairs);
    std::swap(c.cand_offsets, c.kept_offsets);  // the kept pairs by first cell's rank
    c.kept_count = pair_count;
  }
  return touch_count;
}

// Wall touches appended at out[base, base + count); returns count.
std::uint32_t find_walls(Ctx& c, Geometry& geometry, float margin, float epsilon, bool every_face, DBuf<Touch>& out,
                         std::uint32_t base) {
  const std::uint32_t n = c.n;
  if (n == 0 || c.constraint_count == 0) return 0;
  const GeometryView g = view_of(c, geometry);
  c.wall_counts.ensure(n + 1ull);
  c.wall_offsets.ensure(n + 1ull);
  c.temp.ensure(scan_temp_words(n + 1ull) + 64);
  check(cudaMemsetAsync(c.wall_counts.p + n, 0, 4, c.stream), "memset");
  launch_wall_contacts(g, c.constraints.p, c.constraint_count, margin, epsilon, every_face ? 1u : 0u, c.rank.p,
                       c.wall_counts.p, nullptr, nullptr, c.stream);
  exclusive_scan(c.wall_counts.p, c.wall_offsets.p, n + 1ull, c.temp.p, c.stream);
  const std::uint32_t count = read_u32(c, c.wall_offsets.p + n);
  if (count == 0) return 0;
  out.grow(std::size_t(base) + count + 1, base, c.stream);
  launch_wall_contacts(g, c.constraints.p, c.constraint_count, margin, epsilon, every_face ? 1u : 0u, c.rank.p,
                       nullptr, c.wall_offsets.p, out.p + base, c.stream);
  return count;
}

// find_touches (contact_dynamics.cpp:176-210): pairs then constraint faces.
// With `keep` the pair search's candidates (at `candidate_margin`, at least
// `margin`) stay for the substep's re-checks.
std::uint32_t find_touches(Ctx& c, Geometry& geometry, const msb_contact_parameters& cp,
                           const msb_constraint_contact_parameters& wp, float margin, DBuf<Touch>& out,
                           float candidate_margin = -1.0f, bool keep = false) {
  const ContactSearchParams prm{margin, cp.parallel_sine_threshold, cp.degeneracy_epsilon};
  const std::uint32_t pairs = find_pairs(c, geometry, prm, out, candidate_margin, keep);
  const std::uint32_t walls = find_walls(c, geometry, margin, wp.degeneracy_epsilon, true, out, pairs);
  return pairs + walls;
}

// The touches of find_touches at margin 0 on `geometry`, with the pair
// candidates taken from the substep's kept list instead of a new search.
// Exact when no cell's box face moved more than (kept_margin - 1e-6) / 2
// since the kept search: a pair missing from the list had boxes padded by
// kept_margin that did not overlap, so their unpadded boxes, each moved by
// less than half of that, still do not, and the pair is no candidate of the
// search at margin 0 either.  Listed pairs get that search's box test here.
std::uint32_t find_touches_kept(Ctx& c, Geometry& geometry, const msb_contact_parameters& cp,
                                const msb_constraint_contact_parameters& wp, DBuf<Touch>& out) {
  ContactSearchParams prm{0.0f, cp.parallel_sine_threshold, cp.degeneracy_epsilon};
  prm.box_margin = 0.0f;
  const std::uint32_t pairs = narrow_touches(c, view_of(c, geometry), prm, c.kept_pairs.p, c.kept_count, out);
  const std::uint32_t walls = find_walls(c, geometry, 0.0f, wp.degeneracy_epsilon, true, out, pairs);
  return pairs + walls;
}

// Fast cells at most, and new pairs at most, for a partial re-search;
// beyond either the re-check runs a full search.  Below kPartialFromCells
// cells a full search costs less than the partial one's fixed part (the grid
// of the current geometry and the fast cells' queries): at 100k capsules of
// the trap colony 285 us against 320-730 us.  Each fast cell's query is one
// thread's walk of its neighbour boxes, so thousands of them cost more than
// the broad phase of every cell (1M capsules: up to 16k fast cells took
// 1.2 ms a query launch against 0.7 ms for the broad phase): at most 1,024.
constexpr std::uint32_t kPartialPairs = 8192;
constexpr std::uint32_t kPartialFromCells = 262144;
std::uint32_t partial_cells(std::uint32_t n) { return std::clamp<std::uint32_t>(n / 1024, 64, 1024); }

// The touches of find_touches at margin 0 on `geometry` when some cells
// moved further than the kept candidates allow.  The kept pairs of two cells
// that did not are still every such pair of the search (by the argument of
// find_touches_kept); the pairs of the others are searched again on a grid
// of `geometry`, and those the kept list lacks (usually none) are merged in,
// in (first id, second id) order; then the constraint faces.  The same
// touches in the same order as a full search.  Returns false, and no
// touches, when more cells or pairs moved than the partial search takes.
bool find_touches_partial(Ctx& c, Geometry& geometry, const msb_contact_parameters& cp,
                          const msb_constraint_contact_parameters& wp, DBuf<Touch>& out, std::uint32_t& count) {
  const std::uint32_t n = c.n;
  if (!c.kept_valid || n < kPartialFromCells) return false;
  const GeometryView from = view_of(c, c.base);
  const GeometryView g = view_of(c, geometry);
  const std::uint32_t cap = partial_cells(n);
  const std::uint32_t kept = c.kept_count;
  if (kept == 0) return false;  // no kept list (nor its offsets) to search beside
  c.fast_flags.ensure(n);
  c.fast_list.ensure(n);
  check(cudaMemsetAsync(c.scalars.p + kFastCount, 0, 4, c.stream), "memset");
  launch_fast_cells(from, g, double(c.kept_margin) - 1.0e-6, c.fast_flags.p, c.fast_list.p, c.scalars.p + kFastCount,
                    c.stream);
  build_grid(c, g, 0.0f);
  c.fast_counts.ensure(cap + 1ull);
  c.fast_offsets.ensure(cap + 1ull);
  c.temp.ensure(scan_temp_words(std::max<std::uint64_t>(cap, kept) + 1ull) + 64);
  check(cudaMemsetAsync(c.fast_counts.p + cap, 0, 4, c.stream), "memset");
  launch_fast_partners(g, c.bounds.p, c.grid.p, c.bucket_starts.p, c.sorted_lo.p, c.sorted_hi.p, c.sorted_id.p,
                       c.coords.p, c.fast_flags.p, c.fast_list.p, c.scalars.p + kFastCount, cap, c.kept_pairs.p,
                       c.kept_offsets.p, c.rank.p, c.fast_counts.p, nullptr, nullptr, c.stream);
  exclusive_scan(c.fast_counts.p, c.fast_offsets.p, cap + 1ull, c.temp.p, c.stream);
  // The fast cells' number, the new pairs' number and the grid's status in one round trip.
  GridParams grid{};
  check(cudaMemcpyAsync(&c.host_scalars[kScalarCount + 5], c.fast_offsets.p + cap, 4, cudaMemcpyDeviceToHost,
                        c.stream),
        "read");
  check(cudaMemcpyAsync(&grid, c.grid.p, sizeof(GridParams), cudaMemcpyDeviceToHost, c.stream), "read grid");
  read_scalars(c);
  if (grid.status == 1) throw std::invalid_argument("cell geometry is not finite");
  if (grid.status != 0) throw DeviceCheckError("grid bucket capacity exceeded");
  const std::uint32_t fast_count = c.host_scalars[kFastCount];
  const std::uint32_t added = c.host_scalars[kScalarCount + 5];
  if (fast_count > cap || added > kPartialPairs) return false;
  ContactSearchParams prm{0.0f, cp.parallel_sine_threshold, cp.degeneracy_epsilon};
  prm.box_margin = 0.0f;
  std::uint32_t pairs = 0;
  if (added == 0) {
    pairs = narrow_touches(c, g, prm, c.kept_pairs.p, kept, out);
  } else {
    c.fast_pairs.ensure(added + 1ull);
    c.fast_sorted.ensure(added + 1ull);
    launch_fast_partners(g, c.bounds.p, c.grid.p, c.bucket_starts.p, c.sorted_lo.p, c.sorted_hi.p, c.sorted_id.p,
                         c.coords.p, c.fast_flags.p, c.fast_list.p, c.scalars.p + kFastCount, cap, c.kept_pairs.p,
                         c.kept_offsets.p, c.rank.p, nullptr, c.fast_offsets.p, c.fast_pairs.p, c.stream);
    c.shift.ensure(kept + 1ull);
    c.shift_scan.ensure(kept + 1ull);
    c.pairs.ensure(std::size_t(kept) + added + 1);
    launch_merge_fast_pairs(c.fast_pairs.p, added, c.fast_sorted.p, c.kept_pairs.p, kept, c.ids.p, c.shift.p,
                            c.shift_scan.p, c.temp.p, c.pairs.p, c.stream);
    pairs = narrow_touches(c, g, prm, c.pairs.p, kept + added, out);
  }
  const std::uint32_t walls = find_walls(c, geometry, 0.0f, wp.degeneracy_epsilon, true, out, pairs);
  count = pairs + walls;
  return true;
}

// Whether the last move allows find_touches_kept.
bool kept_candidates_hold(const Ctx& c) {
  return c.kept_valid && std::isfinite(c.displacement) &&
         2.0 * double(c.displacement) <= double(c.kept_margin) - 1.0e-6;
}

// ---- solve ---------------------------------------------------------------

#ifndef MSB_GRAPH_CLASSES
#define MSB_GRAPH_CLASSES 1, 4, 16, 74, 148, 296, 444, 592, 1184
#endif

// The solve graph for a system of `items` rows or bodies: one per class of
// grid sizes (the smallest class that gives every thread an item, at most
// one resident wave).
SolveGraph& graph_for(Ctx& c, std::uint32_t items) {
  static constexpr int classes[] = {MSB_GRAPH_CLASSES};
  const std::uint32_t wanted = (items + kSolveThreads - 1) / kSolveThreads;
  int index = 0;
  while (index + 1 < int(std::size(classes)) && std::uint32_t(classes[index]) < wanted) ++index;
  if (c.graphs.size() < std::size(classes)) c.graphs.resize(std::size(classes));
  auto& slot = c.graphs[index];
  if (!slot) {
    slot = std::make_unique<SolveGraph>();
    check(cudaError_t(slot->create(c.desc, classes[index], c.stream)), "solve graph");
  }
  return *slot;
}

// Whether a solve over `items` rows or bodies takes the fused relaxation
// (one cooperative launch) rather than the graph with a WHILE node.
bool use_fused_relaxation(Ctx& c, std::uint32_t items) {
  if (c.relaxation == 1) return false;
  if (c.relax_blocks < 0) c.relax_blocks = relax_resident_blocks();
  if (c.relax_blocks <= 0) return false;
  if (c.relaxation == 2) return true;
  return items <= kFusedRelaxationItems;
}

IncidenceArrays incidence_arrays(Ctx& c) {
  return {c.inc_offsets.p, c.inc_a.p, c.inc_b.p, c.inc_constants.p, c.inc_sides.p};
}

void fill_desc(Ctx& c, std::uint32_t row_count, float dt, const msb_growth_load_response& growth, float tolerance,
               std::uint32_t max_iterations, bool with_state = false) {
  SolveDesc& d = *c.host_desc;
  d.rows = c.rows.arrays();
  d.bodies = {c.body_a.p, c.body_b.p, c.drift_a.p, c.drift_b.p};
  d.incidence = incidence_arrays(c);
  d.response = {c.resp_a.p, c.resp_b.p};
  d.multipliers = c.rows.multipliers.p;
  d.gaps = c.rows.gaps.p;
  d.iterate = c.rows.iterate.p;
  d.partials = c.partials.p;
  d.row_count = row_count;
  d.body_count = c.n;
  d.dt = dt;
  d.law = growth.law;
  d.sensitivity = growth.sensitivity;
  d.free_load = growth.free_load;
  d.stall_load = growth.stall_load;
  d.tolerance = tolerance;
  d.max_iterations = max_iterations;
  d.has_drift = c.has_drift ? 1u : 0u;
  if (with_state) {
    // The fused solve resets nothing itself: copy the state part too.
    d.step = 0.0f;
    d.residual = 0.0f;
    d.bound = 0.0f;
    d.iterations = 0;
    d.status = MSB_SOLVE_CONVERGED;
    d.mode = 0;
    d.ticket = 0;
    d.proceed = 0;
    d.handle = 0;
    d.bound_ticket = 0;
    d.bound_bits = 0;
    d.barrier_count = 0;
    d.barrier_generation = 0;
    d.barrier_abort = 0;
    d.check_status = 0;
    check(cudaMemcpyAsync(c.desc, &d, sizeof(SolveDesc), cudaMemcpyHostToDevice, c.stream), "desc");
    return;
  }
  // Copy only the problem part; the state part is reset in the graph.
  check(cudaMemcpyAsync(c.desc, &d, offsetof(SolveDesc, step), cudaMemcpyHostToDevice, c.stream), "desc");
}

void build_system_incidence(Ctx& c, std::uint32_t row_count) {
  const std::size_t entries = 2ull * std::max<std::uint32_t>(row_count, 1);
  c.inc_offsets.ensure(c.n + 1ull);
  c.inc_a.ensure(entries);
  c.inc_b.ensure(entries);
  c.inc_constants.ensure(entries / 2);
  c.inc_sides.ensure(entries / 2);
  c.sort_keys.ensure(entries);
  c.sort_values.ensure(entries);
  c.counts.ensure(c.n + 1ull);
  c.temp.ensure(sort_temp_words(entries) + scan_temp_words(c.n + 1ull) + 64);
  build_incidence(c.rows.arrays(), row_count, c.n, incidence_arrays(c), c.sort_keys.p,
                  c.sort_values.p, c.counts.p, c.temp.p, c.stream, c.scalars.p + kStatus);
}

void build_row_keys(Ctx& c, RowStore& store) {
  c.sort_keys.ensure(std::max<std::uint32_t>(store.count, 1));
  c.counts.ensure(c.n + 1ull);
  store.keyed_offsets.ensure(c.n + 1ull);
  store.keyed_rows.ensure(std::max<std::uint32_t>(store.count, 1));
  c.temp.ensure(sort_temp_words(store.count + 1ull) + scan_temp_words(c.n + 1ull) + 64);
  build_keyed(store.slots.p, store.count, c.n, store.keyed_offsets.p, store.keyed_rows.p, c.sort_keys.p, c.counts.p,
              c.temp.p, c.stream);
}

// Runs the solve graph on c.rows (multipliers in place).  Requires the
// incidence of c.rows and the bodies.
SolveOutcome solve_batch(Ctx& c, float dt, const msb_growth_load_response& growth, std::uint32_t max_iterations);

SolveOutcome solve(Ctx& c, float dt, const msb_growth_load_response& growth, float tolerance,
                   std::uint32_t max_iterations) {
  if (c.colonies > 0) return solve_batch(c, dt, growth, max_iterations);
  const std::uint32_t rows = c.rows.count;
  c.resp_a.ensure(std::max<std::uint32_t>(c.n, 1));
  c.resp_b.ensure(std::max<std::uint32_t>(c.n, 1));
  if (rows == 0) {
    fill_desc(c, 0, dt, growth, tolerance, max_iterations);
    launch_evaluate(c.desc, std::max(1, grid_for(c.n, kSolveThreads)), false, c.stream);
    return {};
  }
  c.partials.ensure(5ull * kMaxPassBlocks);
  const bool fused = use_fused_relaxation(c, std::max(rows, c.n));
  if (fused) {
    // One cooperative launch runs the whole solve (relax_kernel).
    const std::uint32_t wanted = (std::max(rows, c.n) + kSolveThreads - 1) / kSolveThreads;
    const int blocks = std::max(1, std::min({int(wanted), c.relax_blocks, 1184}));
    c.last_blocks = blocks;
    fill_desc(c, rows, dt, growth, tolerance, max_iterations, true);
    check(cudaError_t(launch_relax(*c.host_desc, c.desc, blocks, c.stream)), "solve launch");
  } else {
    auto& graph = graph_for(c, std::max(rows, c.n));
    c.last_blocks = graph.blocks();
    fill_desc(c, rows, dt, growth, tolerance, max_iterations);
    check(cudaError_t(graph.launch(c.stream)), "solve launch");
  }
  // The final multipliers and gaps, and their response (the passes of a
  // solve write only the rows' side terms).
  launch_unpack_iterate(c.desc, c.last_blocks, c.stream);
  launch_evaluate(c.desc, c.last_blocks, false, c.stream);
  check(cudaMemcpyAsync(c.host_desc, c.desc, sizeof(SolveDesc), cudaMemcpyDeviceToHost, c.stream), "read desc");
  sync(c);
  const SolveDesc& d = *c.host_desc;
  if (d.barrier_abort != 0) throw DeviceCheckError("a grid barrier of the relaxation ran out of time");
  if (d.check_status != 0) throw DeviceCheckError("an index check of the relaxation failed");
  if (!fused) count_launch(SolveGraph::loop_launches(d.iterations));
  c.solve_log.push_back({rows, d.iterations, d.status, d.residual});
  if (d.status == 3) throw std::invalid_argument("contact system has no positive diagonal");
  return {d.status, d.iterations, d.residual};
}

// The batched solve over c.rows: rows grouped by colony, one persistent
// launch of clusters (see batch.h), per-colony state read back.  The outcome
// is the batch's worst status and its largest iteration count; each
// colony's iterations accumulate in c.colony_iterations.
msb::BatchDesc batch_desc(Ctx& c, float dt, const msb_growth_load_response& growth, std::uint32_t max_iterations) {
  msb::BatchDesc d{};
  d.rows = c.rows.arrays();
  d.bodies = {c.body_a.p, c.body_b.p, c.drift_a.p, c.drift_b.p};
  d.incidence = incidence_arrays(c);
  d.response = {c.resp_a.p, c.resp_b.p};
  d.multipliers = c.rows.multipliers.p;
  d.gaps = c.rows.gaps.p;
  d.iterate = c.rows.iterate.p;
  d.colony_rows = c.colony_rows.p;
  d.row_offsets = c.colony_row_offsets.p;
  d.cell_offsets = c.colony_offsets.p;
  d.order = c.colony_order.p;
  d.active = c.colony_active.p;
  d.tolerance = c.colony_solve_tolerance.p;
  d.state = c.colony_state.p;
  d.next = c.batch_next.p;
  d.colonies = c.colonies;
  d.dt = dt;
  d.law = growth.law;
  d.sensitivity = growth.sensitivity;
  d.free_load = growth.free_load;
  d.stall_load = growth.stall_load;
  d.max_iterations = max_iterations;
  d.has_drift = c.has_drift ? 1u : 0u;
  return d;
}

void run_batch(Ctx& c, const msb::BatchDesc& d, msb::BatchShape shape, int clusters) {
  check(cudaMemsetAsync(c.batch_next.p, 0, 4, c.stream), "memset");
  check(cudaError_t(launch_batch_solve(d, shape, clusters, c.stream)), "batched solve launch");
}

// The project's autotuner for the batched solve: times each launch shape
// (CTAs per cluster x threads per CTA) on the system at hand, from the same
// start multipliers, and keeps the fastest.
void tune_batch(Ctx& c, const msb::BatchDesc& d) {
  const std::uint32_t rows = c.rows.count;
  c.batch_saved.ensure(std::max<std::uint32_t>(rows, 1));
  check(cudaMemcpyAsync(c.batch_saved.p, c.rows.multipliers.p, rows * 4ull, cudaMemcpyDeviceToDevice, c.stream),
        "save multipliers");
  cudaEvent_t start, stop;
  check(cudaEventCreate(&start), "event");
  check(cudaEventCreate(&stop), "event");
  float best = -1.0f;
  for (const bool lean : {false, true}) for (const int threads : {256, 512}) {
    for (const int cluster : {1, 2, 4, 8, 16}) {
      const msb::BatchShape shape{cluster, threads, lean};
      const int resident = batch_resident_clusters(shape);
      if (resident <= 0) continue;
      const int clusters = std::min<int>(resident, int(c.colonies));
      check(cudaMemcpyAsync(c.rows.multipliers.p, c.batch_saved.p, rows * 4ull, cudaMemcpyDeviceToDevice, c.stream),
            "restore multipliers");
      check(cudaEventRecord(start, c.stream), "event");
      run_batch(c, d, shape, clusters);
      check(cudaEventRecord(stop, c.stream), "event");
      check(cudaEventSynchronize(stop), "event");
      float ms = 0.0f;
      check(cudaEventElapsedTime(&ms, start, stop), "event");
      if (best < 0.0f || ms < best) {
        best = ms;
        c.batch_shape = shape;
        c.batch_clusters = clusters;
      }
    }
  }
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  if (best < 0.0f) throw std::runtime_error("no launch shape of the batched solve fits the device");
  check(cudaMemcpyAsync(c.rows.multipliers.p, c.batch_saved.p, rows * 4ull, cudaMemcpyDeviceToDevice, c.stream),
        "restore multipliers");
  c.batch_tuned = true;
}

SolveOutcome solve_batch(Ctx& c, float dt, const msb_growth_load_response& growth, std::uint32_t max_iterations) {
  const std::uint32_t rows = c.rows.count;
  const std::uint32_t k = c.colonies;
  c.resp_a.ensure(std::max<std::uint32_t>(c.n, 1));
  c.resp_b.ensure(std::max<std::uint32_t>(c.n, 1));
  c.colony_rows.ensure(std::max<std::uint32_t>(rows, 1));
  c.sort_keys.ensure(std::max<std::uint32_t>(rows, 1));
  c.colony_row_counts.ensure(k + 1ull);
  c.colony_row_offsets.ensure(k + 1ull);
  c.temp.ensure(sort_temp_words(rows + 1ull) + scan_temp_words(k + 1ull) + 64);
  check(cudaMemsetAsync(c.colony_row_counts.p, 0, (k + 1ull) * 4, c.stream), "memset");
  launch_colony_row_keys(c.rows.slots.p, rows, c.colony_of_slot.p, c.sort_keys.p, c.colony_rows.p,
                         c.colony_row_counts.p, c.stream);
  exclusive_scan(c.colony_row_counts.p, c.colony_row_offsets.p, k + 1ull, c.temp.p, c.stream);
  if (rows > 1) radix_sort_pairs(c.sort_keys.p, c.colony_rows.p, rows, std::max(1, int(std::bit_width(k))), c.temp.p,
                                 c.stream);
  const msb::BatchDesc d = batch_desc(c, dt, growth, max_iterations);
  if (!c.batch_tuned) tune_batch(c, d);
  // A solve of few colonies (a step's later refinement rounds, where most
  // colonies have settled) runs them on clusters of 16 CTAs: the largest
  // colonies then set the time, and twice the CTAs halve their iteration
  // (256-colony sweep, 3.0M capsules: 100k-row colonies 131 -> 63 us an
  // iteration; solves of 3 colonies 1.8-2.0 -> 1.1 ms, of 83 5.0 -> 4.8 ms).
  // With many colonies the tuned shape's more clusters serve them better.
  c.host_colony_active.resize(k);
  check(cudaMemcpyAsync(c.host_colony_active.data(), c.colony_active.p, k * 4ull, cudaMemcpyDeviceToHost, c.stream),
        "read active colonies");
  sync(c);
  std::uint32_t active = 0;
  for (const std::uint32_t a : c.host_colony_active) active += a != 0u ? 1u : 0u;
  const msb::BatchShape wide{16, 512, true};
  const int wide_clusters = active > 0 && active <= kFewColonies ? batch_resident_clusters(wide) : 0;
  if (wide_clusters > 0) {
    run_batch(c, d, wide, std::min<int>(wide_clusters, int(active)));
  } else {
    run_batch(c, d, c.batch_shape, c.batch_clusters);
  }
  c.host_colony_state.resize(k);
  check(cudaMemcpyAsync(c.host_colony_state.data(), c.colony_state.p, k * sizeof(msb::ColonyState),
                        cudaMemcpyDeviceToHost, c.stream),
        "read colony states");
  sync(c);
  SolveOutcome out{};
  out.status = MSB_SOLVE_CONVERGED;
  std::uint32_t worst = 0;
  float residual = 0.0f;
  for (std::uint32_t i = 0; i < k; ++i) {
    const auto& st = c.host_colony_state[i];
    if (st.status == 3) throw std::invalid_argument("contact system has no positive diagonal");
    c.colony_iterations[i] += st.iterations;
    c.colony_status[i] = st.status;
    out.iterations = std::max(out.iterations, st.iterations);
    residual = std::max(residual, st.residual);
    if (st.status == MSB_SOLVE_BREAKDOWN) {
      worst = 2;
    } else if (st.status != MSB_SOLVE_CONVERGED && worst < 1) {
      worst = 1;
    }
  }
  out.status = worst == 2 ? MSB_SOLVE_BREAKDOWN : (worst == 1 ? MSB_SOLVE_ITERATION_LIMIT : MSB_SOLVE_CONVERGED);
  out.residual = residual;
  c.solve_log.push_back({rows, out.iterations, out.status, residual});
  return out;
}

// ---- the substep and the step -------------------------------------------

struct Attempt {
  bool accepted = false;
  float rotation = 0.0f;
  std::uint32_t refinements = 0;
  std::uint32_t rows = 0;
  float max_overlap = 0.0f;
};

struct Overlaps {
  std::uint32_t candidates = 0;   // touches in c.found
  std::uint32_t overlapping = 0;  // flagged among them
  float max_overlap = 0.0f;
};

// The overlap test of contact_dynamics.cpp:520-548 on the geometry in
// c.state: touches at margin 0 into c.found, flags and their offsets.
Overlaps flag_overlaps(Ctx& c, const msb_contact_parameters& cp, const msb_constraint_contact_parameters& wp,
                       const msb_contact_dynamics_parameters& p) {
  Overlaps o;
  mark(c, kPhaseSearch);
  if (c.search_reuse < 2 && kept_candidates_hold(c)) {
    o.candidates = find_touches_kept(c, c.state, cp, wp, c.found);
    ++c.searches[1];
  } else if (c.search_reuse < 1 && find_touches_partial(c, c.state, cp, wp, c.found, o.candidates)) {
    ++c.searches[2];
  } else {
    o.candidates = find_touches(c, c.state, cp, wp, 0.0f, c.found);
    ++c.searches[0];
  }
  mark(c, kPhaseMove);
  c.flags.ensure(o.candidates + 1ull);
  c.flag_offsets.ensure(o.candidates + 1ull);
  reset_scalars(c);
  check(cudaMemsetAsync(c.flags.p + o.candidates, 0, 4, c.stream), "memset");
  if (c.colonies > 0) {
    launch_colony_reset_overlap(c.colonies, c.colony_active.p, c.colony_overlap.p, c.stream);
    check(cudaMemsetAsync(c.colony_flagged.p, 0, c.colonies * 4ull, c.stream), "memset");
  }
  launch_recheck(c.found.p, o.candidates, c.rows.keyed(), c.slack.p, p.wall_stiffness, p.contact_stiffness,
                 c.flags.p, c.scalars.p + kOverlapBits, c.stream, colonies_of(c));
  c.temp.ensure(scan_temp_words(o.candidates + 1ull) + 64);
  exclusive_scan(c.flags.p, c.flag_offsets.p, o.candidates + 1ull, c.temp.p, c.stream);
  check(cudaMemcpyAsync(c.host_scalars + kScalarCount + 4, c.flag_offsets.p + o.candidates, 4,
                        cudaMemcpyDeviceToHost, c.stream),
        "read");
  read_scalars(c);
  o.overlapping = c.host_scalars[kScalarCount + 4];
  o.max_overlap = bits_to_float(c.host_scalars[kOverlapBits]);
  // A batch's colonies with nothing flagged leave the following rounds'
  // searches: their rows are final, their solves converge at once and their
  // moves repeat.
  if (c.colonies > 0 && o.overlapping > 0) launch_colony_refine(c.colonies, c.colony_flagged.p, c.colony_active.p, c.stream);
  return o;
}

// Appends rows for the flagged touches, linearized at c.trial, with offsets
// moved by -dt * the rate that `response` predicts.
void append_overlap_rows(Ctx& c, const Overlaps& o, const ResponseArrays& response, const RowBuild& build) {
  mark(c, kPhaseRows);
  c.flagged.ensure(o.overlapping);
  launch_gather_flagged(c.found.p, o.candidates, c.flags.p, c.flag_offsets.p, c.flagged.p, c.stream);
  const std::uint32_t base_row = c.rows.count;
  c.rows.grow(std::size_t(base_row) + o.overlapping, c.stream);
  launch_make_rows(c.flagged.p, o.overlapping, c.trial.view(), build, &response, c.rows.arrays(), base_row,
                   c.rows.partner.p, c.rows.multipliers.p, c.scalars.p + kOverlapBits, c.stream, colonies_of(c));
  c.rows.count = base_row + o.overlapping;
  build_row_keys(c, c.rows);
}

float from_ordered(std::uint32_t u) {
  const std::uint32_t b = (u & 0x80000000u) != 0 ? (u & 0x7FFFFFFFu) : ~u;
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

// Neighbour features of the cells in `geometry` into c.features: a grid of
// mlp::kBinSide bins over the centres (wider when the centres are sparse, so
// that bins never outnumber four per cell), cells counting-sorted by bin.
void compute_features(Ctx& c, GeometryBuffers geometry) {
  const std::uint32_t n = c.n;
  c.features.ensure(std::size_t(std::max<std::uint32_t>(n, 1)) * mlp::kInput);
  if (n == 0) return;
  c.knn_bounds.ensure(4);
  mlp::launch_centre_bounds(n, geometry.pos_len, c.knn_bounds.p, c.stream);
  check(cudaMemcpyAsync(c.host_scalars + kScalarCount + 8, c.knn_bounds.p, 16, cudaMemcpyDeviceToHost, c.stream),
        "read bounds");
  sync(c);
  const float x0 = from_ordered(c.host_scalars[kScalarCount + 8]);
  const float y0 = from_ordered(c.host_scalars[kScalarCount + 9]);
  const float x1 = from_ordered(c.host_scalars[kScalarCount + 10]);
  const float y1 = from_ordered(c.host_scalars[kScalarCount + 11]);
  if (!std::isfinite(x0) || !std::isfinite(y0) || !std::isfinite(x1) || !std::isfinite(y1)) {
    throw std::invalid_argument("cell centres must be finite");
  }
  double side = mlp::kBinSide;
  const double area = (double(x1 - x0) + side) * (double(y1 - y0) + side);
  const double max_bins = 4.0 * n + 64.0;
  if (area / (side * side) > max_bins) side = std::sqrt(area / max_bins) * 1.01;
  const auto nx = std::uint32_t(std::floor(double(x1 - x0) / side)) + 1;
  const auto ny = std::uint32_t(std::floor(double(y1 - y0) / side)) + 1;
  const std::uint32_t bins = nx * ny;
  c.knn_keys.ensure(n);
  c.knn_values.ensure(n);
  c.knn_counts.ensure(bins + 1ull);
  c.knn_offsets.ensure(bins + 1ull);
  c.temp.ensure(sort_temp_words(n) + scan_temp_words(bins + 1ull) + 64);
  check(cudaMemsetAsync(c.knn_counts.p, 0, (bins + 1ull) * 4, c.stream), "memset");
  c.knn_centres.ensure(n);
  mlp::Grid grid{x0, y0, float(1.0 / side), nx, ny, c.knn_offsets.p, c.knn_values.p, c.knn_centres.p};
  mlp::launch_bin_keys(n, geometry.pos_len, grid, c.knn_keys.p, c.knn_values.p, c.knn_counts.p, c.stream);
  exclusive_scan(c.knn_counts.p, c.knn_offsets.p, bins + 1ull, c.temp.p, c.stream);
  const int bits = std::max(1, int(std::bit_width(bins)));
  radix_sort_pairs(c.knn_keys.p, c.knn_values.p, n, bits, c.temp.p, c.stream);
  mlp::launch_sorted_centres(n, geometry.pos_len, c.knn_values.p, c.knn_centres.p, c.stream);
  mlp::launch_features(n, geometry.pos_len, geometry.dir_rad, grid, c.features.p, c.stream);
}

// The network's motion guess for the step from the geometry in c.state.
void learned_guess(Ctx& c, float dt) {
  const std::uint32_t n = c.n;
  mark(c, kPhaseGuess);
  compute_features(c, c.state.view());
  c.net_outputs.ensure(3ull * std::max<std::uint32_t>(n, 1));
  c.guess.ensure(std::max<std::uint32_t>(n, 1));
  check(cudaError_t(mlp::launch_forward_tc(c.net_weights.p, c.net_biases.p, c.features.p, n, c.net_outputs.p,
                                           nullptr, c.scalars.p + kStatus, c.stream)),
        "warm-start network");
  mlp::launch_outputs_to_guess(n, c.net_outputs.p, c.net_scale, c.state.dir_rad.p, c.guess.p, c.stream);
  check(cudaGetLastError(), "warm-start network");
  c.guess_cells = n;
  c.guess_dt = dt;
  c.has_guess = true;
}

// Start multipliers moved toward the forces a motion guess asks of each
// body (guess_forces_kernel): the response of the current multipliers, the
// guessed response, and one distribution pass per body.
void guess_forces(Ctx& c, float dt, const msb_growth_load_response& growth) {
  const std::uint32_t n = c.n;
  const std::uint32_t rows = c.rows.count;
  if (rows == 0) return;
  mark(c, kPhaseRows);
  c.resp_a.ensure(n);
  c.resp_b.ensure(n);
  c.guess_a.ensure(n);
  c.guess_b.ensure(n);
  c.guess_delta.ensure(rows);
  fill_desc(c, rows, dt, growth, 0.0f, 0);
  launch_evaluate(c.desc, std::max(1, grid_for(n, kSolveThreads)), false, c.stream);
  const BodyArrays bodies{c.body_a.p, c.body_b.p, c.drift_a.p, c.drift_b.p};
  const ResponseArrays guess{c.guess_a.p, c.guess_b.p};
  launch_guess_response(n, c.guess.p, bodies, c.guess_dt, guess, c.stream);
  launch_guess_forces(n, rows, incidence_arrays(c), bodies, {c.resp_a.p, c.resp_b.p}, guess,
                      c.rows.slots.p, c.guess_delta.p, c.rows.multipliers.p, c.stream);
}

Attempt advance_substep(Ctx& c, float dt, const msb_contact_dynamics_parameters& p, const msb_contact_parameters& cp,
                        const msb_constraint_contact_parameters& wp, bool probe, std::uint64_t& iterations) {
  const std::uint32_t n = c.n;
  c.has_drift = false;  // no drift unless flow drift writes it below
  if (c.colonies > 0) {
    // Every colony takes part in the substep's first search and test.
    check(cudaMemsetAsync(c.colony_active.p, 0xFF, c.colonies * 4ull, c.stream), "memset");
  }
  c.body_a.ensure(n);
  c.body_b.ensure(n);
  c.drift_a.ensure(n);
  c.drift_b.ensure(n);
  mark(c, kPhaseRows);
  launch_make_bodies(n, c.state.view(), c.growth.p, c.fixed.p, c.initial.view(), p.drag,
                     {c.body_a.p, c.body_b.p, c.drift_a.p, c.drift_b.p}, c.stream, colonies_of(c));
  if (p.flow_drift != 0) {
    // The flow's drift over this substep from its starting geometry
    // (contact_dynamics.cpp:426-431).
    launch_flow_drift(n, c.state.view(), c.fixed.p, c.flow, dt, {c.body_a.p, c.body_b.p, c.drift_a.p, c.drift_b.p},
                      c.scalars.p + kStatus, c.stream);
    c.has_drift = true;
  }
  mark(c, kPhaseSearch);
  // The first search keeps its candidates, padded by kRecheckReach more than
  // the candidate margin, for the overlap re-checks of the refinement rounds
  // (in a batch, those of the colonies still searched).
  const std::uint32_t found = find_touches(c, c.state, cp, wp, p.candidate_margin, c.touches,
                                           p.candidate_margin + (c.colonies > 0 ? kBatchRecheckReach : kRecheckReach), true);
  mark(c, kPhaseRows);
  c.rows.count = 0;
  c.rows.ensure(std::max<std::uint32_t>(found, 1));
  reset_scalars(c);
  const RowBuild build{p.wall_stiffness, p.contact_stiffness, p.max_overlap_recovery, dt};
  if (c.colonies > 0) check(cudaMemsetAsync(c.colony_overlap.p, 0, c.colonies * 4ull, c.stream), "memset");
  launch_make_rows(c.touches.p, found, c.base.view(), build, nullptr, c.rows.arrays(), 0, c.rows.partner.p,
                   c.rows.multipliers.p, c.scalars.p + kOverlapBits, c.stream, colonies_of(c));
  c.rows.count = found;
  const float tolerance = effective_overlap_tolerance(p);
  c.slack.ensure(1);
  launch_slack(c.scalars.p + kOverlapBits, tolerance, p.max_overlap_recovery, c.slack.p, c.stream);
  if (c.colonies > 0) {
    launch_colony_slack(c.colonies, c.colony_overlap.p, c.colony_tolerance.p, p.max_overlap_recovery,
                        c.colony_slack.p, c.stream);
  }
  build_row_keys(c, c.rows);
  const KeyedLists memory = c.memory.keyed();
  const MemoryCells cells{c.memory_first_ids.p, c.memory_partner_ids.p, c.ids.p, c.memory_cells};
  launch_warm_start(found, c.rows.slots.p, c.rows.keyed(), c.has_memory ? &memory : nullptr, cells, c.rows.multipliers.p,
                    c.stream);
  const float solve_tolerance = kSolveToleranceFraction * tolerance;
  Attempt attempt;
  for (std::uint32_t refinement = 0; refinement <= p.max_refinements; ++refinement) {
    mark(c, kPhaseIncidence);
    build_system_incidence(c, c.rows.count);
    if (refinement == 0 && (c.warm_start_mode & (kWarmGuess | kWarmLearned)) != 0 && c.has_guess) {
      guess_forces(c, dt, p.growth);
    }
    mark(c, kPhaseSolve);
    std::uint32_t remaining = p.max_iterations;
    bool solved = false;
    if (probe && refinement == 0 && remaining > kRotationProbeIterations) {
      const auto early = solve(c, dt, p.growth, solve_tolerance, kRotationProbeIterations);
      iterations += early.iterations;
      remaining -= early.iterations;
      if (early.status == MSB_SOLVE_BREAKDOWN) break;
      if (early.status != MSB_SOLVE_CONVERGED) {
        reset_scalars(c);
        launch_largest_rotation(n, {c.resp_a.p, c.resp_b.p}, dt, c.scalars.p + kRotationBits, c.stream);
        read_scalars(c);
        attempt.rotation = bits_to_float(c.host_scalars[kRotationBits]);
        if (attempt.rotation > kMaximumSubstepRotation) break;
      } else {
        // A second solve from converged multipliers takes no iteration.
        solved = true;
      }
    }
    if (!solved) {
      const auto full = solve(c, dt, p.growth, solve_tolerance, remaining);
      iterations += full.iterations;
      if (full.status != MSB_SOLVE_CONVERGED) break;
    }
    // Move from the base geometry under the response of the solution.
    mark(c, kPhaseMove);
    c.trial.ensure(n);
    reset_scalars(c);
    launch_move(n, c.base.view(), {c.resp_a.p, c.resp_b.p}, dt, c.trial.view(), c.scalars.p + kRotationBits,
                c.scalars.p + kInvalid, c.scalars.p + kStatus, c.stream, c.scalars.p + kDisplacementBits);
    read_scalars(c);
    attempt.rotation = bits_to_float(c.host_scalars[kRotationBits]);
    c.displacement = bits_to_float(c.host_scalars[kDisplacementBits]);
    if (c.host_scalars[kInvalid] != 0) break;
    launch_restore(n, c.trial.view(), c.state.view(), c.scalars.p + kStatus, c.stream);

    const Overlaps found_overlaps = flag_overlaps(c, cp, wp, p);
    if (found_overlaps.overlapping == 0) {
      if (c.colonies > 0) {
        // Each colony's deepest overlap at the accepted geometry and its rows.
        std::vector<std::uint32_t> bits(c.colonies);
        c.colony_rows_at_accept.resize(c.colonies);
        check(cudaMemcpyAsync(bits.data(), c.colony_overlap.p, c.colonies * 4ull, cudaMemcpyDeviceToHost, c.stream),
              "read overlaps");
        check(cudaMemcpyAsync(c.colony_rows_at_accept.data(), c.colony_row_counts.p, c.colonies * 4ull,
                              cudaMemcpyDeviceToHost, c.stream),
              "read rows");
        sync(c);
        c.colony_max_overlap.resize(c.colonies);
        for (std::uint32_t i = 0; i < c.colonies; ++i) c.colony_max_overlap[i] = bits_to_float(bits[i]);
      }
      attempt.accepted = true;
      attempt.refinements = refinement;
      attempt.rows = c.rows.count;
      attempt.max_overlap = found_overlaps.max_overlap;
      return attempt;
    }
    // Rows for the new overlaps, linearized at the trial geometry, with
    // offsets that the multipliers of the move predict (contact_dynamics.cpp:567-578).
    append_overlap_rows(c, found_overlaps, {c.resp_a.p, c.resp_b.p}, build);
  }
  launch_restore(n, c.base.view(), c.state.view(), c.scalars.p + kStatus, c.stream);
  reset_scalars(c);
  attempt.accepted = false;
  return attempt;
}

void copy_geometry(Ctx& c, Geometry& dst, Geometry& src) {
  dst.ensure(c.n);
  check(cudaMemcpyAsync(dst.pos_len.p, src.pos_len.p, c.n * sizeof(float4), cudaMemcpyDeviceToDevice, c.stream), "copy");
  check(cudaMemcpyAsync(dst.dir_rad.p, src.dir_rad.p, c.n * sizeof(float4), cudaMemcpyDeviceToDevice, c.stream), "copy");
}

struct StepOutcome {
  msb_contact_dynamics_report report{};
};

// detail::advance_contact_dynamics (contact_dynamics.cpp:676-782) over the
// cells loaded in c.state.  Leaves the final geometry in c.state and the
// outputs in c.out_*.
StepOutcome advance(Ctx& c, float dt, const msb_contact_dynamics_parameters& p, const msb_contact_parameters& cp,
                    const msb_constraint_contact_parameters& wp) {
  StepOutcome out;
  const std::uint32_t n = c.n;
  c.out_velocities.ensure(3ull * std::max<std::uint32_t>(n, 1));
  c.out_loads.ensure(std::max<std::uint32_t>(n, 1));
  c.out_increments.ensure(std::max<std::uint32_t>(n, 1));
  if (n == 0) return out;
  check(cudaMemsetAsync(c.out_velocities.p, 0, 12ull * n, c.stream), "memset");
  check(cudaMemsetAsync(c.out_loads.p, 0, 4ull * n, c.stream), "memset");
  check(cudaMemsetAsync(c.out_increments.p, 0, 4ull * n, c.stream), "memset");
  if (dt == 0.0f) return out;
  copy_geometry(c, c.initial, c.state);
  copy_geometry(c, c.base, c.state);
  if ((c.warm_start_mode & kWarmLearned) != 0) {
    if (!c.has_network) throw std::invalid_argument("the learned warm start needs a network (msb_set_warm_start_network)");
    learned_guess(c, dt);
  }
  if ((c.warm_start_mode & kWarmCarry) == 0) {
    c.has_memory = false;
    c.memory.count = 0;
  }

  reset_scalars(c);
  launch_growth_bound(n, c.state.view(), c.growth.p, dt, c.scalars.p + kGrowthBits, c.stream);
  read_scalars(c);
  const float growth = bits_to_float(c.host_scalars[kGrowthBits]);
  float pieces = std::max(1.0f, std::ceil(growth / p.max_growth_fraction));
  if (p.flow_drift != 0 && c.flow_travel_limit > 0.0f) {
    // No cell drifts more than the travel limit in a substep
    // (contact_dynamics.cpp:708-714).
    reset_scalars(c);
    launch_flow_speed(n, c.state.view(), c.fixed.p, c.flow, c.scalars.p + kGrowthBits, c.scalars.p + kStatus,
                      c.stream);
    read_scalars(c);
    const float speed = bits_to_float(c.host_scalars[kGrowthBits]);
    pieces = std::max(pieces, std::ceil(speed * dt / c.flow_travel_limit));
  }
  if (!std::isfinite(pieces)) throw std::runtime_error("contact dynamics growth per step is not finite");
  const float longest = dt / pieces;
  const float shortest = std::ldexp(longest, -int(p.max_step_halvings));
  double remaining = double(dt);
  float length = longest;
  float proven = 0.0f;
  c.accepted_a.ensure(n);
  c.accepted_b.ensure(n);
  while (remaining > 0.0) {
    if (double(length) >= remaining * (1.0 - 1.0e-6)) length = float(remaining);
    const auto attempt = advance_substep(c, length, p, cp, wp, length > proven, out.report.iterations);
    if (!attempt.accepted) {
      const float excess = attempt.rotation / kPlannedSubstepRotation;
      const std::uint32_t halvings = excess > 2.0f ? std::uint32_t(std::ceil(std::log2(excess))) : 1u;
      const float failed = length;
      length = std::ldexp(length, -int(std::min<std::uint32_t>(halvings, 64)));
      out.report.halvings += halvings;
      if (length < shortest) {
        throw std::runtime_error("contact dynamics did not resolve the contacts of a substep of " +
                                 std::to_string(failed));
      }
      continue;
    }
    remaining -= double(length);
    proven = std::max(proven, length);
    std::swap(c.base, c.trial);  // base <- the accepted trial geometry
    check(cudaMemcpyAsync(c.accepted_a.p, c.resp_a.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, c.stream), "copy");
    check(cudaMemcpyAsync(c.accepted_b.p, c.resp_b.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, c.stream), "copy");
    ++out.report.substeps;
    out.report.refinements += attempt.refinements;
    out.report.max_rows = std::max<std::uint64_t>(out.report.max_rows, attempt.rows);
    out.report.max_overlap = attempt.max_overlap;
    std::swap(c.rows, c.memory);  // forces <- this substep's rows
    c.has_memory = true;
    c.memory_cells = n;
    c.memory_first_ids.ensure(std::max<std::uint32_t>(c.memory.count, 1));
    c.memory_partner_ids.ensure(std::max<std::uint32_t>(c.memory.count, 1));
    launch_memory_ids(c.memory.count, c.memory.slots.p, c.memory.partner.p, c.ids.p, c.memory_first_ids.p,
                      c.memory_partner_ids.p, c.stream);
    if (attempt.refinements <= kEasyRefinements && 2.0f * attempt.rotation <= kPlannedSubstepRotation) {
      length = std::min(longest, length * 2.0f);
    }
  }
  launch_outputs(n, {c.accepted_a.p, c.accepted_b.p}, c.base.view(), c.initial.view(), c.out_velocities.p,
                 c.out_loads.p, c.out_increments.p, c.stream);
  return out;
}

// Pinned download space for a step's results with host buffers: 7 geometry
// arrays and 5 output floats per cell, each array 256-byte aligned.
void prepare_downloads(Ctx& c, bool device_pointers) {
  c.pending.clear();
  if (!device_pointers) c.download.ensure(48ull * c.n + 12 * 256);
}

void write_back(Ctx& c, msb_cell_arrays& cells, bool device_pointers, std::size_t& at) {
  const std::size_t n = c.n;
  if (n == 0) return;
  launch_unpack_cells(c.n, c.state.view(), c.staging[0].p, c.staging[1].p, c.staging[2].p, c.staging[3].p,
                      c.staging[4].p, c.staging[5].p, c.staging[6].p, c.stream);
  float* dst[7] = {cells.position_x,  cells.position_y,  cells.position_z, cells.direction_x,
                   cells.direction_y, cells.direction_z, cells.lengths};
  for (int k = 0; k < 7; ++k) {
    if (device_pointers) {
      check(cudaMemcpyAsync(dst[k], c.staging[k].p, n * 4, cudaMemcpyDeviceToDevice, c.stream), "copy back");
    } else {
      stage_download(c, dst[k], c.staging[k].p, n * 4, at);
    }
  }
}

void write_outputs(Ctx& c, msb_contact_dynamics_outputs* outputs, bool device_pointers, std::size_t& at) {
  if (outputs == nullptr || c.n == 0) return;
  const std::size_t n = c.n;
  const auto copy = [&](void* dst, const void* src, std::size_t bytes) {
    if (dst == nullptr) return;
    if (device_pointers) {
      check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c.stream), "copy out");
    } else {
      stage_download(c, dst, src, bytes, at);
    }
  };
  copy(outputs->center_velocities, c.out_velocities.p, 12 * n);
  copy(outputs->axial_loads, c.out_loads.p, 4 * n);
  copy(outputs->length_increments, c.out_increments.p, 4 * n);
}

// Uploads a ContactSystem's records as the context's rows and bodies.
void load_system(Ctx& c, const msb_contact_system& s, const float* multipliers) {
  validate_system(s);
  c.n = std::uint32_t(s.body_count);
  c.has_drift = false;
  for (std::uint64_t b = 0; b < s.body_count && !c.has_drift; ++b) {
    for (float v : s.bodies[b].drift) c.has_drift = c.has_drift || v != 0.0f || std::signbit(v);
  }
  const std::uint32_t rows = std::uint32_t(s.row_count);
  c.body_a.ensure(std::max<std::uint32_t>(c.n, 1));
  c.body_b.ensure(std::max<std::uint32_t>(c.n, 1));
  c.drift_a.ensure(std::max<std::uint32_t>(c.n, 1));
  c.drift_b.ensure(std::max<std::uint32_t>(c.n, 1));
  c.rows.ensure(std::max<std::uint32_t>(rows, 1));
  c.rows.count = rows;
  const std::size_t bytes = std::max<std::size_t>(rows * sizeof(msb_contact_row), c.n * sizeof(msb_contact_body));
  c.records.ensure(std::max<std::size_t>(bytes, 1));
  if (c.n > 0) {
    check(cudaMemcpyAsync(c.records.p, s.bodies, c.n * sizeof(msb_contact_body), cudaMemcpyHostToDevice, c.stream),
          "copy bodies");
    launch_bodies_from_records(c.records.p, c.n, {c.body_a.p, c.body_b.p, c.drift_a.p, c.drift_b.p}, c.stream);
  }
  if (rows > 0) {
    check(cudaMemcpyAsync(c.records.p, s.rows, rows * sizeof(msb_contact_row), cudaMemcpyHostToDevice, c.stream),
          "copy rows");
    launch_rows_from_records(c.records.p, rows, c.rows.arrays(), c.stream);
    check(cudaMemcpyAsync(c.rows.multipliers.p, multipliers, rows * 4ull, cudaMemcpyHostToDevice, c.stream),
          "copy multipliers");
  }
  build_system_incidence(c, rows);
}

template <typename Body>
int guarded(msb_context* c, Body&& body) {
  if (c == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  try {
    check(cudaSetDevice(c->device), "cudaSetDevice");
    body();
    c->error.clear();
    return MSB_OK;
  } catch (const std::invalid_argument& e) {
    c->error = e.what();
    return MSB_ERR_INVALID_ARGUMENT;
  } catch (const std::overflow_error& e) {
    c->error = e.what();
    return MSB_ERR_OVERFLOW;
  } catch (const CapacityError& e) {
    c->error = e.what();
    return MSB_ERR_CAPACITY;
  } catch (const CudaError& e) {
    c->error = e.what();
    return MSB_ERR_CUDA;
  } catch (const DeviceCheckError& e) {
    c->error = e.what();
    return MSB_ERR_DEVICE_CHECK;
  } catch (const std::exception& e) {
    c->error = e.what();
    return MSB_ERR_RUNTIME;
  }
}

// ---- contact graph index (graph.cu)

// The reference's validate_contact texts, by the reason codes of graph.cu.
constexpr const char* kCellContactReasons[] = {
    "contact is valid",
    "contact cell identifiers are not canonical",
    "contact slots are invalid",
    "cell contact ordinal exceeds the capsule-pair contract",
    "contact contains a non-finite or invalid field",
    "contact normal is not unit length",
};
constexpr const char* kExternalContactReasons[] = {
    "external contact is valid",
    "external contact has an invalid identity",
    "external contact cell slot is invalid",
    "external contact contains an invalid tag",
    "external contact contains a non-finite or invalid field",
    "external contact normal is not unit length",
};

using GraphArrays = GraphIndexArrays;

void check_graph_size(std::uint64_t cell_count, std::uint64_t count, bool external) {
  // checked_offset_count (contact_graph.cpp:209-215)
  if (cell_count > 0xFFFFFFFFull) throw std::overflow_error("contact graph exceeds the slot index space");
  if ((external ? count : 2 * count) >= 0xFFFFFFFFull) {
    throw std::overflow_error("contact incidence exceeds the 32-bit entry index space");
  }
}

// Validates `count` device-resident contacts and builds their index into
// `out`; returns the packed neighbour count (0 without a neighbour index).
std::uint64_t build_graph(Ctx& c, const void* contacts, std::uint64_t count, std::uint64_t cell_count,
                          bool external, const GraphArrays& out) {
  check_graph_size(cell_count, count, external);
  const std::uint64_t entries = external ? count : 2 * count;
  c.graph_words.ensure(4);
  c.graph_scratch.ensure(graph_scratch_words(entries, cell_count));
  launch_validate_contacts(contacts, count, cell_count, external, c.graph_words.p, c.graph_scratch.p, c.stream);
  unsigned long long words[4] = {0, 0, 0, 0};
  check(cudaMemcpyAsync(words, c.graph_words.p, sizeof(words), cudaMemcpyDeviceToHost, c.stream), "copy words");
  sync(c);
  if (words[0] != ~0ull) {
    const unsigned reason = std::min(unsigned(words[0] & 0xFFu), 5u);
    throw std::invalid_argument(external ? kExternalContactReasons[reason] : kCellContactReasons[reason]);
  }
  build_graph_index(contacts, count, cell_count, external, words[1], words[3], out, c.graph_scratch.p,
                    c.graph_words.p, c.stream);
  if (external || out.neighbor_offsets == nullptr) return 0;
  unsigned long long total = 0;
  check(cudaMemcpyAsync(&total, c.graph_words.p + 2, sizeof(total), cudaMemcpyDeviceToHost, c.stream),
        "copy count");
  sync(c);
  return total;
}

// Device staging for an index the caller wants in host memory.
GraphArrays graph_staging(Ctx& c, std::uint64_t cell_count, std::uint64_t entries, bool neighbors) {
  GraphArrays g{};
  g.incidence_offsets = c.graph_incidence_offsets.ensure(cell_count + 1);
  g.incidence = c.graph_incidence.ensure(std::max<std::uint64_t>(entries, 1));
  if (neighbors) {
    g.neighbor_offsets = c.graph_neighbor_offsets.ensure(cell_count + 1);
    g.neighbors = c.graph_neighbors.ensure(std::max<std::uint64_t>(entries, 1));
    g.neighbor_capacity = entries;  // distinct partners never outnumber entries
  }
  return g;
}

void copy_out(Ctx& c, void* host, const void* device, std::uint64_t bytes) {
  if (bytes == 0) return;
  check(cudaMemcpyAsync(host, device, bytes, cudaMemcpyDeviceToHost, c.stream), "copy index");
}

// Copies a staged index to the caller's host arrays (`index` names them).
void copy_graph_out(Ctx& c, const GraphArrays& g, std::uint64_t cell_count, std::uint64_t entries,
                    std::uint64_t neighbors, msb_contact_graph_index& index) {
  copy_out(c, index.incidence_offsets, g.incidence_offsets, (cell_count + 1) * 8);
  copy_out(c, index.incidence_contacts, g.incidence, entries * 8);
  if (g.neighbor_offsets != nullptr) {
    copy_out(c, index.neighbor_offsets, g.neighbor_offsets, (cell_count + 1) * 8);
    copy_out(c, index.neighbor_ids, g.neighbors, neighbors * 8);
  }
  sync(c);
}

// The checks on a caller's index record shared by the graph calls.
bool check_index(const msb_contact_graph_index& index, std::uint64_t count) {
  if (index.incidence_offsets == nullptr || (count > 0 && index.incidence_contacts == nullptr)) {
    throw std::invalid_argument("null incidence array");
  }
  const bool neighbors = index.neighbor_offsets != nullptr || index.neighbor_ids != nullptr;
  if (neighbors && (index.neighbor_offsets == nullptr || (index.neighbor_capacity > 0 && index.neighbor_ids == nullptr))) {
    throw std::invalid_argument("null neighbour array");
  }
  return neighbors;
}

}  // namespace
}  // namespace msb

using namespace msb;

extern "C" {

size_t msb_device_count(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return std::size_t(count);
}

int msb_context_create(uint32_t device_index, msb_context** out) {
  if (out == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return MSB_ERR_NO_DEVICE;
  }
  if (int(device_index) >= count) return MSB_ERR_INVALID_ARGUMENT;
  auto context = std::make_unique<msb_context>();
  context->device = int(device_index);
  try {
    check(cudaSetDevice(context->device), "cudaSetDevice");
    cudaDeviceProp prop{};
    check(cudaGetDeviceProperties(&prop, context->device), "properties");
    context->device_name = prop.name;
    check(cudaStreamCreateWithFlags(&context->stream, cudaStreamNonBlocking), "stream");
    check(cudaMalloc(&context->desc, sizeof(SolveDesc)), "cudaMalloc");
    check(cudaMemset(context->desc, 0, sizeof(SolveDesc)), "memset");
    check(cudaMallocHost(&context->host_scalars, 2 * kScalarCount * sizeof(std::uint32_t)), "cudaMallocHost");
    check(cudaMallocHost(&context->host_desc, sizeof(SolveDesc)), "cudaMallocHost");
    std::memset(context->host_desc, 0, sizeof(SolveDesc));
    context->scalars.ensure(kScalarCount);
    check(cudaMemset(context->scalars.p, 0, kScalarCount * 4), "memset");
  } catch (const std::exception& e) {
    return MSB_ERR_CUDA;
  }
  context->launches_at_create = launches.load();
  *out = context.release();
  return MSB_OK;
}

void msb_context_destroy(msb_context* context) {
  if (context == nullptr) return;
  cudaSetDevice(context->device);
  if (context->stream != nullptr) cudaStreamSynchronize(context->stream);
  for (auto e : context->phase_events) cudaEventDestroy(e);
  for (auto e : context->download_events) cudaEventDestroy(e);
  context->graphs.clear();
  if (context->desc != nullptr) cudaFree(context->desc);
  if (context->host_scalars != nullptr) cudaFreeHost(context->host_scalars);
  if (context->host_desc != nullptr) cudaFreeHost(context->host_desc);
  if (context->stream != nullptr) cudaStreamDestroy(context->stream);
  delete context;
}

const char* msb_last_error(const msb_context* context) {
  return context != nullptr ? context->error.c_str() : "no context";
}

int msb_backend_info(const msb_context* context, char* device_name, size_t capacity) {
  if (context == nullptr || device_name == nullptr || capacity == 0) return MSB_ERR_INVALID_ARGUMENT;
  std::snprintf(device_name, capacity, "%s", context->device_name.c_str());
  return MSB_OK;
}

int msb_last_step_solves(const msb_context* context, msb_solve_record* records, uint32_t capacity,
                         uint32_t* count) {
  if (context == nullptr || count == nullptr || (capacity > 0 && records == nullptr)) return MSB_ERR_INVALID_ARGUMENT;
  const auto& log = context->solve_log;
  *count = std::uint32_t(log.size());
  for (std::size_t k = 0; k < log.size() && k < capacity; ++k) records[k] = log[k];
  return log.size() > capacity ? MSB_ERR_CAPACITY : MSB_OK;
}

int msb_last_step_searches(const msb_context* context, uint32_t* full, uint32_t* kept, uint32_t* partial) {
  if (context == nullptr || full == nullptr || kept == nullptr || partial == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  *full = context->searches[0];
  *kept = context->searches[1];
  *partial = context->searches[2];
  return MSB_OK;
}

int msb_set_search_reuse(msb_context* context, uint32_t mode) {
  return guarded(context, [&] {
    if (mode > 2) throw std::invalid_argument("search reuse must be 0 (all kinds), 1 (no partial re-search) or 2 (full searches)");
    context->search_reuse = mode;
  });
}

int msb_set_flow_field(msb_context* context, const msb_flow_field* field) {
  if (context == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  auto& c = *context;
  return guarded(context, [&] {
    c.has_flow = false;
    if (field == nullptr) return;
    const auto positive_finite = [](float v) { return std::isfinite(v) && v > 0.0f; };
    if (field->shape_x == 0 || field->shape_y == 0 || field->shape_z == 0) {
      throw std::invalid_argument("flow field shape must be positive");
    }
    if (!positive_finite(field->spacing.x) || !positive_finite(field->spacing.y) ||
        !positive_finite(field->spacing.z)) {
      throw std::invalid_argument("flow field spacing must be finite and positive");
    }
    if (!std::isfinite(field->origin.x) || !std::isfinite(field->origin.y) || !std::isfinite(field->origin.z)) {
      throw std::invalid_argument("flow field origin must be finite");
    }
    if (field->x_faces == nullptr || field->y_faces == nullptr || field->z_faces == nullptr) {
      throw std::invalid_argument("flow field faces must not be null");
    }
    const std::size_t sx = field->shape_x, sy = field->shape_y, sz = field->shape_z;
    const std::size_t nx = (sx + 1) * sy * sz, ny = sx * (sy + 1) * sz, nz = sx * sy * (sz + 1);
    const auto finite_all = [](const float* v, std::size_t count) {
      for (std::size_t i = 0; i < count; ++i) {
        if (!std::isfinite(v[i])) return false;
      }
      return true;
    };
    if (!finite_all(field->x_faces, nx) || !finite_all(field->y_faces, ny) || !finite_all(field->z_faces, nz)) {
      throw std::invalid_argument("flow field velocities must be finite");
    }
    c.flow_x.ensure(nx);
    c.flow_y.ensure(ny);
    c.flow_z.ensure(nz);
    check(cudaMemcpyAsync(c.flow_x.p, field->x_faces, nx * 4, cudaMemcpyHostToDevice, c.stream), "copy flow");
    check(cudaMemcpyAsync(c.flow_y.p, field->y_faces, ny * 4, cudaMemcpyHostToDevice, c.stream), "copy flow");
    check(cudaMemcpyAsync(c.flow_z.p, field->z_faces, nz * 4, cudaMemcpyHostToDevice, c.stream), "copy flow");
    const std::uint8_t* obstacles = nullptr;
    if (field->obstacles != nullptr) {
      c.flow_obstacles.ensure(sx * sy * sz);
      check(cudaMemcpyAsync(c.flow_obstacles.p, field->obstacles, sx * sy * sz, cudaMemcpyHostToDevice, c.stream),
            "copy flow");
      obstacles = c.flow_obstacles.p;
    }
    sync(c);
    c.flow = {field->shape_x, field->shape_y, field->shape_z,
              make_float3(field->origin.x, field->origin.y, field->origin.z),
              make_float3(field->spacing.x, field->spacing.y, field->spacing.z),
              c.flow_x.p, c.flow_y.p, c.flow_z.p, obstacles, nullptr};
    c.flow_sites.ensure(std::size_t(field->shape_x) * field->shape_y * field->shape_z);
    launch_flow_sites(c.flow, c.flow_sites.p, c.stream);
    c.flow.sites = c.flow_sites.p;
    check(cudaGetLastError(), "flow sites");
    sync(c);
    c.flow_travel_limit = 0.25f * std::min({field->spacing.x, field->spacing.y, field->spacing.z});
    c.has_flow = true;
  });
}

int msb_set_relaxation(msb_context* context, uint32_t form) {
  return guarded(context, [&] {
    if (form > 2) throw std::invalid_argument("relaxation form must be 0 (automatic), 1 (graph) or 2 (fused)");
    context->relaxation = form;
  });
}

int msb_set_warm_start(msb_context* context, uint32_t mode) {
  if (context == nullptr || (mode & ~kWarmFlags) != 0) return MSB_ERR_INVALID_ARGUMENT;
  context->warm_start_mode = mode;
  if ((mode & kWarmCarry) == 0) context->has_memory = false;
  return MSB_OK;
}

uint64_t msb_mlp_activation_bytes(uint64_t rows) { return mlp::activation_bytes(rows); }
uint64_t msb_mlp_backward_scratch_bytes(uint64_t rows) { return mlp::backward_scratch_bytes(rows); }

namespace {
int cuda_status(cudaError_t e) { return e == cudaSuccess ? MSB_OK : MSB_ERR_CUDA; }
}  // namespace

int msb_mlp_forward(const uint16_t* weights, const float* biases, const uint16_t* features, uint64_t rows,
                    float* outputs, void* activations, void* stream) {
  if (rows > std::numeric_limits<std::uint32_t>::max() / 2) return MSB_ERR_OVERFLOW;
  if (rows > 0 && (weights == nullptr || biases == nullptr || features == nullptr || outputs == nullptr)) {
    return MSB_ERR_INVALID_ARGUMENT;
  }
  // The tcgen05 pass, keeping the activations for training when given them.
  return cuda_status(cudaError_t(mlp::launch_forward_tc(weights, biases, features, std::uint32_t(rows), outputs,
                                                        activations, nullptr, static_cast<cudaStream_t>(stream))));
}

int msb_mlp_backward(const uint16_t* weights, const uint16_t* features, uint64_t rows, const void* activations,
                     const float* output_grad, float* grads, void* scratch, void* stream) {
  if (rows > std::numeric_limits<std::uint32_t>::max() / 2) return MSB_ERR_OVERFLOW;
  if (grads == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  if (rows > 0 && (weights == nullptr || features == nullptr || activations == nullptr || output_grad == nullptr ||
                   scratch == nullptr)) {
    return MSB_ERR_INVALID_ARGUMENT;
  }
  return cuda_status(cudaError_t(mlp::launch_backward(weights, features, std::uint32_t(rows), activations, output_grad,
                                                      grads, scratch, nullptr, static_cast<cudaStream_t>(stream))));
}

int msb_mlp_adam(float* params, const float* grads, float* m, float* v, uint32_t step, float lr, float beta1,
                 float beta2, float epsilon, uint16_t* weights, float* biases, void* stream) {
  if (params == nullptr || grads == nullptr || m == nullptr || v == nullptr || weights == nullptr ||
      biases == nullptr || step == 0 || !(lr > 0.0f) || !(beta1 >= 0.0f && beta1 < 1.0f) ||
      !(beta2 >= 0.0f && beta2 < 1.0f) || !(epsilon > 0.0f)) {
    return MSB_ERR_INVALID_ARGUMENT;
  }
  mlp::launch_adam(params, grads, m, v, step, lr, beta1, beta2, epsilon, weights, biases,
                   static_cast<cudaStream_t>(stream));
  return cuda_status(cudaGetLastError());
}

int msb_cell_features(msb_context* context, const msb_cell_arrays* cells, uint16_t* features) {
  if (context == nullptr || cells == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  auto& c = *context;
  return guarded(context, [&] {
    if (cells->count > 0 && features == nullptr) throw std::invalid_argument("null features");
    msb_cell_arrays copy = *cells;
    load_cells(c, copy, true);
    compute_features(c, c.state.view());
    if (c.n > 0) {
      check(cudaMemcpyAsync(features, c.features.p, std::size_t(c.n) * mlp::kInput * 2, cudaMemcpyDeviceToDevice,
                            c.stream),
            "copy features");
    }
    sync(c);
  });
}

int msb_set_warm_start_network(msb_context* context, const uint16_t* weights, const float* biases,
                               const float* scale) {
  if (context == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  auto& c = *context;
  return guarded(context, [&] {
    c.has_network = false;
    if (weights == nullptr) return;
    if (biases == nullptr || scale == nullptr) throw std::invalid_argument("null network biases or scale");
    for (int k = 0; k < 3; ++k) {
      if (!std::isfinite(scale[k]) || !(scale[k] > 0.0f)) throw std::invalid_argument("network scale must be positive");
      c.net_scale[k] = scale[k];
    }
    c.net_weights.ensure(mlp::kWeights);
    c.net_biases.ensure(mlp::kBiases);
    check(cudaMemcpyAsync(c.net_weights.p, weights, mlp::kWeights * 2ull, cudaMemcpyDefault, c.stream), "weights");
    check(cudaMemcpyAsync(c.net_biases.p, biases, mlp::kBiases * 4ull, cudaMemcpyDefault, c.stream), "biases");
    sync(c);
    c.has_network = true;
  });
}

int msb_set_motion_guess(msb_context* context, const float* guess, uint64_t cell_count, float dt) {
  if (context == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  auto& c = *context;
  return guarded(context, [&] {
    c.has_guess = false;
    if (guess == nullptr || cell_count == 0) return;
    if (cell_count > std::numeric_limits<std::uint32_t>::max()) throw std::overflow_error("too many cells");
    if (!(dt > 0.0f) || !std::isfinite(dt)) throw std::invalid_argument("motion guess dt must be positive");
    std::vector<float4> packed(cell_count);
    for (std::uint64_t s = 0; s < cell_count; ++s) {
      const float x = guess[3 * s], y = guess[3 * s + 1], t = guess[3 * s + 2];
      if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(t)) {
        throw std::invalid_argument("motion guess must be finite");
      }
      packed[s] = make_float4(x, y, t, 0.0f);
    }
    c.guess.ensure(cell_count);
    check(cudaMemcpyAsync(c.guess.p, packed.data(), cell_count * sizeof(float4), cudaMemcpyHostToDevice, c.stream),
          "copy guess");
    sync(c);
    c.guess_cells = std::uint32_t(cell_count);
    c.guess_dt = dt;
    c.has_guess = true;
  });
}

int msb_last_step_phases(const msb_context* context, double* milliseconds, uint32_t capacity) {
  if (context == nullptr || milliseconds == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  for (std::uint32_t k = 0; k < capacity && k < kPhaseEnd; ++k) milliseconds[k] = context->phase_ms[k];
  return MSB_OK;
}

uint64_t msb_launch_count(const msb_context* context) {
  return launches.load() - (context != nullptr ? context->launches_at_create : 0);
}

int msb_find_cell_contacts(msb_context* context, const msb_cell_arrays* cells,
                           const msb_contact_parameters* parameters, msb_cell_contact* contacts, uint64_t capacity,
                           uint64_t* count) {
  return guarded(context, [&] {
    if (cells == nullptr || parameters == nullptr || count == nullptr) throw std::invalid_argument("null argument");
    validate_contact_parameters(*parameters);
    auto& c = *context;
    load_cells(c, *cells, false);
    const ContactSearchParams prm{parameters->activation_margin, parameters->parallel_sine_threshold,
                                  parameters->degeneracy_epsilon};
    const std::uint32_t total = find_pairs(c, c.state, prm, c.touches);
    *count = total;
    if (total > capacity) throw CapacityError("contact array is too small");
    if (total == 0) return;
    if (contacts == nullptr) throw std::invalid_argument("null contact array");
    c.records.ensure(total * sizeof(msb_cell_contact));
    launch_touches_to_cell_contacts(c.touches.p, total, c.ids.p, c.records.p, c.stream);
    check(cudaMemcpyAsync(contacts, c.records.p, total * sizeof(msb_cell_contact), cudaMemcpyDeviceToHost, c.stream),
          "copy contacts");
    sync(c);
  });
}

int msb_find_cell_contact_graph(msb_context* context, const msb_cell_arrays* cells,
                                const msb_contact_parameters* parameters, msb_cell_contact* contacts,
                                uint64_t capacity, uint64_t* count, msb_contact_graph_index* index) {
  return guarded(context, [&] {
    if (cells == nullptr || parameters == nullptr || count == nullptr) throw std::invalid_argument("null argument");
    validate_contact_parameters(*parameters);
    auto& c = *context;
    load_cells(c, *cells, false);
    const ContactSearchParams prm{parameters->activation_margin, parameters->parallel_sine_threshold,
                                  parameters->degeneracy_epsilon};
    const std::uint32_t total = find_pairs(c, c.state, prm, c.touches);
    *count = total;
    if (total > capacity) throw CapacityError("contact array is too small");
    if (total > 0 && contacts == nullptr) throw std::invalid_argument("null contact array");
    const bool neighbors = index != nullptr && check_index(*index, total);
    c.records.ensure(std::max<std::uint64_t>(total, 1) * sizeof(msb_cell_contact));
    if (total > 0) launch_touches_to_cell_contacts(c.touches.p, total, c.ids.p, c.records.p, c.stream);
    if (index != nullptr) {
      const GraphArrays g = graph_staging(c, cells->count, 2ull * total, neighbors);
      const std::uint64_t packed = build_graph(c, c.records.p, total, cells->count, false, g);
      if (neighbors) {
        index->neighbor_count = packed;
        if (packed > index->neighbor_capacity) throw CapacityError("neighbour id array is too small");
      }
      copy_graph_out(c, g, cells->count, 2ull * total, packed, *index);
    }
    if (total > 0) {
      check(cudaMemcpyAsync(contacts, c.records.p, total * sizeof(msb_cell_contact), cudaMemcpyDeviceToHost,
                            c.stream),
            "copy contacts");
    }
    sync(c);
  });
}

int msb_find_external_contact_graph(msb_context* context, const msb_cell_arrays* cells,
                                    const msb_constraint* constraints, uint64_t constraint_count,
                                    const msb_constraint_contact_parameters* parameters, uint32_t every_face,
                                    msb_external_contact* contacts, uint64_t capacity, uint64_t* count,
                                    uint64_t* incidence_offsets, uint64_t* incidence_contacts) {
  return guarded(context, [&] {
    if (cells == nullptr || parameters == nullptr || count == nullptr) throw std::invalid_argument("null argument");
    validate_constraint_parameters(*parameters);
    auto& c = *context;
    load_cells(c, *cells, false);
    load_constraints(c, constraints, constraint_count);
    const std::uint32_t total =
        find_walls(c, c.state, parameters->activation_margin, parameters->degeneracy_epsilon, every_face != 0,
                   c.touches, 0);
    *count = total;
    if (total > capacity) throw CapacityError("contact array is too small");
    if (total > 0 && contacts == nullptr) throw std::invalid_argument("null contact array");
    if (incidence_offsets != nullptr && total > 0 && incidence_contacts == nullptr) {
      throw std::invalid_argument("null incidence array");
    }
    c.records.ensure(std::max<std::uint64_t>(total, 1) * sizeof(msb_external_contact));
    if (total > 0) launch_touches_to_external_contacts(c.touches.p, total, c.ids.p, c.records.p, c.stream);
    if (incidence_offsets != nullptr) {
      const GraphArrays g = graph_staging(c, cells->count, total, false);
      build_graph(c, c.records.p, total, cells->count, true, g);
      copy_out(c, incidence_offsets, g.incidence_offsets, (cells->count + 1) * 8);
      copy_out(c, incidence_contacts, g.incidence, std::uint64_t(total) * 8);
    }
    if (total > 0) {
      check(cudaMemcpyAsync(contacts, c.records.p, total * sizeof(msb_external_contact), cudaMemcpyDeviceToHost,
                            c.stream),
            "copy contacts");
    }
    sync(c);
  });
}

int msb_build_contact_graph(msb_context* context, const msb_cell_contact* contacts, uint64_t count,
                            uint64_t cell_count, uint32_t device_pointers, msb_contact_graph_index* index) {
  return guarded(context, [&] {
    if (index == nullptr || (count > 0 && contacts == nullptr)) throw std::invalid_argument("null argument");
    check_graph_size(cell_count, count, false);  // the constructor's first check (contact_graph.cpp:305-306)
    const bool neighbors = check_index(*index, count);
    auto& c = *context;
    const void* source = contacts;
    if (device_pointers == 0 && count > 0) {
      c.graph_contacts.ensure(count * sizeof(msb_cell_contact));
      check(cudaMemcpyAsync(c.graph_contacts.p, contacts, count * sizeof(msb_cell_contact), cudaMemcpyHostToDevice,
                            c.stream),
            "copy contacts");
      source = c.graph_contacts.p;
    }
    GraphArrays g{};
    if (device_pointers != 0) {
      g = {index->incidence_offsets, index->incidence_contacts, neighbors ? index->neighbor_offsets : nullptr,
           index->neighbor_ids, index->neighbor_capacity};
    } else {
      g = graph_staging(c, cell_count, 2 * count, neighbors);
    }
    const std::uint64_t packed = build_graph(c, source, count, cell_count, false, g);
    if (neighbors) {
      index->neighbor_count = packed;
      if (packed > index->neighbor_capacity) throw CapacityError("neighbour id array is too small");
    }
    if (device_pointers == 0) {
      copy_graph_out(c, g, cell_count, 2 * count, packed, *index);
    } else {
      sync(c);
    }
  });
}

int msb_build_external_contact_graph(msb_context* context, const msb_external_contact* contacts, uint64_t count,
                                     uint64_t cell_count, uint32_t device_pointers, uint64_t* incidence_offsets,
                                     uint64_t* incidence_contacts) {
  return guarded(context, [&] {
    if (count > 0 && contacts == nullptr) throw std::invalid_argument("null argument");
    check_graph_size(cell_count, count, true);
    if (incidence_offsets == nullptr || (count > 0 && incidence_contacts == nullptr)) {
      throw std::invalid_argument("null incidence array");
    }
    auto& c = *context;
    const void* source = contacts;
    if (device_pointers == 0 && count > 0) {
      c.graph_contacts.ensure(count * sizeof(msb_external_contact));
      check(cudaMemcpyAsync(c.graph_contacts.p, contacts, count * sizeof(msb_external_contact),
                            cudaMemcpyHostToDevice, c.stream),
            "copy contacts");
      source = c.graph_contacts.p;
    }
    GraphArrays g{};
    if (device_pointers != 0) {
      g.incidence_offsets = incidence_offsets;
      g.incidence = incidence_contacts;
    } else {
      g = graph_staging(c, cell_count, count, false);
    }
    build_graph(c, source, count, cell_count, true, g);
    if (device_pointers == 0) {
      copy_out(c, incidence_offsets, g.incidence_offsets, (cell_count + 1) * 8);
      copy_out(c, incidence_contacts, g.incidence, count * 8);
    }
    sync(c);
  });
}

int msb_find_external_contacts(msb_context* context, const msb_cell_arrays* cells, const msb_constraint* constraints,
                               uint64_t constraint_count, const msb_constraint_contact_parameters* parameters,
                               uint32_t every_face, msb_external_contact* contacts, uint64_t capacity,
                               uint64_t* count) {
  return guarded(context, [&] {
    if (cells == nullptr || parameters == nullptr || count == nullptr) throw std::invalid_argument("null argument");
    validate_constraint_parameters(*parameters);
    auto& c = *context;
    load_cells(c, *cells, false);
    load_constraints(c, constraints, constraint_count);
    const std::uint32_t total =
        find_walls(c, c.state, parameters->activation_margin, parameters->degeneracy_epsilon, every_face != 0,
                   c.touches, 0);
    *count = total;
    if (total > capacity) throw CapacityError("contact array is too small");
    if (total == 0) return;
    if (contacts == nullptr) throw std::invalid_argument("null contact array");
    c.records.ensure(total * sizeof(msb_external_contact));
    launch_touches_to_external_contacts(c.touches.p, total, c.ids.p, c.records.p, c.stream);
    check(cudaMemcpyAsync(contacts, c.records.p, total * sizeof(msb_external_contact), cudaMemcpyDeviceToHost,
                          c.stream),
          "copy contacts");
    sync(c);
  });
}

int msb_solve_contact_forces(msb_context* context, const msb_contact_system* system, const float* initial,
                             const msb_contact_solve_parameters* parameters, float* multipliers,
                             msb_contact_solve_report* report) {
  return guarded(context, [&] {
    if (system == nullptr || parameters == nullptr || report == nullptr) throw std::invalid_argument("null argument");
    if (system->row_count > 0 && (initial == nullptr || multipliers == nullptr || system->rows == nullptr)) {
      throw std::invalid_argument("null row arrays");
    }
    if (system->body_count > 0 && system->bodies == nullptr) throw std::invalid_argument("null body array");
    validate_system(*system);
    require_multipliers(initial, system->row_count);
    if (!std::isfinite(parameters->tolerance) || parameters->tolerance <= 0.0f) {
      throw std::invalid_argument("contact solve tolerance must be finite and positive");
    }
    *report = {MSB_SOLVE_CONVERGED, 0, 0.0f};
    if (system->row_count == 0) return;
    auto& c = *context;
    load_system(c, *system, initial);
    const auto outcome = solve(c, system->dt, system->growth, parameters->tolerance, parameters->max_iterations);
    check(cudaMemcpyAsync(multipliers, c.rows.multipliers.p, system->row_count * 4, cudaMemcpyDeviceToHost, c.stream),
          "copy multipliers");
    sync(c);
    *report = {outcome.status, outcome.iterations, outcome.residual};
  });
}

int msb_evaluate_contact_response(msb_context* context, const msb_contact_system* system, const float* multipliers,
                                  float* velocities, float* loads, float* length_rates) {
  return guarded(context, [&] {
    if (system == nullptr) throw std::invalid_argument("null argument");
    validate_system(*system);
    if (system->row_count > 0) {
      if (multipliers == nullptr) throw std::invalid_argument("null multipliers");
      require_multipliers(multipliers, system->row_count);
    }
    auto& c = *context;
    load_system(c, *system, multipliers);
    c.resp_a.ensure(std::max<std::uint32_t>(c.n, 1));
    c.resp_b.ensure(std::max<std::uint32_t>(c.n, 1));
    fill_desc(c, c.rows.count, system->dt, system->growth, 1.0f, 0);
    launch_evaluate(c.desc, std::max(1, grid_for(std::max<std::uint32_t>(c.n, 1), kSolveThreads)), false, c.stream);
    if (c.n == 0) return;
    c.out_velocities.ensure(6ull * c.n);
    c.out_loads.ensure(c.n);
    c.out_increments.ensure(c.n);
    launch_response_to_host_layout(c.n, {c.resp_a.p, c.resp_b.p}, c.out_velocities.p, c.out_loads.p,
                                   c.out_increments.p, c.stream);
    if (velocities) check(cudaMemcpyAsync(velocities, c.out_velocities.p, 24ull * c.n, cudaMemcpyDeviceToHost, c.stream), "copy");
    if (loads) check(cudaMemcpyAsync(loads, c.out_loads.p, 4ull * c.n, cudaMemcpyDeviceToHost, c.stream), "copy");
    if (length_rates) check(cudaMemcpyAsync(length_rates, c.out_increments.p, 4ull * c.n, cudaMemcpyDeviceToHost, c.stream), "copy");
    sync(c);
  });
}

int msb_evaluate_contact_gaps(msb_context* context, const msb_contact_system* system, const float* multipliers,
                              float* gaps) {
  return guarded(context, [&] {
    if (system == nullptr) throw std::invalid_argument("null argument");
    validate_system(*system);
    if (system->row_count == 0) return;
    if (multipliers == nullptr || gaps == nullptr) throw std::invalid_argument("null arrays");
    require_multipliers(multipliers, system->row_count);
    auto& c = *context;
    load_system(c, *system, multipliers);
    c.resp_a.ensure(std::max<std::uint32_t>(c.n, 1));
    c.resp_b.ensure(std::max<std::uint32_t>(c.n, 1));
    fill_desc(c, c.rows.count, system->dt, system->growth, 1.0f, 0);
    launch_evaluate(c.desc, std::max(1, grid_for(std::max(c.rows.count, c.n), kSolveThreads)), true, c.stream);
    check(cudaMemcpyAsync(gaps, c.rows.gaps.p, system->row_count * 4, cudaMemcpyDeviceToHost, c.stream), "copy");
    sync(c);
  });
}

int msb_contact_system_diagonal_bound(msb_context* context, const msb_contact_system* system, float* bound) {
  return guarded(context, [&] {
    if (system == nullptr || bound == nullptr) throw std::invalid_argument("null argument");
    validate_system(*system);
    *bound = 0.0f;
    if (system->row_count == 0) return;
    auto& c = *context;
    std::vector<float> zeros(system->row_count, 0.0f);
    load_system(c, *system, zeros.data());
    // A solve capped at zero iterations computes the bound and stops.
    c.resp_a.ensure(std::max<std::uint32_t>(c.n, 1));
    c.resp_b.ensure(std::max<std::uint32_t>(c.n, 1));
    auto& graph = graph_for(c, std::max(c.rows.count, c.n));
    c.partials.ensure(5ull * kMaxPassBlocks);
    fill_desc(c, c.rows.count, system->dt, system->growth, 1.0f, 0);
    check(cudaError_t(graph.launch(c.stream)), "launch");
    check(cudaMemcpyAsync(c.host_desc, c.desc, sizeof(SolveDesc), cudaMemcpyDeviceToHost, c.stream), "read");
    sync(c);
    *bound = c.host_desc->bound;
  });
}

int msb_profile_iterations(msb_context* context, uint32_t iterations, float* body_ms, float* row_ms,
                           uint64_t* rows, uint64_t* bodies) {
  return guarded(context, [&] {
    auto& c = *context;
    if (c.last_blocks == 0 || iterations == 0) throw std::invalid_argument("no solved system to time");
    cudaEvent_t start, between, stop;
    check(cudaEventCreate(&start), "event");
    check(cudaEventCreate(&between), "event");
    check(cudaEventCreate(&stop), "event");
    // Warm the caches as the solve loop does.
    launch_iteration(c.desc, c.last_blocks, nullptr, c.stream);
    double body = 0.0, row = 0.0;
    for (std::uint32_t k = 0; k < iterations; ++k) {
      check(cudaEventRecord(start, c.stream), "event");
      launch_iteration(c.desc, c.last_blocks, between, c.stream);
      check(cudaEventRecord(stop, c.stream), "event");
      check(cudaEventSynchronize(stop), "event");
      float a = 0.0f, b = 0.0f;
      check(cudaEventElapsedTime(&a, start, between), "event");
      check(cudaEventElapsedTime(&b, between, stop), "event");
      body += a;
      row += b;
    }
    cudaEventDestroy(start);
    cudaEventDestroy(between);
    cudaEventDestroy(stop);
    check(cudaMemcpyAsync(c.host_desc, c.desc, sizeof(SolveDesc), cudaMemcpyDeviceToHost, c.stream), "read");
    sync(c);
    *body_ms = float(body / iterations);
    *row_ms = float(row / iterations);
    *rows = c.host_desc->row_count;
    *bodies = c.host_desc->body_count;
  });
}

static int advance_entry(msb_context* context, msb_cell_arrays* cells, const msb_constraint* constraints,
                         uint64_t constraint_count, float dt, const msb_contact_dynamics_parameters* dynamics,
                         const msb_contact_parameters* contacts,
                         const msb_constraint_contact_parameters* constraint_parameters,
                         msb_contact_dynamics_report* report, msb_contact_dynamics_outputs* outputs,
                         bool device_pointers) {
  return guarded(context, [&] {
    if (cells == nullptr || dynamics == nullptr || report == nullptr) throw std::invalid_argument("null argument");
    if (!std::isfinite(dt) || dt < 0.0f) throw std::invalid_argument("time step must be finite and non-negative");
    const msb_contact_parameters cp = contacts != nullptr ? *contacts : msb_contact_parameters{0.01f, 0.1f, 1.0e-6f};
    const msb_constraint_contact_parameters wp =
        constraint_parameters != nullptr ? *constraint_parameters : msb_constraint_contact_parameters{0.0f, 1.0e-6f};
    validate_dynamics(*dynamics);
    validate_contact_parameters(cp);
    validate_constraint_parameters(wp);
    auto& c = *context;
    c.phase_marks.clear();
    c.solve_log.clear();
    std::fill(std::begin(c.searches), std::end(c.searches), 0u);
    mark(c, kPhaseLoad);
    load_cells(c, *cells, device_pointers);
    load_constraints(c, constraints, constraint_count);
    c.has_memory = c.has_memory && (c.warm_start_mode & kWarmCarry) != 0;
    if (dynamics->flow_drift != 0 && !c.has_flow) {
      // Simulation::step's error (simulation.cpp:194), a logic_error: MSB_ERR_RUNTIME.
      throw std::logic_error("flow drift requires a signal grid with a velocity field (msb_set_flow_field)");
    }
    if (c.has_guess && c.guess_cells != c.n) {
      c.has_guess = false;
      throw std::invalid_argument("the motion guess covers " + std::to_string(c.guess_cells) +
                                  " cells; the step has " + std::to_string(c.n));
    }
    StepOutcome outcome;
    try {
      outcome = advance(c, dt, *dynamics, cp, wp);
    } catch (...) {
      c.has_memory = false;  // forces of a step that did not complete
      c.has_guess = false;
      throw;
    }
    c.has_guess = false;  // a guess serves one step
    mark(c, kPhaseOutput);
    prepare_downloads(c, device_pointers);
    std::size_t at = 0;
    write_back(c, *cells, device_pointers, at);
    write_outputs(c, outputs, device_pointers, at);
    mark(c, kPhaseEnd);
    flush_downloads(c);  // each array's host copy starts when its DMA is done
    sync(c);
    collect_phases(c);
    *report = outcome.report;
  });
}

int msb_advance_contact_dynamics(msb_context* context, msb_cell_arrays* cells, const msb_constraint* constraints,
                                 uint64_t constraint_count, float dt, const msb_contact_dynamics_parameters* dynamics,
                                 const msb_contact_parameters* contacts,
                                 const msb_constraint_contact_parameters* constraint_parameters,
                                 msb_contact_dynamics_report* report, msb_contact_dynamics_outputs* outputs) {
  return advance_entry(context, cells, constraints, constraint_count, dt, dynamics, contacts, constraint_parameters,
                       report, outputs, false);
}

int msb_advance_contact_dynamics_batch(msb_context* context, msb_cell_arrays* cells, const uint32_t* colony_cells,
                                       uint32_t colony_count, const msb_colony_parameters* colony_parameters,
                                       float dt, const msb_contact_dynamics_parameters* dynamics,
                                       const msb_contact_parameters* contacts, msb_contact_dynamics_report* report,
                                       msb_colony_report* colony_reports, msb_contact_dynamics_outputs* outputs,
                                       int device_pointers) {
  if (context == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  return guarded(context, [&] {
    if (cells == nullptr || dynamics == nullptr || report == nullptr || colony_cells == nullptr ||
        colony_parameters == nullptr || colony_reports == nullptr) {
      throw std::invalid_argument("null argument");
    }
    if (colony_count == 0 || colony_count > kMaxColonies) {
      throw std::invalid_argument("a batch holds 1 to " + std::to_string(kMaxColonies) + " colonies");
    }
    if (!std::isfinite(dt) || dt < 0.0f) throw std::invalid_argument("time step must be finite and non-negative");
    const msb_contact_parameters cp = contacts != nullptr ? *contacts : msb_contact_parameters{0.01f, 0.1f, 1.0e-6f};
    const msb_constraint_contact_parameters wp{0.0f, 1.0e-6f};
    validate_dynamics(*dynamics);
    validate_contact_parameters(cp);
    auto& c = *context;
    if ((c.warm_start_mode & ~kWarmCarry) != 0) {
      throw std::invalid_argument("a batch takes no motion guess or warm-start network");
    }
    if (dynamics->flow_drift != 0) throw std::invalid_argument("a batch takes no flow drift");
    std::vector<std::uint32_t> offsets(colony_count + 1, 0);
    std::vector<float> drag(colony_count), stiffness(colony_count), tolerance(colony_count), solve_tol(colony_count);
    for (std::uint32_t i = 0; i < colony_count; ++i) {
      offsets[i + 1] = offsets[i] + colony_cells[i];
      if (offsets[i + 1] < offsets[i]) throw std::overflow_error("too many cells");
      const auto& q = colony_parameters[i];
      if (!std::isfinite(q.drag) || !(q.drag > 0.0f) || !std::isfinite(q.contact_stiffness) ||
          !(q.contact_stiffness > 0.0f)) {
        throw std::invalid_argument("colony drag and contact stiffness must be positive and finite");
      }
      msb_contact_dynamics_parameters own = *dynamics;
      own.drag = q.drag;
      own.contact_stiffness = q.contact_stiffness;
      validate_dynamics(own);
      drag[i] = q.drag;
      stiffness[i] = q.contact_stiffness;
      tolerance[i] = effective_overlap_tolerance(own);
      solve_tol[i] = kSolveToleranceFraction * tolerance[i];
    }
    if (offsets.back() != cells->count) throw std::invalid_argument("colony cell counts must sum to the cell count");
    // Largest colonies first in the solve's work queue.
    std::vector<std::uint32_t> order(colony_count);
    for (std::uint32_t i = 0; i < colony_count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](std::uint32_t a, std::uint32_t b) { return colony_cells[a] > colony_cells[b]; });

    struct Reset {
      Ctx& c;
      ~Reset() {
        c.colonies = 0;
        c.box_scale = 1.0f;
      }
    } reset{c};
    c.box_scale = c.batch_box_scale;
    c.phase_marks.clear();
    c.solve_log.clear();
    std::fill(std::begin(c.searches), std::end(c.searches), 0u);
    mark(c, kPhaseLoad);
    load_cells(c, *cells, device_pointers != 0);
    c.constraint_count = 0;
    c.colonies = colony_count;
    c.host_colony_offsets = offsets;
    c.colony_offsets.ensure(colony_count + 1ull);
    c.colony_order.ensure(colony_count);
    c.colony_drag.ensure(colony_count);
    c.colony_stiffness.ensure(colony_count);
    c.colony_tolerance.ensure(colony_count);
    c.colony_solve_tolerance.ensure(colony_count);
    c.colony_overlap.ensure(colony_count);
    c.colony_slack.ensure(colony_count);
    c.colony_active.ensure(colony_count);
    c.colony_flagged.ensure(colony_count);
    check(cudaMemsetAsync(c.colony_active.p, 0xFF, colony_count * 4ull, c.stream), "memset");
    c.colony_state.ensure(colony_count);
    c.batch_next.ensure(1);
    c.colony_of_slot.ensure(std::max<std::uint32_t>(c.n, 1));
    const auto up = [&](void* dst, const void* src, std::size_t bytes) {
      check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream), "copy colonies");
    };
    up(c.colony_offsets.p, offsets.data(), offsets.size() * 4);
    up(c.colony_order.p, order.data(), order.size() * 4);
    up(c.colony_drag.p, drag.data(), drag.size() * 4);
    up(c.colony_stiffness.p, stiffness.data(), stiffness.size() * 4);
    up(c.colony_tolerance.p, tolerance.data(), tolerance.size() * 4);
    up(c.colony_solve_tolerance.p, solve_tol.data(), solve_tol.size() * 4);
    launch_colony_of_slot(colony_count, c.colony_offsets.p, c.n, c.colony_of_slot.p, c.stream);
    c.has_memory = c.has_memory && (c.warm_start_mode & kWarmCarry) != 0;
    c.colony_iterations.assign(colony_count, 0);
    c.colony_status.assign(colony_count, MSB_SOLVE_CONVERGED);
    c.colony_max_overlap.assign(colony_count, 0.0f);
    c.colony_rows_at_accept.assign(colony_count, 0);
    if (c.tune_search && c.n > 1) {
      // The autotuner's search leg: the box scale with the fastest contact
      // search on this batch (every scale finds the same contacts).
      cudaEvent_t start, stop;
      check(cudaEventCreate(&start), "event");
      check(cudaEventCreate(&stop), "event");
      float best = -1.0f, chosen = 1.0f;
      for (const float scale : {1.0f, 1.5f, 2.0f, 3.0f}) {
        c.box_scale = scale;
        find_touches(c, c.state, cp, wp, dynamics->candidate_margin, c.touches);  // warm
        check(cudaEventRecord(start, c.stream), "event");
        find_touches(c, c.state, cp, wp, dynamics->candidate_margin, c.touches);
        check(cudaEventRecord(stop, c.stream), "event");
        check(cudaEventSynchronize(stop), "event");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, start, stop), "event");
        if (best < 0.0f || ms < best) {
          best = ms;
          chosen = scale;
        }
      }
      cudaEventDestroy(start);
      cudaEventDestroy(stop);
      c.box_scale = chosen;
      c.batch_box_scale = chosen;
      c.tune_search = false;
    }
    StepOutcome outcome;
    try {
      outcome = advance(c, dt, *dynamics, cp, wp);
    } catch (...) {
      c.has_memory = false;
      throw;
    }
    mark(c, kPhaseOutput);
    prepare_downloads(c, device_pointers != 0);
    std::size_t at = 0;
    write_back(c, *cells, device_pointers != 0, at);
    write_outputs(c, outputs, device_pointers != 0, at);
    mark(c, kPhaseEnd);
    flush_downloads(c);  // each array's host copy starts when its DMA is done
    sync(c);
    collect_phases(c);
    *report = outcome.report;
    for (std::uint32_t i = 0; i < colony_count; ++i) {
      colony_reports[i] = {c.colony_iterations[i], c.colony_max_overlap[i],
                           i < c.colony_rows_at_accept.size() ? c.colony_rows_at_accept[i] : 0u, colony_cells[i],
                           c.colony_status[i]};
    }
  });
}

int msb_tune_batch(msb_context* context) {
  if (context == nullptr) return MSB_ERR_INVALID_ARGUMENT;
  context->batch_tuned = false;
  context->tune_search = true;
  return MSB_OK;
}

int msb_batch_tuning(const msb_context* context, uint32_t* cluster, uint32_t* threads, uint32_t* lean,
                     float* box_scale) {
  if (context == nullptr || cluster == nullptr || threads == nullptr || lean == nullptr || box_scale == nullptr) {
    return MSB_ERR_INVALID_ARGUMENT;
  }
  *cluster = std::uint32_t(context->batch_shape.cluster);
  *threads = std::uint32_t(context->batch_shape.threads);
  *lean = context->batch_shape.lean ? 1u : 0u;
  *box_scale = context->batch_box_scale;
  return MSB_OK;
}

int msb_advance_contact_dynamics_device(msb_context* context, msb_cell_arrays* cells,
                                        const msb_constraint* constraints, uint64_t constraint_count, float dt,
                                        const msb_contact_dynamics_parameters* dynamics,
                                        const msb_contact_parameters* contacts,
                                        const msb_constraint_contact_parameters* constraint_parameters,
                                        msb_contact_dynamics_report* report, msb_contact_dynamics_outputs* outputs) {
  return advance_entry(context, cells, constraints, constraint_count, dt, dynamics, contacts, constraint_parameters,
                       report, outputs, true);
}

}  // extern "C"
