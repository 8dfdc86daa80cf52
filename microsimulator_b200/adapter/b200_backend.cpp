// The B200 backend as a MicroSimulator ComputeBackend: see b200_backend.hpp.
//
// Compiled against the reference's public headers (cpp/include) and linked
// with the reference's core library and libmsb200.so.

#include "b200_backend.hpp"

#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace microsimulator {
namespace {

// ContactRow and ContactBody (cpp/include/microsimulator/contact_dynamics.hpp:71-92)
// are passed to the C-ABI as they lie in memory: their layouts are those of
// msb_contact_row and msb_contact_body.
static_assert(sizeof(ContactRow) == sizeof(msb_contact_row));
static_assert(offsetof(ContactRow, first_slot) == offsetof(msb_contact_row, first_slot));
static_assert(offsetof(ContactRow, second_slot) == offsetof(msb_contact_row, second_slot));
static_assert(offsetof(ContactRow, first_jacobian) == offsetof(msb_contact_row, first_jacobian));
static_assert(offsetof(ContactRow, second_jacobian) == offsetof(msb_contact_row, second_jacobian));
static_assert(offsetof(ContactRow, first_length_lever) == offsetof(msb_contact_row, first_length_lever));
static_assert(offsetof(ContactRow, second_length_lever) == offsetof(msb_contact_row, second_length_lever));
static_assert(offsetof(ContactRow, offset) == offsetof(msb_contact_row, offset));
static_assert(offsetof(ContactRow, compliance) == offsetof(msb_contact_row, compliance));
static_assert(sizeof(ContactBody) == sizeof(msb_contact_body));
static_assert(offsetof(ContactBody, axis) == offsetof(msb_contact_body, axis));
static_assert(offsetof(ContactBody, translational_mobility) == offsetof(msb_contact_body, translational_mobility));
static_assert(offsetof(ContactBody, transverse_mobility) == offsetof(msb_contact_body, transverse_mobility));
static_assert(offsetof(ContactBody, axial_mobility) == offsetof(msb_contact_body, axial_mobility));
static_assert(offsetof(ContactBody, length_rate) == offsetof(msb_contact_body, length_rate));
static_assert(offsetof(ContactBody, drift) == offsetof(msb_contact_body, drift));
static_assert(sizeof(Vec3) == sizeof(msb_vec3));
static_assert(sizeof(CellId) == sizeof(std::uint64_t) && sizeof(Slot) == sizeof(std::uint32_t));

// The reference's exceptions for the C-ABI's status codes (include/msb200.h).
[[noreturn]] void raise(const msb_context* context, int status) {
  std::string message = context != nullptr ? msb_last_error(context) : "";
  if (message.empty()) message = "B200 backend call failed with status " + std::to_string(status);
  switch (status) {
    case MSB_ERR_INVALID_ARGUMENT:
      throw std::invalid_argument(message);
    case MSB_ERR_OVERFLOW:
      throw std::overflow_error(message);
    default:
      throw std::runtime_error(message);
  }
}

void check(const msb_context* context, int status) {
  if (status != MSB_OK) raise(context, status);
}

// The cells of a WorldState as the C-ABI's host arrays.  The contact
// searches only read them; the stepping call writes positions, directions and
// lengths, so it is given copies (`scratch`).
struct Cells {
  msb_cell_arrays arrays{};
  std::vector<float> scratch;
};

Cells cells_of(const WorldState& state, bool writable) {
  const auto g = state.geometry_state();
  const auto a = state.cell_attributes();
  const std::size_t n = g.size();
  Cells cells;
  auto* px = const_cast<float*>(g.position_x.data());
  auto* py = const_cast<float*>(g.position_y.data());
  auto* pz = const_cast<float*>(g.position_z.data());
  auto* dx = const_cast<float*>(g.direction_x.data());
  auto* dy = const_cast<float*>(g.direction_y.data());
  auto* dz = const_cast<float*>(g.direction_z.data());
  auto* len = const_cast<float*>(g.lengths.data());
  if (writable) {
    cells.scratch.resize(7 * n);
    float* base = cells.scratch.data();
    const std::span<const float> sources[7] = {g.position_x, g.position_y, g.position_z, g.direction_x,
                                               g.direction_y, g.direction_z, g.lengths};
    for (int k = 0; k < 7; ++k) std::copy(sources[k].begin(), sources[k].end(), base + k * n);
    px = base;
    py = base + n;
    pz = base + 2 * n;
    dx = base + 3 * n;
    dy = base + 4 * n;
    dz = base + 5 * n;
    len = base + 6 * n;
  }
  cells.arrays = {n, g.ids.data(), px, py, pz, dx, dy, dz, len, g.radii.data(), a.growth_rates.data(),
                  a.fixed.data()};
  return cells;
}

msb_vec3 vec(Vec3 v) { return {v.x, v.y, v.z}; }
Vec3 vec(msb_vec3 v) { return {v.x, v.y, v.z}; }

// A ConstraintSet's records in the C-ABI's flattened form.
std::vector<msb_constraint> constraints_of(const ConstraintSet& set) {
  std::vector<msb_constraint> out;
  out.reserve(set.size());
  for (const auto& p : set.planes()) {
    out.push_back({p.id, MSB_CONSTRAINT_PLANE, MSB_REGION_OUTSIDE, vec(p.point), vec(p.inward_normal), 0.0F, 0.0F,
                   p.coefficient, 0});
  }
  for (const auto& s : set.spheres()) {
    out.push_back({s.id, MSB_CONSTRAINT_SPHERE, std::uint32_t(s.allowed_region), vec(s.center), {0.0F, 0.0F, 0.0F},
                   s.radius, 0.0F, s.coefficient, 0});
  }
  for (const auto& b : set.boxes()) {
    out.push_back({b.id, MSB_CONSTRAINT_BOX, std::uint32_t(b.allowed_region), vec(b.center), vec(b.half_extents),
                   0.0F, 0.0F, b.coefficient, 0});
  }
  for (const auto& c : set.cylinders()) {
    out.push_back({c.id, MSB_CONSTRAINT_CYLINDER, std::uint32_t(c.allowed_region), vec(c.center),
                   {0.0F, 0.0F, 0.0F}, c.radius, c.half_height, c.coefficient, 0});
  }
  return out;
}

msb_contact_parameters contact_parameters_of(const ContactParameters& p) {
  return {p.activation_margin, p.parallel_sine_threshold, p.degeneracy_epsilon};
}

msb_constraint_contact_parameters constraint_parameters_of(const ConstraintContactParameters& p) {
  return {p.activation_margin, p.degeneracy_epsilon};
}

msb_growth_load_response growth_of(const GrowthLoadResponse& g) {
  return {std::uint32_t(g.law), g.sensitivity, g.free_load, g.stall_load};
}

// Calls `call(buffer, capacity, &count)` once with a guessed capacity and once
// more with the exact one if it was too small.
template <class Record, class Call>
std::vector<Record> grown(const msb_context* context, std::size_t guess, Call&& call) {
  std::vector<Record> out(guess);
  std::uint64_t count = 0;
  int status = call(out.data(), std::uint64_t(out.size()), &count);
  if (status == MSB_ERR_CAPACITY) {
    out.resize(count);
    status = call(out.data(), std::uint64_t(out.size()), &count);
  }
  check(context, status);
  out.resize(count);
  return out;
}

}  // namespace

B200Backend::B200Backend(std::uint32_t device_index, std::unique_ptr<ComputeBackend> host_features)
    : device_index_(device_index), host_features_(std::move(host_features)) {
  const int status = msb_context_create(device_index, &context_);
  if (status != MSB_OK) {
    throw std::runtime_error("cannot open B200 device " + std::to_string(device_index) + " (status " +
                             std::to_string(status) + ")");
  }
}

B200Backend::~B200Backend() { msb_context_destroy(context_); }

BackendInfo B200Backend::info() const {
  char name[256] = {};
  check(context_, msb_backend_info(context_, name, sizeof(name)));
  return {.kind = BackendKind::cuda, .name = "b200", .device = name, .device_index = device_index_, .native = true};
}

bool B200Backend::supports(BackendFeature feature) const noexcept {
  if (feature == BackendFeature::cell_contacts || feature == BackendFeature::external_constraints ||
      feature == BackendFeature::contact_dynamics) {
    return true;
  }
  return host_features_ != nullptr && host_features_->supports(feature);
}

ContactGraph B200Backend::find_cell_contacts(const WorldState& state, const ContactParameters& parameters) {
  auto cells = cells_of(state, false);
  const auto p = contact_parameters_of(parameters);
  const auto records = grown<msb_cell_contact>(context_, 4 * state.size() + 64,
                                               [&](msb_cell_contact* out, std::uint64_t capacity, std::uint64_t* n) {
                                                 return msb_find_cell_contacts(context_, &cells.arrays, &p, out,
                                                                               capacity, n);
                                               });
  std::vector<CellContact> contacts(records.size());
  for (std::size_t i = 0; i < records.size(); ++i) {
    const auto& c = records[i];
    contacts[i] = {c.first_id, c.second_id, c.first_slot, c.second_slot, std::uint8_t(c.ordinal),
                   vec(c.point_on_first), vec(c.normal), c.signed_separation, c.weight};
  }
  return ContactGraph(state.size(), std::move(contacts));
}

ExternalContactGraph B200Backend::find_external_contacts(const WorldState& state, const ConstraintSet& constraints,
                                                         const ConstraintContactParameters& parameters) {
  auto cells = cells_of(state, false);
  const auto set = constraints_of(constraints);
  const auto p = constraint_parameters_of(parameters);
  const auto records = grown<msb_external_contact>(
      context_, 2 * state.size() + 64, [&](msb_external_contact* out, std::uint64_t capacity, std::uint64_t* n) {
        return msb_find_external_contacts(context_, &cells.arrays, set.data(), set.size(), &p, 0, out, capacity, n);
      });
  std::vector<ExternalContact> contacts(records.size());
  for (std::size_t i = 0; i < records.size(); ++i) {
    const auto& c = records[i];
    contacts[i] = {c.cell_id,
                   c.cell_slot,
                   c.constraint_id,
                   ExternalConstraintKind(c.constraint_kind),
                   RodContactLocation(c.location),
                   vec(c.point_on_cell),
                   vec(c.normal),
                   c.signed_separation,
                   c.weight};
  }
  return ExternalContactGraph(state.size(), std::move(contacts));
}

ContactSolveResult B200Backend::solve_contact_forces(const ContactSystem& system,
                                                     std::span<const float> initial_multipliers,
                                                     const ContactSolveParameters& parameters) {
  if (initial_multipliers.size() != system.rows.size()) {
    throw std::invalid_argument("contact multiplier count does not match the contact rows");
  }
  const msb_contact_system s{reinterpret_cast<const msb_contact_row*>(system.rows.data()),
                             system.rows.size(),
                             reinterpret_cast<const msb_contact_body*>(system.bodies.data()),
                             system.bodies.size(),
                             system.dt,
                             growth_of(system.growth)};
  const msb_contact_solve_parameters p{parameters.tolerance, parameters.max_iterations};
  ContactSolveResult result;
  result.multipliers.resize(system.rows.size());
  msb_contact_solve_report report{};
  check(context_,
        msb_solve_contact_forces(context_, &s, initial_multipliers.data(), &p, result.multipliers.data(), &report));
  result.report = {ContactSolveStatus(report.status), report.iterations, report.residual};
  return result;
}

ContactDynamicsResult B200Backend::advance_contact_dynamics(WorldState& state, const ConstraintSet& constraints,
                                                            float dt, const ContactDynamicsParameters& parameters,
                                                            const ContactParameters& contact_parameters,
                                                            const ConstraintContactParameters& constraint_parameters) {
  if (parameters.flow_drift) {
    throw std::logic_error("flow drift requires a signal grid with a velocity field");
  }
  auto cells = cells_of(state, true);
  const std::size_t n = state.size();
  const auto set = constraints_of(constraints);
  const msb_contact_dynamics_parameters d{parameters.drag,
                                          parameters.contact_stiffness,
                                          parameters.wall_stiffness,
                                          parameters.overlap_tolerance,
                                          parameters.candidate_margin,
                                          parameters.max_overlap_recovery,
                                          parameters.max_growth_fraction,
                                          parameters.max_iterations,
                                          parameters.max_refinements,
                                          parameters.max_step_halvings,
                                          0,
                                          growth_of(parameters.growth)};
  const auto c = contact_parameters_of(contact_parameters);
  const auto w = constraint_parameters_of(constraint_parameters);
  std::vector<float> velocities(3 * n), loads(n), increments(n);
  msb_contact_dynamics_outputs outputs{velocities.data(), loads.data(), increments.data()};
  msb_contact_dynamics_report report{};
  check(context_, msb_advance_contact_dynamics(context_, &cells.arrays, set.data(), set.size(), dt, &d, &c, &w,
                                               &report, &outputs));
  ContactDynamicsResult result;
  result.report.substeps = report.substeps;
  result.report.halvings = report.halvings;
  result.report.refinements = report.refinements;
  result.report.iterations = report.iterations;
  result.report.max_rows = report.max_rows;
  result.report.max_overlap = report.max_overlap;
  result.center_velocities.resize(n);
  for (std::size_t i = 0; i < n; ++i) {
    result.center_velocities[i] = {velocities[3 * i], velocities[3 * i + 1], velocities[3 * i + 2]};
  }
  result.axial_loads = std::move(loads);
  result.length_increments = std::move(increments);
  const auto& a = cells.arrays;
  for (std::size_t slot = 0; slot < n; ++slot) {
    state.set_cell_geometry(Slot(slot), Vec3{a.position_x[slot], a.position_y[slot], a.position_z[slot]},
                            Vec3{a.direction_x[slot], a.direction_y[slot], a.direction_z[slot]}, a.lengths[slot]);
  }
  return result;
}

ComputeBackend& B200Backend::host(BackendFeature feature, const char* what) const {
  if (host_features_ == nullptr || !host_features_->supports(feature)) {
    throw std::runtime_error(std::string("the B200 backend does not implement ") + what);
  }
  return *host_features_;
}

void B200Backend::advance_growth(WorldState& state, float dt) {
  host(BackendFeature::growth, "growth").advance_growth(state, dt);
}

void B200Backend::advance_species(WorldState& state, const SpeciesRatePlan& plan,
                                  std::span<const float> previous_lengths, float dt) {
  host(BackendFeature::species, "species integration").advance_species(state, plan, previous_lengths, dt);
}

SignalSolveReport B200Backend::advance_signal_grid(SignalGrid& grid, float dt) {
  return host(BackendFeature::signals, "signal grid integration").advance_signal_grid(grid, dt);
}

SignalSolveReport B200Backend::advance_coupled(WorldState& state, SignalGrid& grid, const CoupledRatePlan& plan,
                                               std::span<const float> previous_lengths, float dt) {
  return host(BackendFeature::coupled_rates, "coupled rates").advance_coupled(state, grid, plan, previous_lengths, dt);
}

DepthAveragedFlowResult B200Backend::solve_depth_averaged_flow(const SignalGridSpec& spec,
                                                               std::span<const float> mobility,
                                                               const DepthAveragedFlowParameters& parameters) {
  return host(BackendFeature::depth_averaged_flow, "depth-averaged flow")
      .solve_depth_averaged_flow(spec, mobility, parameters);
}

DepthAveragedPortFlowResult B200Backend::solve_depth_averaged_port_flow(
    const SignalGridSpec& spec, std::span<const FlowPort> ports, std::span<const float> mobility,
    const DepthAveragedPortFlowParameters& parameters) {
  return host(BackendFeature::depth_averaged_flow, "depth-averaged flow")
      .solve_depth_averaged_port_flow(spec, ports, mobility, parameters);
}

ResolvedFlowResult B200Backend::solve_resolved_flow(const SignalGridSpec& spec, std::span<const float> drag,
                                                    const ResolvedFlowParameters& parameters) {
  return host(BackendFeature::resolved_flow, "resolved flow").solve_resolved_flow(spec, drag, parameters);
}

ResolvedPortFlowResult B200Backend::solve_resolved_port_flow(const SignalGridSpec& spec,
                                                             std::span<const FlowPort> ports,
                                                             std::span<const float> drag,
                                                             const ResolvedPortFlowParameters& parameters) {
  return host(BackendFeature::resolved_flow, "resolved flow").solve_resolved_port_flow(spec, ports, drag, parameters);
}

std::unique_ptr<B200Backend> make_b200_contact_backend(std::uint32_t device_index) {
  return std::make_unique<B200Backend>(device_index);
}

// The factory Simulation(BackendKind::cuda) calls (backend.hpp:60-62;
// simulation.cpp:18-36 under MICROSIMULATOR_HAS_CUDA): the contact path on
// the B200, the other features served by the reference's CPU backend.
std::unique_ptr<ComputeBackend> make_cuda_backend(std::uint32_t device_index) {
  return std::make_unique<B200Backend>(device_index, make_cpu_backend(0));
}

std::size_t cuda_backend_device_count() noexcept { return msb_device_count(); }

}  // namespace microsimulator
