// Test infrastructure, not product code.
//
// A C-ABI driver around the reference MicroSimulator CPU backend, compiled by
// oracle/Makefile together with the reference's own sources (read in place,
// never copied) into oracle/_ref/libmsref.so.  Tests use it to pin the CPU
// restatement (oracle/contact_oracle.cpp) and the CUDA path to the reference's
// actual outputs, and bench.py times it as the CPU baseline.  It speaks the
// same POD types as include/msb200.h.
//
// Reference functions wrapped:
//   find_cell_contacts_cpu / _exhaustive      cpp/cpu/cpu_contacts.cpp:216-242
//   find_cell_contact_candidates              cpp/core/contact_graph.cpp:254-300
//   find_external_contacts_cpu / _faces       cpp/cpu/cpu_constraints.cpp:602-612
//   solve_contact_system_cpu                  cpp/cpu/cpu_contact_dynamics.cpp:262-338
//   evaluate_contact_response / _gaps         cpp/cpu/cpu_contact_dynamics.cpp:222-245
//   contact_system_diagonal_bound             cpp/cpu/cpu_contact_dynamics.cpp:247-260
//   detail::advance_contact_dynamics          cpp/core/contact_dynamics.cpp:676-782
//   WorldState::divide                        cpp/core/world_state.cpp:238-276
//   Simulation::step with flow drift          cpp/core/simulation.cpp:387-488 (a Simulation
//                                             with a signal grid and velocity field)

#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/msb200.h"
#include "core/contact_stepper.hpp"
#include "microsimulator/backend.hpp"
#include "microsimulator/constraints.hpp"
#include "microsimulator/contact_dynamics.hpp"
#include "microsimulator/contact_graph.hpp"
#include "microsimulator/signals.hpp"
#include "microsimulator/simulation.hpp"
#include "microsimulator/threads.hpp"
#include "microsimulator/world_state.hpp"

namespace ms = microsimulator;

namespace {

thread_local std::string last_error;

int fail(int code, const char* message) {
  last_error = message;
  return code;
}

template <typename Body>
int guarded(Body&& body) {
  try {
    body();
    last_error.clear();
    return MSB_OK;
  } catch (const std::invalid_argument& error) {
    return fail(MSB_ERR_INVALID_ARGUMENT, error.what());
  } catch (const std::overflow_error& error) {
    return fail(MSB_ERR_OVERFLOW, error.what());
  } catch (const std::length_error& error) {
    return fail(MSB_ERR_CAPACITY, error.what());
  } catch (const std::exception& error) {
    return fail(MSB_ERR_RUNTIME, error.what());
  }
}

ms::WorldState make_world(const msb_cell_arrays& cells) {
  ms::WorldStateCheckpoint checkpoint;
  checkpoint.species_count = 0;
  ms::CellId next = 1;
  checkpoint.cells.reserve(cells.count);
  for (std::uint64_t slot = 0; slot < cells.count; ++slot) {
    ms::CellSnapshot cell;
    cell.id = cells.ids[slot];
    cell.slot = static_cast<ms::Slot>(slot);
    cell.position = {cells.position_x[slot], cells.position_y[slot], cells.position_z[slot]};
    cell.direction = {cells.direction_x[slot], cells.direction_y[slot], cells.direction_z[slot]};
    cell.length = cells.lengths[slot];
    cell.radius = cells.radii[slot];
    cell.growth_rate = cells.growth_rates != nullptr ? cells.growth_rates[slot] : 0.0F;
    cell.fixed = cells.fixed != nullptr && cells.fixed[slot] != 0;
    next = std::max(next, cell.id + 1);
    checkpoint.cells.push_back(std::move(cell));
  }
  checkpoint.next_id = next;
  return ms::WorldState(checkpoint);
}

void write_back(const ms::WorldState& state, msb_cell_arrays& cells) {
  const auto view = state.geometry_state();
  for (std::size_t slot = 0; slot < view.size(); ++slot) {
    cells.position_x[slot] = view.position_x[slot];
    cells.position_y[slot] = view.position_y[slot];
    cells.position_z[slot] = view.position_z[slot];
    cells.direction_x[slot] = view.direction_x[slot];
    cells.direction_y[slot] = view.direction_y[slot];
    cells.direction_z[slot] = view.direction_z[slot];
    cells.lengths[slot] = view.lengths[slot];
  }
}

ms::ConstraintSet make_constraints(const msb_constraint* constraints, std::uint64_t count) {
  ms::ConstraintSetCheckpoint checkpoint;
  ms::ConstraintId next = 1;
  for (std::uint64_t index = 0; index < count; ++index) {
    const auto& c = constraints[index];
    const ms::Vec3 a{c.a.x, c.a.y, c.a.z};
    const ms::Vec3 b{c.b.x, c.b.y, c.b.z};
    const auto region = c.allowed_region == MSB_REGION_INSIDE ? ms::ConstraintRegion::inside
                                                              : ms::ConstraintRegion::outside;
    switch (c.kind) {
      case MSB_CONSTRAINT_PLANE:
        checkpoint.planes.push_back({c.id, a, b, c.coefficient});
        break;
      case MSB_CONSTRAINT_SPHERE:
        checkpoint.spheres.push_back({c.id, a, c.radius, c.coefficient, region});
        break;
      case MSB_CONSTRAINT_BOX:
        checkpoint.boxes.push_back({c.id, a, b, c.coefficient, region});
        break;
      case MSB_CONSTRAINT_CYLINDER:
        checkpoint.cylinders.push_back({c.id, a, c.radius, c.half_height, c.coefficient, region});
        break;
      default:
        throw std::invalid_argument("constraint kind is invalid");
    }
    next = std::max(next, c.id + 1);
  }
  checkpoint.next_id = next;
  return ms::ConstraintSet(checkpoint);
}

ms::ContactParameters contact_parameters(const msb_contact_parameters* p) {
  ms::ContactParameters result;
  if (p != nullptr) {
    result.activation_margin = p->activation_margin;
    result.parallel_sine_threshold = p->parallel_sine_threshold;
    result.degeneracy_epsilon = p->degeneracy_epsilon;
  }
  return result;
}

ms::ConstraintContactParameters constraint_parameters(const msb_constraint_contact_parameters* p) {
  ms::ConstraintContactParameters result;
  if (p != nullptr) {
    result.activation_margin = p->activation_margin;
    result.degeneracy_epsilon = p->degeneracy_epsilon;
  }
  return result;
}

ms::GrowthLoadResponse growth_response(const msb_growth_load_response& g) {
  ms::GrowthLoadResponse result;
  result.law = static_cast<ms::GrowthLoadLaw>(g.law);
  result.sensitivity = g.sensitivity;
  result.free_load = g.free_load;
  result.stall_load = g.stall_load;
  return result;
}

ms::ContactDynamicsParameters dynamics_parameters(const msb_contact_dynamics_parameters& p) {
  ms::ContactDynamicsParameters result;
  result.drag = p.drag;
  result.contact_stiffness = p.contact_stiffness;
  result.wall_stiffness = p.wall_stiffness;
  result.overlap_tolerance = p.overlap_tolerance;
  result.candidate_margin = p.candidate_margin;
  result.max_overlap_recovery = p.max_overlap_recovery;
  result.max_growth_fraction = p.max_growth_fraction;
  result.max_iterations = p.max_iterations;
  result.max_refinements = p.max_refinements;
  result.max_step_halvings = p.max_step_halvings;
  result.flow_drift = p.flow_drift != 0;
  result.growth = growth_response(p.growth);
  return result;
}

struct SystemStorage {
  std::vector<ms::ContactRow> rows;
  std::vector<ms::ContactBody> bodies;
  ms::ContactSystem system;
};

std::unique_ptr<SystemStorage> make_system(const msb_contact_system& s) {
  auto storage = std::make_unique<SystemStorage>();
  storage->rows.resize(s.row_count);
  for (std::uint64_t i = 0; i < s.row_count; ++i) {
    const auto& r = s.rows[i];
    auto& row = storage->rows[i];
    row.first_slot = r.first_slot;
    row.second_slot = r.second_slot;
    std::copy(r.first_jacobian, r.first_jacobian + 6, row.first_jacobian.begin());
    std::copy(r.second_jacobian, r.second_jacobian + 6, row.second_jacobian.begin());
    row.first_length_lever = r.first_length_lever;
    row.second_length_lever = r.second_length_lever;
    row.offset = r.offset;
    row.compliance = r.compliance;
  }
  storage->bodies.resize(s.body_count);
  for (std::uint64_t i = 0; i < s.body_count; ++i) {
    const auto& b = s.bodies[i];
    auto& body = storage->bodies[i];
    body.axis = {b.axis.x, b.axis.y, b.axis.z};
    body.translational_mobility = b.translational_mobility;
    body.transverse_mobility = b.transverse_mobility;
    body.axial_mobility = b.axial_mobility;
    body.length_rate = b.length_rate;
    std::copy(b.drift, b.drift + 6, body.drift.begin());
  }
  storage->system.rows = storage->rows;
  storage->system.bodies = storage->bodies;
  storage->system.dt = s.dt;
  storage->system.growth = growth_response(s.growth);
  return storage;
}

void copy_contact(const ms::CellContact& c, msb_cell_contact& out) {
  out.first_id = c.first_id;
  out.second_id = c.second_id;
  out.first_slot = c.first_slot;
  out.second_slot = c.second_slot;
  out.ordinal = c.ordinal;
  out.point_on_first = {c.point_on_first.x, c.point_on_first.y, c.point_on_first.z};
  out.normal = {c.normal.x, c.normal.y, c.normal.z};
  out.signed_separation = c.signed_separation;
  out.weight = c.weight;
  out.reserved = 0;
}

void copy_external(const ms::ExternalContact& c, msb_external_contact& out) {
  out.cell_id = c.cell_id;
  out.constraint_id = c.constraint_id;
  out.cell_slot = c.cell_slot;
  out.constraint_kind = static_cast<std::uint32_t>(c.constraint_kind);
  out.location = static_cast<std::uint32_t>(c.location);
  out.point_on_cell = {c.point_on_cell.x, c.point_on_cell.y, c.point_on_cell.z};
  out.normal = {c.normal.x, c.normal.y, c.normal.z};
  out.signed_separation = c.signed_separation;
  out.weight = c.weight;
  out.reserved = 0;
}

// A world kept across calls, so that a benchmark times only the step.
struct RefWorld {
  ms::WorldState state;
  ms::ConstraintSet constraints;
  std::unique_ptr<ms::ComputeBackend> backend;
};

}  // namespace

extern "C" {

const char* ref_last_error(void) {
  return last_error.c_str();
}

uint64_t ref_thread_count(void) {
  return ms::cpu_thread_count();
}

int ref_find_cell_contacts(const msb_cell_arrays* cells, const msb_contact_parameters* parameters,
                           uint32_t exhaustive, msb_cell_contact* contacts, uint64_t capacity,
                           uint64_t* count, uint64_t* incidence_offsets,
                           uint64_t* incidence_indices) {
  return guarded([&] {
    const auto state = make_world(*cells);
    const auto p = contact_parameters(parameters);
    const auto graph = exhaustive != 0 ? ms::find_cell_contacts_cpu_exhaustive(state, p)
                                       : ms::find_cell_contacts_cpu(state, p);
    *count = graph.size();
    if (graph.size() > capacity) {
      throw std::length_error("capacity");
    }
    for (std::size_t i = 0; i < graph.size(); ++i) {
      copy_contact(graph.contacts()[i], contacts[i]);
    }
    if (incidence_offsets != nullptr) {
      std::uint64_t at = 0;
      incidence_offsets[0] = 0;
      for (std::size_t slot = 0; slot < cells->count; ++slot) {
        for (const auto index : graph.incident_contact_indices(static_cast<ms::Slot>(slot))) {
          if (incidence_indices != nullptr) {
            incidence_indices[at] = index;
          }
          ++at;
        }
        incidence_offsets[slot + 1] = at;
      }
    }
  });
}

// ContactGraph(cell_count, contacts) (cpp/core/contact_graph.cpp:302-349) on
// a caller's contact list: its incidence and neighbour arrays, packed.
int ref_contact_graph(const msb_cell_contact* contacts, uint64_t count, uint64_t cell_count,
                      uint64_t* incidence_offsets, uint64_t* incidence_contacts, uint64_t* neighbor_offsets,
                      uint64_t* neighbor_ids, uint64_t neighbor_capacity, uint64_t* neighbor_count) {
  return guarded([&] {
    std::vector<ms::CellContact> list(count);
    for (std::uint64_t i = 0; i < count; ++i) {
      const auto& c = contacts[i];
      auto& r = list[i];
      r.first_id = c.first_id;
      r.second_id = c.second_id;
      r.first_slot = c.first_slot;
      r.second_slot = c.second_slot;
      r.ordinal = static_cast<std::uint8_t>(c.ordinal);
      r.point_on_first = {c.point_on_first.x, c.point_on_first.y, c.point_on_first.z};
      r.normal = {c.normal.x, c.normal.y, c.normal.z};
      r.signed_separation = c.signed_separation;
      r.weight = c.weight;
    }
    const ms::ContactGraph graph(cell_count, std::move(list));
    std::uint64_t incident = 0;
    std::uint64_t neighbors = 0;
    incidence_offsets[0] = 0;
    neighbor_offsets[0] = 0;
    for (std::uint64_t slot = 0; slot < cell_count; ++slot) {
      for (const auto index : graph.incident_contact_indices(static_cast<ms::Slot>(slot))) {
        incidence_contacts[incident++] = index;
      }
      incidence_offsets[slot + 1] = incident;
      for (const auto id : graph.neighbor_ids(static_cast<ms::Slot>(slot))) {
        if (neighbors < neighbor_capacity) neighbor_ids[neighbors] = id;
        ++neighbors;
      }
      neighbor_offsets[slot + 1] = neighbors;
    }
    *neighbor_count = neighbors;
  });
}

// ExternalContactGraph(cell_count, contacts) (cpp/core/constraints.cpp:288-307).
int ref_external_contact_graph(const msb_external_contact* contacts, uint64_t count, uint64_t cell_count,
                               uint64_t* incidence_offsets, uint64_t* incidence_contacts) {
  return guarded([&] {
    std::vector<ms::ExternalContact> list(count);
    for (std::uint64_t i = 0; i < count; ++i) {
      const auto& c = contacts[i];
      auto& r = list[i];
      r.cell_id = c.cell_id;
      r.cell_slot = c.cell_slot;
      r.constraint_id = c.constraint_id;
      r.constraint_kind = static_cast<ms::ExternalConstraintKind>(c.constraint_kind);
      r.location = static_cast<ms::RodContactLocation>(c.location);
      r.point_on_cell = {c.point_on_cell.x, c.point_on_cell.y, c.point_on_cell.z};
      r.normal = {c.normal.x, c.normal.y, c.normal.z};
      r.signed_separation = c.signed_separation;
      r.weight = c.weight;
    }
    const ms::ExternalContactGraph graph(cell_count, std::move(list));
    std::uint64_t incident = 0;
    incidence_offsets[0] = 0;
    for (std::uint64_t slot = 0; slot < cell_count; ++slot) {
      for (const auto index : graph.incident_contact_indices(static_cast<ms::Slot>(slot))) {
        incidence_contacts[incident++] = index;
      }
      incidence_offsets[slot + 1] = incident;
    }
  });
}

int ref_find_cell_contact_candidates(const msb_cell_arrays* cells,
                                     const msb_contact_parameters* parameters, uint32_t* pairs,
                                     uint64_t capacity, uint64_t* count) {
  return guarded([&] {
    const auto state = make_world(*cells);
    const auto candidates = ms::find_cell_contact_candidates(state, contact_parameters(parameters));
    *count = candidates.size();
    if (candidates.size() > capacity) {
      throw std::length_error("capacity");
    }
    for (std::size_t i = 0; i < candidates.size(); ++i) {
      pairs[2 * i] = candidates[i].first_slot;
      pairs[2 * i + 1] = candidates[i].second_slot;
    }
  });
}

int ref_find_external_contacts(const msb_cell_arrays* cells, const msb_constraint* constraints,
                               uint64_t constraint_count,
                               const msb_constraint_contact_parameters* parameters,
                               uint32_t every_face, msb_external_contact* contacts,
                               uint64_t capacity, uint64_t* count) {
  return guarded([&] {
    const auto state = make_world(*cells);
    const auto set = make_constraints(constraints, constraint_count);
    const auto p = constraint_parameters(parameters);
    const auto graph = every_face != 0 ? ms::find_external_contact_faces(state, set, p)
                                       : ms::find_external_contacts_cpu(state, set, p);
    *count = graph.size();
    if (graph.size() > capacity) {
      throw std::length_error("capacity");
    }
    for (std::size_t i = 0; i < graph.size(); ++i) {
      copy_external(graph.contacts()[i], contacts[i]);
    }
  });
}

int ref_solve_contact_forces(const msb_contact_system* system, const float* initial,
                             const msb_contact_solve_parameters* parameters, float* multipliers,
                             msb_contact_solve_report* report) {
  return guarded([&] {
    const auto storage = make_system(*system);
    const ms::ContactSolveParameters p{.tolerance = parameters->tolerance,
                                       .max_iterations = parameters->max_iterations};
    const auto result = ms::solve_contact_system_cpu(
        storage->system, std::span<const float>(initial, system->row_count), p);
    std::copy(result.multipliers.begin(), result.multipliers.end(), multipliers);
    report->status = static_cast<std::uint32_t>(result.report.status);
    report->iterations = result.report.iterations;
    report->residual = result.report.residual;
  });
}

int ref_evaluate_contact_response(const msb_contact_system* system, const float* multipliers,
                                  float* velocities, float* loads, float* length_rates) {
  return guarded([&] {
    const auto storage = make_system(*system);
    const auto response = ms::evaluate_contact_response(
        storage->system, std::span<const float>(multipliers, system->row_count));
    for (std::size_t b = 0; b < response.velocities.size(); ++b) {
      if (velocities != nullptr) {
        std::copy(response.velocities[b].begin(), response.velocities[b].end(),
                  velocities + 6 * b);
      }
      if (loads != nullptr) {
        loads[b] = response.loads[b];
      }
      if (length_rates != nullptr) {
        length_rates[b] = response.length_rates[b];
      }
    }
  });
}

int ref_evaluate_contact_gaps(const msb_contact_system* system, const float* multipliers,
                              float* gaps) {
  return guarded([&] {
    const auto storage = make_system(*system);
    const auto result = ms::evaluate_contact_gaps(
        storage->system, std::span<const float>(multipliers, system->row_count));
    std::copy(result.begin(), result.end(), gaps);
  });
}

int ref_contact_system_diagonal_bound(const msb_contact_system* system, float* bound) {
  return guarded([&] {
    const auto storage = make_system(*system);
    *bound = ms::contact_system_diagonal_bound(storage->system);
  });
}

int ref_advance_contact_dynamics(msb_cell_arrays* cells, const msb_constraint* constraints,
                                 uint64_t constraint_count, float dt,
                                 const msb_contact_dynamics_parameters* dynamics,
                                 const msb_contact_parameters* contacts,
                                 const msb_constraint_contact_parameters* constraint_params,
                                 msb_contact_dynamics_report* report,
                                 msb_contact_dynamics_outputs* outputs) {
  return guarded([&] {
    auto state = make_world(*cells);
    const auto set = make_constraints(constraints, constraint_count);
    auto backend = ms::make_cpu_backend();
    const auto result = ms::detail::advance_contact_dynamics(
        state, set, *backend, dt, dynamics_parameters(*dynamics), contact_parameters(contacts),
        constraint_parameters(constraint_params));
    write_back(state, *cells);
    report->substeps = result.report.substeps;
    report->halvings = result.report.halvings;
    report->refinements = result.report.refinements;
    report->iterations = result.report.iterations;
    report->max_rows = result.report.max_rows;
    report->max_overlap = result.report.max_overlap;
    if (outputs != nullptr) {
      for (std::size_t slot = 0; slot < cells->count; ++slot) {
        if (outputs->center_velocities != nullptr) {
          outputs->center_velocities[3 * slot] = result.center_velocities[slot].x;
          outputs->center_velocities[3 * slot + 1] = result.center_velocities[slot].y;
          outputs->center_velocities[3 * slot + 2] = result.center_velocities[slot].z;
        }
        if (outputs->axial_loads != nullptr) {
          outputs->axial_loads[slot] = result.axial_loads[slot];
        }
        if (outputs->length_increments != nullptr) {
          outputs->length_increments[slot] = result.length_increments[slot];
        }
      }
    }
  });
}

// One Simulation::step(dt, dynamics) of the reference on the given cells
// (ids 1..n in slot order, as Simulation::add_cell assigns them) with a
// signal grid that holds the given velocity field: the flow-drift path.
int ref_flow_step(msb_cell_arrays* cells, const msb_flow_field* field, float dt,
                  const msb_contact_dynamics_parameters* dynamics, msb_contact_dynamics_report* report) {
  return guarded([&] {
    ms::Simulation sim(ms::BackendKind::cpu);
    // The signal grid first: Simulation wants its geometry before cells.
    ms::SignalGridSpec spec;
    // One inert signal: the reference's signal grid needs at least one, and
    // with zero diffusion and advection it leaves the mechanics untouched.
    spec.signal_count = 1;
    spec.diffusion = {0.0F};
    spec.advection = {ms::Vec3{}};
    // Implicit, so that a fast test flow meets no explicit stability bound.
    spec.integration = ms::SignalIntegrationKind::backward_euler;
    spec.shape = {field->shape_x, field->shape_y, field->shape_z};
    spec.origin = {field->origin.x, field->origin.y, field->origin.z};
    spec.spacing = {field->spacing.x, field->spacing.y, field->spacing.z};
    const std::size_t sites = std::size_t(field->shape_x) * field->shape_y * field->shape_z;
    if (field->obstacles != nullptr) spec.obstacles.assign(field->obstacles, field->obstacles + sites);
    ms::SignalGridVelocityField velocity;
    velocity.x_faces.assign(field->x_faces, field->x_faces + std::size_t(field->shape_x + 1) * field->shape_y *
                                                                 field->shape_z);
    velocity.y_faces.assign(field->y_faces, field->y_faces + std::size_t(field->shape_x) * (field->shape_y + 1) *
                                                                 field->shape_z);
    velocity.z_faces.assign(field->z_faces, field->z_faces + std::size_t(field->shape_x) * field->shape_y *
                                                                 (field->shape_z + 1));
    spec.velocity_field = velocity;
    sim.configure_signal_grid(spec);
    for (std::size_t s = 0; s < cells->count; ++s) {
      ms::CellInit init;
      init.position = {cells->position_x[s], cells->position_y[s], cells->position_z[s]};
      init.direction = {cells->direction_x[s], cells->direction_y[s], cells->direction_z[s]};
      init.length = cells->lengths[s];
      init.radius = cells->radii[s];
      init.growth_rate = cells->growth_rates != nullptr ? cells->growth_rates[s] : 0.0F;
      init.fixed = cells->fixed != nullptr && cells->fixed[s] != 0;
      sim.add_cell(init);
    }
    auto p = dynamics_parameters(*dynamics);
    p.flow_drift = true;
    const auto result = sim.step(dt, p);
    for (const auto& cell : sim.cells()) {
      const std::size_t s = cell.slot;
      if (s >= cells->count) continue;
      cells->position_x[s] = cell.position.x;
      cells->position_y[s] = cell.position.y;
      cells->position_z[s] = cell.position.z;
      cells->direction_x[s] = cell.direction.x;
      cells->direction_y[s] = cell.direction.y;
      cells->direction_z[s] = cell.direction.z;
      cells->lengths[s] = cell.length;
    }
    report->substeps = result.report.substeps;
    report->halvings = result.report.halvings;
    report->refinements = result.report.refinements;
    report->iterations = result.report.iterations;
    report->max_rows = result.report.max_rows;
    report->max_overlap = result.report.max_overlap;
  });
}

// --- a world kept across calls -------------------------------------------

void* ref_world_create(const msb_cell_arrays* cells, const msb_constraint* constraints,
                       uint64_t constraint_count) {
  try {
    auto world = new RefWorld{make_world(*cells), make_constraints(constraints, constraint_count),
                              ms::make_cpu_backend()};
    return world;
  } catch (const std::exception& error) {
    last_error = error.what();
    return nullptr;
  }
}

void ref_world_destroy(void* world) {
  delete static_cast<RefWorld*>(world);
}

uint64_t ref_world_size(void* world) {
  return static_cast<RefWorld*>(world)->state.size();
}

int ref_world_step(void* handle, float dt, const msb_contact_dynamics_parameters* dynamics,
                   msb_contact_dynamics_report* report) {
  return guarded([&] {
    auto& world = *static_cast<RefWorld*>(handle);
    const auto result = ms::detail::advance_contact_dynamics(
        world.state, world.constraints, *world.backend, dt, dynamics_parameters(*dynamics), {},
        {});
    report->substeps = result.report.substeps;
    report->halvings = result.report.halvings;
    report->refinements = result.report.refinements;
    report->iterations = result.report.iterations;
    report->max_rows = result.report.max_rows;
    report->max_overlap = result.report.max_overlap;
  });
}

// Divides each listed parent in half and turns the two daughters in the xy
// plane, as the reference's division tests do
// (tests/cpp/contact_dynamics_test.cpp:41-58).  `rotations` holds the cosine
// and sine of each daughter's turn (four floats per parent), so that every
// path that replays the division sees the same float values.
int ref_world_divide(void* handle, const uint64_t* parents, uint64_t count,
                     const float* rotations) {
  return guarded([&] {
    auto& world = *static_cast<RefWorld*>(handle);
    for (std::uint64_t index = 0; index < count; ++index) {
      const auto [first, second] = world.state.divide_equal(parents[index]);
      const ms::CellId daughters[2] = {first, second};
      for (int d = 0; d < 2; ++d) {
        const auto cell = world.state.cell(daughters[d]);
        const float c = rotations[4 * index + 2 * d];
        const float s = rotations[4 * index + 2 * d + 1];
        const ms::Vec3 direction{cell.direction.x * c - cell.direction.y * s,
                                 cell.direction.x * s + cell.direction.y * c, cell.direction.z};
        world.state.set_cell_geometry(daughters[d], cell.position, direction, cell.length);
      }
    }
  });
}

int ref_world_read(void* handle, uint64_t* ids, float* position_x, float* position_y,
                   float* position_z, float* direction_x, float* direction_y, float* direction_z,
                   float* lengths) {
  return guarded([&] {
    const auto& world = *static_cast<RefWorld*>(handle);
    const auto view = world.state.geometry_state();
    for (std::size_t slot = 0; slot < view.size(); ++slot) {
      ids[slot] = view.ids[slot];
      position_x[slot] = view.position_x[slot];
      position_y[slot] = view.position_y[slot];
      position_z[slot] = view.position_z[slot];
      direction_x[slot] = view.direction_x[slot];
      direction_y[slot] = view.direction_y[slot];
      direction_z[slot] = view.direction_z[slot];
      lengths[slot] = view.lengths[slot];
    }
  });
}

}  // extern "C"
