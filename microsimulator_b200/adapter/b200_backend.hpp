// The B200 backend as a MicroSimulator ComputeBackend
// (cpp/include/microsimulator/backend.hpp:21-56 of the reference).
//
// This is the drop-in a MicroSimulator build compiles in place of
// cpp/cuda/cuda_backend.cu: it defines make_cuda_backend and
// cuda_backend_device_count (backend.hpp:60-62), so Simulation(BackendKind::cuda)
// (cpp/core/simulation.cpp:18-36) selects it unchanged.  The contact methods
// call libmsb200.so through its C-ABI (include/msb200.h).
#pragma once

#include <cstdint>
#include <memory>

#include "microsimulator/backend.hpp"
#include "msb200.h"

namespace microsimulator {

class B200Backend final : public ComputeBackend {
 public:
  // A backend on B200 `device_index`.  `host_features`, when given, serves
  // the features outside the contact path (growth, species, signals,
  // coupled rates, flow), which this library does not implement; without it
  // those features are unsupported and their calls throw.
  explicit B200Backend(std::uint32_t device_index, std::unique_ptr<ComputeBackend> host_features = nullptr);
  ~B200Backend() override;
  B200Backend(const B200Backend&) = delete;
  B200Backend& operator=(const B200Backend&) = delete;

  [[nodiscard]] BackendInfo info() const override;
  [[nodiscard]] bool supports(BackendFeature feature) const noexcept override;

  // The contact path, on the GPU.
  [[nodiscard]] ContactGraph find_cell_contacts(const WorldState& state,
                                                const ContactParameters& parameters) override;
  [[nodiscard]] ExternalContactGraph find_external_contacts(const WorldState& state,
                                                            const ConstraintSet& constraints,
                                                            const ConstraintContactParameters& parameters) override;
  [[nodiscard]] ContactSolveResult solve_contact_forces(const ContactSystem& system,
                                                        std::span<const float> initial_multipliers,
                                                        const ContactSolveParameters& parameters) override;

  // The whole contact-dynamics step in one call: what
  // detail::advance_contact_dynamics (cpp/core/contact_stepper.hpp:32-35)
  // computes with this backend, with every per-cell, per-row and per-contact
  // pass on the device and only the substep controller on the host.  It is
  // the override a whole-step virtual on ComputeBackend would take.  A step
  // with parameters.flow_drift throws std::logic_error: its drift rates come
  // from the Simulation's signal grid, which this call does not see, so such
  // steps stay with the host stepper.  The state is unchanged if this throws.
  [[nodiscard]] ContactDynamicsResult advance_contact_dynamics(
      WorldState& state, const ConstraintSet& constraints, float dt, const ContactDynamicsParameters& parameters,
      const ContactParameters& contact_parameters, const ConstraintContactParameters& constraint_parameters);

  // Features outside the contact path: forwarded to `host_features`.
  void advance_growth(WorldState& state, float dt) override;
  void advance_species(WorldState& state, const SpeciesRatePlan& plan, std::span<const float> previous_lengths,
                       float dt) override;
  [[nodiscard]] SignalSolveReport advance_signal_grid(SignalGrid& grid, float dt) override;
  [[nodiscard]] SignalSolveReport advance_coupled(WorldState& state, SignalGrid& grid, const CoupledRatePlan& plan,
                                                  std::span<const float> previous_lengths, float dt) override;
  [[nodiscard]] DepthAveragedFlowResult solve_depth_averaged_flow(
      const SignalGridSpec& spec, std::span<const float> mobility,
      const DepthAveragedFlowParameters& parameters) override;
  [[nodiscard]] DepthAveragedPortFlowResult solve_depth_averaged_port_flow(
      const SignalGridSpec& spec, std::span<const FlowPort> ports, std::span<const float> mobility,
      const DepthAveragedPortFlowParameters& parameters) override;
  [[nodiscard]] ResolvedFlowResult solve_resolved_flow(const SignalGridSpec& spec, std::span<const float> drag,
                                                       const ResolvedFlowParameters& parameters) override;
  [[nodiscard]] ResolvedPortFlowResult solve_resolved_port_flow(const SignalGridSpec& spec,
                                                                std::span<const FlowPort> ports,
                                                                std::span<const float> drag,
                                                                const ResolvedPortFlowParameters& parameters) override;

  [[nodiscard]] msb_context* context() const noexcept { return context_; }

 private:
  ComputeBackend& host(BackendFeature feature, const char* what) const;

  msb_context* context_ = nullptr;
  std::uint32_t device_index_ = 0;
  std::unique_ptr<ComputeBackend> host_features_;
};

// A contact-only backend: the three contact features, nothing else.
[[nodiscard]] std::unique_ptr<B200Backend> make_b200_contact_backend(std::uint32_t device_index);

}  // namespace microsimulator
