// The B200 adapter's whole-step call against the reference's own stepper.
//
// detail::advance_contact_dynamics (cpp/core/contact_dynamics.cpp:676-782 of
// the reference) is run with the reference CPU backend, and
// B200Backend::advance_contact_dynamics on the same WorldState; the host
// stepper is also run with the B200 backend's per-call contact methods (the
// path Simulation(BackendKind::cuda) takes without a whole-step hook).
// Criteria: those of the reference's trajectory conformance test
// (tests/conformance/trajectory_conformance_test.cpp:140-172), geometry within
// 2e-3 absolute plus relative after every step, and positions within 4 x the
// overlap tolerance; at the tight tolerance, positions within 1e-4 capsule
// radius.  Exits 77 without a CUDA device, 0
// when every check passes, 1 on the first failure.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <stdexcept>
#include <tuple>
#include <vector>

#include "b200_backend.hpp"
#include "core/contact_stepper.hpp"

namespace ms = microsimulator;

namespace {

int failures = 0;

void expect(bool ok, const char* what, double value = 0.0) {
  if (!ok) {
    std::fprintf(stderr, "FAIL: %s (%g)\n", what, value);
    ++failures;
  }
}

ms::WorldState colony(std::size_t n, float side, std::uint64_t seed) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<float> position(0.0F, side);
  std::uniform_real_distribution<float> length(2.0F, 4.0F);
  std::uniform_real_distribution<float> angle(0.0F, 3.14159265F);
  ms::WorldState state;
  for (std::size_t i = 0; i < n; ++i) {
    ms::CellInit cell;
    cell.position = {position(rng), position(rng), 0.0F};
    const float a = angle(rng);
    cell.direction = {std::cos(a), std::sin(a), 0.0F};
    cell.length = length(rng);
    cell.radius = 0.5F;
    cell.growth_rate = 0.5F;
    state.add_cell(cell);
  }
  return state;
}

// Largest |a - b| over positions (and directions, lengths when `all`), and
// whether every value is within tol * (1 + |b|).
struct Spread {
  double position = 0.0;
  bool within = true;
};

Spread spread(const ms::WorldState& a, const ms::WorldState& b, float tolerance) {
  const auto x = a.geometry_state();
  const auto y = b.geometry_state();
  Spread s;
  if (x.size() != y.size()) return {1e30, false};
  const std::span<const float> fa[7] = {x.position_x, x.position_y, x.position_z, x.direction_x,
                                        x.direction_y, x.direction_z, x.lengths};
  const std::span<const float> fb[7] = {y.position_x, y.position_y, y.position_z, y.direction_x,
                                        y.direction_y, y.direction_z, y.lengths};
  for (int k = 0; k < 7; ++k) {
    for (std::size_t i = 0; i < x.size(); ++i) {
      const double d = std::abs(double(fa[k][i]) - double(fb[k][i]));
      if (k < 3) s.position = std::max(s.position, d);
      if (d > tolerance + tolerance * std::abs(double(fb[k][i]))) s.within = false;
    }
  }
  return s;
}

// `steps` steps of a colony.  Before each, the whole-step call and the host
// stepper with the B200 backend's per-call methods start from the
// reference's state after the previous step, so that each step is compared
// on its own: a colony relaxing from an overlapping start is chaotic, and a
// one-ulp difference in a turned axis (the device's cosf/sinf against the
// host's) would otherwise grow from step to step.
void steps_from_the_reference(ms::B200Backend& b200, ms::ComputeBackend& cpu, ms::WorldState world,
                              const ms::ConstraintSet& walls, int steps, float tolerance, const char* name) {
  ms::ContactDynamicsParameters p;
  p.overlap_tolerance = tolerance;
  const ms::ContactParameters c{};
  const ms::ConstraintContactParameters w{};
  ms::WorldState reference = world;
  for (int step = 0; step < steps; ++step) {
    ms::WorldState hooked = reference, percall = reference;
    const auto rh = b200.advance_contact_dynamics(hooked, walls, 0.02F, p, c, w);
    const auto rp = ms::detail::advance_contact_dynamics(percall, walls, b200, 0.02F, p, c, w);
    const auto rr = ms::detail::advance_contact_dynamics(reference, walls, cpu, 0.02F, p, c, w);
    const auto sh = spread(hooked, reference, 2.0e-3F);
    const auto sp = spread(percall, reference, 2.0e-3F);
    std::printf("%s step %d: substeps %u/%u/%u, iterations %llu/%llu/%llu, max |position - reference| "
                "whole-step %.3e, per-call %.3e\n",
                name, step, rh.report.substeps, rp.report.substeps, rr.report.substeps,
                (unsigned long long)rh.report.iterations, (unsigned long long)rp.report.iterations,
                (unsigned long long)rr.report.iterations, sh.position, sp.position);
    expect(sh.within, "whole-step geometry within 2e-3 of the reference", sh.position);
    expect(sp.within, "per-call geometry within 2e-3 of the reference", sp.position);
    expect(sh.position <= 4.0 * tolerance, "whole-step positions within 4 x tolerance", sh.position);
    expect(sp.position <= 4.0 * tolerance, "per-call positions within 4 x tolerance", sp.position);
    expect(rh.report.substeps == rr.report.substeps, "whole-step substeps", rh.report.substeps);
    expect(std::abs(rh.report.max_overlap - rr.report.max_overlap) <= 2.0F * tolerance, "max overlap",
           rh.report.max_overlap);
  }
}

}  // namespace

int main() {
  if (ms::cuda_backend_device_count() == 0) {
    std::printf("no CUDA device: skipped\n");
    return 77;
  }
  try {
    ms::B200Backend b200(0);
    auto cpu = ms::make_cpu_backend(0);

    // A growing colony from an overlapping random start.
    steps_from_the_reference(b200, *cpu, colony(120, 16.0F, 42), ms::ConstraintSet{}, 6, 2.0e-4F, "colony");

    // Cells in a closed box chamber and against a plane: wall rows.
    {
      ms::ConstraintSet walls;
      ms::BoxConstraintInit box;
      box.center = {8.0F, 8.0F, 0.0F};
      box.half_extents = {7.0F, 7.0F, 0.6F};
      box.allowed_region = ms::ConstraintRegion::inside;
      walls.add_box(box);
      ms::PlaneConstraintInit plane;
      plane.point = {0.0F, 4.0F, 0.0F};
      plane.inward_normal = {0.0F, 1.0F, 0.0F};
      plane.coefficient = 1.25F;
      walls.add_plane(plane);
      steps_from_the_reference(b200, *cpu, colony(60, 14.0F, 7), walls, 6, 2.0e-4F, "walls");
    }

    // One step at a tight tolerance from a settled colony: positions within
    // 1e-4 capsule radius of the reference's step.
    {
      ms::WorldState world = colony(200, 22.0F, 11);
      ms::ContactDynamicsParameters settle;
      settle.overlap_tolerance = 5.0e-4F;
      for (int k = 0; k < 15; ++k) {
        std::ignore = ms::detail::advance_contact_dynamics(world, {}, *cpu, 0.02F, settle, {}, {});
      }
      ms::ContactDynamicsParameters tight;
      tight.overlap_tolerance = 2.0e-5F;
      ms::WorldState gpu = world, ref = world;
      const auto rg = b200.advance_contact_dynamics(gpu, {}, 0.02F, tight, {}, {});
      const auto rr = ms::detail::advance_contact_dynamics(ref, {}, *cpu, 0.02F, tight, {}, {});
      const auto s = spread(gpu, ref, 2.0e-3F);
      std::printf("tight step: substeps %u/%u, max |position - reference| %.3e um\n", rg.report.substeps,
                  rr.report.substeps, s.position);
      expect(rg.report.substeps == rr.report.substeps, "tight substeps", rg.report.substeps);
      expect(s.position <= 1.0e-4 * 0.5, "tight positions within 1e-4 radius", s.position);
      expect(rg.center_velocities.size() == gpu.size() && rg.axial_loads.size() == gpu.size(), "outputs sized");
    }

    // A step that cannot converge throws and leaves the state unchanged.
    {
      ms::WorldState world;
      for (float x : {-1.5F, 1.5F, 4.5F}) {
        ms::CellInit cell;
        cell.position = {x, 0.0F, 0.0F};
        cell.length = 2.0F;
        world.add_cell(cell);
      }
      const ms::WorldState before = world;
      ms::ContactDynamicsParameters p;
      p.max_iterations = 1;
      p.overlap_tolerance = 1.0e-7F;
      p.max_step_halvings = 2;
      bool threw = false;
      try {
        std::ignore = b200.advance_contact_dynamics(world, {}, 0.1F, p, {}, {});
      } catch (const std::runtime_error&) {
        threw = true;
      }
      expect(threw, "an unresolvable step throws std::runtime_error");
      expect(spread(world, before, 0.0F).within, "a failed step leaves the state unchanged");
      bool invalid = false;
      p = {};
      p.contact_stiffness = 0.0F;
      try {
        std::ignore = b200.advance_contact_dynamics(world, {}, 0.1F, p, {}, {});
      } catch (const std::invalid_argument&) {
        invalid = true;
      }
      expect(invalid, "invalid parameters throw std::invalid_argument");
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "FAIL: unexpected exception: %s\n", e.what());
    return 1;
  }
  if (failures != 0) {
    std::fprintf(stderr, "%d check(s) failed\n", failures);
    return 1;
  }
  std::printf("whole-step checks passed\n");
  return 0;
}
