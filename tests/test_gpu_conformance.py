"""The reference's own conformance tests run unchanged against the B200
backend (tests/conformance/*.cpp of the reference, compiled with their
assertions on by oracle/Makefile's conformance target and linked with the
reference core built with MICROSIMULATOR_HAS_CUDA=1 and the B200 adapter).
Simulation(BackendKind::cuda) there selects make_cuda_backend of
microsimulator_b200/adapter/b200_backend.cpp, whose contact methods run on
the B200 through libmsb200.so and whose other features are the reference's
CPU backend.  Each executable compares the CUDA backend with the CPU
backend in the same process:

* contact_conformance: mixed, dense (31 coincident capsules), margins and
  buffer reuse, ids after a division; fields within 2e-5, ids, slots,
  ordinals and incidence exact;
* constraint_conformance: the ten wall fixtures and empty inputs;
* contact_dynamics_conformance: the make_chain solves (2e-3 response), the
  iteration limit, the closed chamber (500 steps) and the free colony
  (100 steps) through the host stepper calling the backend;
* trajectory_conformance: growth, contacts with a plane and a fixed cell,
  coupled rates and signals, a division, over three steps (geometry 2e-3);
* backend_contract_conformance: all nine features advertised;
* whole_step_test (tests/native/whole_step_test.cpp): the adapter's
  whole-step call against the reference's stepper."""

import subprocess

import pytest

from tests.test_conformance_build import CONFORMANCE, TESTS, built

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", TESTS + ["whole_step_test"])
def test_reference_conformance_through_the_adapter(name):
    built()
    from microsimulator_b200 import backend

    assert backend.device_count() >= 1  # the CUDA backend is enumerated
    run = subprocess.run([str(CONFORMANCE / name)], capture_output=True, text=True, timeout=1800)
    print(run.stdout[-3000:])
    assert run.returncode == 0, (name, run.returncode, run.stderr[-3000:])
