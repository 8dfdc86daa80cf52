"""The reference's conformance tests, built against the B200 adapter
(microsimulator_b200/adapter/b200_backend.cpp) by oracle/Makefile's
conformance target: the adapter compiles against the reference's
ComputeBackend (cpp/include/microsimulator/backend.hpp:21-64) with the layout
checks of its ContactRow and ContactBody, and without a GPU each executable
runs its CPU backend's scenarios and passes (no CUDA device is enumerated).
The GPU runs are in test_gpu_conformance.py."""

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CONFORMANCE = ROOT / "oracle" / "_ref" / "conformance"
TESTS = ["contact_conformance", "constraint_conformance", "contact_dynamics_conformance",
         "trajectory_conformance", "backend_contract_conformance"]


def built():
    if Path("/root/reference/cpp").exists() and (ROOT / "microsimulator_b200" / "libmsb200.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "-j8", "ref", "conformance"], check=True)
    if not all((CONFORMANCE / name).exists() for name in TESTS + ["whole_step_test"]):
        pytest.skip("the conformance executables were not built and the reference sources are absent")


def test_adapter_builds_and_cpu_scenarios_pass():
    built()
    from microsimulator_b200 import backend

    if backend.device_count() > 0:
        pytest.skip("a CUDA device is present: test_gpu_conformance.py runs these")
    for name in TESTS:
        run = subprocess.run([str(CONFORMANCE / name)], capture_output=True, text=True, timeout=600)
        assert run.returncode == 0, (name, run.stderr[-2000:])
    skipped = subprocess.run([str(CONFORMANCE / "whole_step_test")], capture_output=True, text=True, timeout=60)
    assert skipped.returncode == 77
