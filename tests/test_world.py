"""The host-side containers mirror the reference's: ConstraintSet validates
as ConstraintSet::add_* does and stores a plane's inward normal normalized in
FP32 (cpp/core/constraints.cpp:169-234)."""

import numpy as np
import pytest

from microsimulator_b200 import abi
from microsimulator_b200.world import ConstraintSet


def test_plane_normal_is_stored_normalized():
    cs = ConstraintSet()
    cs.add_plane(point=(0.0, 0.0, 0.0), inward_normal=(0.0, 2.0, 0.0), coefficient=3.0)
    cs.add_plane(point=(1.0, 0.0, 0.0), inward_normal=(1.0, 1.0, 0.5))
    assert cs.records["b"][0].tolist() == [0.0, 1.0, 0.0]
    n = np.array([1.0, 1.0, 0.5], np.float32)
    magnitude = np.sqrt(np.float32(np.float32(n[0] * n[0]) + np.float32(n[1] * n[1])) + np.float32(n[2] * n[2]),
                        dtype=np.float32)
    expected = n * np.float32(np.float32(1.0) / magnitude)
    assert np.array_equal(cs.records["b"][1], expected)
    assert cs.records["id"].tolist() == [1, 2]


@pytest.mark.parametrize("call", [
    lambda cs: cs.add_plane(inward_normal=(0.0, 0.0, 0.0)),
    lambda cs: cs.add_plane(point=(np.inf, 0.0, 0.0)),
    lambda cs: cs.add_plane(coefficient=0.0),
    lambda cs: cs.add_sphere(radius=-1.0),
    lambda cs: cs.add_box(half_extents=(1.0, 0.0, 1.0)),
    lambda cs: cs.add_cylinder(half_height=np.nan),
    lambda cs: cs.add_cylinder(coefficient=-2.0),
])
def test_invalid_constraints_are_rejected(call):
    cs = ConstraintSet()
    with pytest.raises(ValueError):
        call(cs)
    assert len(cs) == 0
