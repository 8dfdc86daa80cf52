"""The constraint fixtures of the reference's constraint conformance test
(tests/conformance/constraint_conformance_test.cpp:19-153), as host worlds
and constraint sets.  Each builder returns (WorldState, ConstraintSet)."""

from microsimulator_b200 import abi
from microsimulator_b200.world import ConstraintSet, WorldState


def _cells(*specs):
    w = WorldState()
    for position, direction, length, *radius in specs:
        w.add_cell(position=position, direction=direction, length=length, radius=radius[0] if radius else 0.5)
    return w


def mixed_constraints():
    w = _cells(((0.0, 0.4, 0.0), (1.0, 0.0, 0.0), 2.0), ((1.2, 0.6, 0.0), (0.0, 1.0, 0.0), 0.0),
               ((4.8, 2.0, 0.0), (0.0, 0.0, 1.0), 0.0))
    cs = ConstraintSet()
    assert cs.add_plane(inward_normal=(0.0, 2.0, 0.0), coefficient=1.25) == 1
    assert cs.add_sphere(radius=1.0, coefficient=0.75) == 2
    assert cs.add_sphere(radius=5.0, coefficient=1.5, allowed_region=abi.REGION_INSIDE) == 3
    assert cs.add_plane(point=(6.0, 0.0, 0.0), inward_normal=(-1.0, 0.0, 0.0)) == 4
    assert cs.add_box(center=(0.0, 1.3, 0.0), half_extents=(3.0, 0.5, 1.0), coefficient=0.9) == 5
    return w, cs


def box_regions():
    w = _cells(((1.4, 0.0, 0.0), (0.0, 1.0, 0.0), 2.0), ((1.3, 1.3, 0.0), (0.0, 0.0, 1.0), 0.0),
               ((0.5, 0.6, 0.0), (1.0, 0.0, 0.0), 0.0), ((4.8, 0.0, 0.0), (0.0, 1.0, 0.0), 0.0))
    cs = ConstraintSet()
    cs.add_box(half_extents=(2.0, 1.0, 3.0), coefficient=1.25)
    cs.add_box(half_extents=(5.0, 5.0, 5.0), coefficient=0.5, allowed_region=abi.REGION_INSIDE)
    return w, cs


def cylinder_regions():
    w = _cells(((1.4, 0.0, 0.0), (0.0, 0.0, 1.0), 2.0), ((1.3, 0.0, 1.3), (0.0, 1.0, 0.0), 0.0),
               ((0.5, 0.0, 1.4), (1.0, 0.0, 0.0), 0.0), ((4.8, 0.0, 0.0), (0.0, 1.0, 0.0), 0.0))
    cs = ConstraintSet()
    cs.add_cylinder(coefficient=1.25)
    cs.add_cylinder(radius=5.0, half_height=5.0, coefficient=0.5, allowed_region=abi.REGION_INSIDE)
    return w, cs


def degenerate_sphere():
    w = _cells(((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 0.0))
    cs = ConstraintSet()
    cs.add_sphere(radius=2.0)
    return w, cs


def degenerate_box():
    w = _cells(((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 0.0))
    cs = ConstraintSet()
    cs.add_box()
    return w, cs


def midspan_sphere():
    w = _cells(((0.0, 0.75, 0.0), (1.0, 0.0, 0.0), 3.5))
    cs = ConstraintSet()
    cs.add_sphere()
    return w, cs


def midspan_box():
    w = _cells(((0.0, 0.75, 0.0), (1.0, 0.0, 0.0), 3.5))
    cs = ConstraintSet()
    cs.add_box(half_extents=(1.0, 1.0, 5.0))
    return w, cs


def tilted_face_contacts():
    w = _cells(((1.3, 0.0, 0.0), (0.1, 1.0, 0.0), 1.0), ((1.4, 0.0, 2.0), (0.6, 0.8, 0.0), 1.0),
               ((11.3, 0.0, 0.0), (0.1, 0.0, 1.0), 1.0), ((11.4, 0.0, 0.0), (0.6, 0.0, 0.8), 1.0))
    cs = ConstraintSet()
    cs.add_box(half_extents=(1.0, 2.0, 3.0))
    cs.add_cylinder(center=(10.0, 0.0, 0.0), half_height=3.0)
    return w, cs


def centered_wall_crossing():
    w = _cells(((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 3.5))
    cs = ConstraintSet()
    cs.add_box(half_extents=(1.0, 5.0, 5.0))
    return w, cs


def midspan_cylinder():
    w = _cells(((0.0, 0.75, 0.0), (1.0, 0.0, 0.0), 3.5))
    cs = ConstraintSet()
    cs.add_cylinder(center=(0.4, 0.0, 0.0), half_height=5.0)
    return w, cs


FIXTURES = {f.__name__: f for f in (mixed_constraints, box_regions, cylinder_regions, degenerate_sphere,
                                     degenerate_box, midspan_sphere, midspan_box, tilted_face_contacts,
                                     centered_wall_crossing, midspan_cylinder)}
