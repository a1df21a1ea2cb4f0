"""Failure detection without a GPU fault.

Inputs the device must never see are refused on the host: a non-finite
parameter, contour coordinate, quaternion, Euler angle or stored energy gives
GG_E_NUMERIC before anything is uploaded (boxes, pixel indices and contour
walks are derived from these values on the device).  Capacities that a
network outgrows on the device are detected there and stop the call with
GG_E_CAPACITY: a comparison list longer than the list capacity (a smaller
capacity is set through gg_params.list_capacity), in the initial neighbour
search and in the second-order update of a step; and arenas that the boxes
outgrow (a tighter arena is set through gg_params.arena_factor).  Every list
write on the device is bounded by the capacity, so a list overflow only sets
the status bit; an arena overflow is found by the allocation kernel before
any box is written at the new offsets, and every later kernel returns at
once (GG_S_ARENA_FULL), so the step and the calls after it return the error.
"""
import math
import os

import numpy as np
import pytest

from gragles2d_b200 import dumpfile, gg

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _xml(case):
    return os.path.join(GOLDEN, case, case + ".xml")


def test_nonfinite_parameter_is_refused():
    with pytest.raises(gg.GGError) as e:
        gg.GrainHandler(gg.Settings(_xml("rs_v30"), triple_point_drag=math.nan))
    assert e.value.code == 6


def test_nonfinite_contour_coordinate_is_refused():
    s = gg.Settings(_xml("iso_v20"), microstructure_gen_mode=0, number_of_particles=2)
    h = gg.GrainHandler(s)
    try:
        square = [(0.2, 0.2), (0.4, 0.2), (0.4, 0.4), (0.2, 0.4)]
        bad = [(0.6, 0.6), (0.8, 0.6), (math.nan, 0.8), (0.6, 0.8)]
        q = [(1.0, 0.0, 0.0, 0.0)] * 2
        with pytest.raises(gg.GGError) as e:
            h.load_contours([square, bad], q)
        assert e.value.code == 6
        with pytest.raises(gg.GGError) as e:
            h.load_contours([square, square], [(1.0, 0.0, 0.0, 0.0), (math.inf, 0.0, 0.0, 0.0)])
        assert e.value.code == 6
        h.load_contours([square, [(x + 0.4, y + 0.4) for x, y in square]], q)  # the same call with good values
    finally:
        h.close()


def test_nonfinite_euler_angle_is_refused():
    n = 20
    ids = np.zeros((100, 100), np.int32)
    euler = np.zeros((n, 3))
    euler[3, 1] = np.nan
    bbox = np.zeros((n, 5), np.int32)
    h = gg.GrainHandler(gg.Settings(_xml("iso_v20")))
    try:
        with pytest.raises(gg.GGError) as e:
            h.load_voxels(ids, euler, bbox)
        assert e.value.code == 6
    finally:
        h.close()


@pytest.mark.parametrize("precision", [gg.PRECISION_PLAIN, gg.PRECISION_BATCHED])
def test_list_capacity_overflow_in_the_neighbour_search(precision):
    h = gg.GrainHandler(gg.Settings(_xml("iso_v60"), precision=precision, list_capacity=3))
    try:
        h.load_voxel_files()
        h.distanceInitialisation()
        with pytest.raises(gg.GGError) as e:
            h.find_neighbors()
        assert e.value.code == 5
        assert h.status() & 2  # GG_S_LIST_OVERFLOW
    finally:
        h.close()


@pytest.mark.parametrize("precision", [gg.PRECISION_PLAIN, gg.PRECISION_BATCHED])
def test_list_capacity_overflow_in_a_step(precision):
    """Initial lists of three members fill a capacity of 3; the second-order
    update of the first step adds the members' own members and overflows."""
    ref = dumpfile.read(os.path.join(GOLDEN, "iso_v60", "reference.dump.gz"))
    h = gg.GrainHandler(gg.Settings(_xml("iso_v60"), precision=precision, list_capacity=3))
    try:
        h.load_voxel_files()
        h.distanceInitialisation()
        h.set_neighbours({gid: g.sec[:3] for gid, g in ref.records[0].grains.items() if g.state})
        with pytest.raises(gg.GGError) as e:
            h.step(1)
        assert e.value.code == 5
        assert h.status() & 2
    finally:
        h.close()


def test_list_capacity_out_of_range_is_refused():
    with pytest.raises(gg.GGError) as e:
        gg.GrainHandler(gg.Settings(_xml("iso_v20"), list_capacity=129))
    assert e.value.code == 1


@pytest.mark.parametrize("precision", [gg.PRECISION_PLAIN, gg.PRECISION_BATCHED])
def test_arena_overflow_halts_and_returns(precision):
    """se_v30 (stored energies) grows its total box area above the initial
    total within five steps; with arenas of exactly the initial totals the
    allocation kernel finds the overflow, every kernel halts, the step
    returns GG_E_CAPACITY, and so does the next one."""
    h = gg.GrainHandler(gg.Settings(_xml("se_v30"), precision=precision, arena_factor=1.0))
    try:
        h.load_voxel_files()
        h.distanceInitialisation()
        h.find_neighbors()
        failed_at = None
        for k in range(1, 11):
            try:
                h.step(1)
            except gg.GGError as e:
                assert e.code == 5, e
                failed_at = k
                break
        assert failed_at is not None and failed_at <= 5, failed_at
        assert h.status() & 1  # GG_S_ARENA_FULL
        with pytest.raises(gg.GGError) as e:
            h.step(1)
        assert e.value.code == 5
    finally:
        h.close()


def test_arena_factor_below_one_is_refused():
    with pytest.raises(gg.GGError) as e:
        gg.GrainHandler(gg.Settings(_xml("iso_v20"), arena_factor=0.5))
    assert e.value.code == 1

