"""Host-side statistics of the per-grain area comparison (no GPU).

``area_errors`` compares two area vectors indexed by grain ID - 1, NaN for a
grain that has vanished; these tests fix its counting rules on hand-made
vectors whose answers are known.
"""
import math

import numpy as np

from gragles2d_b200.accuracy import FLOOR_SCALE, area_errors


def test_identical_areas_have_zero_error():
    a = np.array([4.0, 9.0, 16.0])
    e = area_errors(a, a.copy(), cell=1.0)
    assert e["compared"] == 3
    assert e["max"] == 0.0 and e["p99"] == 0.0 and e["p50"] == 0.0
    assert e["over_1e-3"] == 0 and e["max_abs_cells"] == 0.0
    assert e["alive_only_ref"] == 0 and e["alive_only_other"] == 0


def test_worst_grain_is_reported_by_its_one_based_id():
    ref = np.array([100.0, 200.0, 50.0, 400.0])
    other = np.array([100.0, 200.1, 50.5, 400.0])
    e = area_errors(ref, other, cell=0.25)
    assert e["compared"] == 4
    assert math.isclose(e["max"], 0.5 / 50.0)
    assert e["worst"] == {"id": 3, "cells_ref": 200.0, "cells": 202.0}
    assert math.isclose(e["max_abs_cells"], 0.5 / 0.25)
    assert e["over_1e-3"] == 1
    assert e["p50"] == np.median(np.abs(other - ref) / ref)


def test_vanished_grains_are_counted_per_side_and_not_compared():
    ref = np.array([10.0, np.nan, 30.0, 40.0, np.nan])
    other = np.array([10.0, 20.0, np.nan, 40.0, np.nan])
    e = area_errors(ref, other, cell=1.0)
    assert e["compared"] == 2
    assert e["alive_only_ref"] == 1
    assert e["alive_only_other"] == 1
    assert e["max"] == 0.0


def test_zero_reference_area_is_not_divided_by():
    ref = np.array([0.0, 8.0])
    other = np.array([1.0, 8.0])
    e = area_errors(ref, other, cell=1.0)
    assert e["compared"] == 1
    assert e["max"] == 0.0


def test_nothing_in_common_gives_counts_only():
    ref = np.array([np.nan, 5.0])
    other = np.array([3.0, np.nan])
    e = area_errors(ref, other, cell=1.0)
    assert e == {"compared": 0, "alive_only_ref": 1, "alive_only_other": 1}


def test_floor_perturbation_is_a_few_fp64_ulps():
    # The perturbed run scales every boundary energy by 1 - 2^-46: below one
    # FP32 ulp (2^-24) by far, a handful of FP64 ulps (2^-53) of the energy.
    assert FLOOR_SCALE < 1.0
    assert (1.0 - FLOOR_SCALE) == 2.0 ** -46
    assert np.float32(FLOOR_SCALE) == np.float32(1.0)
