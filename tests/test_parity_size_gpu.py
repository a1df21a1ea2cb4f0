"""Parity of the plain FP64 form with the reference's own run at full size.

The reference's C++ (oracle/_ref/gg_ref, built from its sources by
oracle/Makefile with the direct-DFT FFT shim) and the library run the same
seeded voxelized input; the library takes the reference's initial neighbour
order (the reference seeds it from an R-tree walk), then both run the time
loop of src/grainhdl.cpp:1049-1142 and dump their state.

- 1,000 grains on 800^2 (Voronoi of uniform seeds, seed 0), isotropic,
  100 steps: every grain's distance field, IDLocal map, contour, junctions,
  neighbour list, area, energy and perimeter bit for bit, per-pixel
  ownership, surviving-grain count exact.
- 20,000 grains on 3600^2 (seed 1), Read-Shockley energy, 10 steps: every
  discrete output identical (states, boxes, lists, junctions, neighbour
  IDs, ownership, surviving count), fields, contours and areas within the
  anisotropic tolerance of tests/parity.py (the per-pair physics uses the
  device's acos / log, whose last bit can differ from glibc's).
"""
import os
import subprocess

import pytest

from gragles2d_b200 import dumpfile, gg
from gragles2d_b200 import microstructure as ms
from tests.parity import compare_records, ownership_mismatch

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GG_REF = os.path.join(ROOT, "oracle", "_ref", "gg_ref")


def _reference_run(d, name, micro, steps, **params):
    """Writes the case and runs the reference for `steps` steps (loops
    0 .. steps - 1); returns (xml, initial record, final record, delta)."""
    xml = ms.make_case(d, name, micro, NumberOfTimesteps=steps - 1, **params)
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    subprocess.run([GG_REF, os.path.basename(xml), "ref.dump", "0", "1"], cwd=d, env=env, check=True,
                   capture_output=True, timeout=1800)
    ref = dumpfile.read(os.path.join(d, "ref.dump"))
    assert ref.records[-1].steps == steps
    return xml, ref.records[0], ref.records[-1], ref.delta, ref.ngridpoints


def _library_run(xml, first, steps, path):
    h = gg.GrainHandler(gg.Settings(xml, precision=gg.PRECISION_PLAIN), device=0)
    try:
        h.load_voxel_files()
        h.distanceInitialisation()
        h.set_neighbours({gid: g.sec for gid, g in first.grains.items() if g.state})
        h.step(steps)
        assert h.status() == 0
        h.dump(path, steps)
    finally:
        h.close()
    return dumpfile.read(path).records[0]


def _check(want, got, m, exact, delta):
    problems = compare_records(want, got, exact=exact, delta=delta)
    assert not problems, problems[:10]
    assert ownership_mismatch(want, got, m) == 0
    alive_ref = sum(1 for g in want.grains.values() if g.state == 1)
    alive = sum(1 for g in got.grains.values() if g.state == 1)
    assert alive == alive_ref
    return alive


@pytest.mark.skipif(not os.path.exists(GG_REF), reason="oracle/_ref/gg_ref not built (reference sources absent)")
def test_1000_grains_800_isotropic_100_steps_bit_exact(tmp_path):
    d = str(tmp_path / "case1")
    xml, first, last, delta, m = _reference_run(d, "voronoi_1000g_800_iso", ms.voronoi(1000, 800, 0), 100,
                                                IsIsotropicNetwork=1)
    got = _library_run(xml, first, 100, str(tmp_path / "got.dump"))
    alive = _check(last, got, m, True, delta)
    assert alive < 1000  # grains vanished on the way, and the count matched


@pytest.mark.skipif(not os.path.exists(GG_REF), reason="oracle/_ref/gg_ref not built (reference sources absent)")
def test_20000_grains_3600_read_shockley_10_steps(tmp_path):
    d = str(tmp_path / "case2")
    xml, first, last, delta, m = _reference_run(d, "voronoi_20000g_3600_rs15", ms.voronoi(20000, 3600, 1), 10,
                                                IsIsotropicNetwork=0)
    got = _library_run(xml, first, 10, str(tmp_path / "got.dump"))
    _check(last, got, m, False, delta)
