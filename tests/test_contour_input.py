"""Contour input (MicrostructureGenMode 0) on the CPU: the restatement of the
contour constructor's box and of LSbox::calculateDistanceFunction in
oracle/gg_oracle.c against the initial state GraGLeS2D itself built from its
own restart files (tests/golden/rst_*: the restart files of a voxelized run,
then the reference's run from them), bit for bit; the parameters the restart
writer emits parse into a mode-0 gg_params; gg_create refuses the modes that
need voro++ or vertex files."""
import json
import math
import os

import numpy as np
import pytest

from gragles2d_b200 import dumpfile, gg
from oracle import analysis, port

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["rst_iso_v60", "rst_rs_v30", "rst_se_v30", "rst_gc_v80"]


def _case(name):
    d = os.path.join(GOLDEN, name)
    with open(os.path.join(d, "case.json")) as f:
        info = json.load(f)
    return d, info


@pytest.mark.parametrize("name", CASES)
def test_oracle_polygon_initialisation_matches_the_reference(name):
    d, info = _case(name)
    s = gg.Settings(os.path.join(d, info["parameters"]))
    p = s.p
    assert p.microstructure_gen_mode == 0 and p.start_time == info["restart_loop"]
    ref = dumpfile.read(os.path.join(d, "reference.dump.gz"))
    # the grid of setSimulationParameter for file input (src/grainhdl.cpp:74-78)
    nn = int(math.sqrt(p.number_of_particles) * p.number_of_points_per_grain)
    b = p.domain_border_size
    assert ref.ngridpoints == nn + 2 * b
    h, delta = 1.0 / nn, b / nn
    assert ref.h == h and ref.delta == delta
    polys, quats = analysis.read_network(os.path.join(d, p.read_from_filename.decode()), p.number_of_particles)
    rec = ref.records[0]
    assert sorted(rec.grains) == list(range(1, len(polys) + 1))
    m = nn + 2 * b
    for gid, pts in enumerate(polys, start=1):
        g = rec.grains[gid]
        assert g.state == 1
        box = port.new_box(port.polygon_box(pts, m, b, h), m)
        assert tuple(g.box) == box, gid
        phi = port.polygon_phi(pts, box, b, h, delta)
        np.testing.assert_array_equal(phi, g.phi, err_msg=f"grain {gid}")
        np.testing.assert_array_equal(g.contour[:, :2], pts)
        assert not g.contour[:, 2:].any() and len(g.junctions) == 0
        assert g.volume == port.area(pts, h) / (h * h)


def test_reader_numbers_grains_in_file_order(tmp_path):
    f = tmp_path / "net.dat"
    f.write_text("5\t3\t1\t0\t0\t0\n0.1\t0.1\n0.2\t0.1\n0.1\t0.2\n\n"
                 "9\t3\t0.5\t0.5\t0.5\t0.5\n0.5\t0.5\n1.5\t0.5\n0.5\t-0.5\n\n")
    polys, quats = analysis.read_network(str(f), 2)
    # the second record's ID (9) raises the grain count; grains 3..9 have no record
    assert len(polys) == 9 and quats[1] == (0.5, 0.5, 0.5, 0.5)
    np.testing.assert_array_equal(polys[1], [[0.5, 0.5], [1.0, 0.5], [0.5, 0.0]])
    assert all(len(q) == 0 for q in polys[2:])


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_create_rejects_generation_modes(mode):
    s = gg.Settings(os.path.join(GOLDEN, "iso_v20", "iso_v20.xml"), microstructure_gen_mode=mode)
    with pytest.raises(gg.GGError) as e:
        gg.GrainHandler(s)
    assert e.value.code == 1 and "MicrostructureGenMode" in str(e.value)


def test_oracle_polygon_distance_known_answers():
    """A square of side 0.5 centred in the unit domain on a 40-point grid:
    inside, the distance to the nearest side; outside, to the nearest side or
    corner; both clamped to delta."""
    nn, b = 40, 7
    h, delta = 1.0 / nn, b / nn
    sq = np.array([[0.25, 0.25], [0.75, 0.25], [0.75, 0.75], [0.25, 0.75], [0.25, 0.25]])
    m = nn + 2 * b
    box = (0, m, 0, m)
    phi = port.polygon_phi(sq, box, b, h, delta)
    for i in range(m):
        for j in range(m):
            x, y = (j - b) * h, (i - b) * h
            dx = max(0.25 - x, 0.0, x - 0.75)
            dy = max(0.25 - y, 0.0, y - 0.75)
            inside = 0.25 < x < 0.75 and 0.25 < y < 0.75
            d = min(x - 0.25, 0.75 - x, y - 0.25, 0.75 - y) if inside else float(np.hypot(dx, dy))
            want = min(d, delta) * (1 if inside else -1)
            assert abs(phi[i, j] - want) <= 1e-15, (i, j, phi[i, j], want)
