"""Pins the C restatement of the step (oracle/gg_oracle.c) against the
reference's own run: from each dumped record r of the every-step fixture,
restate step r+1 grain by grain and require the reference's record r+1 bit
for bit (IDLocal, bounding boxes, contour, junctions, area, perimeter and the
redistanced field)."""
import os
import sys

import numpy as np
import pytest

from gragles2d_b200 import dumpfile

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
from oracle import port  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def seq():
    port.load()
    return dumpfile.read(os.path.join(GOLDEN, "seq_v24", "reference.dump.gz"))


def _clip(nb, m):
    return (max(nb[0], 0), min(nb[1], m), max(nb[2], 0), min(nb[3], m))


def _restate_step(d, r0, r1):
    """Checks one step; returns (grains compared, irregular ones skipped)."""
    m, nn = d.ngridpoints, d.nn
    b = (m - nn) // 2
    assert m == nn + 2 * b
    conv = {gid: port.convolve(g.phi, d.dt, nn) for gid, g in r0.grains.items() if g.state == 1}
    checked = skipped = 0
    for gid, g0 in r0.grains.items():
        if g0.state != 1:
            continue
        g1 = r1.grains[gid]
        members = [(k, r0.grains[k].box, conv[k]) for k in g1.cmp]
        cmp, idl, nb = port.compare(g0.box, conv[gid], members, g0.id_box, g0.idlocal, m, b, d.h, d.delta)
        assert g1.id_box == g0.box, gid
        np.testing.assert_array_equal(idl, g1.idlocal, err_msg=f"IDLocal of grain {gid}")
        pts, junc = port.contour(cmp, g0.box, idl, gid)
        if len(pts) == 0:
            assert g1.state != 1, gid
            continue
        assert _clip(nb, m) == g1.newbb, gid
        area = port.area(pts, d.h)
        regular, flagged = port.motion_regular(len(g0.contour), len(pts), g0.volume, area, d.dt)
        if not regular:
            skipped += 1
            continue
        np.testing.assert_array_equal(pts, g1.contour[:, :2], err_msg=f"contour of grain {gid}")
        assert len(junc) == len(g1.junctions), gid
        for a, e in zip(junc, g1.junctions):
            assert a[0] == e[0] and a[1][:a[0]] == e[1][:e[0]] and a[2] == e[2], (gid, a, e)
            assert a[3:] == e[3:], (gid, a, e)
        assert port.perimeter(pts, d.h) == g1.perimeter, gid
        if not flagged:
            assert area == g1.volume, gid
        box1 = port.new_box(_clip(nb, m), m)
        assert box1 == g1.box, gid
        phi1 = port.redistance(cmp, g0.box, box1, d.h, d.delta)
        np.testing.assert_array_equal(phi1, g1.phi, err_msg=f"redistanced field of grain {gid}")
        checked += 1
    return checked, skipped


def test_restatement_matches_reference_every_step(seq):
    pairs = [(a, c) for a, c in zip(seq.records, seq.records[1:]) if c.steps == a.steps + 1]
    assert len(pairs) >= 4
    total = skipped = 0
    for r0, r1 in pairs:
        c, s = _restate_step(seq, r0, r1)
        total += c
        skipped += s
    assert total >= 0.9 * sum(1 for r0, _ in pairs for g in r0.grains.values() if g.state == 1)


def test_wall_distance_and_compare_on_boundary(seq):
    """A grain touching the domain wall takes the boundary condition: pixels
    beyond the wall get IDLocal 0 (checked inside the step restatement on the
    fixture's border grains, here made explicit)."""
    d = seq
    m, nn = d.ngridpoints, d.nn
    b = (m - nn) // 2
    r0, r1 = d.records[1], d.records[2]
    border = [gid for gid, g in r0.grains.items()
              if g.state == 1 and (g.box[0] < b or g.box[2] < b or g.box[1] > m - b or g.box[3] > m - b)]
    assert border
    walls = 0
    conv = {gid: port.convolve(g.phi, d.dt, nn) for gid, g in r0.grains.items() if g.state == 1}
    for gid in border:
        g0, g1 = r0.grains[gid], r1.grains[gid]
        members = [(k, r0.grains[k].box, conv[k]) for k in g1.cmp]
        _, idl, _ = port.compare(g0.box, conv[gid], members, g0.id_box, g0.idlocal, m, b, d.h, d.delta)
        walls += int((idl == 0).any())
        np.testing.assert_array_equal(idl, g1.idlocal)
    assert walls > 0


def test_redistance_output_box_and_clamp():
    """The sweeps fill the whole output box (also where it reaches beyond
    the input box) and clamp to [-delta, delta]."""
    n, h, delta = 32, 1.0 / 30, 5.0 / 30
    x = np.arange(n)[None, :].repeat(n, 0)
    phi = np.clip((x - 15.5) * h, -delta, delta)
    out = port.redistance(phi, (10, 10 + n, 20, 20 + n), (4, 4 + n + 8, 16, 16 + n + 8), h, delta)
    assert out.shape == (n + 8, n + 8)
    assert np.all(np.abs(out) <= delta)
    # the interface column keeps its interpolated distance
    np.testing.assert_allclose(out[10:30, 6 + 15], -0.5 * h, rtol=1e-12)


def test_new_box_square_and_inside():
    m = 100
    for nb in [(-3, 20, 5, 60), (10, 120, 40, 45), (0, 99, 0, 99), (40, 50, 40, 50)]:
        b = port.new_box(nb, m)
        assert b[1] - b[0] == b[3] - b[2]
        assert b[0] >= 0 and b[2] >= 0
