"""The larger configurations at full size, through size-independent checks.

- 50,000 grains on 5600^2 (Voronoi, seed 3), Read-Shockley energy with the
  mobility model and triple-junction drag Lambda = 0.1 (TriplePointDrag =
  Lambda / a, a = 0.69 / sqrt(N) the mean edge length of a Poisson-Voronoi
  tessellation of the unit square): batched FP32 and plain FP64 side by side.
- 100,000 grains on 8192^2 from a Matern cluster process (radius 0.01, 100
  daughters per cluster on average, 95% of the seeds) mixed with uniform
  seeds: equivalent diameters lognormal-like with sigma ~0.6 and boxes from
  about 16 to 250 cells; batched FP32.

Checks: no device status bit, the grains still tile the domain (sum of areas
within 2e-3 of the unit square and drifting by less than 1e-3), and for the
first configuration the per-grain area agreement of the two forms (every
grain alive in both, no size cut).
"""
import os

import numpy as np
import pytest

from gragles2d_b200 import gg
from gragles2d_b200 import microstructure as ms

pytestmark = pytest.mark.gpu


def _case(root, name, micro, **params):
    d = os.path.join(root, name)
    return ms.make_case(d, name, micro, NumberOfTimesteps=10, **params)


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    root = str(tmp_path_factory.mktemp("scale"))
    n4 = 50000
    c4 = _case(root, "voronoi_50000g_5600", ms.voronoi(n4, 5600, 3), IsIsotropicNetwork=0, UseMobilityModel=1,
               TriplePointDrag=round(0.1 / (0.69 / np.sqrt(n4)), 3))
    m3 = ms.clustered(100000, 8192, 5, cluster_fraction=0.95, cluster_radius=0.01, mean_daughters=100.0)
    dia = ms.equivalent_diameters(m3)
    c3 = _case(root, "clustered_100000g_8192", m3, IsIsotropicNetwork=0)
    return {"c4": c4, "c3": c3, "c3_dia": dia}


def _run(xml, precision, steps):
    h = gg.GrainHandler(gg.Settings(xml, precision=precision), device=0)
    try:
        h.load_voxel_files()
        h.distanceInitialisation()
        h.find_neighbors()
        a0 = np.nansum([s.area for s in h.grain_stats() if s.state == 1])
        h.step(steps)
        st = h.grain_stats()
        live = [s for s in st if s.state == 1]
        areas = np.array([s.area if s.state == 1 else np.nan for s in st])
        edges = np.array([s.box[1] - s.box[0] for s in live])
        return {"status": h.status(), "a0": a0, "areas": areas, "edges": edges,
                "neighbours": np.array([s.n_neighbours for s in live]),
                "points": np.array([s.contour_points for s in live])}
    finally:
        h.close()


def test_50000_grains_batched_and_plain(cases):
    b = _run(cases["c4"], gg.PRECISION_BATCHED, 5)
    p = _run(cases["c4"], gg.PRECISION_PLAIN, 5)
    for r in (b, p):
        assert r["status"] == 0
        assert abs(r["a0"] - 1.0) < 2e-3
        assert abs(np.nansum(r["areas"]) - r["a0"]) < 1e-3
    assert np.array_equal(np.isfinite(b["areas"]), np.isfinite(p["areas"]))
    m = np.isfinite(b["areas"]) & (p["areas"] > 0)
    rel = np.abs(b["areas"][m] - p["areas"][m]) / p["areas"][m]
    assert np.median(rel) < 1e-6
    assert np.quantile(rel, 0.99) < 1e-5
    assert rel.max() <= 1e-3


def test_100000_clustered_grains_batched(cases):
    dia = cases["c3_dia"]
    assert 0.5 < np.std(np.log(dia[dia > 0])) < 0.7
    r = _run(cases["c3"], gg.PRECISION_BATCHED, 3)
    assert r["status"] == 0
    assert r["edges"].min() <= 24 and r["edges"].max() >= 200
    # headroom of the fixed per-grain capacities on the largest grains: direct
    # neighbours (48 rows), contour points (8 n + 64 for a box of edge n)
    cap_points = 8 * r["edges"] + 64
    print({"max_edge": int(r["edges"].max()), "max_neighbours": int(r["neighbours"].max()),
           "max_points": int(r["points"].max()), "max_points_over_capacity": float((r["points"] / cap_points).max())})
    assert r["neighbours"].max() <= 36  # of 48
    assert (r["points"] / cap_points).max() <= 0.75
    assert abs(r["a0"] - 1.0) < 2e-3
    assert abs(np.nansum(r["areas"]) - r["a0"]) < 1e-3


def test_100000_clustered_autotuned_bins(cases):
    """The launch bins chosen by gg_autotune on the clustered network (box
    edges 16 to ~250): the same areas bit for bit as the default bins after
    the same number of steps, and a step no slower than with the defaults."""
    xml = cases["c3"]

    def start():
        h = gg.GrainHandler(gg.Settings(xml, precision=gg.PRECISION_BATCHED), device=0)
        h.load_voxel_files()
        h.distanceInitialisation()
        h.find_neighbors()
        return h

    hd = start()  # default bins (before any tuning is cached for this network size)
    ht = start()
    try:
        info = ht.autotune(1)
        assert info["steps_run"] >= 2 and info["ms_tuned"] <= info["ms_default"]
        total = info["steps_run"] + 2
        ht.step(2)
        hd.step(total)
        a, b = hd.areas(), ht.areas()
        assert np.array_equal(np.isnan(a), np.isnan(b))
        m = np.isfinite(a)
        assert np.array_equal(a[m].view(np.uint64), b[m].view(np.uint64))
        ms_d, ms_t = hd.step(3) / 3, ht.step(3) / 3
        print({"tuned": info, "ms_default": ms_d, "ms_tuned": ms_t})
        assert ms_t <= 1.03 * ms_d
        assert hd.status() == 0 and ht.status() == 0
    finally:
        hd.close()
        ht.close()
