"""The initial neighbour search (gg_find_neighbors) against all pairs.

The search bins the grains by the cells their boxes cover and tests only
grains sharing a cell; every grain's comparison list must still be every
other grain whose closed box overlaps its own (RTree::Overlap,
src/RTree.h:1092-1105), in ascending ID order (grainhdl::find_neighbors,
src/grainhdl.cpp:1258-1283), as an all-pairs test of the dumped boxes gives
it.  Two networks: uniform Voronoi seeds, and a cluster mix whose large boxes
span several bins.
"""
import os

import numpy as np
import pytest

from gragles2d_b200 import dumpfile, gg
from gragles2d_b200 import microstructure as ms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["voronoi", "clustered"])
def test_binned_search_equals_all_pairs(tmp_path, kind):
    if kind == "voronoi":
        micro = ms.voronoi(5000, 1800, 4)
    else:
        micro = ms.clustered(5000, 2400, 7, cluster_fraction=0.9, cluster_radius=0.02, mean_daughters=40.0)
    xml = ms.make_case(str(tmp_path / kind), kind, micro, NumberOfTimesteps=1, IsIsotropicNetwork=0)
    h = gg.GrainHandler(gg.Settings(xml, precision=gg.PRECISION_BATCHED), device=0)
    path = str(tmp_path / "init.dump")
    try:
        h.load_voxel_files()
        h.distanceInitialisation()
        h.find_neighbors()
        h.find_neighbors()  # a second search on the same bins gives the same lists
        h.dump(path, 0)
    finally:
        h.close()
    rec = dumpfile.read(path).records[0]
    ids = np.array(sorted(g for g, r in rec.grains.items() if r.state != 0))
    x0, x1, y0, y1 = np.array([rec.grains[int(g)].box for g in ids]).T
    overlap = ~((x0[:, None] > x1[None, :]) | (x0[None, :] > x1[:, None]) | (y0[:, None] > y1[None, :]) |
                (y0[None, :] > y1[:, None]))
    np.fill_diagonal(overlap, False)
    assert overlap.sum(axis=1).max() <= 96
    if kind == "clustered":
        assert (x1 - x0).max() > 2 * 64  # boxes spanning several bins
    for row, g in enumerate(ids):
        assert rec.grains[int(g)].sec == ids[overlap[row]].tolist(), int(g)
