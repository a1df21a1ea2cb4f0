"""Seeded synthetic microstructures in GraGLeS2D's voxelized input format.

GraGLeS2D reads a voxelized microstructure (``MicrostructureGenMode 4``) as a
text header ``*.uds`` plus a raw ``int32`` grain-ID field ``*.bin``
(src/grainhdl.cpp:275-334 ``read_HeaderCPG`` and 336-511
``read_voxelized_microstructure``):

* ``.uds`` line 1 is skipped; lines 2-7 are ``<name> \\t <int>`` for the ID
  offset, DX, DY, NX (the grid edge, ``realDomainSize``), NY and the grain
  count; line 8 is skipped; then one line per grain
  ``id x y phi1 PHI phi2 xmin xmax ymin ymax count storedEnergy``, with the
  bounding box in interior pixel coordinates (inclusive);
* ``.bin`` holds NX*NY ``int32`` IDs, row-major with the row (y) outer.

The reference's own example inputs are not shipped, so every workload here is
generated: seeds uniform in [0,1)^2 from ``numpy.random.Generator(PCG64)``,
each pixel centre labelled with its nearest seed (Euclidean, bounded domain,
as the reference's domain is bounded), orientations uniform on SO(3)
(Shoemake's method) written as Bunge ZXZ Euler angles.  The clustered seed
mix (a Matern cluster process plus uniform seeds) gives the broad lognormal
size spread of the uneven-box workload.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np


@dataclass
class Microstructure:
    """A labelled grid: ``labels[y, x]`` in 1..n_grains, Euler angles per grain."""

    labels: np.ndarray  # (nn, nn) int32, 1-based grain IDs
    seeds: np.ndarray  # (n_grains, 2) float64 in [0,1)^2 (x, y)
    euler: np.ndarray  # (n_grains, 3) float64 Bunge phi1, PHI, phi2
    stored: np.ndarray | None = None  # (n_grains,) float64 stored elastic energies (.uds column 12), else 0

    @property
    def nn(self) -> int:
        return int(self.labels.shape[0])

    @property
    def n_grains(self) -> int:
        return int(self.seeds.shape[0])


def shoemake_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random unit quaternions (q0, q1, q2, q3) by Shoemake's method."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    q = np.stack(
        [a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)],
        axis=1,
    )
    # scalar part first and non-negative (q and -q are the same rotation)
    q = q[:, [1, 0, 2, 3]]
    q[q[:, 0] < 0] *= -1.0
    return q


def quaternion_to_bunge(q: np.ndarray) -> np.ndarray:
    """Inverse of the reference's Bunge ZXZ conversion (src/Quaternion.cpp:168-192).

    euler2quaternion sets q0 = cos(P/2)cos((p1+p2)/2), q1 = sin(P/2)cos((p1-p2)/2),
    q2 = sin(P/2)sin((p1-p2)/2), q3 = cos(P/2)sin((p1+p2)/2).
    """
    q0, q1, q2, q3 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    big_phi = 2.0 * np.arctan2(np.sqrt(q1 * q1 + q2 * q2), np.sqrt(q0 * q0 + q3 * q3))
    s = np.arctan2(q3, q0)  # (p1 + p2) / 2
    d = np.arctan2(q2, q1)  # (p1 - p2) / 2
    phi1 = np.mod(s + d, 2 * np.pi)
    phi2 = np.mod(s - d, 2 * np.pi)
    return np.stack([phi1, big_phi, phi2], axis=1)


def _label_nearest(seeds: np.ndarray, nn: int, chunk_rows: int = 256) -> np.ndarray:
    from scipy.spatial import cKDTree

    tree = cKDTree(seeds)
    labels = np.empty((nn, nn), dtype=np.int32)
    xs = (np.arange(nn, dtype=np.float64) + 0.5) / nn
    for y0 in range(0, nn, chunk_rows):
        y1 = min(nn, y0 + chunk_rows)
        ys = (np.arange(y0, y1, dtype=np.float64) + 0.5) / nn
        pts = np.stack(np.meshgrid(xs, ys), axis=-1).reshape(-1, 2)
        _, idx = tree.query(pts, k=1, workers=-1)
        labels[y0:y1] = (idx.astype(np.int32) + 1).reshape(y1 - y0, nn)
    return labels


def voronoi(n_grains: int, nn: int, seed: int) -> Microstructure:
    """Voronoi tessellation of ``n_grains`` uniform seeds on an ``nn`` x ``nn`` grid."""
    rng = np.random.Generator(np.random.PCG64(seed))
    seeds = rng.random((n_grains, 2))
    euler = quaternion_to_bunge(shoemake_quaternions(rng, n_grains))
    return Microstructure(_label_nearest(seeds, nn), seeds, euler)


def clustered(n_grains: int, nn: int, seed: int, cluster_fraction: float = 0.5, cluster_radius: float = 0.01,
              mean_daughters: float = 8.0) -> Microstructure:
    """Matern cluster process (parents uniform, Poisson daughters uniform in a
    disc of ``cluster_radius``) mixed with uniform seeds; ``cluster_fraction``
    of the seeds are daughters."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_clustered = int(round(n_grains * cluster_fraction))
    pts = []
    while sum(len(p) for p in pts) < n_clustered:
        parent = rng.random(2)
        k = max(1, rng.poisson(mean_daughters))
        r = cluster_radius * np.sqrt(rng.random(k))
        t = 2 * np.pi * rng.random(k)
        d = parent + np.stack([r * np.cos(t), r * np.sin(t)], axis=1)
        d = d[(d >= 0).all(axis=1) & (d < 1).all(axis=1)]
        pts.append(d)
    clustered_pts = np.concatenate(pts)[:n_clustered]
    seeds = np.concatenate([clustered_pts, rng.random((n_grains - n_clustered, 2))])
    euler = quaternion_to_bunge(shoemake_quaternions(rng, n_grains))
    return Microstructure(_label_nearest(seeds, nn), seeds, euler)


def grain_table(ms: Microstructure) -> np.ndarray:
    """Per grain: (xmin, xmax, ymin, ymax, count) in interior pixel coordinates."""
    n = ms.n_grains
    lab = ms.labels.astype(np.int64) - 1
    yy, xx = np.indices(lab.shape)
    flat = lab.ravel()
    count = np.bincount(flat, minlength=n)
    big = np.iinfo(np.int64).max
    xmin = np.full(n, big, np.int64)
    ymin = np.full(n, big, np.int64)
    xmax = np.full(n, -1, np.int64)
    ymax = np.full(n, -1, np.int64)
    np.minimum.at(xmin, flat, xx.ravel())
    np.maximum.at(xmax, flat, xx.ravel())
    np.minimum.at(ymin, flat, yy.ravel())
    np.maximum.at(ymax, flat, yy.ravel())
    xmin[count == 0] = 0
    ymin[count == 0] = 0
    xmax[count == 0] = 0
    ymax[count == 0] = 0
    return np.stack([xmin, xmax, ymin, ymax, count], axis=1)


def write_mode4(prefix: str, ms: Microstructure) -> tuple[str, str]:
    """Write ``prefix.uds`` and ``prefix.bin``; returns their paths."""
    uds, binp = prefix + ".uds", prefix + ".bin"
    tab = grain_table(ms)
    nn = ms.nn
    with open(uds, "w") as f:
        f.write("GraGLeS2D voxelized microstructure (synthetic)\n")
        f.write("IDOffset \t 1\n")
        f.write("DX \t 1\n")
        f.write("DY \t 1\n")
        f.write(f"NX \t {nn}\n")
        f.write(f"NY \t {nn}\n")
        f.write(f"Grains \t {ms.n_grains}\n")
        f.write("ID x y phi1 PHI phi2 xmin xmax ymin ymax count storedEnergy\n")
        for g in range(ms.n_grains):
            xmin, xmax, ymin, ymax, cnt = (int(v) for v in tab[g])
            e = ms.euler[g]
            se = f"{ms.stored[g]:.17g}" if ms.stored is not None else "0.0"
            f.write(
                f"{g + 1}\t {ms.seeds[g, 0]:.10f}\t {ms.seeds[g, 1]:.10f}\t {e[0]:.17g}\t {e[1]:.17g}\t {e[2]:.17g}\t "
                f"{xmin}\t {xmax}\t {ymin}\t {ymax}\t {cnt}\t {se} \n"
            )
    ms.labels.astype("<i4").tofile(binp)
    return uds, binp


DEFAULT_PARAMETERS = {
    "StartTime": 0,
    "NumberOfPointsPerGrain": 25,
    "AnalysisTimestep": 100000,
    "PlotInterval": 1,
    "NumberOfTimesteps": 10,
    "BreakupNumber": 0,
    "DiscreteSamplingRate": 31,
    "DomainBorderSize": 7,
    "MicrostructureGenMode": 4,
    "LatticeType": 0,
    "HAGB_Energy": 1.0,
    "HAGB_Mobility": 1.0,
    "DislocEnPerM": 1.0,
    "Physical_Domain_Size": 1.0,
    "TriplePointDrag": 0.0,
    "UseMobilityModel": 0,
    "IdentifyTwins": 0,
    "UseStoredElasticEnergy": 0,
    "UseMagneticField": 0,
    "IsIsotropicNetwork": 1,
    "UseTexture": 0,
    "MaxMisOrientation": 0,
    "ExecuteInParallel": 1,
    "MaximumNumberOfThreads": 8,
    "GridCoarsement": 0,
    "GridCoarsementGradient": 0.95,
    "ConvolutionMode": 2,
    "ResearchMode": 0,
    "ResearchProject": 0,
    "ConstantSectorRadius": 3,
    "InterpolatingSectorRadius": 2,
    "NeighbourTracking": 0,
    "GrainScheduler": 0,
    "DecoupleGrains": 0,
}


def write_parameters(path: str, read_from: str, additional: str, **overrides) -> str:
    """Write a ``parameters.xml`` using the tags of src/Settings.cpp:111-283."""
    p = dict(DEFAULT_PARAMETERS)
    p.update(overrides)
    p["ReadFromFilename"] = read_from
    p["AdditionalFilename"] = additional
    with open(path, "w") as f:
        f.write('<?xml version="1.0" encoding="utf-8"?>\n<Parameters>\n')
        for k, v in p.items():
            # file names must not be padded: the reference uses the raw node text
            f.write(f"   <{k}>{v}</{k}>\n" if isinstance(v, str) else f"   <{k}> {v} </{k}>\n")
        f.write("</Parameters>\n")
    return path


def make_case(directory: str, name: str, ms: Microstructure, **params) -> str:
    """Write the mode-4 pair and a parameters file into ``directory``; returns the XML path."""
    os.makedirs(directory, exist_ok=True)
    prefix = os.path.join(directory, name)
    write_mode4(prefix, ms)
    # The reference sizes its grain schedulers from the XML's particle count
    # before it reads the .uds header (src/grainhdl.cpp:57, 1508-1517), so the
    # XML carries the count and the matching points-per-grain as well.
    params.setdefault("NumberOfParticles", ms.n_grains)
    params.setdefault("NumberOfPointsPerGrain", max(1, int(ms.nn / math.sqrt(ms.n_grains))))
    # file names relative to the XML's directory (run the reference from there)
    return write_parameters(prefix + ".xml", name + ".bin", name + ".uds", **params)


def equivalent_diameters(ms: Microstructure) -> np.ndarray:
    cnt = np.bincount(ms.labels.ravel().astype(np.int64) - 1, minlength=ms.n_grains)
    return 2.0 * np.sqrt(cnt / math.pi)
