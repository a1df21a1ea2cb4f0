"""Per-grain area agreement of the batched FP32 form with the plain FP64 form.

The error of grain g at a step is |A_b(g) - A_p(g)| / A_p(g) over the grains
alive in both forms (areas from the contour, ``LSbox::computeVolume``,
src/grainBoundary.cpp:201-213).  ``trajectory`` runs both forms side by side
from the same input and records the error distribution every few steps.

Next to it, the plain form is run a third time with every boundary energy
scaled by (1 - 2^-46) (``gamma_hagb``), a perturbation of the order of FP64
rounding.  Where the network passes through a configuration that is
sensitive to its own rounding (a quadruple junction that opens and closes
from step to step), this perturbed FP64 run drifts away from the FP64 run as
well; its error is the floor that any arithmetic differing from the
reference's, FP64 included, reaches on those grains.
"""
from __future__ import annotations

import numpy as np

from . import gg

FLOOR_SCALE = 1.0 - 2.0 ** -46


def area_errors(a_ref: np.ndarray, a: np.ndarray, cell: float) -> dict:
    """Error statistics of areas `a` against `a_ref` (NaN = grain gone);
    `cell` is the area of one grid cell (for the absolute error in cells)."""
    both = np.isfinite(a_ref) & np.isfinite(a) & (a_ref > 0)
    rel = np.abs(a - a_ref)[both] / a_ref[both]
    out = {"compared": int(both.sum()),
           "alive_only_ref": int((np.isfinite(a_ref) & ~np.isfinite(a)).sum()),
           "alive_only_other": int((np.isfinite(a) & ~np.isfinite(a_ref)).sum())}
    if not both.any():
        return out
    ids = np.nonzero(both)[0]
    k = int(np.argmax(rel))
    out.update({"max": float(rel.max()), "p99": float(np.quantile(rel, 0.99)), "p50": float(np.median(rel)),
                "over_1e-3": int((rel > 1e-3).sum()),
                "max_abs_cells": float(np.max(np.abs(a - a_ref)[both]) / cell),
                "worst": {"id": int(ids[k]) + 1, "cells_ref": float(a_ref[ids[k]] / cell),
                          "cells": float(a[ids[k]] / cell)}})
    return out


def _areas(h: gg.GrainHandler) -> np.ndarray:
    return np.array([s.area if s.state == 1 else np.nan for s in h.grain_stats()])


def trajectory(xml: str, steps: int, every: int, device: int = 0, floor: bool = True, inputs=None,
               floor_scale: float = FLOOR_SCALE) -> list[dict]:
    """Runs the plain FP64 form, the batched FP32 form and (with `floor`) the
    perturbed plain form (boundary energies times `floor_scale`) for `steps`
    steps from the voxelized input of `xml` (or the host arrays `inputs` =
    (ids, euler, bbox)); every `every` steps records the batched form's
    errors against the plain form ("fp32") and the perturbed plain form's
    ("fp64_perturbed")."""
    runs = {"fp64": gg.Settings(xml, precision=gg.PRECISION_PLAIN),
            "fp32": gg.Settings(xml, precision=gg.PRECISION_BATCHED)}
    if floor:
        s = gg.Settings(xml, precision=gg.PRECISION_PLAIN)
        s.p.gamma_hagb = s.p.gamma_hagb * floor_scale
        runs["fp64_perturbed"] = s
    hs = {}
    try:
        for name, s in runs.items():
            h = gg.GrainHandler(s, device=device)
            hs[name] = h
            if inputs is None:
                h.load_voxel_files()
            else:
                h.load_voxels(*inputs)
            h.distanceInitialisation()
            h.find_neighbors()
        cell = hs["fp64"].dims().h ** 2
        rows = []
        done = 0
        while done < steps:
            n = min(every, steps - done)
            for h in hs.values():
                h.step(n)
            done += n
            ref = _areas(hs["fp64"])
            row = {"step": done, "alive": int(np.isfinite(ref).sum())}
            for name in hs:
                if name != "fp64":
                    row[name] = area_errors(ref, _areas(hs[name]), cell)
            row["status"] = {name: h.status() for name, h in hs.items()}
            rows.append(row)
        return rows
    finally:
        for h in hs.values():
            h.close()
