"""Shared comparison of a product state dump against a reference dump."""
from __future__ import annotations

import numpy as np

from gragles2d_b200 import dumpfile


def compare_records(ref: dumpfile.Record, got: dumpfile.Record, *, exact: bool, delta: float,
                    check_idlocal: bool = True, check_newbb: bool = True) -> list[str]:
    """Returns a list of mismatch descriptions (empty when the states agree).

    exact: FP64 bit-for-bit agreement of fields, contours, areas, energies
    (plain form, isotropic); otherwise fields within 1e-12 delta, contour
    points within 1e-9 grid cells, areas within 1e-9 relative and every
    discrete output (state, box, lists, neighbour IDs, junction grains)
    identical.  check_newbb=False skips the set-comparison bounding box,
    which the reference's contour constructor leaves unset until the first
    comparison (src/box.cpp:108-159: m_newXMin .. m_newYMax hold whatever
    the heap held).
    """
    out = []
    for gid, r in ref.grains.items():
        g = got.grains.get(gid)
        if g is None:
            out.append(f"grain {gid}: missing")
            continue
        if (r.state == 0) != (g.state == 0) or r.state != g.state:
            out.append(f"grain {gid}: state ref {r.state} got {g.state}")
            continue
        if r.state != 1:
            continue
        tag = f"grain {gid}"
        if r.box != g.box:
            out.append(f"{tag}: box ref {r.box} got {g.box}")
            continue
        if r.regular != g.regular:
            out.append(f"{tag}: regular ref {r.regular} got {g.regular}")
        if r.boundary != g.boundary:
            out.append(f"{tag}: boundary flag ref {r.boundary} got {g.boundary}")
        if exact:
            if not np.array_equal(r.phi.view(np.uint64), g.phi.view(np.uint64)):
                d = np.abs(r.phi - g.phi)
                k = np.unravel_index(np.argmax(d), d.shape)
                out.append(f"{tag}: phi differs at {int((d > 0).sum())} px, max {d.max():.3e} at {k}")
        else:
            d = np.abs(r.phi - g.phi).max() if r.phi.size else 0
            if d > 1e-12 * delta * 1e3:
                out.append(f"{tag}: phi max diff {d:.3e}")
        if check_idlocal:
            if r.id_box != g.id_box:
                out.append(f"{tag}: IDLocal box ref {r.id_box} got {g.id_box}")
            elif not np.array_equal(r.idlocal, g.idlocal):
                out.append(f"{tag}: IDLocal differs at {int((r.idlocal != g.idlocal).sum())} px")
        if list(r.cmp) != list(g.cmp):
            out.append(f"{tag}: comparison list ref {list(r.cmp)} got {list(g.cmp)}")
        if list(r.sec) != list(g.sec):
            out.append(f"{tag}: second-order list ref {list(r.sec)} got {list(g.sec)}")
        if r.contour.shape != g.contour.shape:
            out.append(f"{tag}: contour length ref {r.contour.shape[0]} got {g.contour.shape[0]}")
        else:
            if exact:
                if not np.array_equal(r.contour, g.contour):
                    out.append(f"{tag}: contour differs, max {np.abs(r.contour - g.contour).max():.3e}")
            elif r.contour.size and np.abs(r.contour[:, :2] - g.contour[:, :2]).max() > 1e-9:
                out.append(f"{tag}: contour xy max diff {np.abs(r.contour[:, :2] - g.contour[:, :2]).max():.3e}")
        rj = [(j[0], j[1], j[2]) for j in r.junctions]
        gj = [(j[0], j[1], j[2]) for j in g.junctions]
        if rj != gj:
            out.append(f"{tag}: junctions ref {rj} got {gj}")
        rn = [n[0] for n in r.neighbours]
        gn = [n[0] for n in g.neighbours]
        if rn != gn:
            out.append(f"{tag}: neighbour IDs ref {rn} got {gn}")
        elif r.neighbours:
            rl = np.array([n[1] for n in r.neighbours])
            gl = np.array([n[1] for n in g.neighbours])
            re_ = np.array([n[2] for n in r.neighbours])
            ge_ = np.array([n[2] for n in g.neighbours])
            tol = 0 if exact else 1e-9
            if np.abs(rl - gl).max() > tol * max(1, np.abs(rl).max()):
                out.append(f"{tag}: neighbour lengths differ {np.abs(rl - gl).max():.3e}")
            if np.abs(re_ - ge_).max() > (1e-12 if exact else 1e-9):
                out.append(f"{tag}: neighbour energies differ {np.abs(re_ - ge_).max():.3e}")
        for name in ("volume", "energy", "perimeter"):
            a, b = getattr(r, name), getattr(g, name)
            if exact:
                if a != b:
                    out.append(f"{tag}: {name} ref {a!r} got {b!r}")
            elif abs(a - b) > 1e-9 * max(abs(a), 1e-30):
                out.append(f"{tag}: {name} ref {a!r} got {b!r}")
        if check_newbb and r.newbb != g.newbb:
            out.append(f"{tag}: new bbox ref {r.newbb} got {g.newbb}")
    return out


def ownership_mismatch(ref: dumpfile.Record, got: dumpfile.Record, m: int) -> int:
    return int((dumpfile.ownership(ref, m) != dumpfile.ownership(got, m)).sum())
