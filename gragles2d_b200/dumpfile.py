"""Reader for the network-state dump written by ``gg_dump`` (include/gg_step.h)
and by the oracle harness around the reference (oracle/ref_harness.cpp).

Both write the same format, so a product state and a reference state of the
same input and step compare field by field.  Per grain: state (0 removed,
1 exists, 2 vanished), motion-regular and boundary flags, area / energy /
perimeter / mean dA, the current distance field with its box, the IDLocal map
with its box, the comparison and second-order lists, the contour (x, y,
energy, mobility), the junctions, the direct-neighbour characteristics and
the set-comparison bounding box.
"""
from __future__ import annotations

import gzip
import struct
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Grain:
    id: int
    state: int
    regular: int = 0
    boundary: int = 0
    volume: float = 0.0
    energy: float = 0.0
    perimeter: float = 0.0
    mean_da: float = 0.0
    box: tuple = (0, 0, 0, 0)  # xmin, xmax, ymin, ymax
    phi: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))
    id_box: tuple = (0, 0, 0, 0)
    idlocal: np.ndarray = field(default_factory=lambda: np.zeros((0, 0), np.uint32))
    cmp: list = field(default_factory=list)
    sec: list = field(default_factory=list)
    contour: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))
    junctions: list = field(default_factory=list)  # (type, grains[4], segment, lambda, x, y)
    neighbours: list = field(default_factory=list)  # (id, length, energy, misori, mobility)
    newbb: tuple = (0, 0, 0, 0)


@dataclass
class Record:
    steps: int
    live: int
    grains: dict  # id -> Grain


@dataclass
class Dump:
    n_grains: int
    ngridpoints: int
    nn: int
    h: float
    delta: float
    dt: float
    records: list


class _Reader:
    def __init__(self, data: bytes):
        self.b = memoryview(data)
        self.o = 0

    def i32(self) -> int:
        v = struct.unpack_from("<i", self.b, self.o)[0]
        self.o += 4
        return v

    def f64(self) -> float:
        v = struct.unpack_from("<d", self.b, self.o)[0]
        self.o += 8
        return v

    def arr(self, dtype, count):
        a = np.frombuffer(self.b, dtype=dtype, count=count, offset=self.o).copy()
        self.o += a.nbytes
        return a

    def done(self) -> bool:
        return self.o >= len(self.b)


def read(path: str) -> Dump:
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rb") as f:
        data = f.read()
    return parse(data)


def parse(data: bytes) -> Dump:
    r = _Reader(data)
    if bytes(r.b[0:4]) != b"GGD1":
        raise ValueError("not a GGD1 dump")
    r.o = 4
    if r.i32() != 1:
        raise ValueError("unsupported dump version")
    n = r.i32()
    m = r.i32()
    nn = r.i32()
    h, delta, dt = r.f64(), r.f64(), r.f64()
    recs = []
    while not r.done():
        if r.i32() != 0x52454344:
            raise ValueError("bad record tag")
        steps = r.i32()
        live = r.i32()
        grains = {}
        for _ in range(n):
            gid = r.i32()
            st = r.i32()
            if st == 0:
                grains[gid] = Grain(gid, 0)
                continue
            g = Grain(gid, st)
            g.regular = r.i32()
            g.boundary = r.i32()
            g.volume, g.energy, g.perimeter, g.mean_da = r.f64(), r.f64(), r.f64(), r.f64()
            bx = (r.i32(), r.i32(), r.i32(), r.i32())
            g.box = bx
            g.phi = r.arr("<f8", (bx[1] - bx[0]) * (bx[3] - bx[2])).reshape(bx[3] - bx[2], bx[1] - bx[0])
            ib = (r.i32(), r.i32(), r.i32(), r.i32())
            g.id_box = ib
            g.idlocal = r.arr("<u4", (ib[1] - ib[0]) * (ib[3] - ib[2])).reshape(ib[3] - ib[2], ib[1] - ib[0])
            g.cmp = list(r.arr("<i4", r.i32()))
            g.sec = list(r.arr("<i4", r.i32()))
            nc = r.i32()
            g.contour = r.arr("<f8", 4 * nc).reshape(nc, 4)
            nj = r.i32()
            js = []
            for _ in range(nj):
                t = r.i32()
                gr = tuple(int(x) for x in r.arr("<u4", 4))
                seg = r.i32()
                js.append((t, gr, seg, r.f64(), r.f64(), r.f64()))
            g.junctions = js
            nb = r.i32()
            g.neighbours = [(r.i32(), r.f64(), r.f64(), r.f64(), r.f64()) for _ in range(nb)]
            g.newbb = (r.i32(), r.i32(), r.i32(), r.i32())
            grains[gid] = g
        recs.append(Record(steps, live, grains))
    return Dump(n, m, nn, h, delta, dt, recs)


def ownership(rec: Record, ngridpoints: int) -> np.ndarray:
    """Per-pixel owning grain over the global grid: the grain whose current
    distance field is largest where that maximum is >= 0 (0 elsewhere)."""
    best = np.full((ngridpoints, ngridpoints), -np.inf)
    owner = np.zeros((ngridpoints, ngridpoints), np.int32)
    for gid in sorted(rec.grains):
        g = rec.grains[gid]
        if g.state != 1:
            continue
        x0, x1, y0, y1 = g.box
        sub = best[y0:y1, x0:x1]
        win = g.phi > sub
        sub[win] = g.phi[win]
        owner[y0:y1, x0:x1][win] = gid
    owner[best < 0] = 0
    return owner
