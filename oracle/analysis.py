"""Analysis output of one timestep, restated from a state record (test
infrastructure only: the tests check the library's writer, and the committed
reference output, against it; nothing in the product imports it).

Follows grainhdl::save_Texture (src/grainhdl.cpp:871-1023) with
NeighbourTracking and ResearchMode off, grainhdl::save_NrGrainsStats
(src/grainhdl.cpp:1225-1241), ExplicitGrainBoundary::
calculateDiscreteEnergyDistribution (src/grainBoundary.cpp:578-598) and the
quaternion conversions Quaternion::euler2quaternion / quaternion2EulerConst
(src/Quaternion.cpp:168-192, 242-289).  Numbers are formatted as the
reference's streams format them: C++ ostream defaults (six significant digits,
%g style) and printf("%lf") of float-rounded MODF values.
"""
from __future__ import annotations

import math

import numpy as np

PI = 3.14159265358979323846  # src/mymath.h:30
QUAT2EUL_ETA = 1e-20         # src/mymath.h:31


def euler2quaternion(e):
    """Bunge ZXZ angles to (q0, q1, q2, q3) (src/Quaternion.cpp:168-192)."""
    p1, t, p2 = e
    co1 = math.cos(t / 2)
    s1 = math.sin(t / 2)
    return (co1 * math.cos((p1 + p2) / 2), s1 * math.cos((p1 - p2) / 2), s1 * math.sin((p1 - p2) / 2),
            co1 * math.sin((p1 + p2) / 2))


def quaternion2euler(q):
    """(phi1, PHI, phi2) in [0, 2 pi) (src/Quaternion.cpp:242-289)."""
    q0, q1, q2, q3 = q
    cos_phi = q3 * q3 - q2 * q2 - q1 * q1 + q0 * q0
    y0 = 2 * q1 * q3 - 2 * q0 * q2
    x0 = 2 * q2 * q3 + 2 * q0 * q1
    y1 = 2 * q1 * q3 + 2 * q0 * q2
    x1 = -2 * q2 * q3 + 2 * q0 * q1
    if cos_phi > 1.0:
        cos_phi = 1.0
    phi = 0.0 if (1.0 - cos_phi) * (1.0 - cos_phi) <= QUAT2EUL_ETA else math.acos(cos_phi)
    sp = math.sin(phi)
    if sp != 0:
        phi2 = math.atan2(y0 / sp, x0 / sp)
        phi1 = math.atan2(y1 / sp, x1 / sp)
    else:
        phi1 = math.atan2(2 * q1 * q2 + 2 * q0 * q3, q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3)
        phi2 = 0.0
    if phi1 < 0.0:
        phi1 += 2 * PI
    if phi2 < 0.0:
        phi2 += 2 * PI
    return phi1, phi, phi2


def magnetic_energy(euler, vacuum_permeability, vector, delta_mag_sys, force_field, hagb_energy=1.0,
                    physical_domain_size=1.0):
    """LSbox::calculateMagneticEnergy (src/box.cpp:2238-2292) of a grain with
    the given input Bunge angles: the c axis (the sample normal rotated by the
    quaternion round trip of the angles) against the field direction."""
    p1, t, _ = quaternion2euler(euler2quaternion(euler))
    axis = (0.0 + math.sin(p1) * math.sin(t), 0.0 + -math.cos(p1) * math.sin(t), 0.0 + math.cos(t))
    cosine = (vector[0] * axis[0]) + (vector[1] * axis[1]) + (vector[2] * axis[2])
    if cosine > 1:
        cosine = 1.0
    e = 0.5 * vacuum_permeability * delta_mag_sys * force_field * force_field * cosine * cosine
    return e / hagb_energy * physical_domain_size


def g6(x) -> str:
    """A double through an ostream with default flags."""
    return "%.6g" % x


def read_uds_stored(path: str) -> dict:
    """Grain ID -> stored energy (column 12) from a mode-4 .uds header."""
    out = {}
    with open(path) as f:
        lines = f.read().splitlines()
    start = next(i for i, l in enumerate(lines) if l.split()[:2] == ["ID", "x"]) + 1
    for line in lines[start:]:
        parts = line.split()
        if len(parts) >= 12:
            out[int(parts[0])] = float(parts[11])
    return out


def read_uds_euler(path: str) -> dict:
    """Grain ID -> Bunge angles from a mode-4 .uds header."""
    out = {}
    with open(path) as f:
        lines = f.read().splitlines()
    start = next(i for i, l in enumerate(lines) if l.split()[:2] == ["ID", "x"]) + 1
    for line in lines[start:]:
        parts = line.split()
        if len(parts) >= 6:
            out[int(parts[0])] = (float(parts[3]), float(parts[4]), float(parts[5]))
    return out


def texture(record, euler: dict, analysis_timestep: int, nbins: int, stored: dict | None = None):
    """(Texture_<loop>.ori text, MODF values, total energy) of a record taken
    right after the analysed step; `stored` maps grain IDs to their scaled
    stored energies (LSbox's m_StoredElasticEnergy), else 0 is written."""
    lines = []
    modf = [0.0] * nbins
    dh = 62.8 / nbins if nbins else math.inf
    total = 0.0
    for gid in sorted(record.grains):
        g = record.grains[gid]
        if g.state != 1 or not g.regular:
            continue
        total += g.energy
        e = quaternion2euler(euler2quaternion(euler[gid]))
        local = {}
        for nb in g.neighbours:  # (id, length, energy, misori, mobility)
            key = int((nb[3] * 180 / PI) / dh - 0.5)
            local[key] = local[key] + nb[1] if key in local else nb[1]
        for key in sorted(local):
            if 0 <= key < nbins:
                modf[key] += local[key] / 2
        fields = [str(gid), str(len(g.neighbours)), str(int(bool(g.boundary))), g6(g.volume),
                  g6(g.mean_da / float(analysis_timestep)), g6(g.perimeter), g6(g.energy),
                  g6(stored[gid]) if stored else "0",
                  g6(e[0]), g6(e[1]), g6(e[2])]
        lines.append("\t".join(fields) + "\n")
        s = 0.0
        for v in modf:
            s += v
        modf = [v / s if v > 0 else v for v in modf]
    return "".join(lines), modf, total


def modf_text(modf, isotropic: bool) -> str:
    if isotropic:
        return ""
    nbins = len(modf)
    dh = 62.8 / nbins
    return "".join("%f\t%f\n" % (float(np.float32(dh * (i + 1))), float(np.float32(v)))
                   for i, v in enumerate(modf))


def realtime(loop: int, start_time: int, dt: float, physical_domain_size: float, time_slope: float,
             hagb_energy: float, hagb_mobility: float) -> float:
    """Simulated time when step `loop` is analysed (src/grainhdl.cpp:1115-1117)."""
    inc = dt * (physical_domain_size * physical_domain_size) / (time_slope * hagb_energy * hagb_mobility)
    t = 0.0
    for _ in range(start_time, loop):
        t += inc
    return t


def stats_line(time: float, nr_grains: int, total_energy: float, nn: int) -> str:
    return "%s\t%d\t%s\t%d\n" % (g6(time), nr_grains, g6(0.5 * total_energy), nn)


def read_network(path: str, number_of_particles: int):
    """(polygons, quaternions) of a contour file as grainhdl::readMicrostructure
    reads it (src/grainhdl.cpp:605-654): records in file order become grains
    1, 2, ...; a record ID at least the grain count raises the count; points
    clamped to [0, 1].  Grains without a record get an empty polygon."""
    with open(path) as f:
        tok = f.read().split()
    pos, ngrains, polys, quats = 0, number_of_particles, [], []
    k = 1
    while k <= ngrains:
        if pos >= len(tok):
            polys.append(np.zeros((0, 2)))
            quats.append((1.0, 0.0, 0.0, 0.0))
            k += 1
            continue
        gid = int(tok[pos])
        if gid >= ngrains:
            ngrains = gid
        nv = int(tok[pos + 1])
        quats.append(tuple(float(t) for t in tok[pos + 2:pos + 6]))
        pts = np.array([float(t) for t in tok[pos + 6:pos + 6 + 2 * nv]]).reshape(nv, 2)
        polys.append(np.clip(pts, 0.0, 1.0))
        pos += 6 + 2 * nv
        k += 1
    return polys, quats
