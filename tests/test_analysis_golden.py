"""Pins the analysis-output restatement (oracle/analysis.py) against the
reference's own files: the ana_* fixtures hold the state after the last step
and the Texture / MODF / NrGrains&EnergyStatistics files GraGLeS2D wrote on
its AnalysisTimestep schedule during the same run (tests/golden/make_golden.py).
"""
import json
import os
import sys

import pytest

from gragles2d_b200 import dumpfile

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
from oracle import analysis  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = ["ana_iso_v80", "ana_mob_v80", "se_v30", "mag_v30"]


def _case(name):
    d = os.path.join(GOLDEN, name)
    with open(os.path.join(d, "case.json")) as f:
        info = json.load(f)
    dump = dumpfile.read(os.path.join(d, "reference.dump.gz"))
    euler = analysis.read_uds_euler(os.path.join(d, name + ".uds"))
    return d, info, dump, euler


def _read(path):
    with open(path) as f:
        return f.read()


@pytest.mark.parametrize("name", CASES)
def test_last_texture_and_modf_restated_from_the_final_state(name):
    d, info, dump, euler = _case(name)
    steps = info["steps"]  # NumberOfTimesteps; loops 0..steps
    final = dump.records[-1]
    assert final.steps == steps + 1
    iso = info["overrides"]["IsIsotropicNetwork"] == 1
    stored = None
    if info["overrides"].get("UseStoredElasticEnergy"):
        # m_StoredElasticEnergy = value * DislocEnPerM / HAGB_Energy * Physical_Domain_Size (all 1 here)
        stored = {g: v * (info["overrides"]["DislocEnPerM"] / 1.0 * 1.0)
                  for g, v in analysis.read_uds_stored(os.path.join(d, name + ".uds")).items()}
    if info["overrides"].get("UseMagneticField"):
        # the magnetic energy takes the stored energy's column
        import re
        M = {k: float(v) for k, v in re.findall(r"<(\w+)>\s*([^<]+?)\s*</\1>", _read(os.path.join(d, "magnetic.xml")))}
        vec = (M["MagneticVector_x"], M["MagneticVector_y"], M["MagneticVector_z"])
        stored = {g: analysis.magnetic_energy(e, M["VacuumPermeability"], vec, M["deltaMagSys"], M["MagneticForceField"])
                  for g, e in euler.items()}
    text, modf, _ = analysis.texture(final, euler, info["overrides"]["AnalysisTimestep"], 31, stored)
    assert text == _read(os.path.join(d, "analysis", f"Texture_{steps}.ori"))
    assert analysis.modf_text(modf, iso) == _read(os.path.join(d, "analysis", f"MODF_{steps}.txt"))
    if not iso:
        assert abs(sum(modf) - 1.0) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_statistics_lines(name):
    """Time before the step's increment, grains present when the step began
    (the reference's per-step grain counts), half the summed grain energies."""
    d, info, dump, euler = _case(name)
    at = info["overrides"]["AnalysisTimestep"]
    steps = info["steps"]
    lines = _read(os.path.join(d, "analysis", "NrGrains&EnergyStatistics.txt")).splitlines(keepends=True)
    loops = [lp for lp in range(steps + 1) if lp % at == 0 or lp == steps]
    assert len(lines) == len(loops)
    final = dump.records[-1]
    _, _, total = analysis.texture(final, euler, at, 31)
    for lp, line in zip(loops, lines):
        t = analysis.realtime(lp, 0, dump.dt, 1.0, 0.8359, 1.0, 1.0)
        cols = line.rstrip("\n").split("\t")
        assert cols[0] == analysis.g6(t)
        assert int(cols[1]) == info["step_grains"][lp]
        assert int(cols[3]) == dump.nn
    assert lines[-1] == analysis.stats_line(analysis.realtime(steps, 0, dump.dt, 1.0, 0.8359, 1.0, 1.0),
                                            info["step_grains"][steps], total, dump.nn)


def test_vanishing_grains_leave_the_texture():
    d, info, dump, euler = _case("ana_iso_v80")
    counts = info["step_grains"]
    assert counts[0] > counts[-1]  # grains vanish during the run
    steps = info["steps"]
    ids = [int(l.split("\t")[0]) for l in _read(os.path.join(d, "analysis", f"Texture_{steps}.ori")).splitlines()]
    alive = [g for g, r in dump.records[-1].grains.items() if r.state == 1]
    assert set(ids) <= set(alive) and len(ids) >= len(alive) - 2


def test_quaternion_round_trip_and_gimbal_branch():
    for e in [(0.3, 1.2, 5.9), (4.0, 0.0, 0.0), (1.0, 3.0, 2.0)]:
        r = analysis.quaternion2euler(analysis.euler2quaternion(e))
        if e[1] == 0.0:
            assert r[2] == 0.0 and abs(r[0] - (e[0] + e[2]) % (2 * analysis.PI)) < 1e-12
        else:
            assert all(abs(a - b) < 1e-9 for a, b in zip(r, e))
