"""Generates the golden fixtures of the parity tests by running the reference.

For each case: a seeded synthetic voxelized microstructure (``*.uds`` +
``*.bin``), its ``parameters.xml``, and the state dumps of GraGLeS2D's own
C++ (``oracle/_ref/gg_ref``, built by ``make -C oracle ref`` from the
reference sources) after initialisation and after selected steps, gzipped.

The ``rst_*`` cases are contour input (MicrostructureGenMode 0): the restart
files the reference writes during a voxelized run, then the reference's run
from them.

Run from the repository root in the build container (it needs the reference
tree to build the oracle):  python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import gzip
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from gragles2d_b200 import microstructure as ms  # noqa: E402

GG_REF = os.path.join(ROOT, "oracle", "_ref", "gg_ref")

# name: (generator, grains, grid, seed, steps, dump_every, parameter overrides)
CASES = {
    "iso_v20": ("voronoi", 20, 100, 0, 24, 8, {"IsIsotropicNetwork": 1}),
    "iso_v60": ("voronoi", 60, 140, 1, 40, 10, {"IsIsotropicNetwork": 1}),
    "rs_v30": ("voronoi", 30, 120, 2, 20, 5, {"IsIsotropicNetwork": 0}),
    "mob_v30": ("voronoi", 30, 120, 3, 20, 5,
                {"IsIsotropicNetwork": 0, "UseMobilityModel": 1, "TriplePointDrag": 5.0}),
    # every step dumped: the per-routine restatement in oracle/gg_oracle.c is
    # checked on each consecutive pair of records
    "seq_v24": ("voronoi", 24, 100, 5, 6, 1, {"IsIsotropicNetwork": 1}),
    # analysis output (Texture_<loop>.ori, MODF_<loop>.txt,
    # NrGrains&EnergyStatistics.txt) every 5 steps, written by the reference
    # into <case>/analysis
    "ana_iso_v80": ("voronoi", 80, 100, 11, 40, 0, {"IsIsotropicNetwork": 1, "AnalysisTimestep": 5}),
    # stored elastic energies uniform in [0, 3000) (seeded separately), a
    # boundary default of 500: the stored-energy term of the corrector and the
    # time-step correction it implies; analysis files every 5 steps
    "se_v30": ("voronoi", 30, 120, 6, 20, 5,
               {"IsIsotropicNetwork": 0, "UseStoredElasticEnergy": 1, "DislocEnPerM": 1.0,
                "BoxDefaultStoredElasticEnergy": 500.0, "AnalysisTimestep": 5}),
    # grid coarsening: every time the grain count falls below 0.99 of the
    # count at the last coarsening the grid shrinks (first at loop 12: 100 -> 97)
    "gc_v80": ("voronoi", 80, 100, 11, 24, 4,
               {"IsIsotropicNetwork": 1, "GridCoarsement": 1, "GridCoarsementGradient": 0.99,
                "AnalysisTimestep": 4}),
    # magnetic driving force: field direction (0.6, 0, 0.8), 1/2 mu0 dchi B^2 = 800,
    # read from magnetic.xml beside the parameters; analysis files every 5 steps
    "mag_v30": ("voronoi", 30, 120, 7, 20, 5,
                {"IsIsotropicNetwork": 0, "UseMagneticField": 1, "MagneticParams": "magnetic.xml",
                 "AnalysisTimestep": 5}),
    "ana_mob_v80": ("voronoi", 80, 100, 12, 40, 0,
                    {"IsIsotropicNetwork": 0, "UseMobilityModel": 1, "TriplePointDrag": 2.0,
                     "AnalysisTimestep": 5}),
}


# MicrostructureGenMode 0: the reference's own restart files of a voxelized
# run (grains, steps, seed and overrides of that run; the restart loop; the
# dump interval of the contour-input run that follows).  The restart loop is
# one at which no grain has vanished: the reference's reader reads past the
# end of a file whose grain IDs have gaps.
RESTARTS = {
    # isotropic: 60 grains restarted at loop 8 on the grid int(sqrt(60) * 18) = 139
    "rst_iso_v60": (("voronoi", 60, 140, 1, {"IsIsotropicNetwork": 1}), 8, 4),
    # Read-Shockley: the first step after the restart runs the corrector with
    # no junctions and the placeholder neighbours of find_neighbors
    "rst_rs_v30": (("voronoi", 30, 120, 2, {"IsIsotropicNetwork": 0}), 6, 2),
    # stored energy on: every grain restarts with 0, and the first corrector
    # finds no neighbour characteristic for IDLocal (its force term is -1)
    "rst_se_v30": (("voronoi", 30, 120, 6, {"IsIsotropicNetwork": 0, "UseStoredElasticEnergy": 1,
                                             "DislocEnPerM": 1.0, "BoxDefaultStoredElasticEnergy": 500.0}), 5, 5),
    # grid coarsening on: restarted at loop 8 (80 grains, grid int(sqrt(80) * 11) = 98), the run from the
    # contour file coarsens its grid as grains vanish
    "rst_gc_v80": (("voronoi", 80, 100, 11, {"IsIsotropicNetwork": 1, "GridCoarsement": 1,
                                             "GridCoarsementGradient": 0.99}), 8, 2),
}


MAGNETIC = {"VacuumPermeability": 1.0, "MagneticVector_x": 0.6, "MagneticVector_y": 0.0, "MagneticVector_z": 0.8,
            "deltaMagSys": 1.0, "MagneticForceField": 40.0}


def make_case(name: str, spec) -> dict:
    gen, n, nn, seed, steps, every, over = spec
    d = os.path.join(HERE, name)
    if os.path.isdir(d):
        shutil.rmtree(d)
    micro = ms.voronoi(n, nn, seed) if gen == "voronoi" else ms.clustered(n, nn, seed)
    if over.get("UseStoredElasticEnergy"):
        micro.stored = np.random.default_rng(1000 + seed).uniform(0.0, 3000.0, n)
    xml = ms.make_case(d, name, micro, NumberOfTimesteps=steps, **over)
    if over.get("UseMagneticField"):
        with open(os.path.join(d, over["MagneticParams"]), "w") as f:
            f.write('<?xml version="1.0" encoding="utf-8"?>\n<Parameters>\n')
            for k, v in MAGNETIC.items():
                f.write(f"   <{k}> {v} </{k}>\n")
            f.write("</Parameters>\n")
    dump = os.path.join(d, "reference.dump")
    cmd = [GG_REF, os.path.basename(xml), "reference.dump", str(every), "1"]
    if name.startswith("ana_") or "AnalysisTimestep" in over:
        os.makedirs(os.path.join(d, "analysis"))
        cmd.append("analysis")
    out = subprocess.run(cmd, cwd=d, check=True, capture_output=True, text=True)
    info = json.loads(out.stdout.strip().splitlines()[-1])
    with open(dump, "rb") as f, gzip.open(dump + ".gz", "wb", compresslevel=9) as g:
        shutil.copyfileobj(f, g)
    os.remove(dump)
    info.update({"generator": gen, "grains": n, "grid": nn, "seed": seed, "steps": steps, "dump_every": every,
                 "overrides": over})
    with open(os.path.join(d, "case.json"), "w") as f:
        json.dump(info, f, indent=1)
    return info


def make_restart_case(name: str, spec) -> dict:
    (gen, n, nn, seed, over), loop, every = spec
    d = os.path.join(HERE, name)
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(os.path.join(d, "analysis"))
    # the voxelized run that writes the restart files, in a scratch directory
    work = tempfile.mkdtemp(prefix=name + "_")
    try:
        micro = ms.voronoi(n, nn, seed)
        if over.get("UseStoredElasticEnergy"):
            micro.stored = np.random.default_rng(1000 + seed).uniform(0.0, 3000.0, n)
        xml = ms.make_case(work, name + "_src", micro, NumberOfTimesteps=loop, AnalysisTimestep=loop, **over)
        os.makedirs(os.path.join(work, "analysis"))
        subprocess.run([GG_REF, os.path.basename(xml), "-", "0", "1", "analysis"], cwd=work, check=True,
                       capture_output=True)
        src = os.path.join(work, "analysis")
        names = [f for f in os.listdir(src) if f.startswith(("NETWORK_", "PARAMETERS_")) and
                 f"_TIMESTEP_{loop}_" in f]
        for f in names:
            shutil.copy(os.path.join(src, f), d)
    finally:
        shutil.rmtree(work)
    params = next(f for f in os.listdir(d) if f.startswith("PARAMETERS_"))
    network = next(f for f in os.listdir(d) if f.startswith("NETWORK_"))
    with open(os.path.join(d, network)) as f:
        ids = [int(line.split()[0]) for line in f if len(line.split()) == 6]
    if ids != list(range(1, len(ids) + 1)):
        raise RuntimeError(f"{name}: grain IDs of the restart file have gaps")
    cmd = [GG_REF, params, "reference.dump", str(every), "1", "analysis"]
    out = subprocess.run(cmd, cwd=d, check=True, capture_output=True, text=True)
    info = json.loads(out.stdout.strip().splitlines()[-1])
    dump = os.path.join(d, "reference.dump")
    with open(dump, "rb") as f, gzip.open(dump + ".gz", "wb", compresslevel=9) as g:
        shutil.copyfileobj(f, g)
    os.remove(dump)
    info.update({"generator": gen, "grains": n, "grid": nn, "seed": seed, "restart_loop": loop, "dump_every": every,
                 "overrides": over, "parameters": params})
    with open(os.path.join(d, "case.json"), "w") as f:
        json.dump(info, f, indent=1)
    return info


def main():
    if not os.path.exists(GG_REF):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    names = sys.argv[1:] or list(CASES) + list(RESTARTS)
    for name in names:
        info = make_restart_case(name, RESTARTS[name]) if name in RESTARTS else make_case(name, CASES[name])
        print(name, info)


if __name__ == "__main__":
    main()
