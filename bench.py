"""Benchmark: grain-updates/s of the batched FP32 level-set step on one B200
(next to the plain FP64 step on the same GPU and the reference's OpenMP CPU
path on the host cores).

Workload: 20,000 grains, Voronoi tessellation of uniform seeds (seed 1) on a
3600 x 3600 grid (mean grain diameter ~25 cells), random uniform SO(3)
orientations, Read-Shockley boundary energy with a 15 degree cut-off,
isotropic mobility; seeded synthetic input in the reference's voxelized
format (its example inputs are not shipped).  A "step" is one level-set
timestep of the whole network (convolution + corrector, second-order lists,
comparison, contour / level set, redistancing).  The working set (two FP32
distance arenas, two IDLocal arenas, contours) is several times the 126 MB
L2, so no flush is needed between timed steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (the step does not shard; one process per
GPU under torchrun) and reports the sum of their throughput over the
slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grain-updates/s"
WORKLOAD = dict(name="voronoi_20000g_3600_rs15", grains=20000, grid=3600, seed=1, iso=0, mobility=0, tpd=0.0)
SMALL = dict(name="voronoi_1000g_800_iso", grains=1000, grid=800, seed=0, iso=1, mobility=0, tpd=0.0)
CACHE = os.path.join(tempfile.gettempdir(), "gg_bench_cache")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "gg_ref")
REF_BIN_FFT = os.path.join(ROOT, "oracle", "_ref", "gg_ref_fft")


def rank_info():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def workload_case(w: dict) -> tuple[str, dict]:
    """Writes (once) the mode-4 input and its parameters.xml; returns the XML path."""
    from gragles2d_b200 import microstructure as ms

    d = os.path.join(CACHE, w["name"])
    xml = os.path.join(d, w["name"] + ".xml")
    if not os.path.exists(xml):
        micro = ms.voronoi(w["grains"], w["grid"], w["seed"])
        tmp = d + f".tmp{os.getpid()}"
        ms.make_case(tmp, w["name"], micro, NumberOfTimesteps=10, IsIsotropicNetwork=w["iso"],
                     UseMobilityModel=w["mobility"], TriplePointDrag=w["tpd"])
        try:
            os.replace(tmp, d)
        except OSError:
            shutil.rmtree(tmp, ignore_errors=True)
    return xml, w


def workload_config(w: dict, world: int) -> dict:
    """The `config` of both arms' JSON lines (the same workload)."""
    return {"workload": "20000-grain Voronoi (seed 1) on 3600x3600, Read-Shockley 15 deg, "
                        "batched FP32 graph-captured step", "grains": w["grains"], "grid": w["grid"],
            "l2": "working set larger than L2 (no flush)", "parallelism": f"replicas{world}"}


def load_inputs(xml: str):
    """Host buffers of the voxelized input (ids, euler, bbox)."""
    from gragles2d_b200 import microstructure as ms

    d = os.path.dirname(xml)
    name = os.path.basename(xml)[:-4]
    lines = open(os.path.join(d, name + ".uds")).read().splitlines()
    nn = int(lines[4].split()[1])
    rows = np.array([l.split() for l in lines[8:]], dtype=np.float64)
    euler = rows[:, 3:6].copy()
    bbox = rows[:, 6:11].astype(np.int32)
    ids = np.fromfile(os.path.join(d, name + ".bin"), dtype="<i4").reshape(nn, nn)
    return ids, euler, bbox


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                v = [x.strip() for x in out.stdout.strip().split(",")]
                if len(v) == 7:
                    self.samples.append(v)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        return json.load(open(p)).get(kernel)
    except Exception:
        return None


def stage_bytes(stage: str, s: int, area: int, overlap: int, aniso: bool) -> float:
    """Algorithmic bytes of one stage over the network (s bytes per field value,
    u32 IDLocal): convolution reads and writes each box; the corrector reads
    phi_t, the convolution and IDLocal and writes the convolution; the
    comparison reads its own and its neighbours' overlapping convolutions and
    the old IDLocal and writes the compared field and IDLocal; the level set
    reads the compared field and IDLocal; redistancing reads the compared
    field and writes the new one."""
    return {
        "convolution": 2 * s * area,
        "corrector": (3 * s + 4) * area if aniso else 0,
        "comparison": s * (2 * area + overlap) + 8 * area,
        "level_set": (s + 4) * area,
        "redistancing": 2 * s * area,
    }.get(stage, 0)


def max_over_ranks(values, dist, device=None):
    """Element-wise maximum of per-rank timings (every rank calls it once)."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def aggregate_throughput(world: int, updates_per_rank: int, max_ms: float) -> float:
    """Replicas: every rank advances its own network by the same number of
    grain-updates; the job's throughput is their sum over the slowest rank's time."""
    return world * updates_per_rank / (max_ms / 1e3)


def run_ours(args, rank, world, local_rank):
    import torch

    from gragles2d_b200 import accuracy, gg

    dist = None
    if world > 1:
        import torch.distributed as tdist

        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = tdist
    device = local_rank
    xml, w = workload_case(WORKLOAD)
    ids, euler, bbox = load_inputs(xml)
    K, W = args.steps, args.warmup

    def barrier():
        if dist:
            dist.barrier()

    # ---- e2e through the C ABI from host buffers (batched form) ----
    # The inputs sit in pinned (page-locked) host memory, as a caller that
    # streams networks to the GPU holds them; pinning is outside the timed
    # region, the copies to the device inside it.
    pinned_keep = []

    def pinned(a: np.ndarray) -> np.ndarray:
        t = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), pin_memory=True)
        pinned_keep.append(t)
        v = t.numpy()
        v[...] = a
        return v

    ids, euler, bbox = pinned(ids), pinned(euler), pinned(bbox)
    # Warm-up, untimed: the same calls on a throw-away network with W steps
    # (CUDA context creation, module loading and the first graph capture
    # are process start-up costs, as the reference's are outside its loop).
    hw = gg.GrainHandler(gg.Settings(xml, precision=gg.PRECISION_BATCHED), device=device)
    hw.load_voxels(ids, euler, bbox)
    hw.distanceInitialisation()
    hw.find_neighbors()
    for _ in range(W):
        hw.step(1)
        hw.grain_stats()
    # launch bins measured on this network; the library keeps them for the
    # contexts below (same largest box edge and grain count)
    tuning = hw.autotune(1)
    hw.close()
    # Timed: load from the host buffers, initialise, K steps each followed by
    # a read of every grain's statistics.
    barrier()
    t0 = time.perf_counter()
    sb = gg.Settings(xml, precision=gg.PRECISION_BATCHED)
    hb = gg.GrainHandler(sb, device=device)
    hb.load_voxels(ids, euler, bbox)
    hb.distanceInitialisation()
    hb.find_neighbors()
    stats_bytes = 0
    st = None  # one statistics array, filled again every step
    for _ in range(K):
        hb.step(1)
        st = hb.grain_stats(st)
        stats_bytes += len(st) * ctypes.sizeof(gg.GrainStats)
    t_e2e = time.perf_counter() - t0
    upd_e2e = hb.grain_updates()
    st_b = hb.grain_stats()
    areas_b = np.array([s.area if s.state == 1 else np.nan for s in st_b])
    h2d = ids.nbytes + euler.nbytes + bbox.nbytes

    # ---- device-timed batched steps ----
    hb.step(W)
    u0 = hb.grain_updates()
    l0, per_step = hb.kernel_launches()
    barrier()
    with ClockSampler(device) as clk:
        ms_b = hb.step(K)
    barrier()
    upd_b = hb.grain_updates() - u0
    launches = hb.kernel_launches()[0] - l0
    # roofline of the dominant stage
    area, overlap, nex = hb.traffic()
    prof = hb.profile_steps(2)
    area2, overlap2, _ = hb.traffic()
    status_b = hb.status()
    hb.close()

    # ---- plain FP64 on the same GPU ----
    sp = gg.Settings(xml, precision=gg.PRECISION_PLAIN)
    hp = gg.GrainHandler(sp, device=device)
    hp.load_voxels(ids, euler, bbox)
    hp.distanceInitialisation()
    hp.find_neighbors()
    hp.step(K)  # the same steps as the batched network's e2e run, for the area comparison
    st_p = hp.grain_stats()
    hp.step(W)
    areas_p = np.array([s.area if s.state == 1 else np.nan for s in st_p])
    u0p = hp.grain_updates()
    kp = max(1, min(K, args.plain_steps))
    ms_p = hp.step(kp)
    upd_p = hp.grain_updates() - u0p
    hp.close()

    # every grain alive in both forms, no size cut
    area_diag = accuracy.area_errors(areas_p, areas_b, 1.0 / (w["grid"] ** 2))
    area_err = area_diag.get("max")

    # ---- max over ranks ----
    t_ms, t_e2e = max_over_ranks([ms_b, t_e2e], dist, f"cuda:{device}")
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    value = aggregate_throughput(world, upd_b, t_ms)
    aniso = not w["iso"]
    peak, peak_kind = measured_peak_hbm()
    stage_ms = {k: v / 2 for k, v in prof.items()}
    ab = {k: stage_bytes(k, 4, (area + area2) // 2, (overlap + overlap2) // 2, aniso) for k in stage_ms}
    path_bytes = float(sum(ab.values()))
    dom = max(stage_ms, key=lambda k: stage_ms[k])
    dom_bytes = ab.get(dom, 0)
    achieved = dom_bytes / (stage_ms[dom] / 1e3) / 1e9 if dom_bytes else None
    kernel_names = {"convolution": "k_conv_sep", "corrector": "k_corrector_f", "comparison": "k_compare",
                    "level_set": "k_levelset_w", "redistancing": "k_redistance_s",
                    "volume_energy_neighbours": "k_neighbours_w + k_sectors"}
    out = {
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": t_ms / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(w, world),
        "e2e": {"value": aggregate_throughput(world, upd_e2e, t_e2e * 1e3), "unit": METRIC, "h2d_bytes_per_step": h2d / K,
                "d2h_bytes_per_step": stats_bytes / K,
                "includes": "context set-up on the device, load from pinned host buffers, distance initialisation, "
                            "neighbour search, K steps each with a read of all grain statistics (after an untimed "
                            "warm-up pass of the same calls with W steps, so CUDA context creation and module "
                            "loading are not in it)"},
        "roofline": {"bound": "hbm", "kernel": kernel_names.get(dom, dom), "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": committed_traffic(kernel_names.get(dom, dom)),
                     "algorithmic_bytes_per_launch": dom_bytes, "stage_ms": stage_ms,
                     # the whole step: every stage's algorithmic bytes over the graph-timed step
                     "path": {"algorithmic_bytes_per_step": path_bytes,
                              "achieved": path_bytes / (t_ms / K / 1e3) / 1e9,
                              "frac": path_bytes / (t_ms / K / 1e3) / 1e9 / peak}},
        "plain_fp64": {"value": upd_p / (ms_p / 1e3), "ms_per_step": ms_p / kp, "steps": kp},
        "batched_vs_plain": (upd_b / (t_ms / 1e3)) / (upd_p / (ms_p / 1e3)),
        "area_rel_err_max": area_err,
        "area_err_detail": {"steps": K, **area_diag},
        "clocks": clk.summary(),
        # kernel nodes of the captured step graph (counted by the library
        # when it captured the graph) times the timed replays
        "gpu_launches": launches,
        "gpu_launches_per_step": per_step,
        "launch_bins": tuning,
        "status": status_b,
    }
    if world == 1 and not args.no_accuracy:
        rows = accuracy.trajectory(xml, args.accuracy_steps, 50, device=device, inputs=(ids, euler, bbox))
        keys = ("max", "p99", "over_1e-3", "compared")
        out["accuracy_run"] = {
            "workload": f"the same network, {args.accuracy_steps} steps of both forms from the same input "
                        "(outside the timed region)",
            "fp64_perturbed": "plain FP64 with every boundary energy scaled by 1 - 2^-46 (sensitivity floor)",
            "every_50_steps": [{"step": r["step"], "fp32": {k: r["fp32"].get(k) for k in keys},
                                "fp64_perturbed": {k: r["fp64_perturbed"].get(k) for k in keys}} for r in rows]}
    if not args.no_gradient:
        out["gradient"] = gradient_check(device)
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(xml, 1, args.cpu_steps)
    return out


def cpu_baseline(xml: str, warmup: int, steps: int) -> dict:
    """The reference's OpenMP path on the host cores (all of them), on a
    bounded sample of the same workload: loop 0 (the reference runs no
    corrector there), `warmup` untimed loops, then `steps` timed loops; the
    throughput is their grains over their summed loop times (the harness
    times every loop of run_sim's body, src/grainhdl.cpp:1049-1142)."""
    binary = REF_BIN_FFT if os.path.exists(REF_BIN_FFT) else REF_BIN
    if not os.path.exists(binary):
        return {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "reference",
                "sample": "unavailable: oracle/_ref/gg_ref not built"}
    d = tempfile.mkdtemp(prefix="gg_ref_")
    src = os.path.dirname(xml)
    for f in os.listdir(src):
        os.symlink(os.path.join(src, f), os.path.join(d, f))
    name = os.path.basename(xml)
    txt = open(xml).read()
    import re

    total = 1 + warmup + steps  # loops 0 .. total - 1
    txt = re.sub(r"<NumberOfTimesteps>[^<]*</NumberOfTimesteps>", f"<NumberOfTimesteps> {total - 1} </NumberOfTimesteps>",
                 txt)
    os.remove(os.path.join(d, name))
    open(os.path.join(d, name), "w").write(txt)
    env = dict(os.environ)
    cores = os.cpu_count() or 1
    env["OMP_NUM_THREADS"] = str(cores)
    out = subprocess.run([binary, name, "-", "0", "1"], cwd=d, capture_output=True, text=True, env=env,
                         timeout=1800)
    shutil.rmtree(d, ignore_errors=True)
    info = json.loads(out.stdout.strip().splitlines()[-1])
    secs = info["step_s"][1 + warmup:]
    grains = info["step_grains"][1 + warmup:]
    fft = "O(n log n) mixed-radix / Bluestein FFT shim" if binary == REF_BIN_FFT else "direct-DFT FFT shim"
    return {"value": sum(grains) / sum(secs), "unit": METRIC, "cores": info["threads"], "kind": "reference",
            "steps": len(secs), "warmup": warmup,
            "sample": f"loops {1 + warmup}..{total - 1} of the same workload after loop 0 and {warmup} warm-up "
                      f"loops ({sum(grains)} grain-updates in {sum(secs):.2f} s; initialisation excluded); "
                      f"the reference's C++ built with -O3 -fopenmp and the {fft} standing in for FFTW3"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    xml, w = workload_case(WORKLOAD)
    # whole steps of the workload; the reference needs a second or more per step
    steps = max(1, min(args.steps, args.ref_max_steps))
    cb = cpu_baseline(xml, args.warmup, steps)
    if cb["value"] is None:
        return {"impl": "reference", "unavailable": cb["sample"]}
    v = cb["value"]
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": world,
            "steps": cb["steps"], "warmup": cb["warmup"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(w, world),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


PROFILE_CASE = dict(name="voronoi_5000g_1800_rs15", grains=5000, grid=1800, seed=4, iso=0, mobility=0, tpd=0.0)

GRAD_PARAMS = ("theta_ref_deg", "gamma_hagb", "m_hagb", "triple_point_drag")


def gradient_check(device: int) -> dict:
    """Parameter derivatives of the plain FP64 step (tangent mode) against
    central differences (h = 1e-5 relative) on the committed 30-grain
    mobility-model case, 8 steps; and the cost of carrying the four tangents
    on the 5,000-grain Voronoi case (20 steps) next to the plain step."""
    from gragles2d_b200 import gg

    xml = os.path.join(ROOT, "tests", "golden", "mob_v30", "mob_v30.xml")
    steps = 8

    def run(params, tangents=False):
        h = gg.GrainHandler(gg.Settings(xml, precision=gg.PRECISION_PLAIN, **params), device=device)
        h.load_voxel_files()
        if tangents:
            h.enable_tangents()
        h.distanceInitialisation()
        h.find_neighbors()
        h.step(steps)
        a = np.array([x.area if x.state == 1 else np.nan for x in h.grain_stats()])
        t = h.area_tangents() if tangents else None
        h.close()
        return a, t

    s = gg.Settings(xml)
    p0 = {k: float(getattr(s.p, k)) for k in GRAD_PARAMS}
    areas, tang = run(p0, True)
    target, _ = run({**p0, "theta_ref_deg": 12.0, "m_hagb": 0.8, "triple_point_drag": 0.3})
    alive = np.isfinite(areas) & np.isfinite(target)
    per_param = {}
    for k, name in enumerate(GRAD_PARAMS):
        hk = p0[name] * 1e-5
        ap, _ = run({**p0, name: p0[name] + hk})
        am, _ = run({**p0, name: p0[name] - hk})
        fd = (ap - am) / (2 * hk)
        m = np.isfinite(fd) & np.isfinite(tang[:, k])
        rel = np.abs(tang[m, k] - fd[m]) / np.maximum(np.abs(fd[m]), 1e-3 * np.abs(fd[m]).max())
        g_t = float(np.sum(2 * (areas - target)[alive] * tang[alive, k]))
        lp = float(np.nansum(((ap - target)[alive]) ** 2))
        lm = float(np.nansum(((am - target)[alive]) ** 2))
        g_fd = (lp - lm) / (2 * hk)
        per_param[name] = {"area_rel_err_median": float(np.median(rel)), "area_rel_err_max": float(rel.max()),
                           "loss_grad": g_t, "loss_grad_fd": g_fd,
                           "loss_grad_rel_err": abs(g_t - g_fd) / max(abs(g_fd), 1e-300)}
    # cost of the tangents at scale
    pxml, _ = workload_case(PROFILE_CASE)
    cost = {}
    for tangents in (False, True):
        h = gg.GrainHandler(gg.Settings(pxml, precision=gg.PRECISION_PLAIN), device=device)
        h.load_voxel_files()
        if tangents:
            h.enable_tangents()
        h.distanceInitialisation()
        h.find_neighbors()
        h.step(3)
        cost["tangent" if tangents else "plain"] = h.step(20) / 20
        h.close()
    return {"form": "tangent-linear (forward mode), plain FP64", "case": "mob_v30: 30 grains, 120^2, "
            "Read-Shockley + mobility model + drag 5, 8 steps; loss sum (A - A*)^2, A* at (12 deg, 1, 0.8, 0.3)",
            "fd": "central, h = 1e-5 relative", "params": per_param,
            "ms_per_step_5000g": cost}


def run_profile_case(args, local_rank):
    """Small case for ncu captures: 5,000 grains on 1800^2 (Read-Shockley),
    batched form, W graph-captured steps then 2 steps launched stage by stage."""
    from gragles2d_b200 import gg

    xml, _ = workload_case(PROFILE_CASE)
    prec = gg.PRECISION_PLAIN if args.profile_plain else gg.PRECISION_BATCHED
    h = gg.GrainHandler(gg.Settings(xml, precision=prec), device=local_rank)
    h.load_voxel_files()
    h.distanceInitialisation()
    h.find_neighbors()
    h.step(args.warmup)
    area, overlap, nex = h.traffic()
    prof = h.profile_steps(2)
    print(json.dumps({"profile_case": PROFILE_CASE["name"], "stage_ms": prof, "status": h.status(),
                      "sum_box_area": area, "sum_overlap": overlap, "grains": nex}), flush=True)
    h.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--plain-steps", type=int, default=20)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gradient", action="store_true", help="skip the parameter-derivative check")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the whole-run area-error comparison")
    ap.add_argument("--accuracy-steps", type=int, default=500)
    ap.add_argument("--ref-max-steps", type=int, default=40)
    ap.add_argument("--profile-case", action="store_true", help="small stage-by-stage run for ncu captures")
    ap.add_argument("--profile-plain", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local_rank = rank_info()
    os.makedirs(CACHE, exist_ok=True)
    if args.profile_case:
        run_profile_case(args, local_rank)
        return
    res = run_reference(args, rank, world) if args.impl == "reference" else run_ours(args, rank, world, local_rank)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
