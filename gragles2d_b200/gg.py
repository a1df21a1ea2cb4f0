"""Python mirror of the reference's driver API over the C ABI (include/gg_step.h).

``Settings`` reads a ``parameters.xml`` (src/Settings.cpp:84-289);
``GrainHandler`` is the reference's ``grainhdl`` (src/grainhdl.h:48-203) with
the same stage methods, each of which runs every grain of the network on the
GPU through ``libgg_b200.so``.  There is no CPU fallback: constructing a
``GrainHandler`` without the built library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgg_b200.so")

GG_OK = 0
PRECISION_PLAIN = 0
PRECISION_BATCHED = 1
ERRORS = {1: "invalid", 2: "cuda", 3: "io", 4: "state", 5: "capacity", 6: "numeric"}

# Entry points declared in include/gg_step.h, in declaration order.
EXPORTS = (
    "gg_params_default", "gg_params_from_xml", "gg_create", "gg_destroy", "gg_last_error", "gg_load_voxels",
    "gg_load_voxel_files", "gg_load_stored_energy", "gg_load_contours", "gg_load_contour_file",
    "gg_distance_initialisation", "gg_find_neighbors", "gg_set_neighbours",
    "gg_convolution", "gg_update_second_order_neighbors", "gg_comparison", "gg_level_set", "gg_redistancing",
    "gg_grain_count", "gg_step", "gg_status", "gg_read_grain_stats", "gg_tangent_enable", "gg_read_area_tangents",
    "gg_write_analysis", "gg_write_restart", "gg_dims", "gg_dump", "gg_last_step_ms",
    "gg_grain_updates", "gg_profile_steps", "gg_traffic", "gg_autotune", "gg_kernel_launches",
    "gg_convolve_box_static",
)
STATIC_CONV_MAX_N = 128
NSTAGES = 9
STAGE_NAMES = ("convolution", "corrector", "second_order", "comparison", "level_set", "alloc",
               "volume_energy_neighbours", "redistancing", "end_of_step")


class GGError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gg error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("precision", ctypes.c_int32), ("start_time", ctypes.c_int32),
        ("number_of_timesteps", ctypes.c_int32), ("analysis_timestep", ctypes.c_int32),
        ("breakup_number", ctypes.c_int32), ("number_of_particles", ctypes.c_int32),
        ("number_of_points_per_grain", ctypes.c_int32), ("domain_border_size", ctypes.c_int32),
        ("microstructure_gen_mode", ctypes.c_int32), ("convolution_mode", ctypes.c_int32),
        ("lattice_type", ctypes.c_int32), ("is_isotropic_network", ctypes.c_int32),
        ("use_mobility_model", ctypes.c_int32), ("identify_twins", ctypes.c_int32),
        ("research_mode", ctypes.c_int32), ("research_project", ctypes.c_int32),
        ("decouple_grains", ctypes.c_int32), ("grid_coarsement", ctypes.c_int32),
        ("use_stored_elastic_energy", ctypes.c_int32), ("use_magnetic_field", ctypes.c_int32),
        ("discrete_sampling_rate", ctypes.c_int32), ("plot_interval", ctypes.c_int32), ("use_texture", ctypes.c_int32),
        ("execute_in_parallel", ctypes.c_int32), ("maximum_number_of_threads", ctypes.c_int32),
        ("neighbour_tracking", ctypes.c_int32), ("grain_scheduler", ctypes.c_int32),
        ("list_capacity", ctypes.c_int32), ("reserved_i", ctypes.c_int32),
        ("triple_point_drag", ctypes.c_double), ("constant_sector_radius", ctypes.c_double),
        ("interpolating_sector_radius", ctypes.c_double), ("hagb_energy", ctypes.c_double),
        ("hagb_mobility", ctypes.c_double), ("physical_domain_size", ctypes.c_double),
        ("time_slope", ctypes.c_double), ("theta_ref_deg", ctypes.c_double), ("gamma_hagb", ctypes.c_double),
        ("m_hagb", ctypes.c_double), ("dislocation_energy_per_m", ctypes.c_double),
        ("box_default_stored_elastic_energy", ctypes.c_double), ("vacuum_permeability", ctypes.c_double),
        ("magnetic_vector", ctypes.c_double * 3), ("delta_mag_sys", ctypes.c_double),
        ("magnetic_force_field", ctypes.c_double), ("grid_coarsement_gradient", ctypes.c_double),
        ("arena_factor", ctypes.c_double),
        ("read_from_filename", ctypes.c_char * 512), ("additional_filename", ctypes.c_char * 512),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("compare_threads", ctypes.c_int32), ("big_edge", ctypes.c_int32), ("conv_smem_edge", ctypes.c_int32),
        ("steps_run", ctypes.c_int32), ("ms_default", ctypes.c_double), ("ms_tuned", ctypes.c_double),
    ]


class GrainStats(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_int32), ("state", ctypes.c_int32), ("motion_regular", ctypes.c_int32),
        ("intersects_boundary", ctypes.c_int32), ("n_neighbours", ctypes.c_int32),
        ("contour_points", ctypes.c_int32), ("box", ctypes.c_int32 * 4), ("area", ctypes.c_double),
        ("energy", ctypes.c_double), ("perimeter", ctypes.c_double), ("mean_da", ctypes.c_double),
    ]


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libgg_b200.so (raises if it was not built) and declares signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise GGError(2, f"{path} is missing: build it with `python -m gragles2d_b200.build`")
    lib = ctypes.CDLL(path)
    P, V, I, D = ctypes.POINTER, ctypes.c_void_p, ctypes.c_int32, ctypes.c_double
    sig = {
        "gg_params_default": (I, [P(Params)]),
        "gg_params_from_xml": (I, [ctypes.c_char_p, P(Params)]),
        "gg_create": (I, [P(Params), ctypes.c_int, P(V)]),
        "gg_destroy": (None, [V]),
        "gg_last_error": (ctypes.c_char_p, [V]),
        "gg_load_voxels": (I, [V, I, P(I), I, P(D), P(I)]),
        "gg_load_voxel_files": (I, [V, ctypes.c_char_p]),
        "gg_load_stored_energy": (I, [V, P(D), I]),
        "gg_load_contours": (I, [V, I, P(I), P(D), P(D)]),
        "gg_load_contour_file": (I, [V, ctypes.c_char_p]),
        "gg_distance_initialisation": (I, [V]),
        "gg_find_neighbors": (I, [V]),
        "gg_set_neighbours": (I, [V, P(I), P(I)]),
        "gg_convolution": (I, [V, I]),
        "gg_update_second_order_neighbors": (I, [V]),
        "gg_comparison": (I, [V]),
        "gg_level_set": (I, [V, I]),
        "gg_redistancing": (I, [V, I]),
        "gg_grain_count": (I, [V, P(I), P(D)]),
        "gg_step": (I, [V, I, I]),
        "gg_status": (I, [V, P(ctypes.c_uint32), I]),
        "gg_read_grain_stats": (I, [V, P(GrainStats), I]),
        "gg_tangent_enable": (I, [V, I]),
        "gg_read_area_tangents": (I, [V, P(D), I]),
        "gg_write_analysis": (I, [V, ctypes.c_char_p, I]),
        "gg_write_restart": (I, [V, ctypes.c_char_p, I]),
        "gg_dims": (I, [V, P(I), P(I), P(D), P(D), P(D)]),
        "gg_dump": (I, [V, ctypes.c_char_p, I, I]),
        "gg_last_step_ms": (I, [V, P(D)]),
        "gg_grain_updates": (I, [V, P(ctypes.c_int64)]),
        "gg_profile_steps": (I, [V, I, I, P(D)]),
        "gg_traffic": (I, [V, P(ctypes.c_int64), P(ctypes.c_int64), P(I)]),
        "gg_kernel_launches": (I, [V, P(ctypes.c_int64), P(I)]),
        "gg_autotune": (I, [V, I, I, P(Tuning)]),
        "gg_convolve_box_static": (I, [V, V, I, D, I, V]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def convolve_box_static(d_in: int, d_out: int, n: int, dt: float, real_domain_size: int, stream: int = 0) -> None:
    """Allocation-free convolution of one n x n FP64 box (device pointers),
    bit-identical to the plain convolution stage; see gg_convolve_box_static."""
    lib = load_library()
    rc = lib.gg_convolve_box_static(ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), n, dt, real_domain_size,
                                    ctypes.c_void_p(stream))
    if rc != GG_OK:
        raise GGError(rc, f"gg_convolve_box_static(n={n})")


class Settings:
    """Parsed parameters.xml (the reference's static ``Settings``)."""

    def __init__(self, path: str | None = None, **overrides):
        lib = load_library()
        self.p = Params()
        lib.gg_params_default(ctypes.byref(self.p))
        self.base_dir = ""
        if path is not None:
            rc = lib.gg_params_from_xml(path.encode(), ctypes.byref(self.p))
            if rc != GG_OK:
                raise GGError(rc, f"cannot parse {path}")
            self.base_dir = os.path.dirname(os.path.abspath(path))
        for k, v in overrides.items():
            setattr(self.p, k, v)

    def __getattr__(self, k):
        return getattr(self.__dict__["p"], k)


@dataclass
class Dims:
    n_grains: int
    ngridpoints: int
    h: float
    delta: float
    dt: float


class GrainHandler:
    """The reference's ``grainhdl`` on one GPU (src/grainhdl.h:48-203)."""

    def __init__(self, settings: Settings, device: int = 0):
        self.lib = load_library()
        self.settings = settings
        ctx = ctypes.c_void_p()
        rc = self.lib.gg_create(ctypes.byref(settings.p), device, ctypes.byref(ctx))
        self.ctx = ctx
        if rc != GG_OK:
            msg = self.lib.gg_last_error(ctx).decode() if ctx.value else ""
            if ctx.value:
                self.lib.gg_destroy(ctx)
                self.ctx = ctypes.c_void_p()
            raise GGError(rc, msg)
        self.loop = settings.p.start_time

    def close(self):
        if self.ctx and self.ctx.value:
            self.lib.gg_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != GG_OK:
            raise GGError(rc, self.lib.gg_last_error(self.ctx).decode())

    # -- setSimulationParameter / read_voxelized_microstructure --
    def load_voxel_files(self):
        self._check(self.lib.gg_load_voxel_files(self.ctx, self.settings.base_dir.encode()))

    def load_voxels(self, ids: np.ndarray, euler: np.ndarray, bbox: np.ndarray, stored: np.ndarray | None = None):
        """Voxelized input from host arrays; `stored` holds the .uds stored
        energies (one per grain), used when UseStoredElasticEnergy is set."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        euler = np.ascontiguousarray(euler, dtype=np.float64)
        bbox = np.ascontiguousarray(bbox, dtype=np.int32)
        P = ctypes.POINTER
        self._check(self.lib.gg_load_voxels(
            self.ctx, ids.shape[0], ids.ctypes.data_as(P(ctypes.c_int32)), euler.shape[0],
            euler.ctypes.data_as(P(ctypes.c_double)), bbox.ctypes.data_as(P(ctypes.c_int32))))
        if stored is not None:
            stored = np.ascontiguousarray(stored, dtype=np.float64)
            self._check(self.lib.gg_load_stored_energy(self.ctx, stored.ctypes.data_as(P(ctypes.c_double)),
                                                       stored.shape[0]))

    def load_contour_file(self):
        """MicrostructureGenMode 0: the contour file ReadFromFilename names
        (grainhdl::readMicrostructure, src/grainhdl.cpp:605-654)."""
        self._check(self.lib.gg_load_contour_file(self.ctx, self.settings.base_dir.encode()))

    def load_contours(self, contours, quats):
        """Contour input from host arrays: `contours[k]` is grain k+1's polygon
        (points x, y in domain coordinates; empty = absent grain) and
        `quats[k]` its orientation quaternion."""
        offs = np.zeros(len(contours) + 1, np.int32)
        for k, c in enumerate(contours):
            offs[k + 1] = offs[k] + len(c)
        xy = np.ascontiguousarray(np.concatenate([np.asarray(c, np.float64).reshape(-1, 2) for c in contours])
                                  if offs[-1] else np.zeros((1, 2)), dtype=np.float64)
        q = np.ascontiguousarray(quats, dtype=np.float64).reshape(len(contours), 4)
        P = ctypes.POINTER
        self._check(self.lib.gg_load_contours(
            self.ctx, len(contours), offs.ctypes.data_as(P(ctypes.c_int32)), xy.ctypes.data_as(P(ctypes.c_double)),
            q.ctypes.data_as(P(ctypes.c_double))))

    def setSimulationParameter(self):
        """Reads the microstructure the parameters name: a contour file for
        MicrostructureGenMode 0, the .uds/.bin pair for mode 4."""
        if self.settings.p.microstructure_gen_mode == 0:
            self.load_contour_file()
        else:
            self.load_voxel_files()

    # -- run_sim prologue --
    def distanceInitialisation(self):
        self._check(self.lib.gg_distance_initialisation(self.ctx))

    def find_neighbors(self):
        self._check(self.lib.gg_find_neighbors(self.ctx))

    def set_neighbours(self, lists: dict):
        n = self.dims().n_grains
        offs = np.zeros(n + 1, np.int32)
        flat = []
        for g in range(1, n + 1):
            ids = lists.get(g, [])
            flat.extend(ids)
            offs[g] = offs[g - 1] + len(ids)
        flat = np.asarray(flat if flat else [0], np.int32)
        P = ctypes.POINTER
        self._check(self.lib.gg_set_neighbours(self.ctx, offs.ctypes.data_as(P(ctypes.c_int32)),
                                               flat.ctypes.data_as(P(ctypes.c_int32))))

    # -- stage methods of the time loop --
    def convolution(self):
        self._check(self.lib.gg_convolution(self.ctx, self.loop))

    def updateSecondOrderNeighbors(self):
        self._check(self.lib.gg_update_second_order_neighbors(self.ctx))

    def comparison_box(self):
        self._check(self.lib.gg_comparison(self.ctx))

    def level_set(self):
        self._check(self.lib.gg_level_set(self.ctx, self.loop))

    def redistancing(self):
        self._check(self.lib.gg_redistancing(self.ctx, self.loop))
        self.loop += 1

    def get_biggestGrainVol(self):
        cur = ctypes.c_int32()
        mv = ctypes.c_double()
        self._check(self.lib.gg_grain_count(self.ctx, ctypes.byref(cur), ctypes.byref(mv)))
        return cur.value, mv.value

    def step(self, nsteps: int = 1) -> float:
        """Runs whole timesteps; returns device milliseconds."""
        self._check(self.lib.gg_step(self.ctx, self.loop, nsteps))
        self.loop += nsteps
        ms = ctypes.c_double()
        self.lib.gg_last_step_ms(self.ctx, ctypes.byref(ms))
        return ms.value

    def run_sim(self, steps: int | None = None, stage_calls: bool = False, analysis_dir: str | None = None):
        """distanceInitialisation, find_neighbors, then the time loop
        (src/grainhdl.cpp:1035-1142); stops early below BreakupNumber.  With
        `analysis_dir`, writes the texture / MODF / statistics files into it
        every AnalysisTimestep steps and after step NumberOfTimesteps
        (src/grainhdl.cpp:1098-1105)."""
        self.distanceInitialisation()
        self.find_neighbors()
        p = self.settings.p
        total = (p.number_of_timesteps + 1) if steps is None else steps
        for _ in range(total):
            loop = self.loop
            if stage_calls:
                self.convolution()
                self.updateSecondOrderNeighbors()
                self.comparison_box()
                self.level_set()
                self.redistancing()
            else:
                self.step(1)
            if analysis_dir is not None and ((loop - p.start_time) % p.analysis_timestep == 0
                                             or loop == p.number_of_timesteps):
                self.write_analysis(analysis_dir, loop)
                if (p.microstructure_gen_mode == 4 and loop == 0) or loop == p.number_of_timesteps:
                    self.write_restart(analysis_dir, loop)
            live, _ = self.get_biggestGrainVol()
            if live < self.settings.p.breakup_number:
                break

    # -- inspection --
    def dims(self) -> Dims:
        n, m = ctypes.c_int32(), ctypes.c_int32()
        h, d, dt = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.gg_dims(self.ctx, ctypes.byref(n), ctypes.byref(m), ctypes.byref(h), ctypes.byref(d),
                                     ctypes.byref(dt)))
        return Dims(n.value, m.value, h.value, d.value, dt.value)

    def status(self, clear: bool = False) -> int:
        s = ctypes.c_uint32()
        self._check(self.lib.gg_status(self.ctx, ctypes.byref(s), int(clear)))
        return s.value

    def grain_stats(self, out=None):
        """Every grain's statistics (gg_read_grain_stats); `out`, an array
        from an earlier call, is filled again instead of a new one."""
        n = self.dims().n_grains
        arr = out if out is not None and len(out) >= n else (GrainStats * n)()
        self._check(self.lib.gg_read_grain_stats(self.ctx, arr, n))
        return arr

    def areas(self) -> np.ndarray:
        st = self.grain_stats()
        return np.array([s.area if s.state == 1 else np.nan for s in st])

    def enable_tangents(self, on: bool = True):
        """Carry d phi / d p for p = (theta_ref [deg], HAGB energy, HAGB
        mobility, triple-point drag); call before distanceInitialisation."""
        self._check(self.lib.gg_tangent_enable(self.ctx, int(on)))

    def area_tangents(self) -> np.ndarray:
        """d area_g / d p of the last level set, shape (N, 4), row g-1 for grain g."""
        n = self.dims().n_grains
        out = np.zeros(4 * n, np.float64)
        self._check(self.lib.gg_read_area_tangents(self.ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                   out.size))
        return out.reshape(n, 4)

    def write_analysis(self, directory: str, loop: int | None = None):
        """save_Texture + save_NrGrainsStats of the completed step `loop`
        (default: the last one) into `directory`."""
        self._check(self.lib.gg_write_analysis(self.ctx, directory.encode(), self.loop - 1 if loop is None else loop))

    def write_restart(self, directory: str, loop: int | None = None):
        """save_Full_Microstructure_for_Restart of the completed step `loop`
        (default: the last one) into `directory`."""
        self._check(self.lib.gg_write_restart(self.ctx, directory.encode(), self.loop - 1 if loop is None else loop))

    def grain_updates(self) -> int:
        v = ctypes.c_int64()
        self._check(self.lib.gg_grain_updates(self.ctx, ctypes.byref(v)))
        return v.value

    def profile_steps(self, nsteps: int) -> dict:
        """Runs nsteps stage by stage; returns device ms per stage."""
        arr = (ctypes.c_double * NSTAGES)()
        self._check(self.lib.gg_profile_steps(self.ctx, self.loop, nsteps, arr))
        self.loop += nsteps
        return dict(zip(STAGE_NAMES, list(arr)))

    def traffic(self) -> tuple[int, int, int]:
        a, o, n = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        self._check(self.lib.gg_traffic(self.ctx, ctypes.byref(a), ctypes.byref(o), ctypes.byref(n)))
        return a.value, o.value, n.value

    def autotune(self, steps_per_candidate: int = 2) -> dict:
        """Chooses the batched form's launch bins by timing whole steps with
        each candidate (gg_autotune); the steps it runs advance the run."""
        t = Tuning()
        self._check(self.lib.gg_autotune(self.ctx, self.loop, steps_per_candidate, ctypes.byref(t)))
        self.loop += t.steps_run
        return {f: getattr(t, f) for f, _ in Tuning._fields_}

    def kernel_launches(self) -> tuple[int, int]:
        """(kernels launched by step() graph replays so far, kernel nodes per
        step graph); the plain form reports (0, 0)."""
        t, k = ctypes.c_int64(), ctypes.c_int32()
        self._check(self.lib.gg_kernel_launches(self.ctx, ctypes.byref(t), ctypes.byref(k)))
        return t.value, k.value

    def dump(self, path: str, steps_done: int = 0, append: bool = False):
        self._check(self.lib.gg_dump(self.ctx, path.encode(), steps_done, int(append)))
