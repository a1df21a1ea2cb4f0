"""The oracle itself: the FFT shim against the DFT definition, the golden
fixtures against the reference run, and the harness build."""
import ctypes
import gzip
import json
import os
import subprocess

import numpy as np
import pytest

from gragles2d_b200 import dumpfile

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = ["iso_v20", "iso_v60", "rs_v30", "mob_v30"]


def reference_src() -> str:
    """The reference's src/ directory: REF_SRC from the environment, else the
    oracle Makefile's default."""
    out = subprocess.run(["make", "-s", "-C", ORACLE, "print-ref-src"], capture_output=True, text=True, check=True)
    return out.stdout.strip()


@pytest.fixture(scope="module", params=["fft_shim", "fft_fast"])
def shim(request):
    """An FFTW-API shim compiled as a small shared library for direct calls:
    the direct DFT of the parity oracle or the FFT of the timing baseline."""
    out = os.path.join(ORACLE, "_ref", f"lib{request.param}_test.so")
    src = os.path.join(ORACLE, "shim", request.param + ".c")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", src, "-lm", "-o", out], check=True)
    lib = ctypes.CDLL(out)
    P = ctypes.POINTER
    lib.fftw_plan_dft_r2c_2d.restype = ctypes.c_void_p
    lib.fftw_plan_dft_r2c_2d.argtypes = [ctypes.c_int, ctypes.c_int, P(ctypes.c_double), P(ctypes.c_double),
                                         ctypes.c_uint]
    lib.fftw_plan_dft_c2r_2d.restype = ctypes.c_void_p
    lib.fftw_plan_dft_c2r_2d.argtypes = [ctypes.c_int, ctypes.c_int, P(ctypes.c_double), P(ctypes.c_double),
                                         ctypes.c_uint]
    lib.fftw_execute.argtypes = [ctypes.c_void_p]
    lib.fftw_destroy_plan.argtypes = [ctypes.c_void_p]
    return lib


def _r2c(lib, x):
    n0, n1 = x.shape
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros((n0, n1 // 2 + 1, 2))
    P = ctypes.POINTER(ctypes.c_double)
    p = lib.fftw_plan_dft_r2c_2d(n0, n1, x.ctypes.data_as(P), y.ctypes.data_as(P), 64)
    lib.fftw_execute(p)
    lib.fftw_destroy_plan(p)
    return y[..., 0] + 1j * y[..., 1]


def _c2r(lib, y, n1):
    n0 = y.shape[0]
    yy = np.ascontiguousarray(np.stack([y.real, y.imag], -1))
    x = np.zeros((n0, n1))
    P = ctypes.POINTER(ctypes.c_double)
    p = lib.fftw_plan_dft_c2r_2d(n0, n1, yy.ctypes.data_as(P), x.ctypes.data_as(P), 64)
    lib.fftw_execute(p)
    lib.fftw_destroy_plan(p)
    return x


@pytest.mark.parametrize("n", [1, 2, 3, 7, 16, 17, 31, 40, 41, 43, 64, 97, 100])
def test_fft_shim_matches_dft_definition(shim, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n))
    y = _r2c(shim, x)
    ref = np.fft.rfft2(x)  # unnormalised forward DFT, same half-spectrum layout
    np.testing.assert_allclose(y, ref, rtol=0, atol=1e-10 * max(1, n * n))
    back = _c2r(shim, ref, n)  # unnormalised inverse: n^2 * x
    np.testing.assert_allclose(back, x * n * n, rtol=0, atol=1e-9 * max(1, n * n))


def test_fft_shim_c2r_ignores_antihermitian_part(shim):
    n = 12
    rng = np.random.default_rng(5)
    x = rng.standard_normal((n, n))
    y = np.fft.rfft2(x)
    y_bad = y.copy()
    y_bad[0, 0] += 3j  # imaginary DC part: ignored by a c2r transform
    np.testing.assert_allclose(_c2r(shim, y_bad, n), _c2r(shim, y, n), atol=1e-9)


@pytest.mark.parametrize("case", CASES)
def test_golden_dumps_parse_and_conserve_area(case):
    d = dumpfile.read(os.path.join(GOLDEN, case, "reference.dump.gz"))
    info = json.load(open(os.path.join(GOLDEN, case, "case.json")))
    assert d.n_grains == info["grains"]
    assert d.records[0].steps == 0 and d.records[-1].steps == info["steps"] + 1
    for rec in d.records:
        live = [g for g in rec.grains.values() if g.state == 1]
        area = sum(g.volume for g in live)
        # grains tile the domain up to the boundary tube
        assert 0.95 < area < 1.0
        for g in live:
            assert g.contour.shape[0] >= 4
            assert np.all(np.abs(g.phi) <= d.delta + 1e-15)
            x0, x1, y0, y1 = g.box
            assert x1 - x0 == y1 - y0  # square boxes (resizeToSquare)


def test_golden_inputs_regenerate_identically(tmp_path):
    """The committed mode-4 inputs are the generator's output for their seeds."""
    from gragles2d_b200 import microstructure as ms

    info = json.load(open(os.path.join(GOLDEN, "iso_v20", "case.json")))
    micro = ms.voronoi(info["grains"], info["grid"], info["seed"])
    ms.write_mode4(str(tmp_path / "x"), micro)
    assert open(tmp_path / "x.bin", "rb").read() == open(os.path.join(GOLDEN, "iso_v20", "iso_v20.bin"), "rb").read()


@pytest.mark.skipif(not os.path.isdir(reference_src()), reason="reference tree not present")
def test_reference_rerun_matches_committed_fixture(tmp_path):
    """Rebuilds the oracle from the reference sources and reruns one case."""
    subprocess.run(["make", "-s", "-C", ORACLE, "ref"], check=True)
    case = "iso_v20"
    src = os.path.join(GOLDEN, case)
    for f in os.listdir(src):
        if f.endswith((".uds", ".bin", ".xml")):
            (tmp_path / f).write_bytes(open(os.path.join(src, f), "rb").read())
    info = json.load(open(os.path.join(src, "case.json")))
    subprocess.run([os.path.join(ORACLE, "_ref", "gg_ref"), case + ".xml", "d.bin", str(info["dump_every"]), "1"],
                   cwd=tmp_path, check=True, capture_output=True)
    assert (tmp_path / "d.bin").read_bytes() == gzip.open(os.path.join(src, "reference.dump.gz")).read()
