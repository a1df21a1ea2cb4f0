"""ctypes binding of the C restatement (oracle/gg_oracle.c) — test
infrastructure: the tests call it as the checker; the product never does.

``load()`` builds ``oracle/_ref/libgg_oracle.so`` with ``make -C oracle port``
when it is missing or older than its sources (gcc only, no reference tree
needed), then binds every function of ``gg_oracle.h``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libgg_oracle.so")
SOURCES = [os.path.join(HERE, "gg_oracle.c"), os.path.join(HERE, "gg_oracle.h")]

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_U = ctypes.POINTER(ctypes.c_uint)
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    stale = not os.path.exists(LIB) or any(os.path.getmtime(LIB) < os.path.getmtime(s) for s in SOURCES)
    if stale:
        subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    lib = ctypes.CDLL(LIB)
    lib.gg_or_convolve.argtypes = [ctypes.c_int, _D, _D, ctypes.c_double, ctypes.c_int]
    lib.gg_or_compare.argtypes = [_I, _D, ctypes.c_int, _I, ctypes.POINTER(_D), _U, _I, _U, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_double, ctypes.c_double, _D, _U, _I]
    lib.gg_or_contour.restype = ctypes.c_int
    lib.gg_or_contour.argtypes = [_D, _I, _U, ctypes.c_uint, _D, ctypes.c_int, _I, _U, _I, _D, _D, ctypes.c_int, _I]
    lib.gg_or_polygon_phi.argtypes = [_D, ctypes.c_int, _I, ctypes.c_int, ctypes.c_double, ctypes.c_double, _D]
    lib.gg_or_polygon_box.argtypes = [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _I]
    lib.gg_or_area.restype = ctypes.c_double
    lib.gg_or_area.argtypes = [_D, ctypes.c_int, ctypes.c_double]
    lib.gg_or_perimeter.restype = ctypes.c_double
    lib.gg_or_perimeter.argtypes = [_D, ctypes.c_int, ctypes.c_double]
    lib.gg_or_motion_regular.restype = ctypes.c_int
    lib.gg_or_motion_regular.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, _I]
    lib.gg_or_new_box.argtypes = [_I, ctypes.c_int, _I]
    lib.gg_or_redistance.argtypes = [_D, _I, _D, _I, ctypes.c_double, ctypes.c_double]
    _lib = lib
    return lib


def _box(b):
    return np.ascontiguousarray(b, np.int32)


def _p(a, t):
    return a.ctypes.data_as(t)


def convolve(phi: np.ndarray, dt: float, real_domain_size: int) -> np.ndarray:
    """Gaussian convolution of one square box (src/box.cpp:622-695)."""
    lib = load()
    phi = np.ascontiguousarray(phi, np.float64)
    n = phi.shape[0]
    assert phi.shape == (n, n)
    out = np.empty_like(phi)
    lib.gg_or_convolve(n, _p(phi, _D), _p(out, _D), dt, real_domain_size)
    return out


def compare(box, own_conv, members, prev_box, idprev, m, b, h, delta):
    """Comparison + boundary condition + set comparison of one grain.

    ``members`` lists (id, box, convolved field) in comparison-list order.
    Returns (compared field, IDLocal, unclipped new bounding box)."""
    lib = load()
    box = _box(box)
    own_conv = np.ascontiguousarray(own_conv, np.float64)
    k = len(members)
    nbox = _box([list(mb[1]) for mb in members] if k else np.zeros((0, 4))).reshape(-1)
    convs = [np.ascontiguousarray(mb[2], np.float64) for mb in members]
    ptrs = (_D * max(k, 1))(*[_p(c, _D) for c in convs])
    ids = np.ascontiguousarray([mb[0] for mb in members] if k else [0], np.uint32)
    pbox = _box(prev_box)
    idp = np.ascontiguousarray(idprev, np.uint32).reshape(-1)
    if idp.size == 0:
        idp = np.zeros(1, np.uint32)
    out = np.empty_like(own_conv)
    idl = np.empty(own_conv.shape, np.uint32)
    nb = np.zeros(4, np.int32)
    lib.gg_or_compare(_p(box, _I), _p(own_conv, _D), k, _p(nbox, _I), ptrs, _p(ids, _U), _p(pbox, _I),
                      _p(idp, _U), m, b, h, delta, _p(out, _D), _p(idl, _U), _p(nb, _I))
    return out, idl, tuple(int(v) for v in nb)


def contour(phi, box, idlocal, own):
    """Marching-squares contour with junctions projected onto it.

    Returns (points (n, 2), junctions [(type, grains, segment, lambda, x, y)])."""
    lib = load()
    phi = np.ascontiguousarray(phi, np.float64)
    idl = np.ascontiguousarray(idlocal, np.uint32)
    box = _box(box)
    cap = 8 * phi.size + 64
    jcap = 4 * phi.size + 16
    pts = np.zeros((cap, 2))
    jt = np.zeros(jcap, np.int32)
    jg = np.zeros((jcap, 4), np.uint32)
    js = np.zeros(jcap, np.int32)
    jl = np.zeros(jcap)
    jxy = np.zeros((jcap, 2))
    nj = ctypes.c_int(0)
    n = lib.gg_or_contour(_p(phi, _D), _p(box, _I), _p(idl, _U), own, _p(pts, _D), cap, _p(jt, _I), _p(jg, _U),
                          _p(js, _I), _p(jl, _D), _p(jxy, _D), jcap, ctypes.byref(nj))
    junc = [(int(jt[q]), tuple(int(v) for v in jg[q]), int(js[q]), float(jl[q]), float(jxy[q, 0]),
             float(jxy[q, 1])) for q in range(nj.value)]
    return pts[:n].copy(), junc


def area(pts, h):
    pts = np.ascontiguousarray(pts, np.float64)
    return load().gg_or_area(_p(pts, _D), len(pts), h)


def perimeter(pts, h):
    pts = np.ascontiguousarray(pts, np.float64)
    return load().gg_or_perimeter(_p(pts, _D), len(pts), h)


def motion_regular(old_contour, new_contour, old_volume, new_volume, dt):
    """(regular, flagged) of isMotionRegular (src/box.cpp:1155-1189)."""
    flagged = ctypes.c_int(0)
    r = load().gg_or_motion_regular(old_contour, new_contour, old_volume, new_volume, dt, ctypes.byref(flagged))
    return bool(r), bool(flagged.value)


def new_box(newbb, m):
    nb = _box(newbb)
    out = np.zeros(4, np.int32)
    load().gg_or_new_box(_p(nb, _I), m, _p(out, _I))
    return tuple(int(v) for v in out)


def redistance(phi_in, box_in, box_out, h, delta):
    """Four directional sweeps + clamp (src/box.cpp:1259-1399)."""
    lib = load()
    phi_in = np.ascontiguousarray(phi_in, np.float64)
    bi, bo = _box(box_in), _box(box_out)
    out = np.empty((bo[3] - bo[2], bo[1] - bo[0]))
    lib.gg_or_redistance(_p(phi_in, _D), _p(bi, _I), _p(out, _D), _p(bo, _I), h, delta)
    return out


def polygon_phi(pts, box, blowup, h, delta):
    """Signed distance to a polygon, clamped to delta (src/box.cpp:342-400)."""
    pts = np.ascontiguousarray(np.asarray(pts, np.float64)[:, :2])
    bo = _box(box)
    out = np.empty((bo[3] - bo[2], bo[1] - bo[0]))
    load().gg_or_polygon_phi(_p(pts, _D), pts.shape[0], _p(bo, _I), blowup, h, delta, _p(out, _D))
    return out


def polygon_box(pts, m, blowup, h):
    """The contour constructor's box before squaring (src/box.cpp:108-159)."""
    pts = np.ascontiguousarray(np.asarray(pts, np.float64)[:, :2])
    out = np.zeros(4, np.int32)
    load().gg_or_polygon_box(_p(pts, _D), pts.shape[0], m, blowup, h, _p(out, _I))
    return tuple(int(v) for v in out)
