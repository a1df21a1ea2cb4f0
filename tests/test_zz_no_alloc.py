"""The allocation-free box convolution (gg_convolve_box_static).

It exists for callers that cannot allocate device memory, such as a host
application that lends this library buffers from its own device memory pool.
This test calls it through the C ABI on every grain's initial distance field,
two and more calls in a row sharing the library's one static scratch array,
and checks each result against the convolution stage of a plain context
(gg_convolution): the comparison stage that follows turns the convolved
fields into the dumped compared field, so the test rebuilds that comparison
(src/box.cpp:890-1025, 838-879) from the static results and requires the
same bits (the FP64 tests' tolerance is exact agreement).
"""
import os

import numpy as np
import pytest

from gragles2d_b200 import dumpfile

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _wall_distance(i, j, b, m):
    dxmin, dymin, dxmax, dymax = -(j - b), -(i - b), j - (m - b), i - (m - b)
    dx = dxmin if abs(dxmin) < abs(dxmax) else dxmax
    dy = dymin if abs(dymin) < abs(dymax) else dymax
    if dx > 0 and dy > 0:
        return np.sqrt(float(dx) * dx + dy * dy)
    if dx < 0 and dy > 0:
        return float(dy)
    if dx > 0 and dy < 0:
        return float(dx)
    if dx < 0 and dy < 0:
        return float(max(dx, dy))
    if dx == 0:
        return float(dy) if dy > 0 else 0.0
    return float(dx) if dx > 0 else 0.0


def _compare(g, conv, boxes, lst, b, m, h, delta):
    """Comparison + boundary + set-comparison of one grain (plain arithmetic)."""
    x0, x1, y0, y1 = boxes[g]
    out = np.full((y1 - y0, x1 - x0), -1.0)
    for k in lst:
        kx0, kx1, ky0, ky1 = boxes[k]
        ox0, ox1, oy0, oy1 = max(x0, kx0), min(x1, kx1), max(y0, ky0), min(y1, ky1)
        if ox1 <= ox0 or oy1 <= oy0:
            continue
        d = conv[k][oy0 - ky0:oy1 - ky0, ox0 - kx0:ox1 - kx0]
        o = out[oy0 - y0:oy1 - y0, ox0 - x0:ox1 - x0]
        win = d > o
        o[win] = d[win]
    lo, hi = b + b, m - b - b
    if not (x0 > lo and x1 < hi and y0 > lo and y1 < hi):
        for i in range(y0, y1):
            for j in range(x0, x1):
                wall = _wall_distance(i, j, b, m) * h
                if wall > out[i - y0, j - x0]:
                    out[i - y0, j - x0] = wall
    own = conv[g]
    return np.where(np.abs(own) < 0.7 * delta, 0.5 * (own - out), own)


@pytest.mark.gpu
def test_static_box_convolution_matches_the_convolution_stage(tmp_path):
    import torch

    from gragles2d_b200 import gg

    case = "iso_v20"
    d = os.path.join(GOLDEN, case)
    ref = dumpfile.read(os.path.join(d, "reference.dump.gz"))
    h = gg.GrainHandler(gg.Settings(os.path.join(d, case + ".xml"), precision=gg.PRECISION_PLAIN))
    h.load_voxel_files()
    h.distanceInitialisation()
    h.set_neighbours({gid: g.sec for gid, g in ref.records[0].grains.items() if g.state})
    dims = h.dims()
    p0 = str(tmp_path / "init.dump")
    h.dump(p0, 0)
    init = dumpfile.read(p0).records[0]
    # the existing entry point: convolution stage, then the comparison that consumes it
    h.convolution()
    h.updateSecondOrderNeighbors()
    h.comparison_box()
    p1 = str(tmp_path / "cmp.dump")
    h.dump(p1, 0)
    after = dumpfile.read(p1).records[0]
    h.close()

    nn = dims.ngridpoints - 2 * 7
    live = [g for g, r in init.grains.items() if r.state == 1]
    assert len(live) > 10
    conv, boxes = {}, {}
    calls = 0
    for g in live:
        phi0 = init.grains[g].phi
        n = phi0.shape[0]
        assert n <= gg.STATIC_CONV_MAX_N
        src = torch.from_numpy(np.ascontiguousarray(phi0)).cuda()
        dst = torch.full_like(src, np.nan)
        torch.cuda.synchronize()
        gg.convolve_box_static(src.data_ptr(), dst.data_ptr(), n, dims.dt, nn)
        first = dst.cpu().numpy()
        dst.fill_(np.nan)
        torch.cuda.synchronize()
        gg.convolve_box_static(src.data_ptr(), dst.data_ptr(), n, dims.dt, nn)  # second call in a row
        second = dst.cpu().numpy()
        calls += 2
        assert np.array_equal(first.view(np.uint64), second.view(np.uint64)), g
        conv[g] = first
        boxes[g] = init.grains[g].box
    assert calls >= 2
    for g in live:
        got = after.grains[g]
        want = _compare(g, conv, boxes, got.cmp, 7, dims.ngridpoints, dims.h, dims.delta)
        assert np.array_equal(want.view(np.uint64), got.phi.view(np.uint64)), f"grain {g}"


@pytest.mark.gpu
def test_static_box_convolution_rejects_sizes_beyond_the_maximum():
    import torch

    from gragles2d_b200 import gg

    n = gg.STATIC_CONV_MAX_N + 1
    buf = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    with pytest.raises(gg.GGError) as e:
        gg.convolve_box_static(buf.data_ptr(), buf.data_ptr(), n, 1e-5, 100)
    assert e.value.code == 1


def _gaussian_convolution(x, dt, nn):
    """The convolution stage's transform in numpy: the unnormalised 2-D DFT
    times G(i2, j2) = exp(-sqrt(2/pi) (i2^2 + j2^2) 4 dt nn^2 / n^2 pi^2) / n^2
    (i2, j2 the frequencies folded to min(k, n - k), src/box.cpp:674-687),
    then the unnormalised inverse."""
    n = x.shape[0]
    k = np.arange(n)
    f = np.minimum(k, n - k).astype(np.float64)
    half = n // 2 + 1
    g = np.exp(-np.sqrt(2 / np.pi) * (f[:, None] ** 2 + f[None, :half] ** 2) * 4.0 * dt * nn * nn / (n * n)
               * np.pi * np.pi) / (n * n)
    return np.fft.irfft2(np.fft.rfft2(x) * g, s=(n, n)) * n * n


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3, 128])
def test_static_box_convolution_known_answer_at_the_size_limits(n):
    """Random boxes at the smallest sizes and at the maximum, where the two
    spectra fill the scratch's spectrum region exactly, against numpy's FFT
    of the same transform, two calls in a row."""
    import torch

    from gragles2d_b200 import gg

    rng = np.random.default_rng(n)
    x = rng.uniform(-1.0, 1.0, (n, n))
    dt, nn = 3.125e-6, 800
    want = _gaussian_convolution(x, dt, nn)
    src = torch.from_numpy(x).cuda()
    for _ in range(2):
        dst = torch.full_like(src, np.nan)
        torch.cuda.synchronize()
        gg.convolve_box_static(src.data_ptr(), dst.data_ptr(), n, dt, nn)
        got = dst.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)



@pytest.mark.gpu
def test_static_box_convolution_refuses_a_capturing_stream():
    """A call on a stream that is being captured into a CUDA graph returns
    GG_E_INVALID and issues nothing there: the capture around it completes,
    its graph replays, and a call after the capture succeeds."""
    import torch

    from gragles2d_b200 import gg

    gg.load_library()  # loaded before the capture starts
    n = 8
    src = torch.from_numpy(np.random.default_rng(5).uniform(-1.0, 1.0, (n, n))).cuda()
    dst = torch.zeros_like(src)
    x = torch.arange(16, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        y = x * 2.0
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        y = x * 2.0
        with pytest.raises(gg.GGError) as e:
            gg.convolve_box_static(src.data_ptr(), dst.data_ptr(), n, 3.125e-6, 800,
                                   stream=torch.cuda.current_stream().cuda_stream)
        assert e.value.code == 1
    x.add_(1.0)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, (x * 2.0))
    assert torch.count_nonzero(dst).item() == 0
    gg.convolve_box_static(src.data_ptr(), dst.data_ptr(), n, 3.125e-6, 800)
    torch.cuda.synchronize()
    np.testing.assert_allclose(dst.cpu().numpy(), _gaussian_convolution(src.cpu().numpy(), 3.125e-6, 800),
                               rtol=0, atol=1e-12)
