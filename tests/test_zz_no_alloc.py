"""hams_eval_green_static (staging in a fixed device reservation, no device
allocation) against hams_eval_green, through the C ABI.

Tolerance: both entry points launch the same kernel on the same inputs, so
the results must agree to 1e-14 relative (they are expected bit-identical).
This file is collected last so the reservation is also exercised after the
other GPU tests have used the device.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "hams-mrel_b200"))
import hams_b200  # noqa: E402
import meshgen  # noqa: E402

pytestmark = pytest.mark.gpu

MAX_POINTS = 4096  # HAMS_EVAL_STATIC_MAX_POINTS of include/hams_gpu.h
TOL = 1e-14


def _lib():
    lib = hams_b200.load_library()
    P = ctypes.POINTER(ctypes.c_double)
    lib.hams_eval_green_static.argtypes = [ctypes.c_void_p, ctypes.POINTER(hams_b200.HamsWave), ctypes.c_int32, P,
                                           ctypes.POINTER(ctypes.c_int32), P]
    lib.hams_eval_green_static.restype = ctypes.c_int
    lib.hams_last_error.restype = ctypes.c_char_p
    return lib


def eval_static(ctx, wave, pts, flag):
    lib = _lib()
    pts = np.asfortranarray(pts, dtype=np.float64)
    flag = np.ascontiguousarray(flag, dtype=np.int32)
    out = np.zeros((pts.shape[0], 4), dtype=np.complex128, order="F")
    rc = lib.hams_eval_green_static(ctx._h, ctypes.byref(wave), pts.shape[0],
                                    pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                    flag.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return rc, out, lib.hams_last_error().decode()


def context(depth):
    bodies = [meshgen.cylinder(4.0, 8.0, 12, 3, 2, 0.0, 0.0), meshgen.cylinder(4.0, 8.0, 12, 3, 2, 20.0, 0.0)]
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    geom = hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, [[0.0, 0.0, 0.0], [20.0, 0.0, 0.0]])
    return hams_b200.Context(geom, depth, rho=1025.0, g=9.81)


def points(n, depth, seed):
    """Source/field pairs spread over all finite-depth branches (R/h from 1e-4 to 2)."""
    rng = np.random.default_rng(seed)
    h = depth if depth > 0 else 50.0
    r = h * 10.0 ** rng.uniform(-4.0, 0.3, n)
    th = rng.uniform(0.0, 2.0 * np.pi, n)
    zq = -h * rng.uniform(0.01, 0.9, n)
    zp = -h * rng.uniform(0.01, 0.9, n)
    pts = np.zeros((n, 6))
    pts[:, 0], pts[:, 1], pts[:, 2] = r * np.cos(th), r * np.sin(th), zq
    pts[:, 5] = zp
    return pts, (rng.random(n) < 0.5).astype(np.int32)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("depth", [30.0, -1.0])
def test_static_matches_allocating_entry_twice(depth):
    ctx = context(depth)
    w = hams_b200.wave_properties(0.9, depth, 9.81)
    for call, n in enumerate((777, MAX_POINTS)):  # two calls in a row, the second at the limit
        pts, flag = points(n, depth, seed=call)
        ref = ctx.eval_green(w, pts, flag)
        rc, got, msg = eval_static(ctx, w, pts, flag)
        assert rc == 0, msg
        assert np.all(np.isfinite(got))
        assert rel(got, ref) <= TOL
    ctx.close()


def test_static_rejects_more_points_than_reserved():
    ctx = context(30.0)
    w = hams_b200.wave_properties(0.9, 30.0, 9.81)
    pts, flag = points(MAX_POINTS + 1, 30.0, seed=5)
    rc, _, msg = eval_static(ctx, w, pts, flag)
    assert rc == -1  # HAMS_ERR_ARG
    assert "static reservation" in msg
    # the context and the reservation stay usable after the rejection
    pts, flag = points(64, 30.0, seed=6)
    rc, got, msg = eval_static(ctx, w, pts, flag)
    assert rc == 0, msg
    assert rel(got, ctx.eval_green(w, pts, flag)) <= TOL
    ctx.close()


def test_static_allocates_no_device_memory():
    """The property the entry point exists for: after a first call on the device (which looks the
    reservation up), further calls leave the device's free memory exactly as it was."""
    import torch

    ctx = context(30.0)
    w = hams_b200.wave_properties(0.9, 30.0, 9.81)
    pts, flag = points(MAX_POINTS, 30.0, seed=7)
    rc, first, msg = eval_static(ctx, w, pts, flag)
    assert rc == 0, msg
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for k in range(5):
        rc, got, msg = eval_static(ctx, w, pts, flag)
        assert rc == 0, msg
        assert np.array_equal(got, first)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    ctx.close()
