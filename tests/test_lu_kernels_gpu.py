"""The mixed form's own tensor-core kernels: the tcgen05 TF32 GEMM of the
block LU and the block triangular solves, through the C ABI.

GEMM: against the product of the inputs rounded to TF32 the way the tensor
cores read them, computed in FP64 (relative Frobenius 1e-5: only the FP32
accumulation differs), and against the unrounded FP64 product within the
TF32 bound (3e-3); ragged shapes (M, N, K not multiples of the tiles),
alpha / beta, row- and column-major results; the three tile variants of the
autotuner give the same bits.  LU: solves of odd order
and of several 256-column panels, mixed form with the own GEMM and with
cuBLAS's FP32 emulation, against the fp64 form (1e-7), with the block LU
actually used (no fallback to the library LU) and few refinement sweeps.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "hams-mrel_b200"))
import hams_b200  # noqa: E402
import meshgen  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def tf32(x, mode):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    if mode == "round":  # to nearest, ties away from zero in magnitude
        u = u + 0x1000
    return (u & 0xFFFFE000).astype(np.uint32).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("m,n,k,alpha,beta,rowmajor", [
    (128, 128, 32, 1.0, 0.0, False),
    (300, 77, 45, -1.0, 1.0, False),
    (1000, 700, 512, -1.0, 1.0, False),
    (250, 128, 128, 1.0, 0.0, True),
    (129, 260, 96, 0.5, -2.0, True),
])
def test_gemm_tf32(m, n, k, alpha, beta, rowmajor):
    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((k, n)).astype(np.float32)
    c = rng.standard_normal((m, n)).astype(np.float32)
    got = hams_b200.diag_gemm_tf32(a, b, c, alpha, beta, rowmajor).astype(np.float64)
    exact = alpha * (a.astype(np.float64) @ b.astype(np.float64)) + beta * c.astype(np.float64)
    assert rel(got, exact) < 3e-3
    emul = min(rel(got, alpha * (tf32(a, mode) @ tf32(b, mode)) + beta * c.astype(np.float64))
               for mode in ("trunc", "round"))
    assert emul < 1e-5, emul
    # the three tile variants the autotuner chooses from sum over K in the same order: the same bits
    for v in range(3):
        assert np.array_equal(hams_b200.diag_gemm_tf32(a, b, c, alpha, beta, rowmajor, variant=v).astype(np.float64),
                              got), v


def _array(n_theta, n_z, n_r, nx, ny, spacing):
    bodies, centres = [], []
    for iy in range(ny):
        for ix in range(nx):
            bodies.append(meshgen.cylinder(3.0, 6.0, n_theta, n_z, n_r, spacing * ix, spacing * iy))
            centres.append((spacing * ix, spacing * iy, 0.0))
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    return hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, np.array(centres)), int(ncn.size)


@pytest.mark.parametrize("lu_kind", [hams_b200.LU_BLOCK_TF32, hams_b200.LU_BLOCK_EMU])
def test_block_lu_odd_order_several_panels(lu_kind):
    geom, n = _array(13, 8, 5, 5, 1, 14.0)  # 5 x 169 = 845 panels: odd, four 256-column panels, a ragged block
    assert n == 845
    betas = np.radians([0.0, 60.0])
    ref = hams_b200.Context(geom, 30.0, rho=1025.0, g=9.81)
    mix = hams_b200.Context(geom, 30.0, rho=1025.0, g=9.81, precision=hams_b200.PREC_MIXED, lu_kind=lu_kind)
    for om in (0.6, 1.7):
        w = hams_b200.wave_properties(om, 30.0, 9.81)
        r = ref.solve_frequency(w, betas)
        got = mix.solve_frequency(w, betas)
        t = mix.timings()
        assert t["lu_used"] in (hams_b200.LU_BLOCK_TF32, hams_b200.LU_BLOCK_EMU), mix.note()
        assert t["refine_sweeps"] <= 8
        for a, b in zip(got, r):
            assert rel(a, b) < 1e-7
    ref.close()
    mix.close()


def test_block_lu_recorded_graphs_give_the_same_bits():
    """opts.lu_graph: the block LU's factorisation and triangular solves recorded as CUDA graphs
    (once per lane and right-hand-side count) and replayed give the bits of the direct launches,
    one frequency at a time and in a batch of eight lanes, on the odd order with a ragged block."""
    geom, n = _array(13, 8, 5, 5, 1, 14.0)
    betas = np.radians([0.0, 60.0])
    direct = hams_b200.Context(geom, 30.0, rho=1025.0, g=9.81, precision=hams_b200.PREC_MIXED)
    graph = hams_b200.Context(geom, 30.0, rho=1025.0, g=9.81, precision=hams_b200.PREC_MIXED, lu_graph=1)
    for om in (0.6, 1.7, 0.6):
        w = hams_b200.wave_properties(om, 30.0, 9.81)
        a = direct.solve_frequency(w, betas)
        b = graph.solve_frequency(w, betas)
        assert "not recorded" not in graph.note(), graph.note()
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    ws = [hams_b200.wave_properties(om, 30.0, 9.81) for om in np.linspace(0.3, 2.2, 10)]
    for x, y in zip(direct.solve_batch(ws, betas), graph.solve_batch(ws, betas)):
        assert np.array_equal(x, y)
    assert "not recorded" not in graph.note(), graph.note()
    direct.close()
    graph.close()
