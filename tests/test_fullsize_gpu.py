"""Full-size parity of the benchmark workloads against the oracle.

The smaller parity tests (test_gpu_parity.py) use coarsened meshes; these run
the benchmark geometries at their full panel counts, one frequency at a time,
against the CPU oracle (the FP64 restatement of the reference's assembly,
with LAPACK zgetrf/zgetrs as the solve the reference calls through MKL):

  * the 800-panel truncated cylinder in infinite depth (40 x 15 side +
    40 x 5 bottom quads): the plain fp64 form within 1e-6 relative Frobenius
    in added mass, damping and excitation;
  * the 5,400-panel 3 x 3 array of cylinders in 50 m of water: the plain fp64
    form within 1e-6 and the surrogate form as the benchmark runs it
    (network far pairs over the network's whole K domain, each frequency
    judged by the series and taken back by it above the 1e-4 bar, identical
    body blocks, complex64 panel LU with FP64 refinement) within 1e-4, at the
    lowest and highest frequencies of the sweep, one in the middle and one in
    the band before the cylinders' irregular frequency;
  * a second geometry the judgement was not calibrated on: a 2 x 2 array of
    the same cylinders at 30 m spacing in 40 m of water (2,400 panels), the
    surrogate form within 1e-4 of the oracle at long, middle and short waves.

Each oracle frequency of the 3 x 3 array costs about 15 s on 16 host cores.
"""
import os
import sys

import numpy as np
import pytest
import scipy.linalg.lapack as lapack

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "hams-mrel_b200"))
import hams_b200  # noqa: E402
import meshgen  # noqa: E402
import oracle_lib  # noqa: E402
import train_surrogate  # noqa: E402

RHO, G = 1025.0, 9.81


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_solve(oc, omega, betas):
    """The oracle's assembly of the whole system, LAPACK LU and solve, the oracle's reductions."""
    w = oc.wave(omega)
    a, b, d = oc.assemble(w, betas)
    xr, xd = np.zeros_like(b), np.zeros_like(d)
    for ip in range(oc.geom.nsys):
        lu, piv, info = lapack.zgetrf(a[:, :, ip], overwrite_a=True)
        assert info == 0
        xr[:, :, ip] = lapack.zgetrs(lu, piv, b[:, :, ip])[0]
        xd[:, ip, :] = lapack.zgetrs(lu, piv, d[:, ip, :])[0]
    return oc.forces(w, betas, xr, xd)


def surrogate_form(geom, h, blocks=1):
    """The surrogate form as the benchmark runs it."""
    ctx = hams_b200.Context(geom, h, rho=RHO, g=G, precision=hams_b200.PREC_MIXED, refine_tol=1e-7, body_blocks=blocks)
    ctx.set_surrogate(train_surrogate.load(), hams_b200.SURROGATE_FAR, hams_b200.SURROGATE_K_RANGE)
    ctx.set_surrogate_tolerance(hams_b200.SURROGATE_TOL)
    return ctx


def build(case):
    xyz, ncn, ncon, cnt = meshgen.combine(case["bodies"])
    xr = np.array(case["centres"], dtype=np.float64)
    oc = oracle_lib.Case(xyz, ncn, ncon, cnt, xr, case["depth"], rho=RHO, g=G)
    oc.opts.nthread = len(os.sched_getaffinity(0))
    geom = hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, xr)
    return oc, geom


@pytest.mark.gpu
def test_c1_cylinder_full_size():
    case = meshgen.case_c1()
    oc, geom = build(case)
    assert oc.n == 800
    ctx = hams_b200.Context(geom, case["depth"], rho=RHO, g=G)
    betas = np.radians([0.0])
    for om in (0.3, 1.5, 3.0):
        got = ctx.solve_frequency(hams_b200.wave_properties(om, case["depth"], G), betas)
        ref = oracle_solve(oc, om, betas)
        for name, a, b in zip(("added mass", "damping", "excitation"), got, ref):
            assert rel(a, b) < 1e-6, f"omega {om}: {name} {rel(a, b):.3e}"
    ctx.close()


@pytest.mark.gpu
def test_c2_array_full_size_fp64_and_surrogate_form():
    case = meshgen.case_c2()
    oc, geom = build(case)
    assert oc.n == 5400
    h = case["depth"]
    betas = np.radians(case["betas_deg"])
    fp64 = hams_b200.Context(geom, h, rho=RHO, g=G)
    sg = surrogate_form(geom, h)
    oms = case["omegas"]
    for om in (oms[0], oms[len(oms) // 2], oms[31], oms[-1]):
        w = hams_b200.wave_properties(float(om), h, G)
        ref = oracle_solve(oc, float(om), betas)
        got = fp64.solve_frequency(w, betas)
        for name, a, b in zip(("added mass", "damping", "excitation"), got, ref):
            assert rel(a, b) < 1e-6, f"fp64 omega {om}: {name} {rel(a, b):.3e}"
        got = sg.solve_frequency(w, betas)
        for name, a, b in zip(("added mass", "damping", "excitation"), got, ref):
            assert rel(a, b) < 1e-4, f"surrogate form omega {om}: {name} {rel(a, b):.3e}"
    fp64.close()
    sg.close()


@pytest.mark.gpu
def test_surrogate_form_second_geometry():
    bodies, centres = [], []
    for iy in range(2):
        for ix in range(2):
            bodies.append(meshgen.cylinder(4.0, 8.0, 40, 10, 5, 30.0 * ix, 30.0 * iy))
            centres.append((30.0 * ix, 30.0 * iy, 0.0))
    case = dict(bodies=bodies, centres=centres, depth=40.0)
    oc, geom = build(case)
    assert oc.n == 2400
    betas = np.radians([0.0, 45.0, 90.0])
    sg = surrogate_form(geom, 40.0)
    used = 0
    for om in (0.2, 0.7, 1.3, 1.9, 2.3, 2.4):
        got = sg.solve_frequency(hams_b200.wave_properties(om, 40.0, G), betas)
        t = sg.timings()
        used += (not t["judge_resolved"]) and t["pairs_surrogate"] > 0
        ref = oracle_solve(oc, om, betas)
        for name, a, b in zip(("added mass", "damping", "excitation"), got, ref):
            assert rel(a, b) < 1e-4, f"omega {om}: {name} {rel(a, b):.3e} (estimate {t['judge_estimate']:.2e})"
    assert used >= 3  # the network keeps most of these frequencies
    sg.close()
