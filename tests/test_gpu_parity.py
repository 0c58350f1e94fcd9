"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances (relative Frobenius norms unless stated):
  Green functions, single pairs           1e-8 of max(1, |G|)
  assembled A, B (FP64)                   1e-10
  added mass / damping / excitation, FP64 1e-7   (the bar for the plain form is 1e-6)
  same, mixed (complex64 LU + FP64 IR)    1e-6   (bar for the chosen form: 1e-4)
The device and host math libraries differ in the last bit of sin/cos/exp/log;
the Wynn-epsilon extrapolation of the EIGENE/PIDCOCK series (1/(S(i+1)-S(i))
of nearly equal partial sums) amplifies that to ~1e-9 in single Green values.
"""
import os
import sys

import numpy as np
import pytest

import oracle_lib

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "hams-mrel_b200"))
import hams_b200  # noqa: E402
import meshgen  # noqa: E402

GOLDEN = os.path.join(HERE, "golden")
pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def deck_context(deck, precision=hams_b200.PREC_FP64, **kw):
    d = oracle_lib.load_deck(os.path.join(GOLDEN, deck, "input"))
    ctx = hams_b200.Context(d, d["h"], isol=d["isol"], irsp=d["irsp"], precision=precision, **kw)
    return d, ctx


def oracle_case_from_deck(d):
    c = oracle_lib.Case(d["xyz"], d["ncn"], d["ncon"], d["body_nelem"], d["xr"], d["h"], isol=d["isol"],
                        irsp=d["irsp"], prepare=False,
                        ixyz=d.get("ixyz"), incn=d.get("incn"), incon=d.get("incon"), body_inelem=d.get("body_inelem"))
    for k in ("xyz_p", "ds", "pnsz", "dxyz"):
        getattr(c, k)[:] = d[k]
    if d["inelem"] > 0:
        for k in ("ixyz_p", "ids", "ipnsz", "idxyz"):
            getattr(c, k)[:] = d[k]
    return c


def synthetic(case, precision=hams_b200.PREC_FP64, rho=1025.0, g=9.81):
    xyz, ncn, ncon, cnt = meshgen.combine(case["bodies"])
    oc = oracle_lib.Case(xyz, ncn, ncon, cnt, np.array(case["centres"]), case["depth"], rho=rho, g=g)
    geom = dict(xyz=xyz, ncn=ncn, ncon=ncon, xyz_p=oc.xyz_p, ds=oc.ds, pnsz=oc.pnsz, dxyz=oc.dxyz, body_nelem=cnt)
    ctx = hams_b200.Context(geom, case["depth"], rho=rho, g=g, precision=precision)
    return oc, ctx


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("omega,h", [(0.05, 70.0), (0.8, 50.0), (2.5, 50.0), (1.2, 14.5)])
def test_fingreen_pairs_all_branches(omega, h):
    rng = np.random.default_rng(7)
    _, ctx = synthetic(dict(bodies=[meshgen.cylinder(4.0, 8.0, 8, 2, 2)], centres=[(0.0, 0.0, 0.0)], depth=h))
    w = hams_b200.wave_properties(omega, h, 9.80665)
    ow = oracle_lib.OrcWave()
    oracle_lib.load().orc_wave_props(3, omega, h, 9.80665, 0, oracle_lib.ctypes.byref(ow))
    # horizontal distances spread over every branch of FINGREEN3D_R, including R = 0
    rr = np.concatenate([[0.0, 0.0], h * np.array([1e-4, 4.9e-4, 5.1e-4, 0.01, 0.049, 0.051, 0.2, 0.49, 0.51, 1.5]),
                         h * 10 ** rng.uniform(-3.5, 0.5, 40)])
    ang = rng.uniform(0, 2 * np.pi, rr.size)
    zq = -rng.uniform(0.05, 0.6 * h, rr.size)
    zp = -rng.uniform(0.05, 0.6 * h, rr.size)
    xp, yp = rng.uniform(-5, 5, rr.size), rng.uniform(-5, 5, rr.size)
    pts = np.stack([xp + rr * np.cos(ang), yp + rr * np.sin(ang), zq, xp, yp, zp], axis=1)
    flag = (rng.random(rr.size) < 0.5).astype(np.int32)
    got = ctx.eval_green(w, pts, flag)
    for k in range(rr.size):
        ref = oracle_lib.fingreen(pts[k, 0], pts[k, 3], pts[k, 1], pts[k, 4], pts[k, 2], pts[k, 5], ow.v,
                                  np.array(ow.wvn), h, int(flag[k]))
        err = np.abs(got[k] - ref).max() / max(1.0, np.abs(ref).max())
        assert err < 1e-8, (k, rr[k] / h, got[k], ref)


@pytest.mark.parametrize("omega", [0.1, 0.7, 1.5, 3.0])
def test_infgreen_pairs(omega):
    rng = np.random.default_rng(3)
    case = meshgen.case_c1()
    _, ctx = synthetic(dict(case, bodies=[meshgen.cylinder(5.0, 10.0, 8, 3, 2)]))
    w = hams_b200.wave_properties(omega, -1.0, 9.81)
    n = 64
    rr = np.concatenate([[0.0], 10 ** rng.uniform(-3, 2, n - 1)])
    pts = np.stack([rr, np.zeros(n), -rng.uniform(0.01, 20, n), np.zeros(n), np.zeros(n), -rng.uniform(0.01, 20, n)],
                   axis=1)
    flag = (rng.random(n) < 0.5).astype(np.int32)
    got = ctx.eval_green(w, pts, flag)
    for k in range(n):
        ref = oracle_lib.infgreen(pts[k, 0], pts[k, 3], pts[k, 1], pts[k, 4], pts[k, 2], pts[k, 5], w.v, int(flag[k]))
        assert np.abs(got[k] - ref).max() < 1e-10 * max(1.0, np.abs(ref).max()), (k, got[k], ref)


def test_assembly_config1():
    d, ctx = deck_context("config1")
    oc = oracle_case_from_deck(d)
    betas = np.radians(d["wvhd"])
    for omega in d["wvnb"]:
        w = hams_b200.wave_properties(omega, d["h"], 9.80665)
        a, b, dd = ctx.assemble(w, betas)
        oa, ob, od = oc.assemble(oc.wave(omega), betas)
        assert rel(a, oa[:, :, 0]) < 1e-10
        assert rel(b, ob[:, :, 0]) < 1e-10
        assert rel(dd, od[:, 0, :]) < 1e-10


@pytest.mark.parametrize("deck,nfreq", [("config1", 3), ("example2", 1), ("example5", 2)])
def test_solve_matches_oracle(deck, nfreq):
    d, ctx = deck_context(deck)
    oc = oracle_case_from_deck(d)
    betas = np.radians(d["wvhd"])
    for kk in range(nfreq):
        w = hams_b200.wave_properties(d["wvnb"][kk], d["h"], 9.80665, inft=d["inft"])
        ow = oracle_lib.OrcWave()
        oracle_lib.load().orc_wave_props(d["inft"], d["wvnb"][kk], d["h"], 9.80665, 0, oracle_lib.ctypes.byref(ow))
        am, bd, ex = ctx.solve_frequency(w, betas)
        oam, obd, oex, info = oc.solve(ow, betas)
        assert info == 0
        assert rel(am, oam) < 1e-7, rel(am, oam)
        assert rel(bd, obd) < 1e-7, rel(bd, obd)
        assert rel(ex, oex) < 1e-7, rel(ex, oex)


@pytest.mark.parametrize("lu_kind", [hams_b200.LU_BLOCK_EMU, hams_b200.LU_BLOCK_TF32, hams_b200.LU_LIBRARY])
def test_mixed_precision_config1(lu_kind):
    d, ctx = deck_context("config1", precision=hams_b200.PREC_MIXED, lu_kind=lu_kind)
    oc = oracle_case_from_deck(d)
    betas = np.radians(d["wvhd"])
    for omega in d["wvnb"]:
        am, bd, ex = ctx.solve_frequency(hams_b200.wave_properties(omega, d["h"], 9.80665), betas)
        used = ctx.timings()["lu_used"]
        # no fallback to the library LU (the emulated GEMM runs as TF32 under a cuBLAS older than 12.9)
        assert used == lu_kind or (lu_kind == hams_b200.LU_BLOCK_EMU and used == hams_b200.LU_BLOCK_TF32
                                   and "emulation" in ctx.note()), ctx.note()
        oam, obd, oex, _ = oc.solve(oc.wave(omega), betas)
        assert rel(am, oam) < 1e-6 and rel(bd, obd) < 1e-6 and rel(ex, oex) < 1e-6


@pytest.mark.parametrize("lu_kind", [hams_b200.LU_BLOCK_EMU, hams_b200.LU_BLOCK_TF32])
def test_mixed_block_lu_array(lu_kind):
    """2x2 cylinder array (4 x 96 panels, six 64-row blocks) in 40 m: the block LU with
    refinement against the FP64 oracle, and the refinement stays short."""
    bodies, centres = [], []
    for iy in range(2):
        for ix in range(2):
            bodies.append(meshgen.cylinder(3.0, 6.0, 16, 4, 2, 15.0 * ix, 15.0 * iy))
            centres.append((15.0 * ix, 15.0 * iy, 0.0))
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    oc = oracle_lib.Case(xyz, ncn, ncon, cnt, np.array(centres), 40.0, rho=1025.0, g=9.81)
    geom = hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, np.array(centres))
    ctx = hams_b200.Context(geom, 40.0, rho=1025.0, g=9.81, precision=hams_b200.PREC_MIXED, lu_kind=lu_kind)
    betas = np.radians([0.0, 60.0])
    for omega in (0.4, 1.6):
        am, bd, ex = ctx.solve_frequency(hams_b200.wave_properties(omega, 40.0, 9.81), betas)
        t = ctx.timings()
        used = t["lu_used"]
        assert used == lu_kind or (lu_kind == hams_b200.LU_BLOCK_EMU and used == hams_b200.LU_BLOCK_TF32
                                   and "emulation" in ctx.note()), ctx.note()
        assert t["refine_sweeps"] <= (4 if used == hams_b200.LU_BLOCK_EMU else 12)
        oam, obd, oex, _ = oc.solve(oc.wave(omega), betas)
        assert rel(am, oam) < 1e-7 and rel(bd, obd) < 1e-7 and rel(ex, oex) < 1e-7
    ctx.close()


@pytest.mark.parametrize("omega", [0.1, 1.0, 3.0])
def test_infinite_depth_cylinder(omega):
    case = dict(meshgen.case_c1(), bodies=[meshgen.cylinder(5.0, 10.0, 16, 6, 3)])
    oc, ctx = synthetic(case)
    betas = np.radians([0.0, 45.0])
    am, bd, ex = ctx.solve_frequency(hams_b200.wave_properties(omega, -1.0, 9.81), betas)
    oam, obd, oex, _ = oc.solve(oc.wave(omega), betas)
    assert rel(am, oam) < 1e-7 and rel(bd, obd) < 1e-7 and rel(ex, oex) < 1e-7


@pytest.mark.parametrize("kk", [1, 2])
def test_zero_and_infinite_frequency_limits(kk):
    d, ctx = deck_context("config1")
    oc = oracle_case_from_deck(d)
    w = hams_b200.wave_properties(1.0, d["h"], 9.80665, sybo_kk=kk)
    ow = oracle_lib.OrcWave()
    oracle_lib.load().orc_wave_props(3, 1.0, d["h"], 9.80665, kk, oracle_lib.ctypes.byref(ow))
    am, bd, ex = ctx.solve_frequency(w, np.radians([0.0]))
    oam, obd, oex, _ = oc.solve(ow, np.radians([0.0]))
    assert rel(am, oam) < 1e-7


def test_batch_equals_single_calls():
    d, ctx = deck_context("config1")
    betas = np.radians(d["wvhd"])
    waves = [hams_b200.wave_properties(w, d["h"], 9.80665) for w in d["wvnb"]]
    am, bd, ex = ctx.solve_batch(waves, betas)
    for k, w in enumerate(waves):
        a1, b1, e1 = ctx.solve_frequency(w, betas)
        assert np.array_equal(am[k], a1) and np.array_equal(bd[k], b1) and np.array_equal(ex[k], e1)


def test_results_are_deterministic():
    d, ctx = deck_context("config1")
    w = hams_b200.wave_properties(0.06, d["h"], 9.80665)
    r1 = ctx.solve_frequency(w, np.radians(d["wvhd"]))
    r2 = ctx.solve_frequency(w, np.radians(d["wvhd"]))
    for a, b in zip(r1, r2):
        assert np.array_equal(a, b)


def test_array_of_cylinders_finite_depth():
    """A 2 x 2 array with the c2 cylinder geometry, coarsened, against the oracle."""
    bodies, centres = [], []
    for iy in range(2):
        for ix in range(2):
            bodies.append(meshgen.cylinder(4.0, 8.0, 16, 4, 2, 20.0 * ix, 20.0 * iy))
            centres.append((20.0 * ix, 20.0 * iy, 0.0))
    case = dict(bodies=bodies, centres=centres, depth=50.0)
    oc, ctx = synthetic(case)
    betas = np.radians([0.0, 30.0, 60.0, 90.0])
    for omega in (0.2, 1.1, 2.5):
        am, bd, ex = ctx.solve_frequency(hams_b200.wave_properties(omega, 50.0, 9.81), betas)
        oam, obd, oex, _ = oc.solve(oc.wave(omega), betas)
        assert rel(am, oam) < 1e-7 and rel(bd, obd) < 1e-7 and rel(ex, oex) < 1e-7


def test_field_points_on_the_hull_return_the_panel_potentials():
    """At a hull panel's centre (on the body: divided by 2 pi) the field-point potential is the
    boundary integral equation of that panel's row, so it must equal the solved panel potential:
    radiation columns directly, diffraction columns once the incident potential (the last columns)
    is taken off.  In the fluid (4 pi) the result differs."""
    d, ctx = deck_context("config1")
    betas = np.radians(d["wvhd"])
    rows = np.array([0, 117, 300, 555, d["xyz_p"].shape[0] - 1])
    ctx.set_field_points(d["xyz_p"][rows])
    w = hams_b200.wave_properties(d["wvnb"][1], d["h"], 9.80665)
    ctx.solve_frequency(w, betas)
    pot = ctx.field_potentials(len(betas))
    a, b, dd = ctx.assemble(w, betas)
    x = np.linalg.solve(a, np.concatenate([b, dd], axis=1))
    nd = 6 * d["body_nelem"].size
    nb = len(betas)
    assert rel(pot[:, :nd], x[rows, :nd]) < 1e-9
    assert rel(pot[:, nd:nd + nb] - pot[:, nd + nb:], x[rows, nd:]) < 1e-9
    lifted = d["xyz_p"][rows] + 0.5 * d["dxyz"][rows, :3]  # half a metre off the hull along its normal
    ctx.set_field_points(lifted)
    ctx.solve_frequency(w, betas)
    assert rel(ctx.field_potentials(len(betas))[:, :nd], x[rows, :nd]) > 1e-3
