"""GMRES solver (HAMS_SOLVER_GMRES) through the C ABI.

With dense products: against the oracle's direct solve at a tight tolerance
(1e-8 relative Frobenius on added mass, damping, excitation; the lid case
1e-5 as its normal equations square the condition number), and at the
reference's defaults (restart 25, tolerance 1e-4, 100 steps) against the
GMRES restatement of oracle/gmres_ref.py on the same assembled systems: the
iteration count equals the restatement's largest per-column count (+-1, the
last step can fall either side of the tolerance).

With H-matrix products (the reference's choice without lids): at the
reference's defaults the forces stay within the reference's own
GMRES-vs-LU test bounds (test_integration_gmres.f90:48-101: 1e-3 added mass,
5e-2 damping); with ACA at 1e-8 and GMRES at 1e-10 within 1e-5 of the direct
solve, which bounds the H-matrix's own error.
"""
import os
import sys

import numpy as np
import pytest

import oracle_lib

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "hams-mrel_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import gmres_ref  # noqa: E402
import hams_b200  # noqa: E402
import meshgen  # noqa: E402

GOLDEN = os.path.join(HERE, "golden")
pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def array_case():
    bodies, centres = [], []
    for iy in range(2):
        for ix in range(2):
            bodies.append(meshgen.cylinder(3.0, 6.0, 16, 4, 2, 15.0 * ix, 15.0 * iy))
            centres.append((15.0 * ix, 15.0 * iy, 0.0))
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    oc = oracle_lib.Case(xyz, ncn, ncon, cnt, np.array(centres), 40.0, rho=1025.0, g=9.81)
    geom = hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, np.array(centres))
    return oc, geom, cnt


def single_case():
    body = meshgen.cylinder(5.0, 10.0, 16, 6, 3)
    xyz, ncn, ncon, cnt = meshgen.combine([body])
    oc = oracle_lib.Case(xyz, ncn, ncon, cnt, np.array([(0.0, 0.0, 0.0)]), 30.0, rho=1025.0, g=9.81)
    geom = hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, np.array([(0.0, 0.0, 0.0)]))
    return oc, geom, cnt


CASES = {"array": (array_case, 40.0), "single": (single_case, 30.0)}


@pytest.mark.parametrize("name", ["array", "single"])
@pytest.mark.parametrize("precision", [hams_b200.PREC_FP64, hams_b200.PREC_MIXED])
def test_gmres_tight_matches_direct_solve(name, precision):
    make, h = CASES[name]
    oc, geom, _ = make()
    ctx = hams_b200.Context(geom, h, rho=1025.0, g=9.81, precision=precision, solver=hams_b200.SOLVER_GMRES,
                            gmres_restart=40, gmres_maxit=400, gmres_tol=1e-11, gmres_dense=1)
    betas = np.radians([0.0, 60.0])
    for omega in (0.4, 1.6):
        am, bd, ex = ctx.solve_frequency(hams_b200.wave_properties(omega, h, 9.81), betas)
        assert ctx.note() == "", ctx.note()
        assert 0 < ctx.timings()["iterations"] < 400
        oam, obd, oex, _ = oc.solve(oc.wave(omega), betas)
        assert rel(am, oam) < 1e-8 and rel(bd, obd) < 1e-8 and rel(ex, oex) < 1e-8
    ctx.close()


@pytest.mark.parametrize("name", ["array", "single"])
def test_gmres_defaults_follow_the_restatement(name):
    make, h = CASES[name]
    oc, geom, cnt = make()
    ctx = hams_b200.Context(geom, h, rho=1025.0, g=9.81, solver=hams_b200.SOLVER_GMRES, gmres_dense=1)
    betas = np.radians([0.0, 60.0])
    for omega in (0.4, 1.6):
        w = hams_b200.wave_properties(omega, h, 9.81)
        am, bd, ex = ctx.solve_frequency(w, betas)
        its = ctx.timings()["iterations"]
        a, b, d = ctx.assemble(w, betas)
        _, ref_its = gmres_ref.solve(a, np.concatenate([b, d], axis=1), list(cnt))
        assert abs(its - max(ref_its)) <= 1, (its, ref_its)
        oam, obd, oex, _ = oc.solve(oc.wave(omega), betas)
        assert rel(am, oam) < 1e-3 and rel(bd, obd) < 5e-2 and rel(ex, oex) < 1e-3
    ctx.close()


@pytest.mark.parametrize("name", ["array", "single"])
def test_gmres_hmatrix(name):
    make, h = CASES[name]
    oc, geom, _ = make()
    betas = np.radians([0.0, 60.0])
    ref = {om: oc.solve(oc.wave(om), betas) for om in (0.4, 1.6)}
    for kw, bound in ((dict(), (1e-3, 5e-2, 1e-3)),
                      (dict(aca_tol=1e-8, gmres_tol=1e-10, gmres_restart=40, gmres_maxit=400), (1e-5,) * 3)):
        ctx = hams_b200.Context(geom, h, rho=1025.0, g=9.81, solver=hams_b200.SOLVER_GMRES, **kw)
        for om in (0.4, 1.6):
            am, bd, ex = ctx.solve_frequency(hams_b200.wave_properties(om, h, 9.81), betas)
            assert ctx.note() == "", ctx.note()
            oam, obd, oex, _ = ref[om]
            assert rel(am, oam) < bound[0] and rel(bd, obd) < bound[1] and rel(ex, oex) < bound[2], \
                (kw, om, rel(am, oam), rel(bd, obd), rel(ex, oex))
        ctx.close()


def test_gmres_missed_tolerance_keeps_iterate_and_notes():
    oc, geom, _ = array_case()
    ctx = hams_b200.Context(geom, 40.0, rho=1025.0, g=9.81, solver=hams_b200.SOLVER_GMRES, gmres_restart=3,
                            gmres_maxit=3, gmres_tol=1e-14)
    am, bd, ex = ctx.solve_frequency(hams_b200.wave_properties(1.0, 40.0, 9.81), np.radians([0.0]))
    assert "GMRES" in ctx.note() and ctx.timings()["iterations"] == 3
    assert np.isfinite(am).all() and np.isfinite(ex).all()
    oam, _, _, _ = oc.solve(oc.wave(1.0), np.radians([0.0]))
    assert rel(am, oam) < 0.5  # a three-step block-preconditioned iterate, not garbage
    ctx.close()


def test_gmres_lid_normal_equations():
    d = oracle_lib.load_deck(os.path.join(GOLDEN, "example5", "input"))
    ctx = hams_b200.Context(d, d["h"], isol=d["isol"], irsp=d["irsp"], solver=hams_b200.SOLVER_GMRES,
                            gmres_restart=60, gmres_maxit=600, gmres_tol=1e-12)
    c = oracle_lib.Case(d["xyz"], d["ncn"], d["ncon"], d["body_nelem"], d["xr"], d["h"], isol=d["isol"],
                        irsp=d["irsp"], prepare=False, ixyz=d.get("ixyz"), incn=d.get("incn"),
                        incon=d.get("incon"), body_inelem=d.get("body_inelem"))
    for k in ("xyz_p", "ds", "pnsz", "dxyz"):
        getattr(c, k)[:] = d[k]
    for k in ("ixyz_p", "ids", "ipnsz", "idxyz"):
        getattr(c, k)[:] = d[k]
    betas = np.radians(d["wvhd"][:1])
    for omega in d["wvnb"][::4][:2]:
        w = hams_b200.wave_properties(omega, d["h"], 9.80665)
        am, bd, ex = ctx.solve_frequency(w, betas)
        oam, obd, oex, _ = c.solve(c.wave(omega), betas)
        assert rel(am, oam) < 1e-5 and rel(bd, obd) < 1e-5 and rel(ex, oex) < 1e-5
    ctx.close()
