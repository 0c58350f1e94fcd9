"""The batched heterogeneous cases and the large iterative array, on the GPU.

Heterogeneous single / two-body cases (`meshgen.case_c3(seed)`: cylinders or
boxes of random size and panel count, half with water-plane lids, finite or
infinite depth): the six smallest of the 128 seeded cases and the two
smallest with two bodies (together: both depths, lids, two bodies) against
the CPU oracle (added mass, damping, excitation within 1e-6 relative Frobenius, the
plain form's bar), and the four largest (up to 5,757 panels) through the
mixed form against the fp64 form (1e-6); four cases in flight together, one
host thread per case, give the same bits as one by one.  (The seed lists
themselves are checked on the CPU.)

The 6 x 6 array (`meshgen.case_c5()`: 36 cylinders, 20,160 panels, h 40 m)
at full size, one frequency and three headings: GMRES (restart 50,
tolerance 1e-6) with H-matrix products (ACA tolerance 1e-5) against the
mixed-form LU, both with the identical body blocks (121 of the 1,296
blocks computed); the forces agree within 1e-4, the chosen form's bar.
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

RHO, G = 1025.0, 9.81
SMALL = [34, 70, 35, 78, 3, 44, 115, 0]  # the six smallest, the two smallest with two bodies
LARGE = [82, 1, 37, 99]  # the four largest (5,757 to 4,612 panels)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def c3_case(seed, with_oracle=True, **kw):
    c = meshgen.case_c3(seed)
    xyz, ncn, ncon, cnt = meshgen.combine(c["bodies"])
    lid = {}
    if c["lids"]:
        lx, ln, lc, lcnt = meshgen.combine(c["lids"])
        lid = dict(ixyz=lx, incn=ln, incon=lc, body_inelem=lcnt, irsp=1)
    xr = np.array(c["centres"])
    oc = oracle_lib.Case(xyz, ncn, ncon, cnt, xr, c["depth"], rho=RHO, g=G, **lid)
    geom = dict(xyz=xyz, ncn=ncn, ncon=ncon, xyz_p=oc.xyz_p, ds=oc.ds, pnsz=oc.pnsz, dxyz=oc.dxyz, body_nelem=cnt)
    if lid:
        geom["ixyz_p"] = oc.ixyz_p
    ctx = hams_b200.Context(geom, c["depth"], rho=RHO, g=G, irsp=1 if lid else 0, **kw)
    return c, (oc if with_oracle else None), ctx


def test_seed_lists():
    sizes = sorted(((sum(b[1].size for b in meshgen.case_c3(s)["bodies"]), s) for s in range(128)), reverse=True)
    assert [s for _, s in sizes[:4]] == LARGE
    assert [s for _, s in sorted(sizes)[:6]] == SMALL[:6]
    two = sorted((n, s) for n, s in sizes if len(meshgen.case_c3(s)["bodies"]) == 2)
    assert [s for _, s in two[:2]] == SMALL[6:]


@pytest.mark.gpu
@pytest.mark.parametrize("seed", SMALL)
def test_c3_small_cases_against_oracle(seed):
    c, oc, ctx = c3_case(seed)
    betas = np.radians(c["betas_deg"])
    for om in (c["omegas"][2], c["omegas"][12]):
        w = hams_b200.wave_properties(om, c["depth"], G)
        am, bd, ex = ctx.solve_frequency(w, betas)
        oam, obd, oex, _ = oc.solve(oc.wave(om), betas)
        assert rel(am, oam) < 1e-6 and rel(bd, obd) < 1e-6 and rel(ex, oex) < 1e-6, (seed, om)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", LARGE)
def test_c3_large_cases_mixed_against_fp64(seed):
    c, _, full = c3_case(seed, with_oracle=False)
    _, _, mixed = c3_case(seed, with_oracle=False, precision=hams_b200.PREC_MIXED)
    betas = np.radians(c["betas_deg"])
    waves = [hams_b200.wave_properties(om, c["depth"], G) for om in c["omegas"][::5]]
    r0 = full.solve_batch(waves, betas)
    r1 = mixed.solve_batch(waves, betas)
    for k in range(len(waves)):
        for x, y in zip(r1, r0):
            assert rel(x[k], y[k]) < 1e-6, (seed, k)
    full.close()
    mixed.close()


@pytest.mark.gpu
def test_c5_iterative_path_full_size():
    c = meshgen.case_c5()
    xyz, ncn, ncon, cnt = meshgen.combine(c["bodies"])
    geom = hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, np.array(c["centres"]))
    assert hams_b200.body_blocks(geom)[1] == 121
    betas = np.radians(c["betas_deg"])
    w = hams_b200.wave_properties(1.0, c["depth"], G)
    lu = hams_b200.Context(geom, c["depth"], rho=RHO, g=G, precision=hams_b200.PREC_MIXED, body_blocks=1)
    ref = lu.solve_frequency(w, betas)
    assert lu.note() == ""
    lu.close()
    gm = hams_b200.Context(geom, c["depth"], rho=RHO, g=G, solver=hams_b200.SOLVER_GMRES, gmres_restart=50,
                           gmres_maxit=500, gmres_tol=1e-6, aca_tol=1e-5, body_blocks=1)
    got = gm.solve_frequency(w, betas)
    t = gm.timings()
    assert gm.note() == "" and 0 < t["iterations"] < 500
    assert t["pairs_copied"] == (1296 - 121) * 560 * 560
    for x, y in zip(got, ref):
        assert np.all(np.isfinite(x)) and rel(x, y) < 1e-4
    gm.close()


@pytest.mark.gpu
def test_c3_cases_solved_concurrently():
    """Heterogeneous cases in flight together: one context per case, each solved by its own host
    thread (the C calls release the interpreter), gives the same bits as solving them one by one."""
    import threading

    seeds = SMALL[:4]
    cases = [c3_case(s, with_oracle=False) for s in seeds]
    runs = []
    for c, _, ctx in cases:
        waves = [hams_b200.wave_properties(om, c["depth"], G) for om in c["omegas"][::4]]
        runs.append((ctx, waves, np.radians(c["betas_deg"])))
    alone = [ctx.solve_batch(w, b) for ctx, w, b in runs]
    together = [None] * len(runs)

    def work(k):
        ctx, w, b = runs[k]
        together[k] = ctx.solve_batch(w, b)

    th = [threading.Thread(target=work, args=(k,)) for k in range(len(runs))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for a, b in zip(alone, together):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    for ctx, _, _ in runs:
        ctx.close()
