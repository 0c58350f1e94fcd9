"""Edge cases of the input the reference accepts, on the GPU against the oracle.

- triangular panels (NCN = 3: SGLINTBD_TRI, SingularIntgr.f90:44-200), alone
  and mixed with quadrilaterals in one body;
- no wave headings (radiation only: NBETA = 0, the diffraction solve and
  EFORCE skipped), single and batched;
- bodies of different panel counts in one deck.
Added mass, damping and excitation within 1e-7 relative Frobenius of the
oracle (the plain form's parity bound of tests/test_gpu_parity.py).
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


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def triangulate(mesh, every=1):
    """Split every `every`-th quadrilateral [a, b, c, d] into [a, b, c] and [a, c, d] (same
    winding); a quad with a repeated node (the bottom's centre ring) keeps one triangle."""
    nodes, ncn, ncon = mesh
    out_n, out_c = [], []
    for k, (q, m) in enumerate(zip(ncon, ncn)):
        if m == 4 and k % every == 0:
            a, b, c, d = q
            for tri in ([a, b, c], [a, c, d]):
                if len(set(tri)) == 3:
                    out_n.append(3)
                    out_c.append(tri + [0])
        else:
            out_n.append(m)
            out_c.append(list(q))
    return nodes, np.array(out_n, dtype=np.int32), np.array(out_c, dtype=np.int32)


def contexts(bodies, centres, depth):
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    xr = np.array(centres, dtype=np.float64)
    oc = oracle_lib.Case(xyz, ncn, ncon, cnt, xr, depth, rho=RHO, g=G)
    geom = dict(xyz=xyz, ncn=ncn, ncon=ncon, xyz_p=oc.xyz_p, ds=oc.ds, pnsz=oc.pnsz, dxyz=oc.dxyz, body_nelem=cnt)
    return oc, hams_b200.Context(geom, depth, rho=RHO, g=G)


def test_triangulation_keeps_the_surface():
    nodes, ncn, ncon = meshgen.cylinder(4.0, 6.0, 12, 3, 2)
    t = triangulate((nodes, ncn, ncon))
    assert set(t[1]) == {3} and t[1].size == 2 * 12 * 3 + 2 * 12 * 2 - 12
    # the triangles of the side and bottom add up to the quads they split (planar quads)
    xyz, n2, c2, cnt = meshgen.combine([t])
    g = hams_b200.prepare_geometry(xyz, n2, c2, cnt, np.zeros((1, 3)))
    g4 = hams_b200.prepare_geometry(*meshgen.combine([(nodes, ncn, ncon)]), np.zeros((1, 3)))
    assert abs(g["ds"].sum() - g4["ds"].sum()) < 1e-9 * g4["ds"].sum() and np.all(g["ds"] > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("every,depth", [(1, 40.0), (1, -1.0), (3, 40.0)])
def test_triangular_panels(every, depth):
    bodies = [triangulate(meshgen.cylinder(4.0, 6.0, 12, 3, 2), every),
              triangulate(meshgen.box(8.0, 6.0, 5.0, 4, 3, 3, 25.0, 0.0), every)]
    oc, ctx = contexts(bodies, [(0.0, 0.0, 0.0), (25.0, 0.0, 0.0)], depth)
    betas = np.radians([0.0, 60.0])
    for om in (0.5, 1.4):
        got = ctx.solve_frequency(hams_b200.wave_properties(om, depth, G), betas)
        ref = oc.solve(oc.wave(om), betas)
        for x, y in zip(got, ref[:3]):
            assert rel(x, y) < 1e-7, (every, depth, om)
    ctx.close()


@pytest.mark.gpu
def test_no_headings_and_uneven_bodies():
    bodies = [meshgen.cylinder(4.0, 6.0, 16, 4, 2), meshgen.cylinder(2.0, 4.0, 8, 2, 1, 20.0, 5.0)]
    oc, ctx = contexts(bodies, [(0.0, 0.0, 0.0), (20.0, 5.0, 0.0)], 35.0)
    none = np.zeros(0)
    for om in (0.4, 1.6):
        am, bd, ex = ctx.solve_frequency(hams_b200.wave_properties(om, 35.0, G), none)
        assert ex.size == 0 or not np.any(ex)
        oam, obd, _, _ = oc.solve(oc.wave(om), none)
        assert rel(am, oam) < 1e-7 and rel(bd, obd) < 1e-7
    waves = [hams_b200.wave_properties(om, 35.0, G) for om in (0.4, 0.9, 1.6)]
    am, bd, _ = ctx.solve_batch(waves, none)
    for k, om in enumerate((0.4, 0.9, 1.6)):
        oam, obd, _, _ = oc.solve(oc.wave(om), none)
        assert rel(am[k], oam) < 1e-7 and rel(bd[k], obd) < 1e-7
    ctx.close()
