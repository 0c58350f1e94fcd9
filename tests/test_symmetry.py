"""Geometric symmetry (ISX / ISY = 1, NSYS = 2): half meshes.

The reference solves the symmetric and antisymmetric systems of a half mesh
(field points imaged with the SX/SY signs, RXY combinations:
CalGreenFuncMulti.f90:112-318, AssbMatxMulti.f90:53-251,
PotentWavForceMulti.f90:45-226).  Together they are the full body's system
in another basis, which gives a property that pins the oracle's restatement
without a golden (none of the reference's decks is symmetric): the oracle's
NSYS = 2 solve of a half mesh equals its NSYS = 1 solve of the unfolded mesh
(CPU, 1e-12 relative Frobenius of added mass, damping, excitation; 1e-15
seen), when the mirrored panels carry the exact mirror images of the half's
centres, areas, sizes and normals, as the library's unfolding gives them
(n' = M n, (r x n)' = -M (r x n)).  Panel centres recomputed from the
mirrored nodes round differently, and the epsilon extrapolation of the
finite-depth series amplifies that to ~1e-6.

GPU (marked gpu): the library unfolds a half mesh itself (hams_ctx_create)
and matches the oracle's NSYS = 2 solve to 1e-7, for ISX and ISY, finite
and infinite depth, two bodies, and with water-plane lids.
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


def half(mesh, axis):
    """Panels of a mesh whose centre has coordinate `axis` > 0 (the half a symmetric deck holds)."""
    nodes, ncn, ncon = mesh
    c = np.array([nodes[q[:k] - 1].mean(axis=0) for q, k in zip(ncon, ncn)])
    keep = c[:, axis] > 1e-9
    return nodes, ncn[keep], ncon[keep]


def unfold(meshes, axis):
    """Each body's half panels followed by their mirror images, vertex order reversed."""
    out = []
    for nodes, ncn, ncon in meshes:
        m = nodes.copy()
        m[:, axis] *= -1.0
        nt = nodes.shape[0]
        rev = ncon.copy()
        rev[:, 1:] = ncon[:, :0:-1]
        out.append((np.vstack([nodes, m]), np.concatenate([ncn, ncn]), np.vstack([ncon, rev + nt])))
    return out


def two_cylinders(axis):
    """Two cylinders centred on the symmetry plane, 16 x 3 side + 16 x 2 bottom panels each."""
    other = 1 - axis
    pos = [(0.0, 0.0), (0.0, 0.0)]
    pos = [tuple(-15.0 if k == other else 0.0 for k in range(2)), tuple(15.0 if k == other else 0.0 for k in range(2))]
    bodies = [half(meshgen.cylinder(4.0, 6.0, 16, 3, 2, x, y), axis) for x, y in pos]
    lids = [half(meshgen.disc_lid(4.0, 16, 1, x, y), axis) for x, y in pos]
    return bodies, lids, np.array([(x, y, 0.0) for x, y in pos])


def oracle_case(bodies, lids, xr, depth, isx=0, isy=0, with_lids=False):
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    kw = {}
    if with_lids:
        lx, ln, lc, lcnt = meshgen.combine(lids)
        kw = dict(ixyz=lx, incn=ln, incon=lc, body_inelem=lcnt, irsp=1)
    return oracle_lib.Case(xyz, ncn, ncon, cnt, xr, depth, rho=RHO, g=G, isx=isx, isy=isy, **kw), (xyz, ncn, ncon, cnt)


def unfolded_case(sym, bodies, lids, xr, depth, axis, with_lids):
    """The oracle's case of the unfolded mesh, its mirrored panels carrying the exact mirror
    images of the half's geometry."""
    full, _ = oracle_case(unfold(bodies, axis), unfold(lids, axis), xr, depth, with_lids=with_lids)
    sg = np.ones(6)
    sg[axis] = -1.0
    sg[3:] = -1.0
    sg[3 + axis] = 1.0
    o_s = o_f = 0
    for m in (b[1].size for b in bodies):
        for dst in (o_f, o_f + m):
            mirror = dst != o_f
            for k in range(3):
                full.xyz_p[dst:dst + m, k] = (-1.0 if mirror and k == axis else 1.0) * sym.xyz_p[o_s:o_s + m, k]
            full.ds[dst:dst + m] = sym.ds[o_s:o_s + m]
            full.pnsz[dst:dst + m] = sym.pnsz[o_s:o_s + m]
            for k in range(6):
                full.dxyz[dst:dst + m, k] = (sg[k] if mirror else 1.0) * sym.dxyz[o_s:o_s + m, k]
        o_s += m
        o_f += 2 * m
    if with_lids:
        o_s = o_f = 0
        for m in (l[1].size for l in lids):
            for k in range(3):
                v = sym.ixyz_p[o_s:o_s + m, k]
                full.ixyz_p[o_f:o_f + m, k] = v
                full.ixyz_p[o_f + m:o_f + 2 * m, k] = -v if k == axis else v
            o_s += m
            o_f += 2 * m
    return full


@pytest.mark.parametrize("axis,depth,with_lids", [(0, 40.0, False), (1, 40.0, False), (0, -1.0, False),
                                                  (0, 40.0, True)])
def test_oracle_half_mesh_equals_unfolded_mesh(axis, depth, with_lids):
    bodies, lids, xr = two_cylinders(axis)
    flags = dict(isx=1) if axis == 0 else dict(isy=1)
    sym, _ = oracle_case(bodies, lids, xr, depth, with_lids=with_lids, **flags)
    full = unfolded_case(sym, bodies, lids, xr, depth, axis, with_lids)
    betas = np.radians([0.0, 30.0])
    for om in (0.6, 1.5):
        a = sym.solve(sym.wave(om), betas)
        b = full.solve(full.wave(om), betas)
        for x, y in zip(a[:3], b[:3]):
            assert rel(x, y) < 1e-12, (axis, depth, with_lids, om, rel(x, y))


@pytest.mark.gpu
@pytest.mark.parametrize("axis,depth,with_lids", [(0, 40.0, False), (1, 40.0, False), (0, -1.0, False),
                                                  (0, 40.0, True)])
def test_gpu_half_mesh_matches_oracle(axis, depth, with_lids):
    bodies, lids, xr = two_cylinders(axis)
    flags = dict(isx=1) if axis == 0 else dict(isy=1)
    oc, (xyz, ncn, ncon, cnt) = oracle_case(bodies, lids, xr, depth, with_lids=with_lids, **flags)
    geom = dict(xyz=xyz, ncn=ncn, ncon=ncon, xyz_p=oc.xyz_p, ds=oc.ds, pnsz=oc.pnsz, dxyz=oc.dxyz, body_nelem=cnt,
                isx=flags.get("isx", 0), isy=flags.get("isy", 0))
    if with_lids:
        geom["ixyz_p"] = oc.ixyz_p
    ctx = hams_b200.Context(geom, depth, rho=RHO, g=G, irsp=1 if with_lids else 0)
    assert ctx.n == ncn.size  # the caller's half mesh; the library holds the unfolded one
    with pytest.raises(hams_b200.HamsError):  # whose matrices have no caller-sized layout
        ctx.assemble(hams_b200.wave_properties(1.0, depth, G), np.radians([0.0]))
    betas = np.radians([0.0, 30.0])
    for om in (0.6, 1.5):
        got = ctx.solve_frequency(hams_b200.wave_properties(om, depth, G), betas)
        ref = oc.solve(oc.wave(om), betas)
        for x, y in zip(got, ref[:3]):
            assert rel(x, y) < 1e-7, (axis, depth, with_lids, om, rel(x, y))
    ctx.close()


@pytest.mark.gpu
def test_two_symmetry_planes_rejected():
    bodies, _, xr = two_cylinders(0)
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    geom = dict(hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, xr), isx=1, isy=1)
    with pytest.raises(hams_b200.HamsError):
        hams_b200.Context(geom, 40.0)
