"""Identical body blocks (hams_body_blocks, hams_opts.body_blocks).

CPU: which (field body, source body) blocks of the collocation matrices the
library copies instead of computing -- arrays of translated identical bodies
share one block per horizontal offset; different shapes, a moved vertex, a
different panel order or water-plane lids keep their own blocks.
GPU (marked gpu): the copies against the same context computing every pair
(finite and infinite depth, regular and limit frequencies, single and batched
solves).  Every copied block equals its source block bit for bit, and the
source blocks equal the fully computed ones bit for bit.  The fully computed
copies differ from their source blocks only through the rounding of the
translated coordinates; the epsilon extrapolation of the EIGENE / PIDCOCK
series amplifies that in single pairs -- the CPU oracle's own values for a
pair and its translate differ by up to 2e-6 of max(1, |G|) at 0.3 rad/s and
6e-5 at 2.0 rad/s -- and the assembled matrices differ by up to 2.4e-5
(relative Frobenius, at 2.0 rad/s).  The bound here is 1e-4, the accuracy
bar of the surrogate form that uses the blocks, for the matrices, the
right-hand sides and the added mass, damping and excitation.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "hams-mrel_b200"))
import hams_b200  # noqa: E402
import meshgen  # noqa: E402


def rel(a, b):
    """Relative Frobenius difference over the finite entries; non-finite entries (the
    diffraction terms at the zero and infinite frequency limits) must coincide."""
    fa, fb = np.isfinite(a), np.isfinite(b)
    assert np.array_equal(fa, fb)
    return np.linalg.norm(a[fa] - b[fb]) / max(np.linalg.norm(b[fb]), 1e-300)


def array_geom(positions, make=lambda x, y: meshgen.cylinder(4.0, 8.0, 12, 3, 2, x, y), lids=False):
    bodies = [make(x, y) for x, y in positions]
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    xr = np.array([(x, y, 0.0) for x, y in positions])
    geom = hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, xr)
    if lids:
        geom["ixyz_p"] = np.zeros((4, 3))
    return geom


def grid3():
    return [(20.0 * ix, 20.0 * iy) for iy in range(3) for ix in range(3)]


def test_grid_of_identical_bodies_shares_one_block_per_offset():
    pos = grid3()
    rep, distinct = hams_b200.body_blocks(array_geom(pos))
    assert distinct == 25  # offsets (dx, dy) in {-40, -20, 0, 20, 40}^2
    nb = len(pos)
    for b2 in range(nb):
        for b1 in range(nb):
            k = b1 + nb * b2
            r = rep[b1, b2]
            assert r <= k and rep[r % nb, r // nb] == r  # a representative represents itself
            c1, c2 = r % nb, r // nb
            off = np.subtract(pos[b2], pos[b1])
            assert np.allclose(np.subtract(pos[c2], pos[c1]), off)
            # and it is the first block with that offset
            first = min(q for q in range(nb * nb)
                        if np.allclose(np.subtract(pos[q // nb], pos[q % nb]), off))
            assert r == first


def test_large_grid_counts_offsets():
    """144 small bodies on a 12 x 12 grid: one block per offset (23 x 23), found at once."""
    pos = [(10.0 * ix, 10.0 * iy) for iy in range(12) for ix in range(12)]
    rep, distinct = hams_b200.body_blocks(array_geom(pos, make=lambda x, y: meshgen.cylinder(2.0, 3.0, 8, 2, 1, x, y)))
    assert distinct == 23 * 23
    nb = len(pos)
    for k in (1, 13, 143, nb * nb - 1, nb * 77 + 5):
        r = rep.ravel(order="F")[k]
        assert np.allclose(np.subtract(pos[r // nb], pos[r % nb]), np.subtract(pos[k // nb], pos[k % nb]))


def test_uneven_row():
    rep, distinct = hams_b200.body_blocks(array_geom([(0.0, 0.0), (10.0, 0.0), (25.0, 0.0)]))
    assert distinct == 7  # one diagonal block, offsets +-10, +-15, +-25
    assert rep[1, 1] == 0 and rep[2, 2] == 0


def test_blocks_kept_when_bodies_differ():
    # a cylinder and a box
    geom = array_geom([(0.0, 0.0), (30.0, 0.0)],
                      make=lambda x, y: meshgen.cylinder(4.0, 8.0, 12, 3, 2, x, y) if x == 0.0
                      else meshgen.box(8.0, 8.0, 8.0, 4, 4, 3, x, y))
    rep, distinct = hams_b200.body_blocks(geom)
    assert distinct == 4 and np.array_equal(rep.ravel(order="F"), np.arange(4))
    # one vertex of the third body moved by 1e-6 of the mesh size
    pos = [(0.0, 0.0), (20.0, 0.0), (40.0, 0.0)]
    g = array_geom(pos)
    per = g["body_nelem"][0]
    node = g["ncon"][2 * per, 0] - 1
    g["xyz"][node, 2] += 6e-5
    g2 = hams_b200.prepare_geometry(g["xyz"], g["ncn"], g["ncon"], g["body_nelem"],
                                    np.array([(x, y, 0.0) for x, y in pos]))
    rep, distinct = hams_b200.body_blocks(g2)
    assert distinct == 8  # bodies 0 and 1: three blocks; every block with body 2: its own
    assert rep[1, 1] == 0 and rep[1, 0] == 1 and rep[2, 1] == 5 and rep[1, 2] == 7 and rep[2, 2] == 8
    # the same panels in another order
    g3 = array_geom(pos)
    sl = slice(2 * per, 3 * per)
    for k in ("ncn", "ncon", "xyz_p", "ds", "pnsz", "dxyz"):
        g3[k][sl] = g3[k][sl][::-1].copy()
    rep, distinct = hams_b200.body_blocks(g3)
    assert rep[2, 2] == 8 and rep[1, 1] == 0


def test_lids_and_single_body_keep_every_block():
    rep, distinct = hams_b200.body_blocks(array_geom(grid3(), lids=True))
    assert distinct == 81
    rep, distinct = hams_b200.body_blocks(array_geom([(0.0, 0.0)]))
    assert distinct == 1 and rep[0, 0] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("depth", [50.0, -1.0])
def test_copied_blocks_match_every_pair(depth):
    geom = array_geom(grid3())
    betas = np.radians([0.0, 30.0])
    full = hams_b200.Context(geom, depth, rho=1025.0, g=9.81)
    copy = hams_b200.Context(geom, depth, rho=1025.0, g=9.81, body_blocks=1)
    per = int(geom["body_nelem"][0])
    waves = [hams_b200.wave_properties(om, depth, 9.81) for om in (0.3, 1.1, 2.0)]
    if depth > 0:
        waves += [hams_b200.wave_properties(1.0, depth, 9.81, sybo_kk=k) for k in (1, 2)]
    reps, distinct = hams_b200.body_blocks(geom)
    blk = lambda a, k: a[(k % 9) * per:(k % 9 + 1) * per, (k // 9) * per:(k // 9 + 1) * per]
    for w in waves:
        a0, b0, d0 = full.assemble(w, betas)
        a1, b1, d1 = copy.assemble(w, betas)
        for k in range(81):
            r = reps[k % 9, k // 9]
            assert np.array_equal(blk(a1, k), blk(a1, r))
            if r == k:
                assert np.array_equal(blk(a1, k), blk(a0, k))
        # the right-hand sides are sums over S, so they see the copies too
        assert rel(a1, a0) < 1e-4 and rel(b1, b0) < 1e-4 and rel(d1, d0) < 1e-4
        r0 = full.solve_frequency(w, betas)
        r1 = copy.solve_frequency(w, betas)
        assert copy.timings()["pairs_copied"] == (81 - distinct) * per * per
        assert full.timings()["pairs_copied"] == 0
        for x, y in zip(r1, r0):
            assert rel(x, y) < 1e-4
    # batched lanes share the copy lists
    if depth > 0:
        for x, y in zip(copy.solve_batch(waves[:3], betas), full.solve_batch(waves[:3], betas)):
            for k in range(3):
                assert rel(x[k], y[k]) < 1e-4
    full.close()
    copy.close()
