"""Contexts created one after another reuse the device memory, streams and
library handles of the destroyed ones (hams_ctx_destroy keeps them,
hams_release_cached gives them back).  A reused buffer must carry nothing
from its previous owner: a second context on the same deck gives the same
bits as the first, a context of another size in between changes nothing,
and the judged surrogate form with its eight lanes repeats exactly."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "hams-mrel_b200"))
import hams_b200  # noqa: E402
import meshgen  # noqa: E402
import train_surrogate  # noqa: E402


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def array(ncol, nrow, nbot, spacing=20.0):
    bodies, centres = [], []
    for iy in range(3):
        for ix in range(3):
            bodies.append(meshgen.cylinder(4.0, 8.0, ncol, nrow, nbot, spacing * ix, spacing * iy))
            centres.append((spacing * ix, spacing * iy, 0.0))
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    return hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, np.array(centres))


def solve(geom, waves, betas, sg=False, precision=hams_b200.PREC_MIXED, blocks=0):
    ctx = hams_b200.Context(geom, 50.0, rho=1025.0, g=9.81, precision=precision, refine_tol=1e-7 if sg else 0.0,
                            body_blocks=blocks)
    if sg:
        ctx.set_surrogate(train_surrogate.load(), 3.0)
        ctx.set_surrogate_tolerance(1e-4)
    out = ctx.solve_batch(waves, betas)
    note = ctx.note()
    ctx.close()
    return out, note


@pytest.mark.gpu
def test_contexts_in_sequence_reuse_memory_and_repeat_bits():
    import torch

    betas = np.radians([0.0, 45.0])
    small, big = array(20, 5, 3), array(28, 7, 4)
    waves = [hams_b200.wave_properties(om, 50.0, 9.81) for om in (0.4, 0.9, 1.4, 1.9, 2.3)]
    first, _ = solve(small, waves, betas)
    other, _ = solve(big, waves, betas)  # a larger context takes and grows the cached buffers
    again, _ = solve(small, waves, betas)
    for a, b in zip(first, again):
        assert np.array_equal(a, b)
    # the larger deck against its own fp64 solve
    ref, _ = solve(big, waves, betas, precision=hams_b200.PREC_FP64)
    for a, b in zip(other, ref):
        assert rel(a, b) < 1e-6
    # the judged surrogate form, eight lanes, twice
    s1, n1 = solve(small, waves, betas, sg=True, blocks=1)
    s2, n2 = solve(small, waves, betas, sg=True, blocks=1)
    assert n1 == n2
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    # the cache goes back to the driver on request
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    hams_b200.release_cached()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 > free0
