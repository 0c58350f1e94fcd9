"""The GMRES restatement (oracle/gmres_ref.py) on small dense complex systems:
converges to the direct solution, stops on the reference's tests, the
block-diagonal preconditioner inverts a block-diagonal matrix exactly, and the
reference's rotation (IterativeSolvers.f90:490-506) stops early on a complex
system while the complex Givens rotation meets the tolerance."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import gmres_ref  # noqa: E402


def bem_like(n, rng, sizes=None):
    """Diagonally dominant complex matrix with smooth off-diagonal coupling, like a
    collocation matrix (0.5 on the diagonal plus decaying interactions)."""
    p = rng.uniform(-1, 1, (n, 3))
    d = np.linalg.norm(p[:, None] - p[None], axis=2) + 0.3
    a = (0.05 / d) * np.exp(1j * d) / np.sqrt(n / 64)
    a[np.diag_indices(n)] = 0.5 + 0.1j
    return a


def test_converges_to_direct_solution():
    rng = np.random.default_rng(3)
    a = bem_like(120, rng)
    b = rng.standard_normal((120, 3)) + 1j * rng.standard_normal((120, 3))
    x, its = gmres_ref.solve(a, b, [120], tol=1e-12, maxiter=400)
    ref = np.linalg.solve(a, b)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-10
    assert all(0 < k < 400 for k in its)


def test_stops_at_tolerance_and_counts_iterations():
    rng = np.random.default_rng(4)
    a = bem_like(100, rng)
    b = rng.standard_normal(100) + 1j * rng.standard_normal(100)
    pre = gmres_ref.jacobi(a)
    for tol in (1e-3, 1e-6, 1e-9):
        x, it, ok = gmres_ref.gmres(a, b, pre, tol=tol, maxiter=200, m=10)
        assert ok and np.linalg.norm(b - a @ x) / np.linalg.norm(b) < 2 * tol
        # one fewer step misses the tolerance
        x1, it1, ok1 = gmres_ref.gmres(a, b, pre, tol=tol, maxiter=it - 1, m=10)
        assert not ok1 and it1 == it - 1
    # a zero right-hand side returns zero at once (IterativeSolvers.f90:348-352)
    x, it, ok = gmres_ref.gmres(a, np.zeros(100, complex), pre)
    assert ok and it == 0 and not x.any()


def test_block_preconditioner_is_exact_on_block_diagonal():
    rng = np.random.default_rng(5)
    sizes = [30, 50, 20]
    a = np.zeros((100, 100), complex)
    o = 0
    for s in sizes:
        a[o:o + s, o:o + s] = bem_like(s, rng)
        o += s
    b = rng.standard_normal((100, 2)) + 1j * rng.standard_normal((100, 2))
    x, its = gmres_ref.solve(a, b, sizes)
    assert its == [1, 1]
    assert np.linalg.norm(a @ x - b) / np.linalg.norm(b) < 1e-12


def test_reference_rotation_stops_early_on_complex_systems():
    rng = np.random.default_rng(6)
    a = bem_like(100, rng)
    b = rng.standard_normal(100) + 1j * rng.standard_normal(100)
    pre = gmres_ref.jacobi(a)
    x, it, ok = gmres_ref.gmres(a, b, pre, tol=1e-6, rotation="reference")
    res_ref = np.linalg.norm(b - a @ x) / np.linalg.norm(b)
    x, it, ok = gmres_ref.gmres(a, b, pre, tol=1e-6)
    res = np.linalg.norm(b - a @ x) / np.linalg.norm(b)
    assert res < 2e-6 < 1e-3 < res_ref
    # on a real system the two rotations agree
    ar, br = a.real.copy(), b.real.astype(complex)
    x1, it1, _ = gmres_ref.gmres(ar, br, gmres_ref.jacobi(ar), tol=1e-8, rotation="reference")
    x2, it2, _ = gmres_ref.gmres(ar, br, gmres_ref.jacobi(ar), tol=1e-8)
    assert it1 == it2 and np.allclose(x1, x2, rtol=1e-10, atol=1e-12)
