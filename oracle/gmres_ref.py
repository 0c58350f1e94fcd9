"""CPU restatement of the reference's restarted GMRES (test infrastructure).

Checks the library's GMRES solver: same preconditioners, restart length and
stopping tests as src/IterativeSolvers.f90, one right-hand side at a time in
numpy.  Parity is pinned through the LU solution of the same systems (the
oracle's direct solve), which every converged GMRES solution must approach to
its tolerance, and through the reference's own GMRES test (its GMRES output
against its LU output at relative Frobenius 1e-3 for added mass and 5e-2 for
damping, test/test_integration_gmres.f90:48-101).

Rotations.  The reference's ZGIVENS_ROTATION (IterativeSolvers.f90:490-506)
returns cs = a/d, sn = b/d, which zeroes the sub-diagonal entry only when
conj(a) b is real; with a complex diagonal entry of the Hessenberg matrix the
entry it then sets to zero (:433) was not zero, so its residual estimate
|g(j+1)| is not the residual of its iterate and it can stop early.
rotation="reference" restates that form; the default rotation="complex" is
the complex Givens rotation (cs = |a|/d real, sn = (a/|a|) conj(b)/d) that
GMRES (Saad and Schultz, 1986) needs and the library uses.
"""
import numpy as np
import scipy.linalg as sla

# IterativeSolvers.f90:56-58
RESTART, TOL, MAXITER = 25, 1.0e-4, 100


def jacobi(a):
    """SETUP_PRECONDITIONER (IterativeSolvers.f90:154-174): the diagonal, 1 where |a_ii| < 1e-30."""
    d = np.diag(a).copy()
    d[np.abs(d) < 1e-30] = 1.0
    return lambda r: r / d


def block_diagonal(a, sizes):
    """SETUP_BLOCK_PRECONDITIONER / APPLY_PRECONDITIONER case 2 (IterativeSolvers.f90:176-253, :270-284):
    LU factors of each body's diagonal block, applied block by block."""
    off = np.concatenate([[0], np.cumsum(sizes)])
    lus = [sla.lu_factor(a[off[k]:off[k + 1], off[k]:off[k + 1]]) for k in range(len(sizes))]

    def apply(r):
        z = np.empty_like(r)
        for k, lu in enumerate(lus):
            z[off[k]:off[k + 1]] = sla.lu_solve(lu, r[off[k]:off[k + 1]])
        return z

    return apply


def givens(a, b, rotation="complex"):
    """(cs, sn) with [[cs, sn], [-conj(sn), conj(cs)]] [a, b] = [d, 0]; rotation="reference" gives
    ZGIVENS_ROTATION's (IterativeSolvers.f90:490-506) cs = a/d, sn = b/d instead."""
    if abs(b) < 1e-30:
        return 1.0 + 0j, 0j
    if abs(a) < 1e-30:
        return (0j, 1.0 + 0j) if rotation == "reference" else (0j, np.conj(b) / abs(b))
    den = np.sqrt(abs(a) ** 2 + abs(b) ** 2)
    if rotation == "reference":
        return a / den, b / den
    return abs(a) / den + 0j, (a / abs(a)) * np.conj(b) / den


def gmres(a, b, precond, tol=TOL, maxiter=MAXITER, m=RESTART, rotation="complex"):
    """ZGMRES_SOLVE (IterativeSolvers.f90:324-484) for one right-hand side from x = 0.
    Returns (x, iterations, converged)."""
    n = b.size
    x = np.zeros(n, dtype=np.complex128)
    bnorm = np.linalg.norm(b)
    if bnorm < 1e-30:
        return x, 0, True
    it, ok = 0, False
    while it < maxiter:
        r = b - a @ x if it > 0 else b.copy()
        beta = np.linalg.norm(r)
        if beta / bnorm < tol:
            ok = True
            break
        v = np.zeros((n, m + 1), dtype=np.complex128)
        h = np.zeros((m + 1, m), dtype=np.complex128)
        cs, sn = np.zeros(m, dtype=np.complex128), np.zeros(m, dtype=np.complex128)
        g = np.zeros(m + 1, dtype=np.complex128)
        v[:, 0] = r / beta
        g[0] = beta
        k = 0
        for j in range(m):
            it += 1
            if it > maxiter:
                break
            w = a @ precond(v[:, j])
            for i in range(j + 1):  # modified Gram-Schmidt
                h[i, j] = np.vdot(v[:, i], w)
                w = w - h[i, j] * v[:, i]
            h[j + 1, j] = np.linalg.norm(w)
            v[:, j + 1] = w / h[j + 1, j] if abs(h[j + 1, j]) > 1e-30 else 0.0
            for i in range(j):
                t = cs[i] * h[i, j] + sn[i] * h[i + 1, j]
                h[i + 1, j] = -np.conj(sn[i]) * h[i, j] + np.conj(cs[i]) * h[i + 1, j]
                h[i, j] = t
            cs[j], sn[j] = givens(h[j, j], h[j + 1, j], rotation)
            h[j, j] = cs[j] * h[j, j] + sn[j] * h[j + 1, j]
            h[j + 1, j] = 0.0
            t = cs[j] * g[j] + sn[j] * g[j + 1]
            g[j + 1] = -np.conj(sn[j]) * g[j] + np.conj(cs[j]) * g[j + 1]
            g[j] = t
            k = j + 1
            if abs(g[j + 1]) / bnorm < tol:
                ok = True
                break
        if k > 0:
            y = g[:k].copy()
            for i in range(k - 1, -1, -1):
                y[i] = 0.0 if abs(h[i, i]) < 1e-30 else y[i] / h[i, i]
                y[:i] -= h[:i, i] * y[i]
            x = x + precond(v[:, :k] @ y)
        if ok:
            break
    return x, min(it, maxiter), ok


def solve(a, rhs, body_sizes, **kw):
    """ZITER_SOLVE_MULTI (IterativeSolvers.f90:565-579): every column of rhs in turn, the block-diagonal
    preconditioner with two or more bodies (AssbMatxMulti.f90:282-292), the diagonal with one.
    Returns (X, iterations per column)."""
    precond = block_diagonal(a, body_sizes) if len(body_sizes) > 1 else jacobi(a)
    out = [gmres(a, rhs[:, c], precond, **kw) for c in range(rhs.shape[1])]
    return np.stack([o[0] for o in out], axis=1), [o[1] for o in out]
