"""Known-answer tests of the oracle's special functions and Green functions.

Known answers come from the example tables in the reference's comments
(src/FinGrnExtSubs.f90:52-59 erf, :124-132 E_n at x=10, :187-195 E1,
:243-251 Ei) and, as independent mathematics, from scipy.special.  The
Green functions are checked against properties that do not depend on the
reference's approximations: continuity across the FINGREEN3D_R branch
boundaries (FinGreen3D.f90:183-191), the dispersion relations, and the
deep-water limit of the finite-depth function.
"""
import numpy as np
import pytest
import scipy.special as sp

import oracle_lib


@pytest.mark.parametrize("x,ref", [(1.0, .84270079), (2.0, .99532227), (3.0, .99997791), (4.0, .99999998), (5.0, 1.0)])
def test_erf_table(oracle, x, ref):
    assert abs(oracle_lib.special(0, x)[0] - ref) < 1e-8
    assert abs(oracle_lib.special(0, x)[0] - sp.erf(x)) < 1e-14


@pytest.mark.parametrize("n,ref", [(0, .45399930e-05), (1, .41569689e-05), (2, .38302405e-05), (3, .35487626e-05),
                                   (4, .33041014e-05), (5, .30897289e-05)])
def test_en_table_x10(oracle, n, ref):
    # ENXA runs the forward recurrence E_k = (e^-x - x E_{k-1})/(k-1) from the rational E1XA fit;
    # at x = 10 the recurrence amplifies the fit's 2e-8 error by ~x per order (1e-5 at n = 5).
    assert abs(oracle_lib.special(5 + n, 10.0)[0] / ref - 1) < 2e-8 * 12.0 ** n


@pytest.mark.parametrize("x,ref", [(1.0, .2193839), (2.0, .4890051e-01), (3.0, .1304838e-01), (4.0, .3779352e-02),
                                   (5.0, .1148296e-02)])
def test_e1_table(oracle, x, ref):
    assert abs(oracle_lib.special(1, x)[0] / ref - 1) < 2e-6
    assert oracle_lib.special(1, 0.0)[0] == 1e300


@pytest.mark.parametrize("x,ref", [(1.0, .18951178e+01), (2.0, .49542344e+01), (3.0, .99338326e+01),
                                   (4.0, .19630874e+02), (5.0, .40185275e+02)])
def test_ei_table(oracle, x, ref):
    assert abs(oracle_lib.special(2, x)[0] / ref - 1) < 5e-8  # table printed to 8 digits
    assert abs(oracle_lib.special(2, x)[0] / sp.expi(x) - 1) < 1e-13


@pytest.mark.parametrize("x", [1e-3, 0.3, 1.0, 4.5, 8.9, 9.1, 17.0, 19.0, 36.0, 55.0])
def test_k0_k1_against_scipy(oracle, x):
    k0, k1 = oracle_lib.special(3, x)[:2]
    # IK01A switches from the K0 series to the asymptotic form at x = 9: ~3e-9 there
    assert abs(k0 / sp.k0(x) - 1) < 1e-8
    assert abs(k1 / sp.k1(x) - 1) < 1e-8


@pytest.mark.parametrize("x", [1e-2, 0.5, 2.0, 3.99, 4.01, 10.0, 40.0])
def test_j_y_polynomials_against_scipy(oracle, x):
    j0, j1, y0, y1 = oracle_lib.special(4, x)
    # Zhang & Jin polynomial fits: ~1e-8 absolute
    assert abs(j0 - sp.j0(x)) < 1e-8 and abs(j1 - sp.j1(x)) < 1e-8
    assert abs(y0 - sp.y0(x)) < 1e-8 * max(1.0, abs(sp.y0(x)))
    assert abs(y1 - sp.y1(x)) < 1e-8 * max(1.0, abs(sp.y1(x)))


@pytest.mark.parametrize("w,h", [(0.05, 70.0), (0.7, 50.0), (2.5, 50.0), (1.0, 14.5), (3.0, 200.0)])
def test_dispersion_roots(oracle, w, h):
    g = 9.807  # DISPERSION uses its own g (WavDynSubs.f90:58)
    wvn = oracle_lib.dispersion(w, h)
    v = w * w / g
    assert abs(wvn[0] * np.tanh(wvn[0] * h) - v) < 1e-10 * max(v, 1)
    m = wvn[1:]
    assert np.allclose(m * np.tan(m * h), -v, rtol=0, atol=1e-8 * max(v, 1))
    assert np.all(np.diff(wvn[1:]) > 0)


def _branch_points(h):
    """Horizontal distances just either side of the R/h = 0.05 and 0.5 branch edges."""
    out = []
    for b in (0.05, 0.5):
        out.append((b * h * (1 - 1e-9), b * h * (1 + 1e-9)))
    return out


@pytest.mark.parametrize("w,h,zf,zp", [(0.8, 50.0, -3.0, -5.0), (1.6, 50.0, -1.0, -7.5), (0.3, 30.0, -2.0, -2.5)])
def test_fingreen_continuous_across_branches(oracle, w, h, zf, zp):
    wvn = oracle_lib.dispersion(w, h)
    v = w * w / 9.80665
    for lo, hi in _branch_points(h):
        ga = oracle_lib.fingreen(lo, 0.0, 0.0, 0.0, zf, zp, v, wvn, h, 1)
        gb = oracle_lib.fingreen(hi, 0.0, 0.0, 0.0, zf, zp, v, wvn, h, 1)
        # value and vertical derivative continue; the series truncations differ by ~1e-5
        assert abs(ga[0] - gb[0]) < 2e-4 * max(1.0, abs(ga[0]))
        assert abs(ga[3] - gb[3]) < 2e-3 * max(1.0, abs(ga[3]))


@pytest.mark.parametrize("w,h,zf,zp", [(0.3, 30.0, -2.0, -2.5), (0.05, 70.0, -1.0, -3.0), (1.6, 50.0, -1.0, -7.5)])
def test_linton_branch_is_self_consistent(oracle, w, h, zf, zp):
    """LINTON (R/h < 0.0005) is flat in R across its R < 1e-6 (EIX) and series
    (SA0/SAM) sub-paths.  Its real part does not join PIDCOCK's at R/h = 0.0005
    (up to a factor 2 at long waves); the reference has the same jump: every
    LINTON pair of the config1 deck is an R = 0 self pair, and the oracle
    reproduces that deck's printed added mass to 3e-7."""
    wvn = oracle_lib.dispersion(w, h)
    v = w * w / 9.807
    vals = [oracle_lib.fingreen(r, 0.0, 0.0, 0.0, zf, zp, v, wvn, h, 1)[0] - 1 / np.hypot(r, zf + zp)
            for r in (0.0, 1e-7, 1e-5, 1e-3, 0.0004 * h)]
    assert np.allclose(vals, vals[0], rtol=1e-5, atol=1e-9)  # G varies as R^2 here


def test_fingreen_tends_to_infinite_depth(oracle):
    """For kh >> 1 the finite-depth function approaches the deep-water one."""
    w, h = 2.0, 200.0
    wvn = oracle_lib.dispersion(w, h)
    v = w * w / 9.80665
    for r in (3.0, 11.0, 60.0):
        gf = oracle_lib.fingreen(r, 0.0, 0.0, 0.0, -2.0, -4.0, v, wvn, h, 1)
        gi = oracle_lib.infgreen(r, 0.0, 0.0, 0.0, -2.0, -4.0, v, 1)
        # the two use different g for the roots (9.807 vs 9.80665): ~1e-4 relative
        assert abs(gf[0] - gi[0]) < 3e-3 * abs(gi[0]), (r, gf[0], gi[0])


def test_infgreen_symmetry(oracle):
    """G(p, q) depends on the horizontal distance only; dG/dx flips sign with x."""
    v = 0.4
    a = oracle_lib.infgreen(2.0, 0.0, 1.0, 0.0, -1.0, -2.0, v, 1)
    b = oracle_lib.infgreen(-2.0, 0.0, -1.0, 0.0, -1.0, -2.0, v, 1)
    assert np.allclose(a[0], b[0], rtol=1e-14) and np.allclose(a[1], -b[1], rtol=1e-14)
