"""Pin the CPU oracle against the reference's own golden decks.

The reference's regression test (test/test_integration.f90:71,98 and
test/testing_utilities.f90:132-166) reruns the Fortran binary on
test/data/config1 and compares OAMASS/ODAMPING files as printed.  Its
expected files come from an ifx + MKL build (ifx defaults to a fast
floating-point model), so a strict-IEEE restatement cannot reproduce every
last printed digit of the small cross couplings; the tolerances below are
relative Frobenius norms per file, in the style of the reference's own
``test_oamass_files_are_close`` (testing_utilities.f90:178-202), plus a
count of entries printed identically.

Observed with the oracle (relative Frobenius, worst of the six files):
  config1  (3 x 234 panels, h=70 m, omega 0.05-0.07):  A 3.4e-7, B 1.3e-4, X 3.0e-8
  example2 (10 x 234 panels, h=14.5 m, T=0.5, 1 s):   A 4.9e-6, B 2.4e-5, X 3.3e-6
  example5 (1 x 234 + 383 lid panels, h=70 m):        A 1.9e-5, B 9.0e-3, X 3.0e-6
  example3 (2 x 234 panels with lids, a generalized mode, 36 headings; its
            expected files hold the first of the deck's 10 frequencies):
                                                      A 3.7e-5, B 1.8e-5, X 2.7e-5
The Wynn-epsilon extrapolation of the EIGENE/PIDCOCK series turns a one-ulp
difference of sin/cos/exp/log into up to 1e-3 in single Green values; the
oracle evaluates those with correctly rounded functions, as the reference's
compiler library does, which is what brings config1 to these numbers.
Damping at these long waves is ~1e-6 of the added mass, and the lid path
squares the condition number (A^T A), so its last digits are FP noise of the
reference build; the tolerances carry that.
"""
import os

import numpy as np
import pytest

import oracle_lib

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

# (deck, tol A, tol B, tol X, minimum fraction of significant entries printed identically per A/B/X)
# Observed fractions: config1 0.977/0.912/0.968, example2 0.73/0.67/0.63, example5 0.79/0.63/0.71,
# example3 0.63/0.55/0.60.
# The epsilon-accelerated series use correctly rounded sin/cos/exp/log (detmath.h); with
# glibc's versions config1 prints identically for 0.92/0.79/0.90 only.
CASES = [
    ("config1", 1e-6, 5e-4, 2e-7, (0.95, 0.88, 0.94)),
    ("example2", 2e-5, 1e-4, 1e-5, (0.70, 0.63, 0.60)),
    ("example5", 1e-4, 3e-2, 1e-5, (0.76, 0.60, 0.68)),
    ("example3", 1e-4, 1e-4, 1e-4, (0.60, 0.50, 0.57)),
]


def _load(path):
    return [line.split() for line in open(path) if line.strip()]


@pytest.mark.parametrize("deck,tol_a,tol_b,tol_x,min_same", CASES)
def test_oracle_reproduces_reference_outputs(tmp_path, oracle, deck, tol_a, tol_b, tol_x, min_same):
    inp = os.path.join(GOLDEN, deck, "input")
    exp = os.path.join(GOLDEN, deck, "expected")
    rc = oracle.orc_run_case(inp.encode(), str(tmp_path).encode(), 8, os.cpu_count() or 1)
    assert rc == 0
    for kind, tol, frac in (("OAMASS", tol_a, min_same[0]), ("ODAMPING", tol_b, min_same[1]),
                            ("OEXFOR", tol_x, min_same[2])):
        same = total = 0
        for m in range(1, 7):
            ref = _load(os.path.join(exp, f"{kind}{m}.txt"))
            heads = {tuple(row[:2]) for row in ref}
            # the frequencies the expected file holds (example3 keeps the first of its deck's)
            got = [row for row in _load(tmp_path / f"{kind}{m}.txt") if tuple(row[:2]) in heads]
            assert len(got) == len(ref)
            g = np.array([[float(x) for x in r[2:]] for r in got])
            r = np.array([[float(x) for x in row[2:]] for row in ref])
            # wave number and frequency columns print identically
            assert [row[:2] for row in got] == [row[:2] for row in ref]
            rel = np.linalg.norm(g - r) / np.linalg.norm(r)
            assert rel < tol, f"{deck} {kind}{m}: relative Frobenius {rel:.3e} >= {tol}"
            sig = np.abs(r) > 1e-2 * np.abs(r).max(axis=1, keepdims=True)
            tg = np.array([row[2:] for row in got])
            tr = np.array([row[2:] for row in ref])
            same += int((tg == tr)[sig].sum())
            total += int(sig.sum())
        print(deck, kind, f"{same / total:.3f} of significant entries printed identically")
        assert same / total >= frac, f"{deck} {kind}: {same}/{total} significant entries printed identically"


def test_deck_loader_config1(oracle):
    d = oracle_lib.load_deck(os.path.join(GOLDEN, "config1", "input"))
    assert d["nper"] == 3 and d["nbeta"] == 3
    assert np.allclose(d["wvnb"], [0.05, 0.06, 0.07])
    assert np.allclose(d["wvhd"], [0.0, 10.0, 20.0])
    assert d["h"] == 70.0 and d["nsys"] == 1
    assert list(d["body_nelem"]) == [234, 234, 234]
    assert np.allclose(d["xr"][:, 1], [0.0, 54.0, 108.0])
    # bodies translated on read (ReadPanelMeshMulti.f90:57-59)
    assert np.isclose(d["xyz_p"][234:468, 1].mean() - d["xyz_p"][:234, 1].mean(), 54.0)
    # areas positive, unit normals
    assert (d["ds"] > 0).all()
    assert np.allclose(np.linalg.norm(d["dxyz"][:, :3], axis=1), 1.0)


def test_deck_loader_lid_and_single_body(oracle):
    d = oracle_lib.load_deck(os.path.join(GOLDEN, "example5", "input"))
    assert d["irsp"] == 1 and d["inelem"] == 383
    assert list(d["body_nelem"]) == [234]
    assert np.allclose(d["ixyz_p"][:, 2], 0.0)
    assert d["nbeta"] == 36 and d["nper"] == 10
