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


def cut_deck(src, dst, nfreq):
    """Copy the deck in src to dst with its frequency list cut to the first
    nfreq frequencies (the zero- and infinite-frequency limits, when the deck
    asks for them, come on top)."""
    import re
    import shutil

    os.makedirs(dst, exist_ok=True)
    for f in os.listdir(src):
        shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
    ctl = os.path.join(dst, "ControlFile.in")
    text = open(ctl).read()
    text, k = re.subn(r"(Number_of_frequencies\s+)(-?)\d+", lambda m: f"{m.group(1)}{m.group(2)}{nfreq}", text, 1)
    assert k == 1
    open(ctl, "w").write(text)
    return dst


def compare_limit_files(got_dir, exp_dir, tol_a, tol_b, tol_x):
    """Per frequency record of the OAMASS/ODAMPING/OEXFOR files: the heads
    print identically, NaN where the reference printed NaN, exact zeros where
    it printed zeros (damping and excitation at the zero-frequency limit,
    damping at the infinite-frequency limit), and the relative Frobenius
    error of every other record within the tolerance.  Returns the worst
    error per kind."""
    worst = {}
    for kind, tol in (("OAMASS", tol_a), ("ODAMPING", tol_b), ("OEXFOR", tol_x)):
        worst[kind] = 0.0
        for m in range(1, 7):
            ref = _load(os.path.join(exp_dir, f"{kind}{m}.txt"))
            got = _load(os.path.join(got_dir, f"{kind}{m}.txt"))[:len(ref)]
            assert [r[:2] for r in got] == [r[:2] for r in ref]
            r = np.array([[float(x) for x in row[2:]] for row in ref])
            g = np.array([[float(x) for x in row[2:]] for row in got])
            assert np.array_equal(np.isnan(r), np.isnan(g)), f"{kind}{m}: NaN entries differ"
            heads = [tuple(row[:2]) for row in ref]
            for key in dict.fromkeys(heads):
                idx = [i for i, h in enumerate(heads) if h == key]
                rr, gg = r[idx], g[idx]
                if np.isnan(rr).any():
                    continue
                nr = np.linalg.norm(rr)
                if nr == 0.0:
                    assert np.all(gg == 0.0), f"{kind}{m} at {key}: nonzero where the reference prints zero"
                    continue
                e = np.linalg.norm(gg - rr) / nr
                worst[kind] = max(worst[kind], e)
                assert e < tol, f"{kind}{m} at {key}: relative Frobenius {e:.3e} >= {tol}"
    return worst


def test_oracle_zero_and_infinite_frequency_limits(tmp_path, oracle):
    """examples/example1_multi_bodies (5 bodies x 727 panels, h = 0.9 m, 0_inf_frequency_limits = 1):
    the zero- and infinite-frequency added mass prints as the reference's (observed: identically),
    damping is zero at both limits and excitation zero at the zero limit and NaN at the infinite one,
    as the reference prints them (its incident-wave terms divide infinities there,
    PatclVelct.f90:90-110); the first regular frequency (0.2 rad/s) within the tolerances of the
    other decks (observed A 3.9e-5, B 3.8e-3 for the small roll damping, X 1.2e-5)."""
    deck = cut_deck(os.path.join(GOLDEN, "example1", "input"), str(tmp_path / "in"), 1)
    out = tmp_path / "out"
    out.mkdir()
    rc = oracle.orc_run_case(deck.encode(), str(out).encode(), 8, os.cpu_count() or 1)
    assert rc == 0
    worst = compare_limit_files(str(out), os.path.join(GOLDEN, "example1", "expected"), 1e-4, 1e-2, 1e-4)
    print("example1", worst)
    # the limit records print identically
    for kind in ("OAMASS", "ODAMPING"):
        ref = _load(os.path.join(GOLDEN, "example1", "expected", f"{kind}1.txt"))[:50]
        assert _load(out / f"{kind}1.txt")[:50] == ref
