"""CPU checks of the product library: exported C ABI and host-side logic.

No CUDA device is needed: libhams_b200.so loads on a CPU-only machine and its
host functions (wave properties / dispersion roots) run without a GPU.
"""
import ctypes
import os
import re
import sys

import numpy as np
import pytest

import oracle_lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "hams-mrel_b200"))
import hams_b200  # noqa: E402


def declared_functions():
    text = open(os.path.join(REPO, "include", "hams_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hams_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = hams_b200.load_library()
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name


@pytest.mark.parametrize("inft,value,depth", [(3, 0.05, 70.0), (3, 1.0, 50.0), (3, 2.5, 50.0), (4, 0.5, 14.5),
                                              (2, 0.3, 30.0), (1, 0.2, 40.0), (5, 60.0, 25.0), (3, 1.3, -1.0)])
def test_wave_properties_bit_identical_to_checker(inft, value, depth):
    """CalWaveProperts/DISPERSION on the product side give the checker's roots bit for bit:
    the epsilon-accelerated Green series would amplify any last-bit difference."""
    w = hams_b200.wave_properties(value, depth, 9.80665, inft=inft)
    ow = oracle_lib.OrcWave()
    oracle_lib.load().orc_wave_props(inft, value, depth, 9.80665, 0, ctypes.byref(ow))
    for k in ("v", "wk", "w1"):
        assert getattr(w, k) == getattr(ow, k), k
    if depth > 0:
        assert np.array_equal(np.array(w.wvn), np.array(ow.wvn))


def test_wave_properties_limits_and_errors():
    z = hams_b200.wave_properties(1.0, 50.0, sybo_kk=1)
    assert z.v == 0.0 and z.w1 == 0.0 and z.tp == -1.0
    inf = hams_b200.wave_properties(1.0, 50.0, sybo_kk=2)
    assert inf.v == -1.0 and inf.wk == -1.0
    with pytest.raises(hams_b200.HamsError):
        hams_b200.wave_properties(-1.0, 50.0)
    with pytest.raises(hams_b200.HamsError):
        hams_b200.wave_properties(1.0, 50.0, inft=9)


@pytest.mark.parametrize("deck", ["config1", "example5"])
def test_prepare_geometry_matches_checker(deck):
    d = oracle_lib.load_deck(os.path.join(REPO, "tests", "golden", deck, "input"))
    g = hams_b200.prepare_geometry(d["xyz"], d["ncn"], d["ncon"], d["body_nelem"], d["xr"])
    for k in ("xyz_p", "ds", "pnsz"):
        assert np.array_equal(g[k], d[k]), k
    # generalized-mode files would override dxyz; these decks have none
    assert np.array_equal(g["dxyz"], d["dxyz"])


def test_prepare_geometry_rejects_bad_connectivity():
    xyz = np.zeros((4, 3))
    with pytest.raises(hams_b200.HamsError):
        hams_b200.prepare_geometry(xyz, [4], [[1, 2, 3, 9]], [1], [[0, 0, 0]])
