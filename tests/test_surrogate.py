"""MLP surrogate of the far-field finite-depth Green function.

CPU: the FP64 reference network (oracle/mlp_ref.py) against finite
differences, and the shipped parameter file.  GPU (marked gpu): the
library's training gradient against the FP64 reference (relative 1e-4, FP32
accumulation), its training samples against the CPU oracle's FINGREEN3D
(1e-6 of the sample scale), the shipped network's accuracy on fresh samples,
and the surrogate form (the series judging each frequency) against the plain
series (relative 1e-4 in added mass, damping and excitation) together with
what the network saves.
"""
import os
import sys

import numpy as np
import pytest
import scipy.special as sp

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "hams-mrel_b200"))
import hams_b200  # noqa: E402
import meshgen  # noqa: E402
import mlp_ref  # noqa: E402
import oracle_lib  # noqa: E402
import train_surrogate  # noqa: E402


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def random_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    p = np.zeros(mlp_ref.count())
    off = 0
    for l in range(mlp_ref.LAYERS):
        fi, fo = mlp_ref.dims(l)
        p[off:off + fi * fo] = rng.uniform(-1, 1, fi * fo) * scale * np.sqrt(6.0 / (fi + fo))
        off += fi * fo
        p[off:off + fo] = rng.uniform(-0.1, 0.1, fo)
        off += fo
    p[off:off + 3] = [0.1, -0.2, 0.0]
    p[off + 3:off + 6] = [0.5, 0.3, 0.2]
    return p


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = random_params(1)
    x = rng.uniform(-1, 1, (4, 16))
    t = rng.normal(size=(3, 16))
    _, g = mlp_ref.loss_grad(p, x, t)
    for k in rng.choice(p.size - 6, 12, replace=False):
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (mlp_ref.loss_grad(p + e, x, t)[0] - mlp_ref.loss_grad(p - e, x, t)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-9


def test_shipped_parameters_load():
    p = train_surrogate.load()
    assert p.size == hams_b200.surrogate_param_count() == mlp_ref.count()
    assert np.all(np.isfinite(p))
    assert np.all(p[-3:] > 0)  # output scales


@pytest.mark.gpu
def test_training_gradient_matches_reference():
    rng = np.random.default_rng(5)
    p = random_params(2).astype(np.float32)
    x = rng.uniform(-1, 1, (4, 512)).astype(np.float32)
    t = rng.normal(size=(3, 512)).astype(np.float32)
    loss, g = hams_b200.surrogate_grad(p, x, t)
    rloss, rg = mlp_ref.loss_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - rloss) <= 1e-5 * rloss
    gw = rg[:-6]  # the output normalisation is not trained
    assert rel(g[:-6].astype(np.float64), gw) <= 1e-4


@pytest.mark.gpu
def test_training_samples_match_checker():
    raw = hams_b200.surrogate_samples(40, seed=7, nslice=64)
    h, g = 1.0, 9.807
    for X, Zq, Zp, K, t0, t1, t2 in raw:
        w = np.sqrt(K * g)
        ow = oracle_lib.OrcWave()
        oracle_lib.load().orc_wave_props(3, w, h, g, 0, oracle_lib.ctypes.byref(ow))
        wvn = np.array(ow.wvn)
        zq, zp = Zq - h, Zp - h
        G = oracle_lib.fingreen(X, 0.0, 0.0, 0.0, zq, zp, ow.v, wvn, h, 0)
        k = wvn[0]
        nm0 = h / 2 * (1 + np.sinh(2 * k * h) / (2 * k * h))
        p0 = np.pi / nm0 * np.cosh(k * Zq) * np.cosh(k * Zp)
        dp0 = np.pi / nm0 * np.sinh(k * Zq) * np.cosh(k * Zp)
        r0 = X * (G[0].real + p0 * sp.y0(k * X))
        r1 = X * X * (G[1].real - k * p0 * sp.y1(k * X))
        r2 = X * X * (G[3].real + k * dp0 * sp.y0(k * X))
        scale = max(1.0, abs(t0), abs(t1), abs(t2))
        assert abs(r0 - t0) <= 1e-6 * scale and abs(r1 - t1) <= 1e-6 * scale and abs(r2 - t2) <= 1e-6 * scale


@pytest.mark.gpu
def test_shipped_network_accuracy_on_fresh_samples():
    p = train_surrogate.load()
    raw = hams_b200.surrogate_samples(50_000, seed=2024, nslice=1024)
    t = hams_b200.surrogate_eval(p, raw[:, :4])
    for k in range(3):
        e = t[:, k] - raw[:, 4 + k]
        assert np.sqrt(np.mean(e ** 2) / np.mean(raw[:, 4 + k] ** 2)) < 2e-3
    # the library's FP32 evaluation against the FP64 reference network
    x = raw[:2000, :4]
    feats = np.stack([2 * np.log(x[:, 0] / 0.05) / np.log(3.0 / 0.05) - 1, 2 * (x[:, 1] - 0.5) / 0.5 - 1,
                      2 * (x[:, 2] - 0.5) / 0.5 - 1, 2 * np.log(x[:, 3] / 0.04) / np.log(40.0 / 0.04) - 1])
    y, _, _ = mlp_ref.forward(p.astype(np.float64), feats)
    _, mean, scale = mlp_ref.unpack(p)
    ref = (mean[:, None] + scale[:, None] * y).T
    assert rel(t[:2000], ref) < 1e-5


def _array_context(precision=hams_b200.PREC_FP64):
    bodies, centres = [], []
    for iy in range(3):
        for ix in range(3):
            bodies.append(meshgen.cylinder(4.0, 8.0, 20, 5, 3, 20.0 * ix, 20.0 * iy))
            centres.append((20.0 * ix, 20.0 * iy, 0.0))
    xyz, ncn, ncon, cnt = meshgen.combine(bodies)
    geom = hams_b200.prepare_geometry(xyz, ncn, ncon, cnt, np.array(centres))
    return hams_b200.Context(geom, 50.0, rho=1025.0, g=9.81, precision=precision)


@pytest.mark.gpu
def test_surrogate_assembly_against_series_and_gain():
    """3x3 array (9 x 160 panels) in 50 m: the surrogate replaces the series for the far pairs, the
    series judges each frequency (re-solving it above the 1e-4 bar), the outputs agree with the
    series to 1e-4, and the network's kernel takes less time than the series it replaces."""
    betas = np.radians([0.0, 45.0])
    ctx = _array_context()
    ref, series_ms = {}, {}
    for om in (0.5, 1.5):
        ref[om] = ctx.solve_frequency(hams_b200.wave_properties(om, 50.0, 9.81), betas)
        ctx.solve_frequency(hams_b200.wave_properties(om, 50.0, 9.81), betas)  # warm timing
        t = ctx.timings()
        series_ms[om] = t["green_eigene"] + t["green_eigen"]
    n_series = t["pairs_eigene"] + t["pairs_eigen"]
    # the surrogate form: mixed precision, the series judging each frequency
    mix = _array_context(hams_b200.PREC_MIXED)
    mix.set_surrogate(train_surrogate.load(), 3.0)
    mix.set_surrogate_tolerance(1e-4)
    kept = 0
    for om in (0.5, 1.5):
        mix.solve_frequency(hams_b200.wave_properties(om, 50.0, 9.81), betas)
        got = mix.solve_frequency(hams_b200.wave_properties(om, 50.0, 9.81), betas)
        t = mix.timings()
        assert t["judge_samples"] > 0 and t["judge_estimate"] > 0.0
        for a, b in zip(got, ref[om]):
            assert rel(a, b) < 1e-4
        if t["judge_resolved"]:
            assert t["judge_estimate"] > 1e-4 and "surrogate estimate" in mix.note()
            continue
        kept += 1
        assert t["pairs_surrogate"] > 0.5 * n_series
        # the series left for the near pairs plus the network cost less than the series alone
        assert t["green_surrogate"] + t["green_eigene"] + t["green_eigen"] < series_ms[om]
    assert kept >= 1
    mix.close()
    # a frequency outside the surrogate's K range keeps the series for every pair: the same bits
    # as the series path (K = 1.25 at 0.5 rad/s, 11.4 at 1.5 rad/s in 50 m)
    ctx.set_surrogate(train_surrogate.load(), 3.0, k_range=(2.0, 40.0))
    low = ctx.solve_frequency(hams_b200.wave_properties(0.5, 50.0, 9.81), betas)
    assert ctx.timings()["pairs_surrogate"] == 0
    for a, b in zip(low, ref[0.5]):
        assert np.array_equal(a, b)
    ctx.solve_frequency(hams_b200.wave_properties(1.5, 50.0, 9.81), betas)
    assert ctx.timings()["pairs_surrogate"] > 0.5 * n_series
    with pytest.raises(hams_b200.HamsError):
        ctx.set_surrogate(train_surrogate.load(), 3.0, k_range=(0.01, 40.0))
    # switched off, the plain series path gives the same bits again
    ctx.set_surrogate(None)
    again = ctx.solve_frequency(hams_b200.wave_properties(1.5, 50.0, 9.81), betas)
    for a, b in zip(again, ref[1.5]):
        assert np.array_equal(a, b)
    ctx.close()


@pytest.mark.gpu
def test_series_takes_back_a_frequency_without_refactoring():
    """A frequency the judgement gives back to the series: the far pairs again from the series, then
    refinement from the network's solution with the network's factors.  The outputs are the series'
    (the mixed form without the network, refined to the same tolerance) to 1e-6, and the library
    says which way it went."""
    betas = np.radians([0.0, 45.0])
    plain = _array_context(hams_b200.PREC_MIXED)
    mix = _array_context(hams_b200.PREC_MIXED)
    mix.set_surrogate(train_surrogate.load(), 3.0)
    mix.set_surrogate_tolerance(1e-12)  # every frequency goes back to the series
    for om in (0.5, 1.5, 2.3):
        w = hams_b200.wave_properties(om, 50.0, 9.81)
        ref = plain.solve_frequency(w, betas)
        got = mix.solve_frequency(w, betas)
        t = mix.timings()
        assert t["judge_resolved"] and t["pairs_surrogate"] > 0
        assert "refined to the series" in mix.note()
        for a, b in zip(got, ref):
            assert rel(a, b) < 1e-6
    # a batch takes the same way frequency by frequency
    ws = [hams_b200.wave_properties(om, 50.0, 9.81) for om in (0.5, 1.5, 2.3)]
    ra = plain.solve_batch(ws, betas)
    rb = mix.solve_batch(ws, betas)
    for a, b in zip(rb, ra):
        assert rel(a, b) < 1e-6
    assert mix.note().count("refined to the series") == 3
    plain.close()
    mix.close()
