"""Throughput of the per-frequency BEM build-and-solve on B200.

Workload: the 3 x 3 array of truncated cylinders (radius 4 m, draft 8 m,
20 m spacing, 600 quad panels each, 5,400 panels) in 50 m of water,
rho = 1025, g = 9.81, frequencies 0.2-2.5 rad/s (40), headings 0/30/60/90 deg
(54 radiation + 4 diffraction right-hand sides).  A step is one frequency:
Green functions and assembly of the 5,400 x 5,400 complex system, the LU
factorisation and solve, and the added-mass / damping / excitation
reductions.  Synthetic parametric mesh (no external data).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form surrogate|mixed|fp64]
  python bench.py --impl reference ...   # the CPU implementation on the host cores

The default form is the surrogate form (network far pairs, the Green
functions of identical body pairs computed once, complex64 panel LU on the
tensor cores with FP64 refinement); the mixed and fp64 forms run on the same
frequencies for the comparison and the error.  Each rank solves its own K
frequencies (weak scaling, no data-path collective); the timed region is the
max over ranks of the device time between two events on the library's
stream.  `e2e` repeats the main form through the C ABI from host buffers,
context set-up included.  Rank 0 prints one JSON line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "hams-mrel_b200"))

import meshgen  # noqa: E402

METRIC = "freq-solves/s @5.4k panels: surrogate+mixed vs plain FP64 GPU @≤1e-4 rel err"
UNIT = "freq-solves/s"
RHO, G = 1025.0, 9.81
LANES = 8  # frequencies in flight in hams_solve_batch (the library's default)
SG_FAR = 3.0  # surrogate pairs: centre distance beyond 3 source-panel sizes
# Frequencies the surrogate serves, by K = k0 h tanh(k0 h): on this array the
# damping below 0.26 rad/s (K < 0.3) and the excitation above 2.05 rad/s
# (K > 21.5, up to the first irregular frequency of the cylinders, 2.43 rad/s)
# are small differences of large terms that amplify the network's error past
# 1e-4; those frequencies keep the series.
SG_K_RANGE = (0.3, 21.5)


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return dict(json.load(f), source="of measured")
    except (OSError, ValueError):
        # an earlier measurement on this pool, used when the measured file is absent
        return {"bf16_tflops": 1590.0, "hbm_gbs": 6650.0, "source": "of fallback"}


PEAKS = _peaks()
WORKLOAD = "3x3 cylinder array R=4 T=8 spacing 20 m, 5400 quad panels, depth 50 m, 40 freq 0.2-2.5 rad/s, " \
           "headings 0/30/60/90 deg (54 rad + 4 dif RHS)"

# FP64 operations per EIGENE panel pair of the series Green kernel, from the
# executed-instruction counters of one ncu capture of that kernel on the
# 3,240-panel profiling case: dadd + dmul + 2 dfma
# (smsp__sass_thread_inst_executed_op_d*), and its DRAM bytes per pair
# (dram__bytes_read.sum + dram__bytes_write.sum over the launch's 4,093,706
# pairs), scaled to a full launch by its pair count
# (profiles/k_green_series_eigene_c2_array.md).
EIGENE_FP64_FLOPS_PER_PAIR = 44_410
EIGENE_DRAM_BYTES_PER_PAIR = 2_381
# DRAM bytes per pair of the surrogate kernel: ncu's dram__bytes_read.sum +
# dram__bytes_write.sum on the 3,240-panel profiling case (642.0 MB for
# 10,233,540 pairs), scaled to a full launch by its pair count
# (profiles/k_green_sg_c2_array.md)
SG_DRAM_BYTES_PER_PAIR = 62.73


# A coarser copy of the array (3,240 panels, 10.2 M far pairs) that profilers
# capture in full in a minute; never a bench line.
PROFILE_WORKLOAD = "3x3 cylinder array R=4 T=8 spacing 20 m, 9 x 360 quad panels (profiling case), depth 50 m"


def build_case(profile_case=False):
    if profile_case:
        bodies, centres = [], []
        for iy in range(3):
            for ix in range(3):
                bodies.append(meshgen.cylinder(4.0, 8.0, 30, 8, 4, 20.0 * ix, 20.0 * iy))
                centres.append((20.0 * ix, 20.0 * iy, 0.0))
        base = meshgen.case_c2()
        case = dict(base, name="c2-coarse", bodies=bodies, centres=centres)
        xyz, ncn, ncon, cnt = meshgen.combine(bodies)
        return case, xyz, ncn, ncon, cnt, np.array(centres, dtype=np.float64)
    case = meshgen.case_c2()
    xyz, ncn, ncon, cnt = meshgen.combine(case["bodies"])
    return case, xyz, ncn, ncon, cnt, np.array(case["centres"], dtype=np.float64)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.proc = None
        self.out = None
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(device).uuid)
            self.sel = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            self.sel = str(device)

    def start(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.sel, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.count(",") >= 8]
        self.out.close()
        os.unlink(self.out.name)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, smax, reasons = [], None, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------- CPU (oracle) timing
def cpu_sample_time(case, xyz, ncn, ncon, cnt, xr, omega, target_s=8.0, threads=None):
    """Seconds per frequency of the CPU implementation, from a bounded sample.

    Assembly: the oracle's OpenMP row assembly (every `stride`-th hull row,
    all host threads), scaled by n / rows.  LU and solve: LAPACK zgetrf /
    zgetrs (the reference calls the same routines through MKL) on the
    n x n system, or on a leading m x m block scaled by (n/m)^3 and (n/m)^2
    when the full factorisation would take longer than a few seconds.
    Force reductions (O(n * modes)) are left out; they are < 0.1 % of a step.
    """
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle_lib
    import scipy.linalg.lapack as lapack

    threads = threads or len(os.sched_getaffinity(0))
    oc = oracle_lib.Case(xyz, ncn, ncon, cnt, xr, case["depth"], rho=RHO, g=G)
    oc.opts.nthread = threads
    n = oc.n
    betas = np.radians(case["betas_deg"])
    w = oc.wave(omega)
    # calibrate the stride on a handful of rows, then time the sample
    stride = max(1, n // max(threads, 8))
    t = time.perf_counter()
    oc.assemble_rows(w, betas, stride, 0)
    t_probe = time.perf_counter() - t
    rows_probe = (n + stride - 1) // stride
    per_row = t_probe / rows_probe
    want = max(rows_probe, min(n, int(0.6 * target_s / max(per_row, 1e-9))))
    stride = max(1, n // want)
    t = time.perf_counter()
    a, _, _ = oc.assemble_rows(w, betas, stride, 1 % stride if stride > 1 else 0)
    t_rows = time.perf_counter() - t
    nr = a.shape[0]
    t_asm = t_rows * n / nr
    # LU + solve on a diagonally dominant complex matrix of the same size
    rng = np.random.default_rng(0)
    m = min(n, 1350)
    while True:
        mat = (rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))).astype(np.complex128)
        mat[np.diag_indices(m)] += 4.0 * np.sqrt(m)
        rhs = np.asfortranarray(rng.standard_normal((m, 58)) + 0j)
        mat = np.asfortranarray(mat)
        t = time.perf_counter()
        lu, piv, info = lapack.zgetrf(mat, overwrite_a=True)
        lapack.zgetrs(lu, piv, rhs, overwrite_b=True)
        t_lu = time.perf_counter() - t
        if m == n or t_lu * (n / m) ** 3 > 0.4 * target_s:
            break
        m = n if (n / m) ** 3 * t_lu < 0.25 * target_s else min(n, 2 * m)
    t_lin = t_lu * (n / m) ** 3
    sample = f"oracle assembly of {nr}/{n} rows (stride {stride}) x {n / nr:.1f}; LAPACK zgetrf+zgetrs " \
             f"(58 RHS) {m}x{m}" + (f" x (n/m)^3 = {(n / m) ** 3:.1f}" if m < n else "") + f"; omega={omega:.3f}"
    return t_asm + t_lin, threads, sample, dict(assembly_s=t_asm, lu_s=t_lin)


def reference_arm(args):
    """The CPU implementation of the path on the host cores (rank 0 only)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    case, xyz, ncn, ncon, cnt, xr = build_case()
    omegas = case["omegas"]
    per = []
    cores, sample = None, None
    for s in range(args.warmup + args.steps):
        om = omegas[s % len(omegas)]
        sec, cores, sample, _ = cpu_sample_time(case, xyz, ncn, ncon, cnt, xr, om,
                                                target_s=args.cpu_seconds or 3.0)
        if s >= args.warmup:
            per.append(sec)
    total = sum(per)
    value = len(per) / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(per),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": "cpu"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "per step: " + sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm
def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_form(hb, dev, geom, case, prec, omegas, betas, warmup, steps, barrier, want_results, sampler=None, sg=None,
             tol=0.0, blocks=0):
    """K frequencies through hams_solve_batch (frequencies in flight on several streams), timed
    between two events on the context's stream."""
    ctx = hb.Context(geom, case["depth"], rho=RHO, g=G, precision=prec, device=dev, refine_tol=tol,
                     body_blocks=blocks)
    if sg is not None:
        ctx.set_surrogate(sg, SG_FAR, SG_K_RANGE)
    waves = [hb.wave_properties(om, case["depth"], G) for om in omegas]
    if warmup:  # at least one frequency per lane, so that no lane is created inside the timed region
        ctx.solve_batch([waves[s % len(waves)] for s in range(max(warmup, LANES))], betas)
    barrier()
    if sampler:
        sampler.start()
    l0, lib0 = ctx.launch_count(), ctx.library_call_count()
    ctx.mark(0)
    res = ctx.solve_batch(waves[:steps], betas) if steps else None
    ctx.mark(1)
    ms = ctx.elapsed_ms(0, 1)
    launches, libcalls = ctx.launch_count() - l0, ctx.library_call_count() - lib0
    clocks = sampler.stop() if sampler else None
    tm = ctx.timings()  # the context's own last frequency
    barrier()
    ctx.close()
    results = [tuple(r[k] for r in res) for k in range(steps)] if (want_results and res is not None) else []
    return dict(ms=ms, launches=launches, lib_calls=libcalls, timings=tm, results=results, clocks=clocks)


def surrogate_kernel_time(hb, dev, geom, case, betas, sg, tol, blocks=0, reps=5):
    """Average duration of the surrogate kernel alone (one lane), CUDA events on its stream."""
    ctx = hb.Context(geom, case["depth"], rho=RHO, g=G, precision=hb.PREC_MIXED, device=dev, refine_tol=tol,
                     batch_lanes=1, body_blocks=blocks)
    ctx.set_surrogate(sg, SG_FAR, SG_K_RANGE)
    w = hb.wave_properties(1.2, case["depth"], G)
    ctx.solve_frequency(w, betas)
    ms, pairs = [], 0
    for _ in range(reps):
        ctx.solve_frequency(w, betas)
        t = ctx.timings()
        ms.append(t["green_surrogate"])
        pairs = t["pairs_surrogate"]
    ctx.close()
    return float(np.mean(ms)), int(pairs), None


def e2e_form(hb, dev, case, xyz, ncn, ncon, cnt, xr, prec, omegas, betas, steps, barrier, sg=None, tol=0.0,
             blocks=0):
    """Deck through the C ABI from host buffers: geometry, context, K frequencies."""
    import torch

    torch.cuda.synchronize()
    barrier()
    t = time.perf_counter()
    geom = hb.prepare_geometry(xyz, ncn, ncon, cnt, xr)
    ctx = hb.Context(geom, case["depth"], rho=RHO, g=G, precision=prec, device=dev, refine_tol=tol,
                     body_blocks=blocks)
    if sg is not None:
        ctx.set_surrogate(sg, SG_FAR, SG_K_RANGE)
    t1 = time.perf_counter()
    # the results are in host memory when solve_batch returns; freeing the context is not timed
    ctx.solve_batch([hb.wave_properties(omegas[s % len(omegas)], case["depth"], G) for s in range(steps)], betas)
    el = time.perf_counter() - t
    t2 = time.perf_counter()
    ctx.close()
    torch.cuda.synchronize()
    parts = {"setup_s": t1 - t, "solves_s": el - (t1 - t), "close_s_untimed": time.perf_counter() - t2}
    n, nb, ndof = ncn.size, cnt.size, 6 * cnt.size
    geom_bytes = xyz.nbytes + ncn.astype(np.int32).nbytes + 4 * 4 * n + 8 * (3 + 1 + 1 + 6) * n + 4 * nb
    wave_bytes = 8 * 205 + 8 * len(betas)
    sg_bytes = 4 * hb.surrogate_param_count() if sg is not None else 0
    h2d = (geom_bytes + sg_bytes) / steps + wave_bytes
    d2h = 8 * 2 * ndof * ndof + 16 * len(betas) * ndof
    return el, int(round(h2d)), int(d2h), parts


# forms: precision, surrogate on, dtype, refinement target, identical body
# blocks computed once.  The surrogate form's accuracy is set by the network
# (~1e-5 in the outputs), so its refinement stops at a relative residual of
# 1e-7; it also computes the Green functions of each of the 25 distinct
# (field, source) body blocks of the array once (hams_opts.body_blocks).  The
# plain forms compute every pair, as the reference does.
FORMS = {"surrogate": ("mixed", True, "f64 near + f16/f32 MLP far, c64 LU + f64 refinement", 1e-7, 1),
         "mixed": ("mixed", False, "f64, c64 LU + f64 refinement", 1e-12, 0),
         "fp64": ("fp64", False, "f64", 0.0, 0)}


def gpu_arm(args):
    import torch
    import torch.distributed as dist

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    import hams_b200 as hb
    import shard
    import train_surrogate

    def max_over_ranks(x):
        return shard.max_over_ranks(x, dist if ws > 1 else None, device="cuda")

    case, xyz, ncn, ncon, cnt, xr = build_case(args.profile_case)
    geom = hb.prepare_geometry(xyz, ncn, ncon, cnt, xr)
    betas = np.radians(case["betas_deg"])
    allom = case["omegas"]
    # weak scaling: the ws*K solves spread evenly over the sweep (cycling through it when ws*K
    # exceeds its 40 frequencies), rank r taking every ws-th, so that every K samples the whole range
    ntot = ws * args.steps
    pick = (lambda q: (q * len(allom)) // ntot) if ntot <= len(allom) else (lambda q: q % len(allom))
    om_rank = np.array([allom[pick(rank + ws * s)] for s in range(args.steps)])
    om_warm = np.array([allom[(s * 7 + 3) % len(allom)] for s in range(args.warmup)])
    sgp = train_surrogate.load()
    prec = {"mixed": hb.PREC_MIXED, "fp64": hb.PREC_FP64}

    def form_args(name):
        pr, on, _, tol, blocks = FORMS[name]
        return prec[pr], (sgp if on else None), tol, blocks

    sampler = ClockSampler(local)
    p_main, sg_main, tol_main, blk_main = form_args(args.form)
    run_form(hb, local, geom, case, p_main, np.concatenate([om_warm, om_rank]), betas, args.warmup, 0, barrier,
             False, sg=sg_main, tol=tol_main, blocks=blk_main)  # warm the library and caches on this deck
    runs = {args.form: run_form(hb, local, geom, case, p_main, om_rank, betas, args.warmup, args.steps, barrier, True,
                                sampler, sg=sg_main, tol=tol_main, blocks=blk_main)}
    # end to end through the C ABI right after the main form's timed batch, as a user's process would
    # run it (before the comparison forms below)
    e2e_s, h2d, d2h, e2e_parts = e2e_form(hb, local, case, xyz, ncn, ncon, cnt, xr, p_main, om_rank, betas, args.steps,
                               barrier, sg=sg_main, tol=tol_main, blocks=blk_main)
    e2e_s = max_over_ranks(e2e_s)
    for other in FORMS:
        if other != args.form and not args.only_form:
            pr, sg, tol, blocks = form_args(other)
            runs[other] = run_form(hb, local, geom, case, pr, om_rank, betas, args.warmup, args.steps, barrier, True,
                                   sg=sg, tol=tol, blocks=blocks)
    main = runs[args.form]
    ms = max_over_ranks(main["ms"])
    forms = {}
    for name, r in runs.items():
        v = ws * args.steps / (max_over_ranks(r["ms"]) * 1e-3)
        err = None
        if "fp64" in runs and name != "fp64":
            e = [max(rel(a[0], b[0]), rel(a[1], b[1]), rel(a[2], b[2])) for a, b in
                 zip(r["results"], runs["fp64"]["results"])]
            err = max_over_ranks(max(e))
            med = float(np.median(e))
        forms[name] = {"value": v, "rel_err_vs_fp64": err}
        if err is not None:
            forms[name]["rel_err_median"] = med

    value = ws * args.steps / (ms * 1e-3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": FORMS[args.form][2], "data": "synthetic",
            "config": {"workload": PROFILE_WORKLOAD if args.profile_case else WORKLOAD, "form": args.form,
                       "panels": int(ncn.size),
                       "rhs_per_step": 6 * int(cnt.size) + len(betas),
                       "l2": "no flush: the 5400x5400 complex system (0.47 GB) and pair tables exceed the 126 MB L2",
                       "parallelism": f"frequency shards x{ws}, {LANES} frequencies in flight per GPU",
                       "frequencies": "K solves per rank spread evenly over the 40-frequency sweep",
                       "surrogate": (f"far pairs beyond {SG_FAR} panel sizes, frequencies with K = k0 h tanh(k0 h) in "
                                     f"[{SG_K_RANGE[0]}, {SG_K_RANGE[1]}]") if sg_main is not None else None,
                       "body_blocks": ("Green functions of the 25 distinct (field body, source body) blocks of the "
                                       "81 computed, the others copied (identical translated cylinders)")
                                      if blk_main else None},
            "clocks": main["clocks"], "gpu_launches": main["launches"], "library_calls": main["lib_calls"],
            "e2e": {"value": ws * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "includes": "host geometry prep, context set-up (upload, Rankine tables, pair sort, surrogate "
                                "upload) and K frequency solves through the C ABI from host buffers",
                    "parts_rank0": {k: round(v, 4) for k, v in e2e_parts.items()}},
            "forms": forms}
    if "fp64" in forms and args.form != "fp64":
        line["speedup_vs_fp64"] = value / forms["fp64"]["value"]
        line["rel_err_vs_fp64"] = forms[args.form]["rel_err_vs_fp64"]
    tm = main["timings"]
    if sg_main is not None:
        # dominant kernel: the surrogate (tensor cores: 3 hidden 128 x 128 layers and the 16-row output
        # layer per pair), timed alone with CUDA events on one lane at a mid-range frequency
        flops = 2.0 * (3 * 128 * 128 + 128 * 16)
        sg_ms, sg_pairs, conc_ms = surrogate_kernel_time(hb, local, geom, case, betas, sg_main, tol_main, blk_main)
        ach = flops * sg_pairs / (sg_ms * 1e-3) / 1e12
        peak = PEAKS.get("bf16_tflops")
        line["roofline"] = {"kernel": "k_green_sg", "bound": "tensor", "unit": "TFLOP/s", "achieved": ach,
                            "peak": peak, "frac": ach / peak if peak else None, "traffic": SG_DRAM_BYTES_PER_PAIR * sg_pairs,
                            "peak_source": PEAKS["source"] + ": dense bf16 cuBLAS burst (MEASURED_PEAKS.json, else the "
                                           "pool's earlier 1,590 TFLOP/s); the kernel "
                                           "runs tcgen05.mma kind::f16 (FP16 operands, FP32 accumulation)",
                            "launch_ms": sg_ms,
                            "launch_ms_in_timed_region": tm["green_surrogate"] if tm["pairs_surrogate"] else None,
                            "pairs_per_launch": sg_pairs, "flops_per_pair": flops,
                            "timing": "mean of 5 launches on one lane (nothing else running), CUDA events on the "
                                      "launching stream"}
    else:
        eig_ms = tm["green_eigene"]
        peak = hb.measure_fp64_peak(local) if rank == 0 else None
        roof = {"kernel": "k_green_series<EIGENE>", "bound": "fp64", "unit": "TFLOP/s", "launch_ms": eig_ms,
                "pairs_per_launch": tm["pairs_eigene"], "peak": peak,
                "peak_source": "measured in this run: FP64 FMA loop on all SMs (no FP64 figure in "
                               "MEASURED_PEAKS.json)", "achieved": None, "frac": None,
                "traffic": EIGENE_DRAM_BYTES_PER_PAIR * tm["pairs_eigene"]}
        if EIGENE_FP64_FLOPS_PER_PAIR and peak and eig_ms > 0:
            ach = EIGENE_FP64_FLOPS_PER_PAIR * tm["pairs_eigene"] / (eig_ms * 1e-3) / 1e12
            roof.update(achieved=ach, frac=ach / peak, flops_per_pair=EIGENE_FP64_FLOPS_PER_PAIR)
        line["roofline"] = roof
    if rank == 0 and ws == 1 and not args.no_cpu:
        sec, cores, sample, parts = cpu_sample_time(case, xyz, ncn, ncon, cnt, xr, float(allom[len(allom) // 2]),
                                                    target_s=args.cpu_seconds or 8.0)
        line["cpu_baseline"] = {"value": 1.0 / sec, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                                **{k: round(v, 3) for k, v in parts.items()}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--form", choices=list(FORMS), default="surrogate")
    ap.add_argument("--only-form", action="store_true", help="time only --form (no fp64 / other forms beside it)")
    ap.add_argument("--cpu-seconds", type=float, default=None,
                    help="CPU work per baseline sample (default 8 s; 3 s per step of --impl reference)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--profile-case", action="store_true",
                    help="the coarser 3,240-panel array, for profiler captures (not a bench line)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
