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
tensor cores with FP64 refinement); the surrogate form without body blocks,
the mixed form and the fp64 form with and without body blocks run on the
same frequencies for the like-for-like comparison and the error.  Each rank solves its own K
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

import hams_b200  # noqa: E402
import meshgen  # noqa: E402

METRIC = "freq-solves/s @5.4k panels: surrogate+mixed vs plain FP64 GPU @≤1e-4 rel err"
UNIT = "freq-solves/s"
RHO, G = 1025.0, 9.81
LANES = 8  # frequencies in flight in hams_solve_batch (the library's default)
SG_FAR = hams_b200.SURROGATE_FAR  # surrogate pairs: centre distance beyond 3 source-panel sizes
SG_K_RANGE = hams_b200.SURROGATE_K_RANGE  # the network's whole domain
SG_TOL = hams_b200.SURROGATE_TOL  # the series judges each frequency against this bar


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
# 3,240-panel profiling case (`--profile-case --form fp64`): dadd + dmul +
# 2 dfma (smsp__sass_thread_inst_executed_op_d*), and its DRAM bytes per pair
# (dram__bytes_read.sum + dram__bytes_write.sum over the launch's 4,093,706
# pairs), scaled to a full launch by its pair count.
EIGENE_FP64_FLOPS_PER_PAIR = 44_410
EIGENE_DRAM_BYTES_PER_PAIR = 2_381
# DRAM bytes per pair of the surrogate kernel: ncu's dram__bytes_read.sum +
# dram__bytes_write.sum on the 3,240-panel profiling case with identical body
# blocks (125.5 MB for 3,210,660 pairs), scaled to a full launch by its pair
# count.
SG_DRAM_BYTES_PER_PAIR = 39.10


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
def oracle_for_timing():
    """The oracle, built for this host's cores (-O3 -march=native) in a
    temporary directory, for the timed CPU legs; the portable build if that
    fails.  Returns (module, build description)."""
    if not os.environ.get("HAMS_ORACLE_SO"):
        out = os.path.join(tempfile.mkdtemp(prefix="hams_oracle_"), "libhams_oracle_native.so")
        r = subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "native", f"NATIVE_OUT={out}"],
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        if r.returncode == 0 and os.path.exists(out):
            os.environ["HAMS_ORACLE_SO"] = out
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle_lib

    native = bool(os.environ.get("HAMS_ORACLE_SO"))
    return oracle_lib, ("gcc -O3 -march=native -fopenmp" if native else "gcc -O3 -fopenmp (portable build)")


def cpu_frequency(oc, omega, betas, threads):
    """One frequency solved on the host cores, every part of it run in full:
    the oracle's OpenMP assembly of all rows of the system (the reference's
    CALGREEN_MULTI, BODINT_MULTI_LEFT, ASSB_LEFT_MULTI, ASSB_RBC_MULTI and
    ASSB_DBC_MULTI), LAPACK zgetrf / zgetrs on that assembled system (the
    routines RADIATION_SOLVER_MULTI and DIFFRACTION_SOLVER_MULTI call through
    MKL; OpenBLAS here) and the oracle's force reductions (RFORCE_MULTI,
    EFORCE_MULTI).  Returns seconds and the split."""
    import scipy.linalg.lapack as lapack

    oc.opts.nthread = threads
    t0 = time.perf_counter()
    w = oc.wave(omega)
    a, b, d = oc.assemble(w, betas)
    t1 = time.perf_counter()
    n, nsys = oc.n, oc.geom.nsys
    xr = np.zeros_like(b)
    xd = np.zeros_like(d)
    for ip in range(nsys):
        lu, piv, info = lapack.zgetrf(a[:, :, ip], overwrite_a=True)
        xr[:, :, ip] = lapack.zgetrs(lu, piv, b[:, :, ip])[0]
        xd[:, ip, :] = lapack.zgetrs(lu, piv, d[:, ip, :])[0]
    t2 = time.perf_counter()
    oc.forces(w, betas, xr, xd)
    t3 = time.perf_counter()
    return t3 - t0, dict(assembly_s=t1 - t0, lu_s=t2 - t1, forces_s=t3 - t2)


def cpu_case(case, xyz, ncn, ncon, cnt, xr):
    orc, build = oracle_for_timing()
    oc = orc.Case(xyz, ncn, ncon, cnt, xr, case["depth"], rho=RHO, g=G)
    return oc, build


def reference_arm(args):
    """The CPU implementation of the path on the host cores (rank 0 only):
    whole frequencies, nothing scaled.  A step is one frequency of the
    sweep; as many of the K steps run as fit --cpu-seconds (at least two),
    and the line's `steps` is the number that ran."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    case, xyz, ncn, ncon, cnt, xr = build_case()
    oc, build = cpu_case(case, xyz, ncn, ncon, cnt, xr)
    threads = len(os.sched_getaffinity(0))
    betas = np.radians(case["betas_deg"])
    omegas = case["omegas"]
    budget = args.cpu_seconds or 120.0
    per, parts, om_run = [], [], []
    t_start = time.perf_counter()
    # the sweep in an order whose every prefix is spread over the whole range (the
    # GPU arm's K steps are spread over it too): 0, 1/2, 1/4, 3/4, 1/8, ... of the sweep
    order, seen = [], set()
    for d in range(12):
        for q in range(2 ** max(d - 1, 0)):
            k = ((2 * q + 1) * len(omegas)) // 2 ** d if d else 0
            if k not in seen and k < len(omegas):
                seen.add(k)
                order.append(k)
    order += [k for k in range(len(omegas)) if k not in seen]
    for s in range(args.steps):
        om = float(omegas[order[s % len(order)]])
        sec, part = cpu_frequency(oc, om, betas, threads)
        per.append(sec)
        parts.append(part)
        om_run.append(round(om, 4))
        elapsed = time.perf_counter() - t_start
        if len(per) >= 2 and elapsed + sec > budget:
            break
    total = sum(per)
    value = len(per) / total
    mean = {k: round(float(np.mean([p[k] for p in parts])), 3) for k in parts[0]}
    sample = (f"{len(per)} whole frequencies ({', '.join(map(str, om_run))} rad/s) of the {len(omegas)}-frequency "
              f"sweep, each fully assembled ({oc.n} x {oc.n}), factored and reduced; oracle {build}, "
              f"LAPACK zgetrf/zgetrs (OpenBLAS); no warm-up (no compilation or caches to warm on the host)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(per), "steps_requested": args.steps, "warmup": 0, "ms_per_step": 1e3 * total / len(per),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": "cpu"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             **mean},
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
        ctx.set_surrogate_tolerance(SG_TOL)
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
    resolved = ctx.note().count("surrogate estimate")  # frequencies the series judgement took back
    barrier()
    ctx.close()
    results = [tuple(r[k] for r in res) for k in range(steps)] if (want_results and res is not None) else []
    return dict(ms=ms, launches=launches, lib_calls=libcalls, timings=tm, results=results, clocks=clocks,
                resolved=resolved)


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
        ctx.set_surrogate_tolerance(SG_TOL)
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
# 1e-7; the mixed form refines to 1e-12.  Body blocks (the Green functions of
# each of the 25 distinct (field, source) body blocks of the array computed
# once, hams_opts.body_blocks) are an exact geometric reuse that any form can
# use, so the surrogate and fp64 forms run both with and without them and the
# speed-ups are reported like for like.
FORMS = {"surrogate": ("mixed", True, "f64 near + f16/f32 MLP far, c64 LU + f64 refinement", 1e-7, 1),
         "surrogate_noblocks": ("mixed", True, "f64 near + f16/f32 MLP far, c64 LU + f64 refinement", 1e-7, 0),
         "mixed": ("mixed", False, "f64, c64 LU + f64 refinement", 1e-12, 0),
         "fp64": ("fp64", False, "f64", 0.0, 0),
         "fp64_blocks": ("fp64", False, "f64", 0.0, 1)}
# the plain drop-in each form is compared with, like for like (body blocks on or off)
PLAIN_OF = {"surrogate": "fp64_blocks", "surrogate_noblocks": "fp64", "mixed": "fp64", "fp64_blocks": "fp64"}


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
        pr, on, _, tol, blocks = FORMS[name]
        forms[name] = {"value": v, "precision": pr, "surrogate": on, "body_blocks": bool(blocks),
                       "refine_tol": tol if pr == "mixed" else None, "rel_err_vs_fp64": None}
        if on:
            forms[name]["resolved_with_series"] = f"{r['resolved']} of {args.steps}"
        if "fp64" in runs and name != "fp64":
            # worst of the relative Frobenius errors of added mass, damping and excitation against the
            # plain fp64 form (every pair computed), per frequency
            e = [[rel(a[k], b[k]) for k in range(3)] for a, b in zip(r["results"], runs["fp64"]["results"])]
            worst = [max(x) for x in e]
            forms[name].update(rel_err_vs_fp64=max_over_ranks(max(worst)), rel_err_median=float(np.median(worst)),
                               rel_err_amas_bdmp_exfc=[max_over_ranks(max(x[k] for x in e)) for k in range(3)])

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
                       "surrogate": (f"far pairs beyond {SG_FAR} panel sizes over the network's K = k0 h tanh(k0 h) "
                                     f"domain [{SG_K_RANGE[0]}, {SG_K_RANGE[1]}]; each frequency judged by the series "
                                     f"(sampled far pairs, error model carried through the solve); above {SG_TOL:g} the series "
                                     f"takes it back: far pairs from the series, refined from the network's solution "
                                     f"with the network's factors") if sg_main is not None else None,
                       "body_blocks": ("Green functions of the 25 distinct (field body, source body) blocks of the "
                                       "81 computed, the others copied (identical translated cylinders)")
                                      if blk_main else None},
            "clocks": main["clocks"], "gpu_launches": main["launches"], "library_calls": main["lib_calls"],
            "e2e": {"value": ws * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "includes": "host geometry prep, context set-up (upload, Rankine tables, pair sort, surrogate "
                                "upload; device buffers, streams and library handles from the library's caches, "
                                "which the timed context destroyed before left) and K frequency solves through "
                                "the C ABI from host buffers",
                    "parts_rank0": {k: round(v, 4) for k, v in e2e_parts.items()}},
            "forms": forms}
    if "fp64" in forms and args.form != "fp64":
        sp = {}
        for name, plain in (("surrogate", "fp64_blocks"), ("surrogate_noblocks", "fp64")):
            if name in forms and plain in forms:
                sp[f"{name}_vs_{plain}"] = forms[name]["value"] / forms[plain]["value"]
        sp["headline_form_vs_plain_fp64"] = value / forms["fp64"]["value"]
        sp["note"] = ("like for like: body blocks on against on, off against off; the blocks-off ratio is the "
                      "speed-up of the network and the tensor-core solve alone")
        line["speedup_vs_fp64"] = sp
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
        # one whole frequency of the same workload on the host cores (about 15 s), nothing scaled
        oc, build = cpu_case(case, xyz, ncn, ncon, cnt, xr)
        cores = len(os.sched_getaffinity(0))
        om = float(allom[len(allom) // 2])
        sec, parts = cpu_frequency(oc, om, betas, cores)
        line["cpu_baseline"] = {"value": 1.0 / sec, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"one whole frequency (omega = {om:.3f} rad/s, {oc.n} x {oc.n} system "
                                          f"fully assembled, factored and reduced); oracle {build}, LAPACK "
                                          f"zgetrf/zgetrs (OpenBLAS)",
                                **{k: round(v, 3) for k, v in parts.items()}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def c3_arm(args):
    """The batched heterogeneous workload: the 128 seeded single / two-body cases
    (cylinders or boxes of 200-3000 panels each, half with water-plane lids,
    finite or infinite depth), 16 frequencies each, in the mixed form.  Cases
    run on a pool of host threads (largest first), each case's frequencies in
    flight on its context's lanes; the tile variants of the block LU's GEMMs
    come from the library's autotuner.  Timed from the first context to the
    last result (wall clock around a device synchronisation: the work spans
    many contexts and streams), geometry preparation included."""
    import threading

    import torch

    import hams_b200 as hb

    torch.cuda.set_device(0)
    cases = []
    for seed in range(128):
        c = meshgen.case_c3(seed)
        xyz, ncn, ncon, cnt = meshgen.combine(c["bodies"])
        xr = np.array(c["centres"], dtype=np.float64)
        lid = None
        if c["lids"]:
            lid = meshgen.combine(c["lids"])
        cases.append((c, xyz, ncn, ncon, cnt, xr, lid, int(ncn.size) + (int(lid[1].size) if lid else 0)))
    order = sorted(range(len(cases)), key=lambda k: -cases[k][-1])

    def solve_case(k):
        c, xyz, ncn, ncon, cnt, xr, lid, _ = cases[k]
        geom = hb.prepare_geometry(xyz, ncn, ncon, cnt, xr)
        irsp = 0
        if lid:
            lg = hb.prepare_geometry(lid[0], lid[1], lid[2], lid[3], xr)
            geom = dict(geom, ixyz_p=lg["xyz_p"])
            irsp = 1
        ctx = hb.Context(geom, c["depth"], rho=RHO, g=G, irsp=irsp, precision=hb.PREC_MIXED)
        waves = [hb.wave_properties(float(om), c["depth"], G) for om in c["omegas"]]
        res = ctx.solve_batch(waves, np.radians(c["betas_deg"]))
        ctx.close()
        return res

    solve_case(order[-1])  # load the library, tune the smallest case's GEMM classes
    torch.cuda.synchronize()
    nxt = [0]
    lock = threading.Lock()
    failures = []

    def worker():
        while True:
            with lock:
                if nxt[0] >= len(order):
                    return
                k = order[nxt[0]]
                nxt[0] += 1
            try:
                res = solve_case(k)
                if not all(np.all(np.isfinite(r)) for r in res):
                    failures.append(f"case {k}: non-finite result")
            except Exception as e:  # noqa: BLE001
                failures.append(f"case {k}: {e}")

    sampler = ClockSampler(0)
    sampler.start()
    t0 = time.perf_counter()
    th = [threading.Thread(target=worker) for _ in range(args.c3_workers)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    clocks = sampler.stop()
    nsolve = sum(len(c[0]["omegas"]) for c in cases)
    line = {"metric": "freq-solves/s, 128 heterogeneous seeded cases (one or two bodies, 220-5,757 panels)", "value": nsolve / el,
            "unit": UNIT, "n_gpus": 1, "steps": nsolve, "warmup": 1, "ms_per_step": 1e3 * el / nsolve,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 assembly, c64 LU + f64 refinement",
            "data": "synthetic",
            "config": {"workload": "128 seeded single/two-body cases (cylinders R U[2,8] T U[3,12] or boxes, 200-3000 "
                                   "panels per body, half with water-plane lids, depth infinite or U[30,200] m), 16 "
                                   "frequencies 0.1-3 rad/s, heading 0", "form": "mixed",
                       "panels": [min(c[-1] for c in cases), max(c[-1] for c in cases)],
                       "parallelism": f"{args.c3_workers} cases at a time, each case's frequencies on its lanes",
                       "timing": "wall clock from the first context to the last result, device synchronised; "
                                 "geometry preparation and context set-up included"},
            "clocks": clocks, "failures": failures[:5]}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--form", choices=list(FORMS), default="surrogate")
    ap.add_argument("--only-form", action="store_true", help="time only --form (no fp64 / other forms beside it)")
    ap.add_argument("--cpu-seconds", type=float, default=None,
                    help="time budget of --impl reference (default 120 s; at least two whole frequencies run)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--profile-case", action="store_true",
                    help="the coarser 3,240-panel array, for profiler captures (not a bench line)")
    ap.add_argument("--workload", choices=["c2", "c3"], default="c2",
                    help="c3: the 128 heterogeneous cases of the batched form (its own line)")
    ap.add_argument("--c3-workers", type=int, default=4, help="cases in flight at once (--workload c3)")
    args = ap.parse_args()
    if args.workload == "c3" and args.impl != "reference":
        c3_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
