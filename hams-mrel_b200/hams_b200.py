"""Python binding of the B200 per-frequency BEM library (libhams_b200.so).

Mirrors the per-frequency operator calls of HAMS-MREL's frequency loop
(src/HAMS_Prog.f90:613-733): CalWaveProperts -> ``wave_properties``;
CALGREEN_MULTI + ASSB_* + *_SOLVER_MULTI + RFORCE/EFORCE_MULTI ->
``Context.solve_frequency``.  Arrays follow the reference's Fortran module
arrays (column-major, 1-based connectivity).  The CUDA library is required:
importing this module on a machine without it raises, there is no CPU
fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhams_b200.so")

HAMS_NK = 200
PREC_FP64 = 0
PREC_MIXED = 1
LU_BLOCK_TF32, LU_BLOCK_EMU, LU_LIBRARY = 0, 1, 2
SOLVER_LU, SOLVER_GMRES = 1, 2
# The surrogate form's defaults: network for pairs farther apart than 3 source-panel sizes, over
# the network's whole K = k0 h tanh(k0 h) domain, each frequency judged by the series against the
# 1e-4 bar (hams_ctx_set_surrogate_tolerance) and taken back by the series above it.
SURROGATE_FAR = 3.0
SURROGATE_K_RANGE = (0.04, 40.0)
SURROGATE_TOL = 1e-4

c_int = ctypes.c_int32
c_dbl = ctypes.c_double
P_dbl = ctypes.POINTER(ctypes.c_double)
P_int = ctypes.POINTER(ctypes.c_int32)


class HamsGeom(ctypes.Structure):
    _fields_ = [("nelem", c_int), ("ntnd", c_int), ("nbody", c_int), ("isx", c_int), ("isy", c_int),
                ("xyz", P_dbl), ("ncn", P_int), ("ncon", P_int), ("xyz_p", P_dbl), ("ds", P_dbl), ("pnsz", P_dbl),
                ("dxyz", P_dbl), ("body_nelem", P_int), ("inelem", c_int), ("ixyz_p", P_dbl)]


class HamsOpts(ctypes.Structure):
    _fields_ = [("depth", c_dbl), ("rho", c_dbl), ("g", c_dbl), ("xw", c_dbl * 2), ("amp", c_dbl), ("isol", c_int),
                ("irsp", c_int), ("precision", c_int), ("device", c_int), ("refine_tol", c_dbl),
                ("refine_max", c_int), ("lu_kind", c_int), ("batch_lanes", c_int),
                ("solver", c_int), ("gmres_restart", c_int), ("gmres_maxit", c_int), ("gmres_tol", c_dbl),
                ("aca_tol", c_dbl), ("gmres_dense", c_int), ("body_blocks", c_int), ("lu_graph", c_int), ("reserved", c_int)]


class HamsWave(ctypes.Structure):
    _fields_ = [("v", c_dbl), ("wk", c_dbl), ("w1", c_dbl), ("tp", c_dbl), ("wl", c_dbl), ("wvn", c_dbl * HAMS_NK)]


class SgTrain(ctypes.Structure):
    _fields_ = [("n_train", c_int), ("n_test", c_int), ("batch", c_int), ("steps", c_int), ("nslice", c_int),
                ("reserved0", c_int), ("seed", ctypes.c_uint64), ("lr", c_dbl), ("reserved", c_dbl * 4)]


class HamsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hams error {code}: {msg}")
        self.code = code


_LIB = None


def load_library(path=LIB_PATH):
    """Load libhams_b200.so (raises OSError if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with `make -C {os.path.dirname(path)}`")
    lib = ctypes.CDLL(path)
    lib.hams_wave_properties.argtypes = [c_int, c_dbl, c_dbl, c_dbl, c_int, ctypes.POINTER(HamsWave)]
    lib.hams_ctx_create.argtypes = [ctypes.POINTER(HamsGeom), ctypes.POINTER(HamsOpts), ctypes.POINTER(ctypes.c_void_p)]
    lib.hams_ctx_destroy.argtypes = [ctypes.c_void_p]
    lib.hams_release_cached.argtypes = []
    lib.hams_release_cached.restype = None
    lib.hams_solve_frequency.argtypes = [ctypes.c_void_p, ctypes.POINTER(HamsWave), c_int, P_dbl, P_dbl, P_dbl, P_dbl]
    lib.hams_solve_batch.argtypes = [ctypes.c_void_p, c_int, ctypes.POINTER(HamsWave), c_int, P_dbl, P_dbl, P_dbl,
                                     P_dbl]
    lib.hams_assemble.argtypes = [ctypes.c_void_p, ctypes.POINTER(HamsWave), c_int, P_dbl, P_dbl, P_dbl, P_dbl]
    lib.hams_eval_green.argtypes = [ctypes.c_void_p, ctypes.POINTER(HamsWave), c_int, P_dbl, P_int, P_dbl]
    lib.hams_last_timings.argtypes = [ctypes.c_void_p, P_dbl, c_int]
    lib.hams_launch_count.argtypes = [ctypes.c_void_p]
    lib.hams_launch_count.restype = ctypes.c_int64
    lib.hams_last_error.restype = ctypes.c_char_p
    lib.hams_last_note.argtypes = [ctypes.c_void_p]
    lib.hams_last_note.restype = ctypes.c_char_p
    lib.hams_library_call_count.argtypes = [ctypes.c_void_p]
    lib.hams_library_call_count.restype = ctypes.c_int64
    lib.hams_mark.argtypes = [ctypes.c_void_p, c_int]
    lib.hams_mark_elapsed.argtypes = [ctypes.c_void_p, c_int, c_int, P_dbl]
    lib.hams_measure_fp64_peak.argtypes = [c_int, P_dbl]
    lib.hams_body_blocks.argtypes = [ctypes.POINTER(HamsGeom), c_dbl, P_int]
    lib.hams_prepare_geometry.argtypes = [c_int, P_dbl, c_int, P_int, P_int, c_int, P_int, P_dbl, P_dbl, P_dbl, P_dbl,
                                          P_dbl]
    P_flt = ctypes.POINTER(ctypes.c_float)
    lib.hams_surrogate_param_count.restype = c_int
    lib.hams_ctx_set_surrogate.argtypes = [ctypes.c_void_p, P_flt, c_int, c_dbl]
    lib.hams_ctx_set_surrogate_range.argtypes = [ctypes.c_void_p, c_dbl, c_dbl]
    lib.hams_ctx_set_surrogate_tolerance.argtypes = [ctypes.c_void_p, c_dbl]
    lib.hams_ctx_set_field_points.argtypes = [ctypes.c_void_p, c_int, P_dbl]
    lib.hams_field_potentials.argtypes = [ctypes.c_void_p, c_int, P_dbl]
    lib.hams_surrogate_samples.argtypes = [c_int, c_int, ctypes.c_uint64, c_int, P_dbl]
    lib.hams_surrogate_train.argtypes = [c_int, ctypes.POINTER(SgTrain), P_flt, P_dbl]
    lib.hams_surrogate_eval.argtypes = [c_int, P_flt, c_int, P_dbl, P_dbl]
    lib.hams_surrogate_grad.argtypes = [c_int, P_flt, c_int, P_flt, P_flt, P_dbl, P_flt]
    lib.hams_diag_gemm_tf32.argtypes = [c_int, c_int, c_int, c_int, ctypes.c_float, P_flt, c_int, P_flt, c_int,
                                        ctypes.c_float, P_flt, c_int, c_int, c_int]
    lib.hams_diag_gemm_tf32_time.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int, P_dbl]
    _LIB = lib
    return lib


def _check(rc, allow_pivot=False):
    if rc < 0 or (rc > 0 and not allow_pivot):
        msg = load_library().hams_last_error().decode()
        raise HamsError(rc, msg or ("singular pivot %d" % rc))
    return rc


def _d(a):
    return a.ctypes.data_as(P_dbl)


def _i(a):
    return a.ctypes.data_as(P_int)


def wave_properties(value, depth, g=9.80665, inft=3, sybo_kk=0):
    """CalWaveProperts for one input value (inft: 1 V, 2 k, 3 omega, 4 T, 5 lambda)."""
    w = HamsWave()
    _check(load_library().hams_wave_properties(inft, float(value), float(depth), float(g), sybo_kk, ctypes.byref(w)))
    return w


def prepare_geometry(xyz, ncn, ncon, body_nelem, xr):
    """CalNormals[Multi]: panel centres, areas, sizes and generalized normals from the nodes.

    Returns a geometry dict ready for Context (arrays in Fortran order).
    """
    xyz = np.asfortranarray(xyz, dtype=np.float64)
    ncn = np.ascontiguousarray(ncn, dtype=np.int32)
    ncon = np.asfortranarray(ncon, dtype=np.int32)
    bn = np.ascontiguousarray(body_nelem, dtype=np.int32)
    xr = np.asfortranarray(np.asarray(xr, dtype=np.float64).reshape(len(bn), 3))
    n = ncn.size
    xyz_p, ds, pnsz, dxyz = np.zeros((n, 3), order="F"), np.zeros(n), np.zeros(n), np.zeros((n, 6), order="F")
    _check(load_library().hams_prepare_geometry(xyz.shape[0], _d(xyz), n, _i(ncn), _i(ncon), bn.size, _i(bn), _d(xr),
                                                _d(xyz_p), _d(ds), _d(pnsz), _d(dxyz)))
    return dict(xyz=xyz, ncn=ncn, ncon=ncon, xyz_p=xyz_p, ds=ds, pnsz=pnsz, dxyz=dxyz, body_nelem=bn)


def body_blocks(geom, tol=1e-9):
    """Blocks of identical body pairs (hams_body_blocks): rep (nbody, nbody), rep[b1, b2] = the
    column-major index b1' + nbody b2' of the block that (field b1, source b2) copies (its own
    index when computed in full), and the number of distinct blocks."""
    lib = load_library()
    keep = {k: np.asfortranarray(geom[k], dtype=np.int32 if k in ("ncn", "ncon", "body_nelem") else np.float64)
            for k in ("xyz", "ncn", "ncon", "xyz_p", "ds", "pnsz", "dxyz", "body_nelem")}
    nb = keep["body_nelem"].size
    g = HamsGeom(nelem=keep["ncn"].size, ntnd=keep["xyz"].shape[0], nbody=nb, xyz=_d(keep["xyz"]),
                 ncn=_i(keep["ncn"]), ncon=_i(keep["ncon"]), xyz_p=_d(keep["xyz_p"]), ds=_d(keep["ds"]),
                 pnsz=_d(keep["pnsz"]), dxyz=_d(keep["dxyz"]), body_nelem=_i(keep["body_nelem"]),
                 inelem=int(len(geom.get("ixyz_p", ()))), ixyz_p=None)
    rep = np.zeros((nb, nb), dtype=np.int32, order="F")
    distinct = lib.hams_body_blocks(ctypes.byref(g), float(tol), _i(rep))
    if distinct < 0:
        raise HamsError(distinct, "hams_body_blocks: null argument")
    return rep, distinct


class Context:
    """Device-resident geometry of one deck; solves frequencies on one GPU.

    geom: dict with xyz (ntnd,3), ncn (n), ncon (n,4) 1-based, xyz_p (n,3),
    ds (n), pnsz (n), dxyz (n,6), body_nelem (nb) and, for irsp=1, ixyz_p.
    """

    def __init__(self, geom, depth, rho=1000.0, g=9.80665, isol=1, irsp=0, precision=PREC_FP64, device=0,
                 xw=(0.0, 0.0), amp=1.0, refine_tol=0.0, refine_max=0, lu_kind=0,
                 batch_lanes=0, solver=SOLVER_LU, gmres_restart=0, gmres_maxit=0, gmres_tol=0.0, aca_tol=0.0,
                 gmres_dense=0, body_blocks=0, lu_graph=0):
        lib = load_library()
        self._keep = {}
        f = lambda k, dt: self._keep.setdefault(k, np.asfortranarray(geom[k], dtype=dt))
        xyz, ncn, ncon = f("xyz", np.float64), f("ncn", np.int32), f("ncon", np.int32)
        xyz_p, ds, pnsz, dxyz = f("xyz_p", np.float64), f("ds", np.float64), f("pnsz", np.float64), f("dxyz", np.float64)
        bn = f("body_nelem", np.int32)
        self.n = int(ncn.size)
        self.nbody = int(bn.size)
        self.ndof = 6 * self.nbody
        g_ = HamsGeom(nelem=self.n, ntnd=xyz.shape[0], nbody=self.nbody, isx=int(geom.get("isx", 0)),
                      isy=int(geom.get("isy", 0)), xyz=_d(xyz), ncn=_i(ncn), ncon=_i(ncon), xyz_p=_d(xyz_p), ds=_d(ds),
                      pnsz=_d(pnsz), dxyz=_d(dxyz), body_nelem=_i(bn), inelem=0, ixyz_p=None)
        if irsp == 1:
            ixyz_p = f("ixyz_p", np.float64)
            g_.inelem = ixyz_p.shape[0]
            g_.ixyz_p = _d(ixyz_p)
        o = HamsOpts(depth=float(depth), rho=float(rho), g=float(g), amp=float(amp), isol=int(isol), irsp=int(irsp),
                     precision=int(precision), device=int(device), refine_tol=float(refine_tol),
                     refine_max=int(refine_max), lu_kind=int(lu_kind), batch_lanes=int(batch_lanes), solver=int(solver),
                     gmres_restart=int(gmres_restart), gmres_maxit=int(gmres_maxit), gmres_tol=float(gmres_tol),
                     aca_tol=float(aca_tol), gmres_dense=int(gmres_dense), body_blocks=int(body_blocks),
                     lu_graph=int(lu_graph))
        o.xw[0], o.xw[1] = xw
        self.depth, self.g = float(depth), float(g)
        self._h = ctypes.c_void_p()
        _check(lib.hams_ctx_create(ctypes.byref(g_), ctypes.byref(o), ctypes.byref(self._h)))

    def close(self):
        if self._h:
            load_library().hams_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def wave(self, omega, inft=3):
        return wave_properties(omega, self.depth, self.g, inft)

    def solve_frequency(self, wave, betas):
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        amas = np.zeros((self.ndof, self.ndof), order="F")
        bdmp = np.zeros((self.ndof, self.ndof), order="F")
        exfc = np.zeros((max(len(betas), 1), self.ndof), dtype=np.complex128, order="F")
        _check(load_library().hams_solve_frequency(self._h, ctypes.byref(wave), len(betas), _d(betas), _d(amas),
                                                   _d(bdmp), exfc.ctypes.data_as(P_dbl)))
        return amas, bdmp, exfc[:len(betas)]

    def solve_batch(self, waves, betas):
        nf = len(waves)
        arr = (HamsWave * nf)(*waves)
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        amas = np.zeros((nf, self.ndof, self.ndof), order="F")
        bdmp = np.zeros((nf, self.ndof, self.ndof), order="F")
        exfc = np.zeros((nf, max(len(betas), 1), self.ndof), dtype=np.complex128, order="F")
        _check(load_library().hams_solve_batch(self._h, nf, arr, len(betas), _d(betas), _d(amas), _d(bdmp),
                                               exfc.ctypes.data_as(P_dbl)))
        return amas, bdmp, exfc[:, :len(betas)]

    def assemble(self, wave, betas):
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        a = np.zeros((self.n, self.n), dtype=np.complex128, order="F")
        b = np.zeros((self.n, self.ndof), dtype=np.complex128, order="F")
        d = np.zeros((self.n, max(len(betas), 1)), dtype=np.complex128, order="F")
        _check(load_library().hams_assemble(self._h, ctypes.byref(wave), len(betas), _d(betas),
                                            a.ctypes.data_as(P_dbl), b.ctypes.data_as(P_dbl), d.ctypes.data_as(P_dbl)))
        return a, b, d[:, :len(betas)]

    def eval_green(self, wave, pts, flag):
        pts = np.asfortranarray(pts, dtype=np.float64)
        flag = np.ascontiguousarray(flag, dtype=np.int32)
        out = np.zeros((pts.shape[0], 4), dtype=np.complex128, order="F")
        _check(load_library().hams_eval_green(self._h, ctypes.byref(wave), pts.shape[0], _d(pts), _i(flag),
                                              out.ctypes.data_as(P_dbl)))
        return out

    def timings(self):
        """Stage times of the last solve (ms), per-branch Green kernel times and pair counts."""
        ms = np.zeros(28)
        load_library().hams_last_timings(self._h, _d(ms), 28)
        return dict(green=ms[0], rhs=ms[1], solve=ms[2], forces=ms[3], total=ms[4], green_linton=ms[5],
                    green_pidcock=ms[6], green_eigene=ms[7], green_eigen=ms[8], factor=ms[9], refine_sweeps=int(ms[10]),
                    iterations=int(ms[10]),
                    pairs_linton=int(ms[11]), pairs_pidcock=int(ms[12]), pairs_eigene=int(ms[13]),
                    pairs_eigen=int(ms[14]), lu_used=int(ms[15]), green_surrogate=ms[16],
                    pairs_surrogate=int(ms[17]), ir_rate=ms[18], pairs_copied=int(ms[19]),
                    judge_err_a=ms[20], judge_err_s=ms[21], judge_errors=(ms[22], ms[23], ms[24]),
                    judge_estimate=ms[25], judge_resolved=bool(ms[26]), judge_samples=int(ms[27]))

    def set_surrogate(self, params, far_factor=3.0, k_range=None):
        """Far pairs from the trained network (params float32), or the series again (params None);
        k_range (kmin, kmax): the frequencies, by K = k0 h tanh(k0 h), the network serves."""
        lib = load_library()
        if params is None:
            _check(lib.hams_ctx_set_surrogate(self._h, None, 0, 0.0))
            return
        self._sg = np.ascontiguousarray(params, dtype=np.float32)
        _check(lib.hams_ctx_set_surrogate(self._h, _f(self._sg), self._sg.size, float(far_factor)))
        kmin, kmax = k_range if k_range is not None else (0.04, 40.0)
        _check(lib.hams_ctx_set_surrogate_range(self._h, float(kmin), float(kmax)))

    def set_surrogate_tolerance(self, tol):
        """The series judges each frequency the network serves; above tol the series takes the frequency
        back (0 switches the judgement off)."""
        _check(load_library().hams_ctx_set_surrogate_tolerance(self._h, float(tol)))

    def set_field_points(self, xfp):
        """Field points (nfp, 3) whose potentials every later solve evaluates (None: off)."""
        if xfp is None or len(xfp) == 0:
            self._fp = None
            _check(load_library().hams_ctx_set_field_points(self._h, 0, None))
            return
        self._fp = np.asfortranarray(xfp, dtype=np.float64)
        _check(load_library().hams_ctx_set_field_points(self._h, self._fp.shape[0], _d(self._fp)))

    def field_potentials(self, nbeta, k=0):
        """(nfp, 6 nb + 2 nbeta) complex potentials of frequency k of the last batch (0 after a single
        solve): radiation modes, diffraction per heading, incident per heading."""
        out = np.zeros((self._fp.shape[0], self.ndof + 2 * nbeta), dtype=np.complex128, order="F")
        _check(load_library().hams_field_potentials(self._h, int(k), out.ctypes.data_as(P_dbl)))
        return out

    def note(self):
        """What the last solve decided on its own (e.g. a fallback to the library LU), or ''."""
        return load_library().hams_last_note(self._h).decode()

    def launch_count(self):
        """Kernels of this library launched so far on this context."""
        return int(load_library().hams_launch_count(self._h))

    def library_call_count(self):
        """cuBLAS / cuSOLVER / CUB calls issued so far on this context."""
        return int(load_library().hams_library_call_count(self._h))

    def mark(self, slot):
        _check(load_library().hams_mark(self._h, slot))

    def elapsed_ms(self, a, b):
        ms = ctypes.c_double()
        _check(load_library().hams_mark_elapsed(self._h, a, b, ctypes.byref(ms)))
        return ms.value


def measure_fp64_peak(device=0):
    """FP64 FMA throughput of the device, TFLOP/s."""
    t = ctypes.c_double()
    _check(load_library().hams_measure_fp64_peak(device, ctypes.byref(t)))
    return t.value


def diag_gemm_tf32(a, b, c=None, alpha=1.0, beta=0.0, c_rowmajor=False, variant=-1, device=0):
    """The block LU's tensor-core GEMM: alpha a @ b + beta c for float32 a (m x k), b (k x n), c (m x n);
    variant 0/1/2 = tiles of 64/128/256 columns, -1 = the autotuner's pick."""
    m, k = a.shape
    n = b.shape[1]
    ld = (k + 3) // 4 * 4
    A = np.zeros((m, ld), dtype=np.float32)
    A[:, :k] = a
    B = np.zeros((n, ld), dtype=np.float32)  # column-major k x n
    B[:, :k] = b.T
    C = np.zeros((m, n), dtype=np.float32) if c is None else np.array(c, dtype=np.float32)  # a copy
    Cbuf = np.ascontiguousarray(C) if c_rowmajor else np.ascontiguousarray(C.T)
    _check(load_library().hams_diag_gemm_tf32(device, m, n, k, alpha, _f(A), ld, _f(B), ld, beta, _f(Cbuf),
                                               n if c_rowmajor else m, int(c_rowmajor), int(variant)))
    return Cbuf if c_rowmajor else Cbuf.T


def diag_gemm_tf32_time(m, n, k, variant=-1, reps=10, device=0):
    """Mean device time (ms) of the block LU's GEMM on device operands of shape m x n x k."""
    ms = ctypes.c_double()
    _check(load_library().hams_diag_gemm_tf32_time(device, variant, m, n, k, reps, ctypes.byref(ms)))
    return ms.value


# ---------------------------------------------------------------------------
# MLP surrogate of the finite-depth evanescent Green function
# ---------------------------------------------------------------------------
def _f(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def release_cached():
    """Give the device memory, streams and library handles that closed contexts left to the library
    (kept for the next contexts) back to the driver."""
    load_library().hams_release_cached()


def surrogate_param_count():
    return int(load_library().hams_surrogate_param_count())


def surrogate_samples(n, seed=1, nslice=256, device=0):
    """n samples of the series: columns X, Zq, Zp, K, t0, t1, t2."""
    raw = np.zeros((n, 7), order="F")
    _check(load_library().hams_surrogate_samples(device, n, seed, nslice, _d(raw)))
    return raw


def surrogate_train(n_train=4_000_000, n_test=200_000, batch=4096, steps=20000, nslice=256, seed=1, lr=2e-3,
                    device=0):
    """Generate samples and train on the GPU; returns (params float32, stats dict)."""
    cfg = SgTrain(n_train=n_train, n_test=n_test, batch=batch, steps=steps, nslice=nslice, seed=seed, lr=lr)
    params = np.zeros(surrogate_param_count(), dtype=np.float32)
    st = np.zeros(9)
    _check(load_library().hams_surrogate_train(device, ctypes.byref(cfg), _f(params), _d(st)))
    stats = dict(rms_rel=st[0:3].tolist(), max_rel=st[3:6].tolist(), loss=float(st[6]), train_ms=float(st[7]),
                 sample_ms=float(st[8]))
    return params, stats


def surrogate_eval(params, x, device=0):
    """FP32 network outputs t (n,3) for inputs x (n,4) = X, Zq, Zp, K."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    x = np.asfortranarray(x, dtype=np.float64)
    t = np.zeros((x.shape[0], 3), order="F")
    _check(load_library().hams_surrogate_eval(device, _f(params), x.shape[0], _d(x), _d(t)))
    return t


def surrogate_grad(params, feats, targ, device=0):
    """Loss and gradient of the normalised MSE for feats (4,n), targ (3,n)."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    feats = np.asfortranarray(feats, dtype=np.float32)
    targ = np.asfortranarray(targ, dtype=np.float32)
    grad = np.zeros_like(params)
    loss = ctypes.c_double()
    _check(load_library().hams_surrogate_grad(device, _f(params), feats.shape[1], _f(feats), _f(targ),
                                              ctypes.byref(loss), _f(grad)))
    return loss.value, grad
