"""ctypes binding of the CPU oracle (oracle/libhams_oracle.so).

The oracle is test infrastructure: a plain-C FP64 restatement of HAMS-MREL's
per-frequency build-and-solve.  Only the tests, ``__graft_entry__.smoke`` and
the CPU-baseline leg of ``bench.py`` load it, as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "libhams_oracle.so")

c_int = ctypes.c_int32
c_dbl = ctypes.c_double
P_dbl = ctypes.POINTER(ctypes.c_double)
P_int = ctypes.POINTER(ctypes.c_int32)


class OrcGeom(ctypes.Structure):
    _fields_ = [
        ("nelem", c_int), ("ntnd", c_int), ("nbody", c_int), ("isx", c_int), ("isy", c_int), ("nsys", c_int),
        ("xyz", P_dbl), ("ncn", P_int), ("ncon", P_int), ("xyz_p", P_dbl), ("ds", P_dbl), ("pnsz", P_dbl),
        ("dxyz", P_dbl), ("body_nelem", P_int),
        ("inelem", c_int), ("intnd", c_int),
        ("ixyz", P_dbl), ("incn", P_int), ("incon", P_int), ("ixyz_p", P_dbl), ("ids", P_dbl), ("ipnsz", P_dbl),
        ("idxyz", P_dbl), ("body_inelem", P_int),
    ]


class OrcOpts(ctypes.Structure):
    _fields_ = [("h", c_dbl), ("rho", c_dbl), ("g", c_dbl), ("xw", c_dbl * 2), ("amp", c_dbl), ("isol", c_int),
                ("irsp", c_int), ("grn_kind", c_int), ("nthread", c_int)]


class OrcWave(ctypes.Structure):
    _fields_ = [("v", c_dbl), ("wk", c_dbl), ("w1", c_dbl), ("tp", c_dbl), ("wl", c_dbl), ("wvn", c_dbl * 200)]


class OrcDeck(ctypes.Structure):
    _fields_ = [("opts", OrcOpts), ("geom", OrcGeom), ("sybo", c_int), ("inft", c_int), ("ouft", c_int),
                ("nper", c_int), ("nbeta", c_int), ("wvnb", P_dbl), ("wvhd", P_dbl), ("xr", P_dbl), ("lcs", P_dbl),
                ("refl", c_dbl), ("isolv", c_int)]


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


_LIB = None


def load():
    """The oracle library: ``oracle/libhams_oracle.so``, or the build named by
    HAMS_ORACLE_SO (the host-tuned build the timed CPU baseline uses)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.environ.get("HAMS_ORACLE_SO") or ORACLE_SO
    if path == ORACLE_SO and not os.path.exists(ORACLE_SO):
        build()
    lib = ctypes.CDLL(path)
    lib.orc_wave_props.argtypes = [c_int, c_dbl, c_dbl, c_dbl, c_int, ctypes.POINTER(OrcWave)]
    lib.orc_dispersion_c.argtypes = [P_dbl, c_int, c_dbl, c_dbl]
    lib.orc_fingreen3d_c.argtypes = [c_dbl] * 7 + [P_dbl, c_int, c_dbl, P_dbl, c_int]
    lib.orc_infgreen3d_c.argtypes = [c_dbl] * 7 + [P_dbl, c_int]
    lib.orc_fin_branch_c.argtypes = [c_dbl, c_dbl]
    lib.orc_fin_branch_c.restype = c_int
    lib.orc_special_c.argtypes = [c_int, c_dbl, P_dbl]
    lib.orc_sglint_c.argtypes = [ctypes.POINTER(OrcGeom), c_int, P_dbl, P_dbl]
    lib.orc_assemble.argtypes = [ctypes.POINTER(OrcGeom), ctypes.POINTER(OrcOpts), ctypes.POINTER(OrcWave), c_int,
                                 P_dbl, P_dbl, P_dbl, P_dbl]
    lib.orc_assemble_rows.argtypes = [ctypes.POINTER(OrcGeom), ctypes.POINTER(OrcOpts), ctypes.POINTER(OrcWave),
                                      c_int, P_dbl, c_int, c_int, P_dbl, P_dbl, P_dbl]
    lib.orc_assemble_rows.restype = c_int
    lib.orc_zgetrf.argtypes = [c_int, P_dbl, P_int, c_int]
    lib.orc_zgetrs.argtypes = [c_int, c_int, P_dbl, P_int, P_dbl]
    lib.orc_forces.argtypes = [ctypes.POINTER(OrcGeom), ctypes.POINTER(OrcOpts), ctypes.POINTER(OrcWave), c_int,
                               P_dbl, P_dbl, P_dbl, P_dbl, P_dbl, P_dbl]
    lib.orc_solve_frequency.argtypes = [ctypes.POINTER(OrcGeom), ctypes.POINTER(OrcOpts), ctypes.POINTER(OrcWave),
                                        c_int, P_dbl, P_dbl, P_dbl, P_dbl]
    lib.orc_run_case.argtypes = [ctypes.c_char_p, ctypes.c_char_p, c_int, c_int]
    lib.orc_load_deck.argtypes = [ctypes.c_char_p, ctypes.POINTER(OrcDeck)]
    lib.orc_geom_prepare.argtypes = [ctypes.POINTER(OrcGeom), P_dbl]
    lib.orc_free_deck.argtypes = [ctypes.POINTER(OrcDeck)]
    _LIB = lib
    return lib


def dptr(a):
    return a.ctypes.data_as(P_dbl)


def iptr(a):
    return a.ctypes.data_as(P_int)


class Case:
    """Geometry + options held in numpy arrays, viewable as an OrcGeom."""

    def __init__(self, xyz, ncn, ncon, body_nelem, xr, h, rho=1000.0, g=9.80665, isx=0, isy=0, isol=1,
                 ixyz=None, incn=None, incon=None, body_inelem=None, irsp=0, prepare=True, dxyz=None):
        self.xyz = np.asfortranarray(xyz, dtype=np.float64)
        self.ncn = np.ascontiguousarray(ncn, dtype=np.int32)
        self.ncon = np.asfortranarray(ncon, dtype=np.int32)
        self.body_nelem = np.ascontiguousarray(body_nelem, dtype=np.int32)
        n = self.ncn.size
        self.xyz_p = np.zeros((n, 3), order="F")
        self.ds = np.zeros(n)
        self.pnsz = np.zeros(n)
        self.dxyz = np.zeros((n, 6), order="F")
        self.xr = np.asfortranarray(xr, dtype=np.float64).reshape(len(self.body_nelem), 3, order="F")
        nb = len(self.body_nelem)
        if ixyz is not None:
            self.ixyz = np.asfortranarray(ixyz, dtype=np.float64)
            self.incn = np.ascontiguousarray(incn, dtype=np.int32)
            self.incon = np.asfortranarray(incon, dtype=np.int32)
            self.body_inelem = np.ascontiguousarray(body_inelem, dtype=np.int32)
        else:
            self.ixyz = np.zeros((1, 3), order="F")
            self.incn = np.zeros(1, dtype=np.int32)
            self.incon = np.zeros((1, 4), dtype=np.int32, order="F")
            self.body_inelem = np.zeros(nb, dtype=np.int32)
        ni = int(self.body_inelem.sum())
        self.ixyz_p = np.zeros((max(ni, 1), 3), order="F")
        self.ids = np.zeros(max(ni, 1))
        self.ipnsz = np.zeros(max(ni, 1))
        self.idxyz = np.zeros((max(ni, 1), 6), order="F")
        self.geom = OrcGeom(
            nelem=n, ntnd=self.xyz.shape[0], nbody=nb, isx=isx, isy=isy, nsys=1 if (isx == 0 and isy == 0) else 2,
            xyz=dptr(self.xyz), ncn=iptr(self.ncn), ncon=iptr(self.ncon), xyz_p=dptr(self.xyz_p), ds=dptr(self.ds),
            pnsz=dptr(self.pnsz), dxyz=dptr(self.dxyz), body_nelem=iptr(self.body_nelem),
            inelem=ni, intnd=self.ixyz.shape[0] if ni else 0,
            ixyz=dptr(self.ixyz), incn=iptr(self.incn), incon=iptr(self.incon), ixyz_p=dptr(self.ixyz_p),
            ids=dptr(self.ids), ipnsz=dptr(self.ipnsz), idxyz=dptr(self.idxyz), body_inelem=iptr(self.body_inelem))
        self.opts = OrcOpts(h=h, rho=rho, g=g, amp=1.0, isol=isol, irsp=irsp, grn_kind=8, nthread=0)
        self.opts.xw[0] = 0.0
        self.opts.xw[1] = 0.0
        if prepare:
            load().orc_geom_prepare(ctypes.byref(self.geom), dptr(self.xr))
        if dxyz is not None:
            self.dxyz[:] = dxyz

    @property
    def n(self):
        return int(self.geom.nelem)

    @property
    def nbody(self):
        return int(self.geom.nbody)

    def wave(self, omega, inft=3):
        w = OrcWave()
        load().orc_wave_props(inft, omega, self.opts.h, self.opts.g, 0, ctypes.byref(w))
        return w

    def assemble(self, w, betas):
        lib = load()
        n, nsys, ndof = self.n, self.geom.nsys, 6 * self.nbody
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        a = np.zeros((n, n, nsys), dtype=np.complex128, order="F")
        b = np.zeros((n, ndof, nsys), dtype=np.complex128, order="F")
        d = np.zeros((n, nsys, max(len(betas), 1)), dtype=np.complex128, order="F")
        lib.orc_assemble(ctypes.byref(self.geom), ctypes.byref(self.opts), ctypes.byref(w), len(betas), dptr(betas),
                         a.ctypes.data_as(P_dbl), b.ctypes.data_as(P_dbl), d.ctypes.data_as(P_dbl))
        return a, b, d

    def assemble_rows(self, w, betas, stride, offset=0):
        """Hull rows offset, offset+stride, ... of the system (the timed CPU sample)."""
        lib = load()
        n, nsys, ndof = self.n, self.geom.nsys, 6 * self.nbody
        nr = (n - offset + stride - 1) // stride
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        a = np.zeros((nr, n, nsys), dtype=np.complex128, order="F")
        b = np.zeros((nr, ndof, nsys), dtype=np.complex128, order="F")
        d = np.zeros((nr, nsys, max(len(betas), 1)), dtype=np.complex128, order="F")
        got = lib.orc_assemble_rows(ctypes.byref(self.geom), ctypes.byref(self.opts), ctypes.byref(w), len(betas),
                                    dptr(betas), stride, offset, a.ctypes.data_as(P_dbl), b.ctypes.data_as(P_dbl),
                                    d.ctypes.data_as(P_dbl))
        assert got == nr
        return a, b, d

    def forces(self, w, betas, xrad, xdif):
        lib = load()
        ndof = 6 * self.nbody
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        amas = np.zeros((ndof, ndof), order="F")
        bdmp = np.zeros((ndof, ndof), order="F")
        exfc = np.zeros((len(betas), ndof), dtype=np.complex128, order="F")
        xrad = np.asfortranarray(xrad, dtype=np.complex128)
        xdif = np.asfortranarray(xdif, dtype=np.complex128)
        lib.orc_forces(ctypes.byref(self.geom), ctypes.byref(self.opts), ctypes.byref(w), len(betas), dptr(betas),
                       xrad.ctypes.data_as(P_dbl), xdif.ctypes.data_as(P_dbl), dptr(amas), dptr(bdmp),
                       exfc.ctypes.data_as(P_dbl))
        return amas, bdmp, exfc

    def solve(self, w, betas):
        lib = load()
        ndof = 6 * self.nbody
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        amas = np.zeros((ndof, ndof), order="F")
        bdmp = np.zeros((ndof, ndof), order="F")
        exfc = np.zeros((len(betas), ndof), dtype=np.complex128, order="F")
        info = lib.orc_solve_frequency(ctypes.byref(self.geom), ctypes.byref(self.opts), ctypes.byref(w), len(betas),
                                       dptr(betas), dptr(amas), dptr(bdmp), exfc.ctypes.data_as(P_dbl))
        return amas, bdmp, exfc, info


def fingreen(xf, xp, yf, yp, zf, zp, v, wvn, h, flag):
    g = np.zeros(8)
    wvn = np.ascontiguousarray(wvn, dtype=np.float64)
    load().orc_fingreen3d_c(xf, xp, yf, yp, zf, zp, v, dptr(wvn), 200, h, dptr(g), flag)
    return g[0::2] + 1j * g[1::2]


def infgreen(xf, xp, yf, yp, zf, zp, v, flag):
    g = np.zeros(8)
    load().orc_infgreen3d_c(xf, xp, yf, yp, zf, zp, v, dptr(g), flag)
    return g[0::2] + 1j * g[1::2]


def special(which, x):
    out = np.zeros(4)
    load().orc_special_c(which, x, dptr(out))
    return out


def dispersion(w, h, n=200):
    wvn = np.zeros(n)
    load().orc_dispersion_c(dptr(wvn), n, w, h)
    return wvn


def load_deck(inputdir):
    """Parse a HAMS deck with the oracle's reader; returns plain numpy arrays."""
    lib = load()
    d = OrcDeck()
    rc = lib.orc_load_deck(inputdir.encode(), ctypes.byref(d))
    if rc != 0:
        raise RuntimeError(f"orc_load_deck({inputdir}) failed with {rc}")
    g = d.geom
    n, nt, nb = g.nelem, g.ntnd, g.nbody

    def arr(p, count, dtype=np.float64):
        return np.ctypeslib.as_array(p, shape=(count,)).astype(dtype).copy()

    out = dict(
        h=d.opts.h, isol=d.opts.isol, irsp=d.opts.irsp, isx=g.isx, isy=g.isy, nsys=g.nsys,
        sybo=d.sybo, inft=d.inft, ouft=d.ouft, nper=d.nper, nbeta=d.nbeta,
        wvnb=arr(d.wvnb, d.nper), wvhd=arr(d.wvhd, d.nbeta), xr=arr(d.xr, 3 * nb).reshape(nb, 3, order="F"),
        xyz=arr(g.xyz, 3 * nt).reshape(nt, 3, order="F"), ncn=arr(g.ncn, n, np.int32),
        ncon=arr(g.ncon, 4 * n, np.int32).reshape(n, 4, order="F"),
        xyz_p=arr(g.xyz_p, 3 * n).reshape(n, 3, order="F"), ds=arr(g.ds, n), pnsz=arr(g.pnsz, n),
        dxyz=arr(g.dxyz, 6 * n).reshape(n, 6, order="F"), body_nelem=arr(g.body_nelem, nb, np.int32),
        inelem=g.inelem)
    if g.inelem > 0:
        ni, nti = g.inelem, g.intnd
        out.update(ixyz=arr(g.ixyz, 3 * nti).reshape(nti, 3, order="F"), incn=arr(g.incn, ni, np.int32),
                   incon=arr(g.incon, 4 * ni, np.int32).reshape(ni, 4, order="F"),
                   ixyz_p=arr(g.ixyz_p, 3 * ni).reshape(ni, 3, order="F"), ids=arr(g.ids, ni),
                   ipnsz=arr(g.ipnsz, ni), idxyz=arr(g.idxyz, 6 * ni).reshape(ni, 6, order="F"),
                   body_inelem=arr(g.body_inelem, nb, np.int32))
    lib.orc_free_deck(ctypes.byref(d))
    return out


def fortran_e(v, d):
    """Fortran Ew.d output text of v (0.ddddE+xx form) without padding."""
    if v == 0.0:
        return "0." + "0" * d + "E+00"
    m = "%.*e" % (d - 1, abs(v))
    mant, ex = m.split("e")
    e = int(ex) + 1
    body = "0." + mant.replace(".", "")
    sign = "-" if v < 0 else ""
    if -99 <= e <= 99:
        return f"{sign}{body}E{'-' if e < 0 else '+'}{abs(e):02d}"
    return f"{sign}{body}{'-' if e < 0 else '+'}{abs(e):03d}"
