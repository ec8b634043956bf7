"""ctypes bindings for the CPU oracle (oracle/liboracle.so) and for the reference's own
host functions built from its sources (oracle/_ref/librefhost_*.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py, always as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
# the reference tree, for building oracle/_ref: the SWD_REFERENCE environment variable
REFERENCE_SRC = Path(os.environ["SWD_REFERENCE"]) if os.environ.get("SWD_REFERENCE") else None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build(reference: bool = False) -> None:
    """Build liboracle.so (and, if asked and the reference sources exist, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if reference and REFERENCE_SRC is not None and REFERENCE_SRC.exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REFERENCE_SRC}"], check=True)


class OrcModel(C.Structure):
    _fields_ = [("ntx", C.c_int), ("ntz", C.c_int), ("pmlc", C.c_int), ("Lc", C.c_int), ("nt", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("dt", C.c_float),
                ("rc", C.c_void_p), ("vp", C.c_void_p), ("rho", C.c_void_p),
                ("a_x", C.c_void_p), ("a_x_half", C.c_void_p), ("a_z", C.c_void_p), ("a_z_half", C.c_void_p),
                ("b_x", C.c_void_p), ("b_x_half", C.c_void_p), ("b_z", C.c_void_p), ("b_z_half", C.c_void_p)]


class OrcGeom(C.Structure):
    _fields_ = [("s_ix", C.c_int), ("s_iz", C.c_int), ("nrec", C.c_int),
                ("r_ix", C.c_void_p), ("r_iz", C.c_void_p)]


class OrcDeconParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("psfwinx", C.c_int), ("psfwinz", C.c_int),
                ("filterwinx", C.c_int), ("filterwinz", C.c_int), ("snapwinx", C.c_int), ("snapwinz", C.c_int),
                ("epsilon", C.c_float), ("fft_n0", C.c_int), ("fft_n1", C.c_int), ("psf_interp", C.c_int),
                ("iters", C.c_int), ("reg_l1", C.c_float), ("reg_l2", C.c_float)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.orc_cal_xishu.argtypes = [C.c_int, _f32p]
        L.orc_cpml.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float] + [_f32p] * 8
        L.orc_ricker2.argtypes = [C.c_int, C.c_float, C.c_float, _f32p]
        L.orc_pad_model.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f32p]
        L.orc_smooth.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_pow2_len.argtypes = [C.c_int]
        L.orc_pow2_len.restype = C.c_int
        L.orc_kz_taper.argtypes = [C.c_int, C.c_float, _f32p]
        L.orc_kz_taper.restype = C.c_int
        L.orc_hilbert1d.argtypes = [C.c_int, _f32p, _f32p]
        L.orc_well_count.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]
        L.orc_well_count.restype = C.c_int
        L.orc_well_geometry.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, _i32p, _i32p]
        L.orc_strip_len.argtypes = [C.POINTER(OrcModel)]
        L.orc_strip_len.restype = C.c_int
        L.orc_edge_zero.argtypes = [C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_decon.argtypes = [C.POINTER(OrcDeconParams), _f32p, _f32p, _f32p, _f32p, C.c_int]
        L.orc_decon.restype = C.c_int
        L.orc_decon_geometry.argtypes = [C.POINTER(OrcDeconParams), _i32p]
        L.orc_decon_geometry.restype = C.c_int
        for sfx, tp in (("f32", _f32p), ("f64", _f64p)):
            getattr(L, f"orc_forward_{sfx}").argtypes = [C.POINTER(OrcModel), C.POINTER(OrcGeom), _f32p, C.c_void_p,
                                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
            getattr(L, f"orc_kzsep_{sfx}").argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, tp, _f32p, C.c_int,
                                                       _i32p, _i32p, tp, tp]
            getattr(L, f"orc_preprocess_{sfx}").argtypes = [C.c_int, C.c_int, C.c_float, _f32p, tp]
            getattr(L, f"orc_rtm_backward_{sfx}").argtypes = [C.POINTER(OrcModel), C.POINTER(OrcGeom), _f32p, tp, tp,
                                                              tp, tp, tp, C.c_void_p, C.c_int, C.c_int,
                                                              C.c_void_p]
            getattr(L, f"orc_rtm_post_{sfx}").argtypes = [C.POINTER(OrcModel), tp, tp, tp, tp]
            getattr(L, f"orc_born_{sfx}").argtypes = [C.POINTER(OrcModel), C.POINTER(OrcGeom), _f32p, _f32p, tp]
            getattr(L, f"orc_born_adjoint_{sfx}").argtypes = [C.POINTER(OrcModel), C.POINTER(OrcGeom), _f32p, _f32p, tp]
        _lib = L
    return _lib


# ---------------------------------------------------------------- host preparation
def cal_xishu(Lc):
    rc = np.zeros(Lc, np.float32)
    lib().orc_cal_xishu(Lc, rc)
    return rc


def cpml(ntx, ntz, pmlc, dx, dz, dt):
    arrs = [np.zeros(ntx, np.float32), np.zeros(ntx, np.float32), np.zeros(ntz, np.float32), np.zeros(ntz, np.float32),
            np.zeros(ntx, np.float32), np.zeros(ntx, np.float32), np.zeros(ntz, np.float32), np.zeros(ntz, np.float32)]
    lib().orc_cpml(ntx, ntz, pmlc, dx, dz, dt, *arrs)
    keys = ["a_x", "a_x_half", "a_z", "a_z_half", "b_x", "b_x_half", "b_z", "b_z_half"]
    return dict(zip(keys, arrs))


def ricker(nt, f0, dt):
    r = np.zeros(nt, np.float32)
    lib().orc_ricker2(nt, f0, dt, r)
    return r


def pad_model(v, pmlc):
    nx, nz = v.shape
    out = np.zeros((nx + 2 * pmlc, nz + 2 * pmlc), np.float32)
    lib().orc_pad_model(nx, nz, pmlc, np.ascontiguousarray(v, np.float32), out)
    return out


def smooth(vpad, pmlc, window):
    v = np.ascontiguousarray(vpad, np.float32).copy()
    lib().orc_smooth(v.shape[0], v.shape[1], pmlc, window, v)
    return v


def pow2_len(n):
    return lib().orc_pow2_len(n)


def kz_taper(nfftz, dz):
    c = np.zeros(nfftz, np.float32)
    layer = lib().orc_kz_taper(nfftz, dz, c)
    return c, layer


def hilbert1d(rick):
    r = np.ascontiguousarray(rick, np.float32)
    h = np.zeros_like(r)
    lib().orc_hilbert1d(len(r), r, h)
    return h


def well_geometry(nx, nz, pmlc, dz, shotdep, offsetz):
    n = lib().orc_well_count(nz, pmlc, dz, shotdep, offsetz)
    rix = np.zeros(n, np.int32)
    riz = np.zeros(n, np.int32)
    lib().orc_well_geometry(nx, nz, pmlc, dz, shotdep, offsetz, rix, riz)
    return rix, riz


# ---------------------------------------------------------------- loops
class Model:
    """Holds the arrays an OrcModel points into (so they stay alive)."""

    def __init__(self, vp, rho, cp, rc, pmlc, Lc, nt, dx, dz, dt):
        self.vp = np.ascontiguousarray(vp, np.float32)
        self.rho = np.ascontiguousarray(rho, np.float32)
        self.cp = {k: np.ascontiguousarray(v, np.float32) for k, v in cp.items()}
        self.rc = np.ascontiguousarray(rc, np.float32)
        self.ntx, self.ntz = self.vp.shape
        self.pmlc, self.Lc, self.nt = pmlc, Lc, nt
        self.dx, self.dz, self.dt = dx, dz, dt
        p = lambda a: a.ctypes.data
        self.s = OrcModel(self.ntx, self.ntz, pmlc, Lc, nt, dx, dz, dt, p(self.rc), p(self.vp), p(self.rho),
                          *[p(self.cp[k]) for k in ["a_x", "a_x_half", "a_z", "a_z_half",
                                                      "b_x", "b_x_half", "b_z", "b_z_half"]])

    @property
    def strip_len(self):
        return lib().orc_strip_len(C.byref(self.s))


class Geom:
    def __init__(self, s_ix, s_iz, r_ix, r_iz):
        self.r_ix = np.ascontiguousarray(r_ix, np.int32)
        self.r_iz = np.ascontiguousarray(r_iz, np.int32)
        self.s = OrcGeom(int(s_ix), int(s_iz), len(self.r_ix), self.r_ix.ctypes.data, self.r_iz.ctypes.data)


def _ptr(a):
    return None if a is None else a.ctypes.data


def forward(model: Model, geom: Geom, rick, hrick=None, strips=False, final=False, col_ix=None, dtype=np.float32):
    sfx = "f32" if dtype == np.float32 else "f64"
    nt, ntp = model.nt, model.ntx * model.ntz
    seis = np.zeros((len(geom.r_ix), nt), dtype)
    st = np.zeros((nt, model.strip_len), dtype) if strips else None
    fs = np.zeros((3, model.ntx, model.ntz), dtype) if final else None
    cix = None if col_ix is None else np.ascontiguousarray(col_ix, np.int32)
    cols = None if cix is None else np.zeros((len(cix), nt, model.ntz, 2), dtype)
    hr = None if hrick is None else np.ascontiguousarray(hrick, np.float32)
    getattr(lib(), f"orc_forward_{sfx}")(C.byref(model.s), C.byref(geom.s), np.ascontiguousarray(rick, np.float32),
                                         _ptr(hr), _ptr(seis), _ptr(st), _ptr(fs),
                                         0 if cix is None else len(cix), _ptr(cix), _ptr(cols))
    return dict(seis=seis, strips=st, final=fs, cols=cols)


def born(model: Model, geom: Geom, rick, dkappa, dtype=np.float64):
    """Born data [nrec][nt] for a bulk-modulus perturbation dkappa (ntx, ntz)."""
    sfx = "f32" if dtype == np.float32 else "f64"
    out = np.zeros((len(geom.r_ix), model.nt), dtype)
    getattr(lib(), f"orc_born_{sfx}")(C.byref(model.s), C.byref(geom.s), np.ascontiguousarray(rick, np.float32),
                                      np.ascontiguousarray(dkappa, np.float32), out)
    return out


def born_adjoint(model: Model, geom: Geom, rick, resid, dtype=np.float64):
    """Adjoint of born(): gradient (ntx, ntz) of <resid, born(dkappa)> with respect to dkappa."""
    sfx = "f32" if dtype == np.float32 else "f64"
    out = np.zeros((model.ntx, model.ntz), dtype)
    getattr(lib(), f"orc_born_adjoint_{sfx}")(C.byref(model.s), C.byref(geom.s), np.ascontiguousarray(rick, np.float32),
                                              np.ascontiguousarray(resid, np.float32), out)
    return out


def kzsep(cols, ntz, nfftz, coef, rec_col, r_iz, dtype=np.float32):
    sfx = "f32" if dtype == np.float32 else "f64"
    ncol, nt = cols.shape[0], cols.shape[1]
    nrec = len(r_iz)
    up = np.zeros((nrec, nt), dtype)
    down = np.zeros((nrec, nt), dtype)
    getattr(lib(), f"orc_kzsep_{sfx}")(ntz, nfftz, nt, ncol, np.ascontiguousarray(cols, dtype),
                                       np.ascontiguousarray(coef, np.float32), nrec,
                                       np.ascontiguousarray(rec_col, np.int32), np.ascontiguousarray(r_iz, np.int32),
                                       up, down)
    return up, down


def preprocess(d, dt, dtype=np.float32):
    sfx = "f32" if dtype == np.float32 else "f64"
    d = np.ascontiguousarray(d, np.float32)
    out = np.zeros(d.shape, dtype)
    getattr(lib(), f"orc_preprocess_{sfx}")(d.shape[0], d.shape[1], dt, d, out)
    return out


def rtm_backward(model: Model, geom: Geom, rick, rms, strips, final, dtype=np.float32, illum_r=False, cig=None):
    """cig = (thetan, delt) also returns the angle gathers (ntx, ntz, thetan) as a 4th value."""
    sfx = "f32" if dtype == np.float32 else "f64"
    shp = (model.ntx, model.ntz)
    img, s = np.zeros(shp, dtype), np.zeros(shp, dtype)
    r = np.zeros(shp, dtype) if illum_r else None
    thetan, delt = cig if cig else (0, 1)
    g = np.zeros(shp + (thetan,), np.float32) if cig else None
    getattr(lib(), f"orc_rtm_backward_{sfx}")(C.byref(model.s), C.byref(geom.s), np.ascontiguousarray(rick, np.float32),
                                              np.ascontiguousarray(rms, dtype), np.ascontiguousarray(strips, dtype),
                                              np.ascontiguousarray(final, dtype), img, s, _ptr(r), thetan, delt, _ptr(g))
    return (img, s, r, g) if cig else (img, s, r)


def rtm_post(model: Model, img, illum, dtype=np.float32):
    sfx = "f32" if dtype == np.float32 else "f64"
    nx, nz = model.ntx - 2 * model.pmlc, model.ntz - 2 * model.pmlc
    norm = np.zeros(img.shape, dtype)
    fim = np.zeros((nx, nz), dtype)
    getattr(lib(), f"orc_rtm_post_{sfx}")(C.byref(model.s), np.ascontiguousarray(img, dtype),
                                          np.ascontiguousarray(illum, dtype), norm, fim)
    return norm, fim


def edge_zero(img, Lc):
    a = np.ascontiguousarray(img, np.float32).copy()
    lib().orc_edge_zero(a.shape[0], a.shape[1], Lc, a)
    return a


def rtm_shot(model: Model, geom: Geom, rick, data, dtype=np.float32, cig=None):
    """One reference RTM shot: forward with strips -> -integral-integral data -> backward;
    cig = (thetan, delt) adds the angle gathers under key "cig"."""
    fw = forward(model, geom, rick, strips=True, final=True, dtype=dtype)
    rms = preprocess(data, model.dt, dtype)
    out = rtm_backward(model, geom, rick, rms, fw["strips"], fw["final"], dtype, cig=cig)
    res = dict(img=out[0], illum=out[1], syn=fw["seis"], rms=rms)
    if cig:
        res["cig"] = out[3]
    return res


def decon(nx, nz, migreal, migpsf, psfwin, filterwin, snapwin, epsilon, fft_n=(0, 0), nthreads=0, psf_interp=0,
          iters=0, reg_l1=0.0, reg_l2=0.0):
    p = OrcDeconParams(nx, nz, psfwin[0], psfwin[1], filterwin[0], filterwin[1], snapwin[0], snapwin[1],
                       epsilon, fft_n[0], fft_n[1], psf_interp, iters, reg_l1, reg_l2)
    dec = np.zeros((nx, nz), np.float32)
    coef = np.zeros((nx, nz), np.float32)
    rc = lib().orc_decon(C.byref(p), np.ascontiguousarray(migreal, np.float32), np.ascontiguousarray(migpsf, np.float32),
                         dec, coef, nthreads)
    if rc:
        raise ValueError(f"orc_decon: invalid geometry ({rc})")
    return dec, coef


def decon_geometry(nx, nz, psfwin, filterwin, snapwin, fft_n=(0, 0)):
    p = OrcDeconParams(nx, nz, psfwin[0], psfwin[1], filterwin[0], filterwin[1], snapwin[0], snapwin[1],
                       0.0, fft_n[0], fft_n[1])
    out = np.zeros(16, np.int32)
    rc = lib().orc_decon_geometry(C.byref(p), out)
    if rc:
        raise ValueError(f"invalid decon geometry ({rc})")
    keys = ["fullwx", "fullwz", "FX", "FZ", "outwinx", "outwinz", "stepwinx", "stepwinz", "stepnumx", "stepnumz",
            "totalnum", "nxp", "nzp", "nxwpsf", "nzwpsf", "n0"]
    return dict(zip(keys, [int(v) for v in out]))


# ---------------------------------------------------------------- reference host functions
class RefHost:
    """The reference's own host functions (acoustic_HLVSPRTMC.cpp), built from its sources by
    oracle/Makefile; only present where the reference sources were available at build time."""

    def __init__(self, which="rtm"):
        path = REF_DIR / f"librefhost_{which}.so"
        if not path.exists():
            raise FileNotFoundError(path)
        self.L = C.CDLL(str(path))
        L = self.L
        L._Z9cal_xishuiPf.argtypes = [C.c_int, _f32p]
        L._Z24get_absorbing_parametersPfS_S_S_S_S_S_S_S_S_S_S_S_S_S_S_iiiiiffffff.argtypes = \
            [_f32p] * 16 + [C.c_int] * 5 + [C.c_float] * 6
        L._Z11ricker_wavePfifffi.argtypes = [_f32p, C.c_int, C.c_float, C.c_float, C.c_float, C.c_int]
        L._Z14ini_model_minePfS_iiiii.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]

    def cal_xishu(self, Lc):
        rc = np.zeros(Lc, np.float32)
        self.L._Z9cal_xishuiPf(Lc, rc)
        return rc

    def cpml(self, ntx, ntz, pmlc, dx, dz, dt, f0=20.0):
        nx, nz = ntx - 2 * pmlc, ntz - 2 * pmlc
        bufs = {}
        order = ["d_x", "d_x_half", "d_z", "d_z_half", "a_x", "a_x_half", "a_z", "a_z_half",
                 "b_x", "b_x_half", "b_z", "b_z_half", "k_x", "k_x_half", "k_z", "k_z_half"]
        for k in order:
            bufs[k] = np.zeros(ntx if "_x" in k else ntz, np.float32)
        self.L._Z24get_absorbing_parametersPfS_S_S_S_S_S_S_S_S_S_S_S_S_S_S_iiiiiffffff(
            *[bufs[k] for k in order], ntz, ntx, nz, nx, pmlc, dx, dz, f0, 1.0 / f0, dt, 5500.0)
        return bufs

    def ricker(self, nt, f0, dt, workdir):
        r = np.zeros(nt, np.float32)
        cwd = os.getcwd()
        os.makedirs(os.path.join(workdir, "output"), exist_ok=True)
        os.chdir(workdir)
        try:
            self.L._Z11ricker_wavePfifffi(r, nt, f0, np.float32(1.0 / np.float64(np.float32(f0))), dt, 2)
        finally:
            os.chdir(cwd)
        return r

    def smooth(self, vpad, pmlc, window):
        v = np.ascontiguousarray(vpad, np.float32).copy()
        vn = np.zeros_like(v)
        ntx, ntz = v.shape
        self.L._Z14ini_model_minePfS_iiiii(v, vn, ntx * ntz, ntz, ntx, pmlc, window)
        return v
