"""swd_b200 -- Python host layer over libswd (the sm_100a engine's C ABI, include/swd.h).

The product is the C ABI and the drop-in programs AFor / AVSPRTM / decon2d_mine built next
to this file; this module is the thin Python view of the same ABI used by the tests, the
benchmark and the torch autograd path.  Every call goes through libswd.so: there is no
Python or CPU implementation of the hot path here, and loading fails loudly when the
library is missing.

Array conventions follow the reference: padded grids are (ntx, ntz) float32 arrays,
C-contiguous, x-major with z fastest; seismograms are (r_n, nt); images are (nx, nz).
Arrays may be numpy arrays (host) or torch CUDA tensors (device pointers are passed
straight through; the library detects which).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libswd.so"

SWD_OK, SWD_ERR_ARG, SWD_ERR_CUDA, SWD_ERR_ALLOC, SWD_ERR_STATE, SWD_ERR_DEVICE, SWD_ERR_CAPACITY = range(7)
STRIP_F32, STRIP_F16, STRIP_BF16, STRIP_I16 = 0, 1, 2, 3
PATH_PLAIN, PATH_FUSED = 0, 1
RTM_PREPROCESS, RTM_ILLUM_RCV, RTM_NO_STACK, RTM_CIG = 1, 2, 4, 8
OPT_GRAPHS, OPT_BATCH, OPT_BATCH_TUNED, OPT_IMAGE_BLOCKS, OPT_BWD_BY_KIND, OPT_TMA, OPT_PDL, OPT_STAGED = 1, 2, 3, 4, 5, 6, 7, 8
OPT_AUTOTUNE, OPT_TUNED_FWD, OPT_TUNED_BWD, OPT_LEAN = 9, 10, 11, 12


class SwdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libswd error {code}: {msg}")
        self.code = code


def build(drivers: bool = True) -> None:
    """Compile libswd.so (sm_100a) and, optionally, the drop-in programs, in place."""
    subprocess.run(["make", "-s", "-C", str(PKG_DIR), "all" if drivers else "lib"], check=True)


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("pml", C.c_int), ("Lc", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("dt", C.c_float), ("nt_max", C.c_int), ("device", C.c_int)]


class Shot(C.Structure):
    _fields_ = [("s_ix", C.c_int), ("s_iz", C.c_int), ("nt", C.c_int), ("r_n", C.c_int),
                ("r_ix", C.c_void_p), ("r_iz", C.c_void_p)]


class DeconParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("psfwinx", C.c_int), ("psfwinz", C.c_int),
                ("filterwinx", C.c_int), ("filterwinz", C.c_int), ("snapwinx", C.c_int), ("snapwinz", C.c_int),
                ("epsilon", C.c_float), ("fft_nx", C.c_int), ("fft_nz", C.c_int), ("psf_interp", C.c_int),
                ("workspace", C.c_int), ("iters", C.c_int), ("reg_l1", C.c_float), ("reg_l2", C.c_float)]


_lib = None
_fp = C.POINTER(C.c_float)


def lib():
    """Load libswd.so; raises if it was not built (no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with swd_b200.build() or make -C {PKG_DIR}")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        L.swd_version.restype = C.c_int
        L.swd_device_count.argtypes = [C.POINTER(C.c_int)]
        L.swd_create.argtypes = [C.POINTER(vp), C.POINTER(Grid)]
        L.swd_destroy.argtypes = [vp]
        L.swd_last_error.argtypes = [vp]
        L.swd_last_error.restype = C.c_char_p
        L.swd_set_stream.argtypes = [vp, vp]
        L.swd_synchronize.argtypes = [vp]
        L.swd_device_bytes.argtypes = [vp]
        L.swd_device_bytes.restype = C.c_size_t
        L.swd_set_stencil.argtypes = [vp, vp]
        L.swd_set_cpml.argtypes = [vp] + [vp] * 8
        L.swd_set_model.argtypes = [vp, vp, vp]
        L.swd_set_strip_precision.argtypes = [vp, C.c_int]
        L.swd_set_kernel_path.argtypes = [vp, C.c_int]
        L.swd_set_source_storage.argtypes = [vp, C.c_int, C.c_int]
        L.swd_set_cig.argtypes = [vp, C.c_int, C.c_int]
        L.swd_rtm_cig.argtypes = [vp, vp]
        L.swd_forward.argtypes = [vp, C.POINTER(Shot), vp, vp, vp, vp, vp, vp]
        L.swd_set_scatter_model.argtypes = [vp, vp, vp]
        L.swd_forward_scatter.argtypes = [vp, C.POINTER(Shot), vp, vp, vp, vp, vp, vp]
        L.swd_rtm_shot.argtypes = [vp, C.POINTER(Shot), vp, vp, C.c_uint, vp, vp, vp, vp]
        L.swd_rtm_raw.argtypes = [vp, vp, vp, vp]
        L.swd_rtm_forward.argtypes = [vp, C.POINTER(Shot), vp, vp]
        L.swd_rtm_backward.argtypes = [vp, C.POINTER(Shot), vp, C.c_uint, vp, vp, vp]
        L.swd_stack_get.argtypes = [vp, C.c_int, vp]
        L.swd_stack_reset.argtypes = [vp]
        L.swd_rtm_batch.argtypes = [vp, C.c_int, C.POINTER(Shot), C.POINTER(vp), C.POINTER(vp), C.c_uint]
        L.swd_hilbert.argtypes = [vp, C.c_int, vp, vp]
        L.swd_smooth.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]
        L.swd_preprocess.argtypes = [vp, C.c_int, C.c_int, C.c_float, vp, vp]
        L.swd_decon_geometry.argtypes = [C.POINTER(DeconParams), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.swd_decon.argtypes = [vp, C.POINTER(DeconParams), vp, vp, vp, vp]
        L.swd_set_option.argtypes = [vp, C.c_int, C.c_int]
        L.swd_get_option.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
        L.swd_set_checkpointing.argtypes = [vp, C.c_int, C.c_int]
        L.swd_checkpoint_bytes.argtypes = [vp, C.c_int, C.POINTER(C.c_size_t)]
        L.swd_born.argtypes = [vp, C.POINTER(Shot), vp, vp, vp, vp, C.c_size_t]
        L.swd_born_adjoint.argtypes = [vp, C.POINTER(Shot), vp, vp, vp, vp, C.c_size_t]
        L.swd_profile.argtypes = [vp, C.c_int]
        L.swd_profile_read.argtypes = [vp, vp, vp]
        L.swd_launch_count.argtypes = [vp]
        L.swd_launch_count.restype = C.c_longlong
        L.swd_prep_xishu.argtypes = [C.c_int, vp]
        L.swd_prep_xishu.restype = None
        L.swd_prep_cpml.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float] + [vp] * 8
        L.swd_prep_cpml.restype = None
        L.swd_prep_ricker.argtypes = [C.c_int, C.c_float, C.c_float, vp]
        L.swd_prep_ricker.restype = None
        L.swd_prep_pad.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp]
        L.swd_prep_pad.restype = None
        L.swd_prep_pow2.argtypes = [C.c_int]
        L.swd_prep_kz_taper.argtypes = [C.c_int, C.c_float, vp]
        L.swd_prep_wells.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    """Raw pointer of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


def _nbytes(a) -> int:
    """Size in bytes of a numpy array or torch tensor (0 for None)."""
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return a.numel() * a.element_size()
    return a.nbytes


def _f32(a):
    if hasattr(a, "data_ptr"):
        return a.contiguous()
    return np.ascontiguousarray(a, np.float32)


def _i32(a):
    if hasattr(a, "data_ptr"):
        return a.contiguous()
    return np.ascontiguousarray(a, np.int32)


# ------------------------------------------------------------------ host preparation
def cal_xishu(Lc: int) -> np.ndarray:
    rc = np.zeros(Lc, np.float32)
    lib().swd_prep_xishu(Lc, _ptr(rc))
    return rc


def get_absorbing_parameters(ntx, ntz, pmlc, dx, dz, dt) -> dict:
    keys = ["a_x", "a_x_half", "a_z", "a_z_half", "b_x", "b_x_half", "b_z", "b_z_half"]
    arrs = {k: np.zeros(ntx if "_x" in k else ntz, np.float32) for k in keys}
    lib().swd_prep_cpml(ntx, ntz, pmlc, dx, dz, dt, *[_ptr(arrs[k]) for k in keys])
    return arrs


def ricker_wave(nt, f0, dt) -> np.ndarray:
    r = np.zeros(nt, np.float32)
    lib().swd_prep_ricker(nt, f0, dt, _ptr(r))
    return r


def pad_model(v, pmlc) -> np.ndarray:
    v = np.ascontiguousarray(v, np.float32)
    out = np.zeros((v.shape[0] + 2 * pmlc, v.shape[1] + 2 * pmlc), np.float32)
    lib().swd_prep_pad(v.shape[0], v.shape[1], pmlc, _ptr(v), _ptr(out))
    return out


def pow2(n) -> int:
    return lib().swd_prep_pow2(n)


def kz_taper(nfftz, dz):
    c = np.zeros(nfftz, np.float32)
    layer = lib().swd_prep_kz_taper(nfftz, dz, _ptr(c))
    return c, layer


def well_geometry(nx, nz, pmlc, dz, shotdep, offsetz):
    n = lib().swd_prep_wells(nx, nz, pmlc, dz, shotdep, offsetz, None, None)
    rix, riz = np.zeros(n, np.int32), np.zeros(n, np.int32)
    lib().swd_prep_wells(nx, nz, pmlc, dz, shotdep, offsetz, _ptr(rix), _ptr(riz))
    return rix, riz


def device_count() -> int:
    n = C.c_int(0)
    lib().swd_device_count(C.byref(n))
    return n.value


# ------------------------------------------------------------------ engine
@dataclass
class ShotSpec:
    s_ix: int
    s_iz: int
    r_ix: np.ndarray
    r_iz: np.ndarray
    nt: int


class Engine:
    """One libswd context: a padded grid on one GPU (see include/swd.h)."""

    def __init__(self, nx, nz, pml, Lc, dx, dz, dt, nt_max, device=0):
        self.nx, self.nz, self.pml, self.Lc = nx, nz, pml, Lc
        self.pmlc = pml + Lc
        self.ntx, self.ntz = nx + 2 * self.pmlc, nz + 2 * self.pmlc
        self.dx, self.dz, self.dt, self.nt_max = dx, dz, dt, nt_max
        self._h = C.c_void_p()
        g = Grid(nx, nz, pml, Lc, dx, dz, dt, nt_max, device)
        rc = lib().swd_create(C.byref(self._h), C.byref(g))
        if rc != SWD_OK:
            raise SwdError(rc, "swd_create failed (invalid grid or no CUDA device)")

    def close(self):
        if self._h:
            lib().swd_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != SWD_OK:
            raise SwdError(rc, lib().swd_last_error(self._h).decode())

    # setup -------------------------------------------------------------------------
    def set_stencil(self, rc):
        self._rc = _f32(rc)
        self._ck(lib().swd_set_stencil(self._h, _ptr(self._rc)))

    def set_cpml(self, cp: dict):
        keys = ["a_x", "a_x_half", "a_z", "a_z_half", "b_x", "b_x_half", "b_z", "b_z_half"]
        arrs = [_f32(cp[k]) for k in keys]
        self._ck(lib().swd_set_cpml(self._h, *[_ptr(a) for a in arrs]))

    def set_model(self, vp, rho):
        vp, rho = _f32(vp), _f32(rho)
        self._ck(lib().swd_set_model(self._h, _ptr(vp), _ptr(rho)))

    def set_strip_precision(self, prec: int):
        self._ck(lib().swd_set_strip_precision(self._h, prec))

    def set_source_storage(self, store: int, prec: int = STRIP_I16):
        """store=1: the RTM forward pass stores dp/dt at `prec` and the backward pass propagates
        only the receiver wavefield; store=0 reconstructs the source wavefield from strips."""
        self._ck(lib().swd_set_source_storage(self._h, store, prec))

    def set_kernel_path(self, path: int):
        """PATH_PLAIN: one cell per thread, two launches per step; PATH_FUSED: one launch per step."""
        self._ck(lib().swd_set_kernel_path(self._h, path))

    def set_option(self, option: int, value: int):
        """OPT_GRAPHS (1: time loops as CUDA graphs, 0: host launches), OPT_BATCH (shots per
        batched launch of rtm_batch, 0 = autotune)."""
        self._ck(lib().swd_set_option(self._h, option, int(value)))

    def get_option(self, option: int) -> int:
        v = C.c_int(0)
        self._ck(lib().swd_get_option(self._h, option, C.byref(v)))
        return v.value

    def set_stream(self, stream_handle: int):
        self._ck(lib().swd_set_stream(self._h, C.c_void_p(stream_handle)))

    def setup_default(self, vp, rho):
        """Stencil coefficients, CPML profiles and model, computed as the reference does."""
        self.set_stencil(cal_xishu(self.Lc))
        self.set_cpml(get_absorbing_parameters(self.ntx, self.ntz, self.pmlc, self.dx, self.dz, self.dt))
        self.set_model(vp, rho)

    def profile(self, every: int):
        """Time every kernel launch of every `every`-th step with CUDA events (0 = off)."""
        self._ck(lib().swd_profile(self._h, every))

    PROFILE_NAMES = ["fwd_v", "fwd_p", "bwd_1", "bwd_2", "fwd_step", "bwd_step", "fwd_pass_step", "bwd_pass_step",
                     "adj_v", "adj_p", "adj_pass_step"]

    def profile_read(self):
        """{kernel: (summed ms, timed launches)} for every profiling id of include/swd.h."""
        ms = np.zeros(len(self.PROFILE_NAMES), np.float64)
        n = np.zeros(len(self.PROFILE_NAMES), np.int64)
        self._ck(lib().swd_profile_read(self._h, _ptr(ms), _ptr(n)))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.PROFILE_NAMES)}

    def launch_count(self) -> int:
        return int(lib().swd_launch_count(self._h))

    def device_bytes(self) -> int:
        return lib().swd_device_bytes(self._h)

    def synchronize(self):
        self._ck(lib().swd_synchronize(self._h))

    # shots ---------------------------------------------------------------------------
    def _shot(self, s: ShotSpec):
        rix, riz = _i32(s.r_ix), _i32(s.r_iz)
        sh = Shot(int(s.s_ix), int(s.s_iz), int(s.nt), int(len(rix)), _ptr(rix).value, _ptr(riz).value)
        return sh, (rix, riz)

    def forward(self, shot: ShotSpec, rick, hrick=None, kz_coef=None, out=None):
        sh, keep = self._shot(shot)
        r_n, nt = sh.r_n, sh.nt
        seis = np.zeros((r_n, nt), np.float32) if out is None else out
        twin = hrick is not None and kz_coef is not None
        up = np.zeros((r_n, nt), np.float32) if twin else None
        dn = np.zeros((r_n, nt), np.float32) if twin else None
        rk = _f32(rick)
        hr = None if hrick is None else _f32(hrick)
        kc = None if kz_coef is None else _f32(kz_coef)
        self._ck(lib().swd_forward(self._h, C.byref(sh), _ptr(rk), _ptr(hr), _ptr(kc), _ptr(seis), _ptr(up), _ptr(dn)))
        return (seis, up, dn) if twin else seis

    def set_scatter_model(self, vp1, rho1):
        """Perturbed model of forward_scatter (padded like set_model, which must come first);
        None, None clears it."""
        if vp1 is None and rho1 is None:
            self._ck(lib().swd_set_scatter_model(self._h, None, None))
            return
        vp1, rho1 = _f32(vp1), _f32(rho1)
        self._ck(lib().swd_set_scatter_model(self._h, _ptr(vp1), _ptr(rho1)))

    def forward_scatter(self, shot: ShotSpec, rick, hrick=None, kz_coef=None):
        """Scatter record u(perturbed) - u(background) at the receivers, propagated as an exact
        scattered field; with hrick and kz_coef also its up/down traces: (seis, up, down)."""
        sh, keep = self._shot(shot)
        r_n, nt = sh.r_n, sh.nt
        seis = np.zeros((r_n, nt), np.float32)
        split = hrick is not None and kz_coef is not None
        up = np.zeros((r_n, nt), np.float32) if split else None
        dn = np.zeros((r_n, nt), np.float32) if split else None
        rk = _f32(rick)
        hr = None if hrick is None else _f32(hrick)
        kc = None if kz_coef is None else _f32(kz_coef)
        self._ck(lib().swd_forward_scatter(self._h, C.byref(sh), _ptr(rk), _ptr(hr), _ptr(kc), _ptr(seis), _ptr(up),
                                           _ptr(dn)))
        return (seis, up, dn) if split else seis

    def rtm_shot(self, shot: ShotSpec, rick, data, flags=RTM_PREPROCESS, want=("image_pp", "image_src", "fimage")):
        sh, keep = self._shot(shot)
        shape = (self.nx, self.nz)
        outs = {k: np.zeros(shape, np.float32) for k in want if k in ("image_pp", "image_src", "fimage")}
        syn = np.zeros((sh.r_n, sh.nt), np.float32) if "syn" in want else None
        rk, d = _f32(rick), _f32(data)
        self._ck(lib().swd_rtm_shot(self._h, C.byref(sh), _ptr(rk), _ptr(d), flags, _ptr(syn),
                                    _ptr(outs.get("image_pp")), _ptr(outs.get("image_src")), _ptr(outs.get("fimage"))))
        if syn is not None:
            outs["syn"] = syn
        return outs

    def rtm_forward(self, shot: ShotSpec, rick, syn=False):
        """Forward pass of an RTM shot; its final wavefield and strips stay for rtm_backward."""
        sh, keep = self._shot(shot)
        out = np.zeros((sh.r_n, sh.nt), np.float32) if syn else None
        rk = _f32(rick)
        self._ck(lib().swd_rtm_forward(self._h, C.byref(sh), _ptr(rk), _ptr(out)))
        return out

    def rtm_backward(self, shot: ShotSpec, data, flags=RTM_PREPROCESS, want=("image_pp", "image_src", "fimage")):
        """Backward pass of the shot whose rtm_forward ran just before."""
        sh, keep = self._shot(shot)
        outs = {k: np.zeros((self.nx, self.nz), np.float32) for k in want}
        d = _f32(data)
        self._ck(lib().swd_rtm_backward(self._h, C.byref(sh), _ptr(d), flags, _ptr(outs.get("image_pp")),
                                        _ptr(outs.get("image_src")), _ptr(outs.get("fimage"))))
        return outs

    def set_cig(self, thetan=10, delt=1):
        """Angle gathers for RTM shots run with flags | RTM_CIG: thetan 1-degree bins, Poynting
        vectors averaged over delt steps."""
        self._ck(lib().swd_set_cig(self._h, thetan, delt))
        self._cig_thetan = thetan

    def rtm_cig(self):
        """The last shot's angle gathers, (nx, nz, thetan) float32."""
        out = np.zeros((self.nx, self.nz, self._cig_thetan), np.float32)
        self._ck(lib().swd_rtm_cig(self._h, _ptr(out)))
        return out

    def rtm_raw(self, rcv=False):
        shp = (self.ntx, self.ntz)
        I, S = np.zeros(shp, np.float64), np.zeros(shp, np.float64)
        R = np.zeros(shp, np.float64) if rcv else None
        self._ck(lib().swd_rtm_raw(self._h, _ptr(I), _ptr(S), _ptr(R)))
        return I, S, R

    def stack(self, edge_zero=True):
        out = np.zeros((self.nx, self.nz), np.float32)
        self._ck(lib().swd_stack_get(self._h, 1 if edge_zero else 0, _ptr(out)))
        return out

    def stack_reset(self):
        self._ck(lib().swd_stack_reset(self._h))

    def rtm_batch(self, shots, ricks, datas, flags=RTM_PREPROCESS):
        n = len(shots)
        arr = (Shot * n)()
        keep = []
        for i, s in enumerate(shots):
            sh, k = self._shot(s)
            arr[i] = sh
            keep.append(k)
        rk = [_f32(r) for r in ricks]
        dd = [_f32(d) for d in datas]
        rp = (C.c_void_p * n)(*[_ptr(r).value for r in rk])
        dp = (C.c_void_p * n)(*[_ptr(d).value for d in dd])
        self._ck(lib().swd_rtm_batch(self._h, n, arr, rp, dp, flags))

    # Born modelling and its adjoint -----------------------------------------------------
    def set_checkpointing(self, every: int, prec: int = STRIP_BF16):
        """every = 0: store the background p-update sums of all steps (FP32); every > 0:
        checkpoint the background state every `every` steps at `prec` and recompute."""
        self._ck(lib().swd_set_checkpointing(self._h, every, prec))

    def checkpoint_bytes(self, nt: int) -> int:
        b = C.c_size_t(0)
        self._ck(lib().swd_checkpoint_bytes(self._h, nt, C.byref(b)))
        return b.value

    def born(self, shot: ShotSpec, rick, dkappa, out=None, ckpt=None):
        """Born data (r_n, nt) of the bulk-modulus perturbation dkappa (ntx, ntz).  `ckpt`
        (device memory of checkpoint_bytes(nt) bytes) receives the background checkpoints."""
        sh, keep = self._shot(shot)
        d = np.zeros((sh.r_n, sh.nt), np.float32) if out is None else out
        rk, dk = _f32(rick), _f32(dkappa)
        self._ck(lib().swd_born(self._h, C.byref(sh), _ptr(rk), _ptr(dk), _ptr(d), _ptr(ckpt), _nbytes(ckpt)))
        return d

    def born_adjoint(self, shot: ShotSpec, rick, resid, out=None, ckpt=None):
        """Exact adjoint of born(): (ntx, ntz) float64 gradient of <resid, born(dkappa)>."""
        sh, keep = self._shot(shot)
        g = np.zeros((self.ntx, self.ntz), np.float64) if out is None else out
        rk, r = _f32(rick), _f32(resid)
        self._ck(lib().swd_born_adjoint(self._h, C.byref(sh), _ptr(rk), _ptr(r), _ptr(g), _ptr(ckpt), _nbytes(ckpt)))
        return g

    # helpers ---------------------------------------------------------------------------
    def hilbert(self, rick):
        r = _f32(rick)
        h = np.zeros(len(r), np.float32)
        self._ck(lib().swd_hilbert(self._h, len(r), _ptr(r), _ptr(h)))
        return h

    def smooth(self, vpad, pmlc, window):
        v = _f32(vpad).copy()
        self._ck(lib().swd_smooth(self._h, v.shape[0], v.shape[1], pmlc, window, _ptr(v)))
        return v

    def preprocess(self, d, dt):
        d = _f32(d)
        out = np.zeros_like(d)
        self._ck(lib().swd_preprocess(self._h, d.shape[0], d.shape[1], dt, _ptr(d), _ptr(out)))
        return out

    def decon(self, migreal, migpsf, psfwin, filterwin, snapwin, epsilon, fft_n=(0, 0), psf_interp=0, workspace=0,
              iters=0, reg_l1=0.0, reg_l2=0.0):
        return decon(migreal, migpsf, psfwin, filterwin, snapwin, epsilon, fft_n, ctx=self._h, psf_interp=psf_interp,
                     workspace=workspace, iters=iters, reg_l1=reg_l1, reg_l2=reg_l2)


def decon_geometry(nx, nz, psfwin, filterwin, snapwin, fft_n=(0, 0)):
    p = DeconParams(nx, nz, psfwin[0], psfwin[1], filterwin[0], filterwin[1], snapwin[0], snapwin[1], 0.0,
                    fft_n[0], fft_n[1])
    w, fx, fz = C.c_int(), C.c_int(), C.c_int()
    rc = lib().swd_decon_geometry(C.byref(p), C.byref(w), C.byref(fx), C.byref(fz))
    if rc != SWD_OK:
        raise SwdError(rc, "invalid decon geometry")
    return w.value, fx.value, fz.value


def decon(migreal, migpsf, psfwin, filterwin, snapwin, epsilon, fft_n=(0, 0), ctx=None, psf_interp=0, workspace=0,
          iters=0, reg_l1=0.0, reg_l2=0.0):
    """Windowed wavenumber PSF deconvolution on the GPU (decon2d_mine's window loop);
    psf_interp=1 blends the four lattice PSFs around each window bilinearly; workspace=1 keeps
    every window's transform buffer in global memory (automatic for windows too large for
    shared memory); iters > 0 refines each window by FISTA with the L1 threshold reg_l1 (a
    fraction of the damped solution's peak) and the Tikhonov weight reg_l2 (a fraction of the
    PSF spectrum's peak power)."""
    migreal, migpsf = _f32(migreal), _f32(migpsf)
    nx, nz = migreal.shape
    p = DeconParams(nx, nz, psfwin[0], psfwin[1], filterwin[0], filterwin[1], snapwin[0], snapwin[1],
                    float(epsilon), fft_n[0], fft_n[1], int(psf_interp), int(workspace), int(iters), float(reg_l1),
                    float(reg_l2))
    dec = np.zeros((nx, nz), np.float32)
    coef = np.zeros((nx, nz), np.float32)
    rc = lib().swd_decon(ctx, C.byref(p), _ptr(migreal), _ptr(migpsf), _ptr(dec), _ptr(coef))
    if rc != SWD_OK:
        raise SwdError(rc, lib().swd_last_error(ctx).decode() if ctx else "swd_decon failed")
    return dec, coef


from . import configs  # noqa: E402  (synthetic workloads of the benchmark configurations)
