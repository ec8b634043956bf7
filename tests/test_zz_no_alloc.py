"""GPU test of swd_decon_noalloc, the deconvolution entry point that allocates nothing.

It exists for callers that cannot allocate device memory while they run (plug-in hosts that
own the device memory pool, services that reserve memory up front because cudaFree
synchronises the whole device).  Its scratch is a fixed 16 MiB static device array, so the
caller passes device buffers for the inputs and outputs.  The test calls it several times in
a row through the C ABI, on different inputs, and checks each result against the allocating
swd_decon within the decon tolerance used by the other tests.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_DECON = 1e-3


def _inputs(seed, nx, nz, psfwin):
    rng = np.random.default_rng(seed)
    mig = rng.standard_normal((nx, nz)).astype(np.float32)
    psf = np.zeros((nx, nz), np.float32)
    psf[psfwin[0] // 2::psfwin[0], psfwin[1] // 2::psfwin[1]] = 1.0
    psf[psfwin[0] // 2 + 1::psfwin[0], psfwin[1] // 2::psfwin[1]] = rng.uniform(-0.5, 0.5)
    return mig, psf


def test_noalloc_decon_matches_allocating_decon_twice(swd):
    import torch
    L = swd.lib()
    L.swd_decon_noalloc.argtypes = [C.POINTER(swd.DeconParams)] + [C.c_void_p] * 5
    L.swd_decon_noalloc.restype = C.c_int
    # (nx, nz, psf, filter, snap, eps, seed, workspace, iterations)
    cases = [(845, 702, (31, 31), (71, 71), (11, 11), 5e-4, 21, 0, 0),   # the reference's own window geometry
             (300, 257, (11, 9), (25, 21), (5, 4), 1e-3, 22, 0, 0),
             (300, 257, (11, 9), (25, 21), (5, 4), 1e-3, 23, 1, 0),      # buffers in the scratch workspace
             # The reference geometry's 2484 window slots take half of the static array, so the
             # per-CTA workspaces that fit in the rest are fewer than the CTAs the allocating
             # entry point runs (one or more per SM): 103 CTAs of two 101^2 buffers with workspace = 1,
             # 41 CTAs of five with the iterative option.  Fewer CTAs then walk more windows.
             (845, 702, (31, 31), (71, 71), (11, 11), 5e-4, 24, 1, 0),
             (845, 702, (31, 31), (71, 71), (11, 11), 5e-4, 25, 0, 3)]
    stream = torch.cuda.current_stream()
    for nx, nz, psfw, fltw, snapw, eps, seed, ws, iters in cases:
        mig, psf = _inputs(seed, nx, nz, psfw)
        ref_dec, ref_coef = swd.decon(mig, psf, psfw, fltw, snapw, eps, workspace=ws, iters=iters, reg_l1=0.02,
                                      reg_l2=0.05)
        d_mig, d_psf = torch.from_numpy(mig).cuda(), torch.from_numpy(psf).cuda()
        d_dec = torch.full((nx, nz), float("nan"), device="cuda")
        d_coef = torch.full((nx, nz), float("nan"), device="cuda")
        p = swd.DeconParams(nx, nz, psfw[0], psfw[1], fltw[0], fltw[1], snapw[0], snapw[1], eps, 0, 0, 0, ws, iters,
                            0.02, 0.05)
        rc = L.swd_decon_noalloc(C.byref(p), d_mig.data_ptr(), d_psf.data_ptr(), d_dec.data_ptr(),
                                 d_coef.data_ptr(), stream.cuda_stream)
        assert rc == swd.SWD_OK
        torch.cuda.synchronize()
        dec, coef = d_dec.cpu().numpy(), d_coef.cpu().numpy()
        assert np.all(np.isfinite(dec))
        assert rel_l2(coef, ref_coef) < 1e-6
        assert rel_l2(dec, ref_dec) < TOL_DECON


def test_noalloc_decon_rejects_oversize_and_host_pointers(swd):
    import torch
    L = swd.lib()
    L.swd_decon_noalloc.argtypes = [C.POINTER(swd.DeconParams)] + [C.c_void_p] * 5
    L.swd_decon_noalloc.restype = C.c_int
    # 4000 x 4000 with small windows needs far more than the 16 MiB of static scratch
    big = swd.DeconParams(4000, 4000, 11, 11, 21, 21, 5, 5, 1e-3, 0, 0)
    d = torch.zeros(16, device="cuda")
    assert L.swd_decon_noalloc(C.byref(big), d.data_ptr(), d.data_ptr(), d.data_ptr(), d.data_ptr(), None) == 6
    small = swd.DeconParams(120, 100, 11, 11, 21, 21, 5, 5, 1e-3, 0, 0)
    h = np.zeros((120, 100), np.float32)
    assert L.swd_decon_noalloc(C.byref(small), h.ctypes.data, h.ctypes.data, h.ctypes.data, h.ctypes.data,
                               None) == swd.SWD_ERR_ARG
