"""CPU tests of the oracle itself: pinned against the reference's shipped data, the
reference's own sources compiled here, numpy.fft, and its own FP64 twin."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rel_l2

REF_HOST = ROOT / "oracle" / "_ref" / "librefhost_rtm.so"
REF_FWD = ROOT / "oracle" / "_ref" / "librefhost_fwd.so"
REF_DECON = ROOT / "oracle" / "_ref" / "decon2d_mine"


def test_smoothing_known_answer(orc):
    """ini_vp.bin shipped with the reference == ini_model_mine(acc_vp, window=5): interior and
    corner crops, bit for bit (acoustic_HLVSPRTMC.cpp:1473-1569)."""
    kat = np.load(GOLDEN / "ini_vp_kat.npz")
    pmlc = 21
    # interior crop: smoothing a crop reproduces the centre exactly (11x11 support)
    a = kat["acc_int"]
    s = orc.smooth(orc.pad_model(a, pmlc), pmlc, 5)[pmlc:-pmlc, pmlc:-pmlc]
    assert np.array_equal(s[5:45, 10:50].view(np.uint32), kat["ini_int"].view(np.uint32))
    # corner crop: true top/left edges -> replication and the unsmoothed first 8 rows
    c = kat["acc_corner"]
    s = orc.smooth(orc.pad_model(c, pmlc), pmlc, 5)[pmlc:-pmlc, pmlc:-pmlc]
    assert np.array_equal(s[0:40, 0:40].view(np.uint32), kat["ini_corner"].view(np.uint32))


@pytest.mark.parametrize("n", [1, 2, 3, 7, 32, 64, 101, 128, 256, 1000, 2048])
def test_fft_matches_numpy(orc, n):
    import ctypes as C
    L = orc.lib()
    L.orc_fft.argtypes = [C.c_int, np.ctypeslib.ndpointer(np.float64), C.c_int]
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign, ref in ((-1, np.fft.fft(x)), (+1, np.fft.ifft(x) * n)):
        a = np.ascontiguousarray(np.stack([x.real, x.imag], -1).ravel())
        L.orc_fft(n, a, sign)
        y = a[0::2] + 1j * a[1::2]
        assert np.abs(y - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


@pytest.mark.skipif(not REF_HOST.exists(), reason="reference host functions not built (needs the reference sources)")
def test_host_prep_bit_exact_vs_reference(orc):
    R, Fw = orc.RefHost("rtm"), orc.RefHost("fwd")
    for Lc in range(1, 8):
        assert np.array_equal(orc.cal_xishu(Lc).view(np.uint32), R.cal_xishu(Lc).view(np.uint32))
    for args in [(469, 269, 34, 5.0, 5.0, 5e-4), (128, 88, 14, 5.0, 5.0, 5e-4), (917, 766, 21, 10.0, 10.0, 1e-3),
                 (1669, 869, 34, 5.0, 5.0, 4e-4)]:
        a, b = orc.cpml(*args), R.cpml(*args)
        for k in a:
            assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k
    with tempfile.TemporaryDirectory() as d:
        for nt, f0, dt in [(2000, 25.0, 5e-4), (7000, 20.0, 1e-3), (6000, 30.0, 4e-4), (8000, 28.0, 3.5e-4)]:
            assert np.array_equal(orc.ricker(nt, f0, dt).view(np.uint32), R.ricker(nt, f0, dt, d).view(np.uint32))
    v = np.random.default_rng(3).uniform(1500, 4500, (70, 53)).astype(np.float32)
    vp = orc.pad_model(v, 12)
    for w in (1, 3, 5):
        s = orc.smooth(vp, 12, w)
        assert np.array_equal(s.view(np.uint32), R.smooth(vp, 12, w).view(np.uint32))
        assert np.array_equal(s.view(np.uint32), Fw.smooth(vp, 12, w).view(np.uint32))


def test_host_prep_random_cases_vs_reference(orc):
    """The oracle's CPML profiles, Gaussian smoothing and Ricker wavelets on random grids,
    spacings, time steps, frames, windows and frequencies equal the reference's own host
    functions (built from its sources) bit for bit, beyond the fixed cases above."""
    from hypothesis import given, settings, strategies as st
    R, Fw = orc.RefHost("rtm"), orc.RefHost("fwd")

    @settings(max_examples=60, derandomize=True, deadline=None)
    @given(ntx=st.integers(40, 1200), ntz=st.integers(40, 1200), pmlc=st.integers(6, 48),
           dx=st.sampled_from([2.0, 2.5, 4.0, 5.0, 10.0]), dz=st.sampled_from([2.0, 4.0, 5.0, 7.5]),
           dt=st.floats(2.0 ** -13, 2.0 ** -10, width=32))
    def cpml(ntx, ntz, pmlc, dx, dz, dt):
        a, b = orc.cpml(ntx, ntz, pmlc, dx, dz, dt), R.cpml(ntx, ntz, pmlc, dx, dz, dt)
        for k in a:
            assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k

    @settings(max_examples=20, derandomize=True, deadline=None)
    @given(nx=st.integers(20, 90), nz=st.integers(20, 90), pmlc=st.integers(9, 20), w=st.integers(1, 6),
           seed=st.integers(0, 2 ** 16))
    def smooth(nx, nz, pmlc, w, seed):
        v = np.random.default_rng(seed).uniform(1500, 4500, (nx, nz)).astype(np.float32)
        vp = orc.pad_model(v, pmlc)
        s = orc.smooth(vp, pmlc, w)
        assert np.array_equal(s.view(np.uint32), R.smooth(vp, pmlc, w).view(np.uint32))
        assert np.array_equal(s.view(np.uint32), Fw.smooth(vp, pmlc, w).view(np.uint32))

    @settings(max_examples=20, derandomize=True, deadline=None)
    @given(nt=st.integers(16, 9000), f0=st.floats(5.0, 60.0, width=32), dt=st.floats(2.0 ** -13, 2.0 ** -10, width=32))
    def ricker(nt, f0, dt):
        with tempfile.TemporaryDirectory() as d:
            assert np.array_equal(orc.ricker(nt, f0, dt).view(np.uint32), R.ricker(nt, f0, dt, d).view(np.uint32))

    cpml()
    smooth()
    ricker()


def test_decon_oracle_matches_reference_golden(orc):
    """Oracle decon vs the reference decon2d_mine (built from its source) on the committed
    cases; both use the same FFT, so they agree bit for bit."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mkg", GOLDEN / "make_golden.py")
    mkg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mkg)
    g = np.load(GOLDEN / "decon_ref.npz")
    for k, (nx, nz, psf, flt, snap, eps, seed) in enumerate(mkg.DECON_CASES):
        dec, coef = orc.decon(nx, nz, g[f"mig{k}"], g[f"psf{k}"], psf, flt, snap, eps)
        assert np.array_equal(coef, g[f"coef{k}"])
        assert rel_l2(dec, g[f"dec{k}"]) < 1e-12


@pytest.mark.skipif(not REF_DECON.exists(), reason="reference decon not built")
def test_decon_oracle_live_vs_reference_build(orc):
    import importlib.util
    spec = importlib.util.spec_from_file_location("mkg", GOLDEN / "make_golden.py")
    mkg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mkg)
    nx, nz, psf, flt, snap, eps = 90, 77, (9, 11), (19, 23), (4, 5), 2e-3
    mig, p, vp = mkg.synthetic_decon_inputs(nx, nz, psf, 99)
    ref_dec, ref_coef = mkg.run_ref_decon(nx, nz, mig, p, vp, psf, flt, snap, eps)
    dec, coef = orc.decon(nx, nz, mig, p, psf, flt, snap, eps)
    assert np.array_equal(coef, ref_coef)
    assert np.array_equal(dec.view(np.uint32), ref_dec.view(np.uint32))


@pytest.mark.skipif(not REF_DECON.exists(), reason="reference decon not built")
def test_decon_oracle_random_cases_vs_reference_build(orc):
    """The oracle's deconvolution on random image sizes, window sizes and damping equals the
    reference's decon2d_mine (built from its source, same FFT shim) bit for bit."""
    import importlib.util
    from hypothesis import assume, given, settings, strategies as st
    spec = importlib.util.spec_from_file_location("mkg", GOLDEN / "make_golden.py")
    mkg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mkg)
    odd = lambda lo, hi: st.integers(lo // 2, hi // 2).map(lambda k: 2 * k + 1)
    done = []

    @settings(max_examples=10, derandomize=True, deadline=None)
    @given(nx=st.integers(60, 130), nz=st.integers(60, 130), px=odd(5, 13), pz=odd(5, 13),
           kx=st.integers(2, 7), kz=st.integers(2, 7), sx=st.integers(3, 6), sz=st.integers(3, 6),
           eps=st.sampled_from([1e-3, 2e-3, 5e-3]), seed=st.integers(0, 1000))
    def check(nx, nz, px, pz, kx, kz, sx, sz, eps, seed):
        psf, flt, snap = (px, pz), (px + 2 * kx, pz + 2 * kz), (sx, sz)
        try:
            orc.decon_geometry(nx, nz, psf, flt, snap)
        except ValueError:
            assume(False)
        mig, p, vp = mkg.synthetic_decon_inputs(nx, nz, psf, seed)
        ref_dec, ref_coef = mkg.run_ref_decon(nx, nz, mig, p, vp, psf, flt, snap, eps)
        dec, coef = orc.decon(nx, nz, mig, p, psf, flt, snap, eps)
        assert np.array_equal(coef, ref_coef)
        assert np.array_equal(dec.view(np.uint32), ref_dec.view(np.uint32))
        done.append(1)

    check()
    assert len(done) >= 5


def _small_model(orc, nt=300, nx=60, nz=44, pml=8, Lc=4):
    rng = np.random.default_rng(5)
    v = np.full((nx, nz), 2000.0, np.float32)
    v[:, nz // 2:] = 2600.0
    v += rng.uniform(-30, 30, v.shape).astype(np.float32)
    pmlc = pml + Lc
    vp = orc.pad_model(v, pmlc)
    rho = np.full_like(vp, 1000.0)
    dx = dz = 5.0
    dt = 5e-4
    M = orc.Model(vp, rho, orc.cpml(vp.shape[0], vp.shape[1], pmlc, dx, dz, dt), orc.cal_xishu(Lc), pmlc, Lc, nt,
                  dx, dz, dt)
    rix, riz = orc.well_geometry(nx, nz, pmlc, dz, 0.0, 1e9)
    return M, orc.Geom(pmlc + 12, pmlc, rix, riz), orc.ricker(nt, 25.0, dt)


def test_oracle_fp32_vs_fp64(orc):
    M, G, rick = _small_model(orc)
    d = orc.forward(M, G, rick)["seis"]
    a = orc.rtm_shot(M, G, rick, d)
    b = orc.rtm_shot(M, G, rick, d, dtype=np.float64)
    assert rel_l2(a["syn"], b["syn"]) < 1e-5
    assert rel_l2(a["img"], b["img"]) < 1e-4
    assert rel_l2(a["illum"], b["illum"]) < 1e-4


def test_oracle_reconstruction_reversible(orc):
    """With the receiver data set to zero the backward pass is pure reconstruction; the
    reconstructed source wavefield must reproduce the forward illumination."""
    M, G, rick = _small_model(orc, nt=250)
    fw = orc.forward(M, G, rick, strips=True, final=True, dtype=np.float64)
    img, ill, _ = orc.rtm_backward(M, G, rick, np.zeros_like(fw["seis"]), fw["strips"], fw["final"], np.float64)
    assert np.all(img == 0)
    assert ill.max() > 0


@pytest.mark.skipif(not (GOLDEN / "ref_gpu_small.npz").exists(), reason="reference-GPU golden not generated")
def test_oracle_matches_reference_cuda_build(orc):
    """Pins the forward/RTM restatement: the oracle on the golden case reproduces the outputs
    of the reference's own CUDA programs run on a B200 (tests/golden/make_golden_ref_gpu.py)."""
    g = np.load(GOLDEN / "ref_gpu_small.npz")
    nx, nz, pml, Lc, nt, swin, window = [int(v) for v in g["case"]]
    pmlc = pml + Lc
    dx = dz = 5.0
    dt, f0 = 5e-4, 25.0
    vp = orc.pad_model(g["acc_vp"], pmlc)
    rho = np.full_like(vp, 1000.0)
    cp = orc.cpml(vp.shape[0], vp.shape[1], pmlc, dx, dz, dt)
    rc = orc.cal_xishu(Lc)
    rick = orc.ricker(nt, f0, dt)
    rix, riz = orc.well_geometry(nx, nz, pmlc, dz, 0.0, 100.0)
    G = orc.Geom(pmlc + 20, pmlc, rix, riz)
    M = orc.Model(vp, rho, cp, rc, pmlc, Lc, nt, dx, dz, dt)
    # forward (obs) and the up/down split, using the reference's own Hilbert wavelet
    hr = g["rick_hilbert"]
    nfftz = orc.pow2_len(vp.shape[1])
    coef, _ = orc.kz_taper(nfftz, dz)
    fw = orc.forward(M, G, rick, hrick=hr, col_ix=[pmlc, vp.shape[0] - pmlc - 1], dtype=np.float64)
    assert rel_l2(fw["seis"], g["obs"]) < 1e-5
    rec_col = (rix != pmlc).astype(np.int32)
    up, dn = orc.kzsep(fw["cols"], vp.shape[1], nfftz, coef, rec_col, riz, np.float64)
    assert rel_l2(up, g["obsup"]) < 1e-4
    assert rel_l2(dn, g["obsdown"]) < 1e-4
    assert rel_l2(orc.hilbert1d(rick), hr) < 1e-5
    # RTM on the smoothed model with the up-going data
    vs = orc.smooth(vp, pmlc, window)
    assert np.array_equal(vs[pmlc:-pmlc, pmlc:-pmlc], g["ini_vp"])
    Ms = orc.Model(vs, rho, cp, rc, pmlc, Lc, nt, dx, dz, dt)
    sh = orc.rtm_shot(Ms, G, rick, g["obsup"], dtype=np.float64)
    assert rel_l2(sh["syn"], g["syn"]) < 1e-5
    norm, fim = orc.rtm_post(Ms, sh["img"], sh["illum"], np.float64)
    assert rel_l2(norm[pmlc:-pmlc, pmlc:-pmlc], g["image_pp"]) < 1e-4
    assert rel_l2(sh["illum"][pmlc:-pmlc, pmlc:-pmlc], g["image_sources"]) < 1e-4
    assert rel_l2(fim, g["fimage_pp"]) < 1e-4
    mig = orc.edge_zero(fim.astype(np.float32), Lc)
    assert rel_l2(mig, g["migration_pp"]) < 1e-4


def test_oracle_born_adjoint_dot_product(orc):
    """The oracle's adjoint (written as scatters of each forward loop body, in reverse) is the
    exact transpose of its Born operator: <r, L dk> = <L^T r, dk> to FP64 rounding."""
    M, G, rick = _small_model(orc, nt=300)
    rng = np.random.default_rng(1)
    for trial in range(2):
        dk = (rng.standard_normal((M.ntx, M.ntz)) * 1e7).astype(np.float32)
        d = orc.born(M, G, rick, dk)
        r = rng.standard_normal(d.shape).astype(np.float32)
        g = orc.born_adjoint(M, G, rick, r)
        lhs = float(np.dot(r.astype(np.float64).ravel(), d.ravel()))
        rhs = float(np.dot(g.ravel(), dk.astype(np.float64).ravel()))
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_oracle_born_is_the_linearised_forward(orc):
    """Born data of dkappa = 2 kappa dv/v equal the central difference of the nonlinear
    forward modelling in vp; the mismatch falls as eps^2."""
    M, G, rick = _small_model(orc, nt=300)
    rng = np.random.default_rng(2)
    kap = M.rho.astype(np.float64) * M.vp.astype(np.float64) ** 2
    dv_rel = np.zeros_like(kap)
    p = M.pmlc
    dv_rel[p:-p, p:-p] = rng.standard_normal((M.ntx - 2 * p, M.ntz - 2 * p))
    d_born = orc.born(M, G, rick, (2 * kap * dv_rel).astype(np.float32))
    errs = []
    for eps in (1e-2, 1e-3):
        outs = []
        for s in (1, -1):
            vp2 = (M.vp.astype(np.float64) * (1 + s * eps * dv_rel)).astype(np.float32)
            M2 = orc.Model(vp2, M.rho, M.cp, M.rc, M.pmlc, M.Lc, M.nt, M.dx, M.dz, M.dt)
            outs.append(orc.forward(M2, G, rick, dtype=np.float64)["seis"])
        errs.append(rel_l2((outs[0] - outs[1]) / (2 * eps), d_born))
    assert errs[1] < 1e-4 and errs[0] / errs[1] > 30


def _decon_case():
    rng = np.random.default_rng(31)
    nx, nz = 120, 100
    mig = rng.standard_normal((nx, nz)).astype(np.float32)
    psf = np.zeros((nx, nz), np.float32)
    psf[5::11, 5::11] = 1.0
    psf[6::11, 5::11] = -0.5
    psf[5::11, 7::11] = 0.3
    return nx, nz, mig, psf


def test_decon_oracle_iterations_fixed_point_and_tikhonov_limit(orc):
    """The iterative option's oracle: started at the damped solution of the same damping and
    without the L1 term, FISTA stays at it (it is the minimiser); with a different damping
    reg_l2 it converges to the direct solution of epsilon = reg_l2."""
    nx, nz, mig, psf = _decon_case()
    geo = ((11, 11), (21, 21), (5, 5))
    d1, c1 = orc.decon(nx, nz, mig, psf, *geo, 1e-2)
    it1, ic1 = orc.decon(nx, nz, mig, psf, *geo, 1e-2, iters=20, reg_l1=0.0, reg_l2=1e-2)
    assert np.array_equal(c1, ic1)
    assert rel_l2(it1, d1) < 1e-6
    d5, _ = orc.decon(nx, nz, mig, psf, *geo, 5e-2)
    it5, _ = orc.decon(nx, nz, mig, psf, *geo, 1e-3, iters=200, reg_l1=0.0, reg_l2=5e-2)
    d3, _ = orc.decon(nx, nz, mig, psf, *geo, 1e-3)
    assert rel_l2(d3, d5) > 1e-2            # the two dampings differ visibly
    assert rel_l2(it5, d5) < 1e-5


def test_decon_oracle_l1_threshold_sparsifies(orc):
    """A positive L1 threshold shrinks the deconvolved image (smaller L1 norm, more exact
    zeros) and leaves it close to the damped solution for a small threshold."""
    nx, nz, mig, psf = _decon_case()
    geo = ((11, 11), (21, 21), (5, 5))
    base, _ = orc.decon(nx, nz, mig, psf, *geo, 5e-2, iters=60, reg_l1=0.0, reg_l2=5e-2)
    small, _ = orc.decon(nx, nz, mig, psf, *geo, 5e-2, iters=60, reg_l1=1e-3, reg_l2=5e-2)
    big, _ = orc.decon(nx, nz, mig, psf, *geo, 5e-2, iters=60, reg_l1=5e-2, reg_l2=5e-2)
    assert rel_l2(small, base) < 5e-2
    assert np.abs(big).sum() < np.abs(small).sum() < np.abs(base).sum()
