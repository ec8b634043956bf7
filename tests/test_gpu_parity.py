"""GPU parity tests: libswd (through its C ABI) against the CPU oracle on the same seeded
inputs, and against the outputs of the reference's own CUDA build.

Tolerances (relative L2): seismograms, RTM images and PSF images 1e-4 against the FP32 and
FP64 oracles; deconvolved image 1e-3; integer/index work, smoothing and preprocessing exact.
"""
import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4        # FP32 seismograms / images
TOL_DECON = 1e-3  # deconvolved image


class Case:
    """One small model set up identically for the engine and the oracle."""

    def __init__(self, swd, orc, nx=100, nz=60, pml=10, Lc=4, nt=400, dx=5.0, dz=5.0, dt=5e-4, f0=25.0,
                 seed=7, geometry="wells", smooth=0, rho_pert=False, path=1):
        rng = np.random.default_rng(seed)
        v = np.full((nx, nz), 1900.0, np.float32)
        v[:, nz // 3:] = 2400.0
        v[:, 2 * nz // 3:] = 3000.0
        v += rng.uniform(-60, 60, v.shape).astype(np.float32)
        self.nx, self.nz, self.pml, self.Lc, self.nt = nx, nz, pml, Lc, nt
        self.pmlc = pmlc = pml + Lc
        self.dx, self.dz, self.dt, self.f0 = dx, dz, dt, f0
        self.vp = orc.pad_model(v, pmlc)
        if smooth:
            self.vp = orc.smooth(self.vp, pmlc, smooth)
        self.rho = np.full_like(self.vp, 1000.0)
        if rho_pert:
            self.rho[pmlc + 20::11, pmlc + 20:-pmlc - 5:11] += self.vp[pmlc + 20::11, pmlc + 20:-pmlc - 5:11] * 1e-3
        self.ntx, self.ntz = self.vp.shape
        self.cp = orc.cpml(self.ntx, self.ntz, pmlc, dx, dz, dt)
        self.rc = orc.cal_xishu(Lc)
        self.rick = orc.ricker(nt, f0, dt)
        if geometry == "wells":
            self.rix, self.riz = orc.well_geometry(nx, nz, pmlc, dz, 0.0, 1e9)
        else:   # scattered receivers incl. a duplicated cell and cells on the PML edge
            self.rix = np.array([pmlc + 40, pmlc + 40, pmlc + 41, pmlc + 7, self.ntx - 1, 3, pmlc + 40], np.int32)
            self.riz = np.array([pmlc + 5, pmlc + 30, pmlc + 5, pmlc + 50, self.ntz // 2, 2, pmlc + 5], np.int32)
        self.sx, self.sz = pmlc + nx // 4, pmlc
        self.M = orc.Model(self.vp, self.rho, self.cp, self.rc, pmlc, Lc, nt, dx, dz, dt)
        self.G = orc.Geom(self.sx, self.sz, self.rix, self.riz)
        self.E = swd.Engine(nx, nz, pml, Lc, dx, dz, dt, nt)
        self.E.set_stencil(self.rc)
        self.E.set_cpml(self.cp)
        self.E.set_model(self.vp, self.rho)
        self.E.set_kernel_path(path)
        self.path = path
        self.shot = swd.ShotSpec(self.sx, self.sz, self.rix, self.riz, nt)


@pytest.fixture(scope="module", params=[1, 0], ids=["fused", "plain"])
def case(swd, orc, request):
    """Both kernel paths: one launch per step on shared-memory tiles, and one cell per thread."""
    return Case(swd, orc, path=request.param)


def test_forward_matches_oracle(case, orc):
    seis = case.E.forward(case.shot, case.rick)
    o32 = orc.forward(case.M, case.G, case.rick)["seis"]
    o64 = orc.forward(case.M, case.G, case.rick, dtype=np.float64)["seis"]
    assert np.abs(seis).max() > 0
    assert rel_l2(seis, o32) < TOL
    assert rel_l2(seis, o64) < TOL


@pytest.mark.parametrize("path", [1, 0], ids=["fused", "plain"])
@pytest.mark.parametrize("shape", [(37, 29, 5, 4), (64, 48, 10, 5), (97, 33, 3, 2), (130, 71, 30, 4), (70, 45, 6, 6),
                                   (41, 39, 2, 7)])
def test_forward_odd_grids_and_orders(swd, orc, shape, path):
    nx, nz, pml, Lc = shape
    c = Case(swd, orc, nx=nx, nz=nz, pml=pml, Lc=Lc, nt=220, path=path)
    seis = c.E.forward(c.shot, c.rick)
    o64 = orc.forward(c.M, c.G, c.rick, dtype=np.float64)["seis"]
    assert rel_l2(seis, o64) < TOL


@pytest.mark.parametrize("path", [1, 0], ids=["fused", "plain"])
def test_forward_scattered_receivers_and_duplicates(swd, orc, path):
    c = Case(swd, orc, geometry="scattered", nt=260, path=path)
    seis = c.E.forward(c.shot, c.rick)
    o64 = orc.forward(c.M, c.G, c.rick, dtype=np.float64)["seis"]
    assert rel_l2(seis, o64) < TOL
    assert np.array_equal(seis[0], seis[6])        # same cell -> same trace


def test_hilbert_matches_oracle(case, orc):
    for nt in (400, 2000, 2048, 6000):
        r = orc.ricker(nt, 25.0, 5e-4)
        assert rel_l2(case.E.hilbert(r), orc.hilbert1d(r)) < 1e-5


def test_kz_separation_matches_oracle(case, swd, orc):
    hr = orc.hilbert1d(case.rick)
    nfftz = swd.pow2(case.ntz)
    coef, layer = swd.kz_taper(nfftz, case.dz)
    assert layer > 0
    seis, up, dn = case.E.forward(case.shot, case.rick, hrick=hr, kz_coef=coef)
    cols = [case.pmlc, case.ntx - case.pmlc - 1]
    fw = orc.forward(case.M, case.G, case.rick, hrick=hr, col_ix=cols, dtype=np.float64)
    rec_col = (case.rix != case.pmlc).astype(np.int32)
    oup, odn = orc.kzsep(fw["cols"], case.ntz, nfftz, coef, rec_col, case.riz, np.float64)
    assert rel_l2(seis, fw["seis"]) < TOL
    assert rel_l2(up, oup) < TOL
    assert rel_l2(dn, odn) < TOL
    # with a flat taper the two halves partition the kz axis: up + down = nfftz * p
    _, up1, dn1 = case.E.forward(case.shot, case.rick, hrick=hr, kz_coef=np.ones(nfftz, np.float32))
    assert rel_l2(up1 + dn1, nfftz * seis) < 1e-5


def test_smoothing_bit_exact(case, orc):
    kat = np.load(GOLDEN / "ini_vp_kat.npz")
    a = kat["acc_corner"]
    pmlc = 21
    s = case.E.smooth(orc.pad_model(a, pmlc), pmlc, 5)[pmlc:-pmlc, pmlc:-pmlc]
    assert np.array_equal(s[0:40, 0:40].view(np.uint32), kat["ini_corner"].view(np.uint32))
    v = orc.pad_model(np.random.default_rng(2).uniform(1500, 4500, (83, 61)).astype(np.float32), 17)
    for w in (2, 5, 7):
        assert np.array_equal(case.E.smooth(v, 17, w).view(np.uint32), orc.smooth(v, 17, w).view(np.uint32))


def test_preprocess_bit_exact(case, orc):
    d = np.random.default_rng(3).standard_normal((23, 517)).astype(np.float32)
    a = case.E.preprocess(d, case.dt)
    b = orc.preprocess(d, case.dt)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def _rtm(case, orc, data, dtype):
    sh = orc.rtm_shot(case.M, case.G, case.rick, data, dtype=dtype)
    norm, fim = orc.rtm_post(case.M, sh["img"], sh["illum"], dtype)
    return sh, norm, fim


def test_rtm_shot_matches_oracle(case, swd, orc):
    data = orc.forward(case.M, case.G, case.rick)["seis"] * 1.3
    case.E.stack_reset()
    out = case.E.rtm_shot(case.shot, case.rick, data, want=("image_pp", "image_src", "fimage", "syn"))
    I, S, _ = case.E.rtm_raw()
    p = case.pmlc
    for dt in (np.float32, np.float64):
        sh, norm, fim = _rtm(case, orc, data, dt)
        assert rel_l2(out["syn"], sh["syn"]) < TOL
        assert rel_l2(I, sh["img"]) < TOL
        assert rel_l2(S, sh["illum"]) < TOL
        assert rel_l2(out["image_pp"], norm[p:-p, p:-p]) < TOL
        assert rel_l2(out["image_src"], sh["illum"][p:-p, p:-p]) < TOL
        assert rel_l2(out["fimage"], fim) < TOL
    stack = case.E.stack(edge_zero=True)
    assert rel_l2(stack, orc.edge_zero(fim.astype(np.float32), case.Lc)) < TOL


@pytest.mark.parametrize("path", [1, 0], ids=["fused", "plain"])
@pytest.mark.parametrize("shape", [(53, 41, 7, 4), (90, 37, 4, 5), (64, 64, 3, 3)])
def test_rtm_odd_grids(swd, orc, shape, path):
    nx, nz, pml, Lc = shape
    c = Case(swd, orc, nx=nx, nz=nz, pml=pml, Lc=Lc, nt=240, path=path, geometry="scattered" if nx == 64 else "wells")
    data = orc.forward(c.M, c.G, c.rick)["seis"]
    c.E.rtm_shot(c.shot, c.rick, data, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK)
    I, S, _ = c.E.rtm_raw()
    sh = orc.rtm_shot(c.M, c.G, c.rick, data, dtype=np.float64)
    assert rel_l2(I, sh["img"]) < TOL
    assert rel_l2(S, sh["illum"]) < TOL


def test_rtm_receiver_illumination_and_stack_of_two(case, swd, orc):
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    case.E.stack_reset()
    f1 = case.E.rtm_shot(case.shot, case.rick, data, flags=swd.RTM_PREPROCESS | swd.RTM_ILLUM_RCV)["fimage"]
    _, _, R = case.E.rtm_raw(rcv=True)
    assert R.max() > 0
    f2 = case.E.rtm_shot(case.shot, case.rick, 2 * data)["fimage"]
    st = case.E.stack(edge_zero=False)
    assert rel_l2(st, f1.astype(np.float64) + f2) < 1e-6


@pytest.mark.parametrize("prec,tol", [(1, 5e-3), (2, 5e-2), (3, 1e-3)], ids=["f16", "bf16", "i16"])
def test_compressed_strips(case, swd, orc, prec, tol):
    """16-bit boundary strips (per-(step, block) scale) against FP32 strips; the image error
    is printed and bounded per format."""
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    case.E.set_strip_precision(0)
    ref = case.E.rtm_shot(case.shot, case.rick, data, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK)["image_pp"]
    case.E.set_strip_precision(prec)
    got = case.E.rtm_shot(case.shot, case.rick, data, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK)["image_pp"]
    case.E.set_strip_precision(0)
    e = rel_l2(got, ref)
    print(f"strip precision {prec}: image rel-L2 vs FP32 strips {e:.3e}")
    assert 0 < e < tol


@pytest.mark.parametrize("path", [1, 0], ids=["fused", "plain"])
def test_psf_density_scatterers(swd, orc, path):
    c = Case(swd, orc, rho_pert=True, nt=300, smooth=5, path=path)
    seis = c.E.forward(c.shot, c.rick)
    o64 = orc.forward(c.M, c.G, c.rick, dtype=np.float64)["seis"]
    assert rel_l2(seis, o64) < TOL


def test_decon_matches_oracle(swd, orc):
    g = np.load(GOLDEN / "decon_ref.npz")
    cases = [(120, 100, (11, 11), (21, 21), (5, 5), 5e-4), (130, 97, (11, 9), (25, 21), (5, 4), 1e-3)]
    for k, (nx, nz, psf, flt, snap, eps) in enumerate(cases):
        dec, coef = swd.decon(g[f"mig{k}"], g[f"psf{k}"], psf, flt, snap, eps)
        assert np.array_equal(coef, g[f"coef{k}"])
        assert rel_l2(dec, g[f"dec{k}"]) < TOL_DECON


def test_decon_shipped_geometry(swd, orc):
    """The reference's own parameters (31^2 PSFs, 71^2 filter, 101^2 prime FFT, 2484 windows)
    on a seeded 845 x 702 image/PSF pair, against the oracle."""
    rng = np.random.default_rng(11)
    nx, nz = 845, 702
    mig = rng.standard_normal((nx, nz)).astype(np.float32)
    psf = np.zeros((nx, nz), np.float32)
    psf[15::31, 15::31] = 1.0
    psf[16::31, 15::31] = -0.5
    psf[15::31, 16::31] = 0.25
    dec, coef = swd.decon(mig, psf, (31, 31), (71, 71), (11, 11), 5e-4)
    odec, ocoef = orc.decon(nx, nz, mig, psf, (31, 31), (71, 71), (11, 11), 5e-4)
    assert np.array_equal(coef, ocoef)
    assert rel_l2(dec, odec) < TOL_DECON


def test_decon_workspace_variant_same_bits(swd):
    """The staged variant (transform buffer in a global workspace, passes through shared
    memory) against the shared-memory one on the reference's window geometry: same bits."""
    rng = np.random.default_rng(12)
    nx, nz = 845, 702
    mig = rng.standard_normal((nx, nz)).astype(np.float32)
    psf = np.zeros((nx, nz), np.float32)
    psf[15::31, 15::31] = 1.0
    psf[16::31, 15::31] = -0.5
    a, ca = swd.decon(mig, psf, (31, 31), (71, 71), (11, 11), 5e-4)
    b, cb = swd.decon(mig, psf, (31, 31), (71, 71), (11, 11), 5e-4, workspace=1)
    assert np.array_equal(a, b) and np.array_equal(ca, cb)


@pytest.mark.parametrize("nx,nz,psf,flt,snap,fft_n", [
    (300, 260, (31, 31), (71, 71), (11, 11), (128, 128)),   # padded to 128: the radix-2 path
    (120, 100, (5, 5), (11, 11), (3, 3), (0, 0)),           # 15-point transforms: Bluestein through 32
    (160, 150, (9, 7), (25, 19), (5, 4), (0, 0)),           # 33 x 25: 64- and 128-point, two lengths
    (600, 500, (41, 41), (241, 241), (60, 60), (0, 0)),     # 281-point: 1024, the largest register width
], ids=["pow2-128", "L15", "L33x25", "L281"])
def test_decon_transform_lengths_match_oracle(swd, orc, nx, nz, psf, flt, snap, fft_n):
    """The window transforms at the register widths the other decon tests do not reach (transform
    buffers of 32, 64, 128 and 1024 points; radix 2 and Bluestein; equal and unequal lengths per
    axis) against the oracle's FP64 FFTs."""
    rng = np.random.default_rng(31)
    mig = rng.standard_normal((nx, nz)).astype(np.float32)
    img_psf = np.zeros((nx, nz), np.float32)
    img_psf[psf[0] // 2::psf[0], psf[1] // 2::psf[1]] = 1.0
    img_psf[psf[0] // 2 + 1::psf[0], psf[1] // 2::psf[1]] = -0.3
    dec, coef = swd.decon(mig, img_psf, psf, flt, snap, 1e-3, fft_n=fft_n)
    odec, ocoef = orc.decon(nx, nz, mig, img_psf, psf, flt, snap, 1e-3, fft_n=fft_n)
    assert np.array_equal(coef, ocoef)
    assert rel_l2(dec, odec) < TOL_DECON


def test_decon_large_windows_match_oracle(swd, orc):
    """Windows whose 181 x 181 transform buffer (262 KB) exceeds shared memory take the
    workspace variant automatically; against the oracle."""
    rng = np.random.default_rng(13)
    nx, nz = 300, 260
    mig = rng.standard_normal((nx, nz)).astype(np.float32)
    psf = np.zeros((nx, nz), np.float32)
    psf[20::41, 20::41] = 1.0
    psf[21::41, 20::41] = -0.4
    psf[20::41, 22::41] = 0.3
    assert swd.decon_geometry(nx, nz, (41, 41), (141, 141), (20, 20))[1:] == (181, 181)
    dec, coef = swd.decon(mig, psf, (41, 41), (141, 141), (20, 20), 1e-3)
    odec, ocoef = orc.decon(nx, nz, mig, psf, (41, 41), (141, 141), (20, 20), 1e-3)
    assert np.array_equal(coef, ocoef)
    assert rel_l2(dec, odec) < TOL_DECON


@pytest.mark.skipif(not (GOLDEN / "ref_gpu_small.npz").exists(), reason="reference-GPU golden not generated")
def test_engine_matches_reference_cuda_build(swd, orc):
    """libswd vs the reference's own CUDA programs (AFor + AVSPRTM) on the golden case."""
    g = np.load(GOLDEN / "ref_gpu_small.npz")
    nx, nz, pml, Lc, nt, swin, window = [int(v) for v in g["case"]]
    pmlc = pml + Lc
    dx = dz = 5.0
    dt, f0 = 5e-4, 25.0
    E = swd.Engine(nx, nz, pml, Lc, dx, dz, dt, nt)
    vp = swd.pad_model(g["acc_vp"], pmlc)
    rho = np.full_like(vp, 1000.0)
    E.setup_default(vp, rho)
    rick = swd.ricker_wave(nt, f0, dt)
    hr = E.hilbert(rick)
    assert rel_l2(hr, g["rick_hilbert"]) < 1e-5
    rix, riz = swd.well_geometry(nx, nz, pmlc, dz, 0.0, 100.0)
    shot = swd.ShotSpec(pmlc + 20, pmlc, rix, riz, nt)
    coef, _ = swd.kz_taper(swd.pow2(vp.shape[1]), dz)
    obs, up, dn = E.forward(shot, rick, hrick=hr, kz_coef=coef)
    assert rel_l2(obs, g["obs"]) < TOL
    assert rel_l2(up, g["obsup"]) < TOL
    assert rel_l2(dn, g["obsdown"]) < TOL
    vs = E.smooth(vp, pmlc, window)
    assert np.array_equal(vs[pmlc:-pmlc, pmlc:-pmlc], g["ini_vp"])
    E.set_model(vs, rho)
    E.stack_reset()
    out = E.rtm_shot(shot, rick, g["obsup"], want=("image_pp", "image_src", "fimage", "syn"))
    assert rel_l2(out["syn"], g["syn"]) < TOL
    assert rel_l2(out["image_pp"], g["image_pp"]) < TOL
    assert rel_l2(out["image_src"], g["image_sources"]) < TOL
    assert rel_l2(out["fimage"], g["fimage_pp"]) < TOL
    assert rel_l2(E.stack(edge_zero=True), g["migration_pp"]) < TOL
    # PSF path: density scatterers on the smoothed model (forward/...HLForC.cpp:697-705)
    rho_s = rho.copy()
    for ix in range(pmlc + swin // 2, vp.shape[0] - pmlc - swin // 2):
        for iz in range(pmlc + swin // 2, vp.shape[1] - pmlc - 5):
            if (ix - (pmlc + swin // 2)) % swin == 0 and (iz - (pmlc + swin // 2)) % swin == 0:
                rho_s[ix, iz] += vs[ix, iz] * np.float32(1.0e-3)
    assert np.array_equal(rho_s[pmlc:-pmlc, pmlc:-pmlc], g["rho_scatter"])
    E.set_model(vs, rho)
    s0, u0, _ = E.forward(shot, rick, hrick=hr, kz_coef=coef)
    E.set_model(vs, rho_s)
    s1, u1, _ = E.forward(shot, rick, hrick=hr, kz_coef=coef)
    # the scatter data is a small difference of two large records: compare on its own scale
    assert rel_l2(s1 - s0, g["scatter"]) < 1e-2
    assert rel_l2(u1 - u0, g["scatterup"]) < 1e-2
    E.set_model(vs, rho)
    E.stack_reset()
    out = E.rtm_shot(shot, rick, g["scatterup"])
    assert rel_l2(out["image_pp"], g["image_psf"]) < TOL
    assert rel_l2(out["fimage"], g["fimage_psf"]) < TOL


def test_rtm_in_two_calls_equals_one(case, swd, orc):
    """swd_rtm_forward + swd_rtm_backward (the reference's forward/backward pair) give the images
    of swd_rtm_shot; a backward pass without its forward pass is refused."""
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    one = case.E.rtm_shot(case.shot, case.rick, data, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK, want=("image_pp", "fimage", "syn"))
    syn = case.E.rtm_forward(case.shot, case.rick, syn=True)
    two = case.E.rtm_backward(case.shot, data, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK, want=("image_pp", "fimage"))
    assert np.array_equal(syn, one["syn"])
    assert np.array_equal(two["image_pp"], one["image_pp"])
    assert np.array_equal(two["fimage"], one["fimage"])
    with pytest.raises(swd.SwdError):          # state consumed by the backward pass
        case.E.rtm_backward(case.shot, data)
    case.E.rtm_forward(case.shot, case.rick)
    case.E.forward(case.shot, case.rick)       # another pass reuses the buffers
    with pytest.raises(swd.SwdError):
        case.E.rtm_backward(case.shot, data)


@pytest.mark.parametrize("prec,tol", [(0, 1e-3), (3, 1e-3), (1, 1e-3), (2, 3e-3)], ids=["f32", "i16", "f16", "bf16"])
def test_stored_source_rtm(case, swd, orc, prec, tol):
    """RTM whose forward pass stores dp/dt (the backward pass propagates only the receiver
    wavefield) against the FP64 oracle of the reference's method, on the raw images I and S
    away from the Lc-wide band at the interior edge.  In that band the reference's interior-only
    reconstruction reads velocities of the absorbing frame frozen at the final forward state,
    so its dp/dt there is not the forward one; the stored mode keeps the forward dp/dt, and the
    reconstruction's error also reaches into the interior at the few 1e-4 level."""
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK
    case.E.set_source_storage(1, prec)
    try:
        case.E.rtm_shot(case.shot, case.rick, data, flags=flags)
        I, S, _ = case.E.rtm_raw()
    finally:
        case.E.set_source_storage(0)
    sh = orc.rtm_shot(case.M, case.G, case.rick, data, dtype=np.float64)
    m = case.pmlc + case.Lc
    sl = (slice(m, -m), slice(m, -m))
    eI, eS = rel_l2(I[sl], sh["img"][sl]), rel_l2(S[sl], sh["illum"][sl])
    print(f"stored dp/dt precision {prec}: interior I {eI:.3e}, S {eS:.3e} vs the FP64 oracle")
    assert eI < tol and eS < tol


def test_decon_psf_interpolation_matches_oracle(swd, orc):
    """The bilinear PSF interpolation option against the oracle's restatement of it, and a
    check that it differs from the nearest-PSF result where the lattice PSFs differ."""
    import importlib.util
    from conftest import GOLDEN
    spec = importlib.util.spec_from_file_location("mk", GOLDEN / "make_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    nx, nz, psf, flt, snap, eps, seed = mk.DECON_CASES[0]
    mig, psfimg, _ = mk.synthetic_decon_inputs(nx, nz, psf, seed)
    near, _ = swd.decon(mig, psfimg, psf, flt, snap, eps)
    got, coef = swd.decon(mig, psfimg, psf, flt, snap, eps, psf_interp=1)
    ref, ref_coef = orc.decon(nx, nz, mig, psfimg, psf, flt, snap, eps, psf_interp=1)
    assert np.array_equal(coef, ref_coef)
    assert rel_l2(got, ref) < TOL_DECON
    assert rel_l2(got, near) > 1e-6


@pytest.mark.parametrize("thetan,delt", [(10, 1), (40, 3)])
def test_rtm_angle_gathers_match_oracle(case, swd, orc, thetan, delt):
    """Angle-domain gathers (SWD_RTM_CIG) against the oracle's restatement of the reference's
    Poynting-vector gather kernel.  The bin of a cell is ceil(angle + ii - 0.5), so a cell whose
    angle sits within rounding of a half degree may land one bin over between two float
    implementations: the gathers and their sums over the angle axis agree in relative L2 to
    1e-2."""
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK | swd.RTM_CIG
    case.E.set_cig(thetan, delt)
    if case.path == 1:                      # the one-launch step has no gather hook
        with pytest.raises(swd.SwdError):
            case.E.rtm_shot(case.shot, case.rick, data, flags=flags)
    case.E.set_kernel_path(0)
    try:
        out = case.E.rtm_shot(case.shot, case.rick, data, flags=flags, want=("image_pp",))
        got = case.E.rtm_cig()
        plain = case.E.rtm_shot(case.shot, case.rick, data, flags=flags & ~swd.RTM_CIG, want=("image_pp",))
    finally:
        case.E.set_kernel_path(case.path)
    sh = orc.rtm_shot(case.M, case.G, case.rick, data, cig=(thetan, delt))
    p = case.pmlc
    ref = sh["cig"][p:-p, p:-p]
    assert got.shape == ref.shape
    assert np.abs(ref).max() > 0
    assert rel_l2(got, ref) < 1e-2
    assert rel_l2(got.sum(axis=2), ref.sum(axis=2)) < 1e-2
    assert np.all(got[:, :, :2] == 0)
    # the image itself is unchanged by the gathers
    assert np.array_equal(out["image_pp"], plain["image_pp"])
    with pytest.raises(swd.SwdError):
        case.E.rtm_cig()                    # the last shot accumulated none


def test_rtm_angle_gathers_reject_stored_source(case, swd, orc):
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    case.E.set_cig(10, 1)
    case.E.set_source_storage(1, 0)
    try:
        with pytest.raises(swd.SwdError):
            case.E.rtm_shot(case.shot, case.rick, data, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK | swd.RTM_CIG)
    finally:
        case.E.set_source_storage(0)


@pytest.mark.parametrize("ws", [0, 1], ids=["shared", "workspace"])
def test_decon_iterative_matches_oracle(swd, orc, ws):
    """The iterative regularised deconvolution (FISTA, L1 threshold and Tikhonov damping)
    against the oracle's FP64 restatement, with the transform buffer in shared memory and in
    the global workspace (same bits)."""
    rng = np.random.default_rng(14)
    nx, nz = 160, 130
    mig = rng.standard_normal((nx, nz)).astype(np.float32)
    psf = np.zeros((nx, nz), np.float32)
    psf[5::11, 5::11] = 1.0
    psf[6::11, 5::11] = -0.5
    psf[5::11, 7::11] = 0.3
    geo = ((11, 11), (21, 21), (5, 5))
    kw = dict(iters=40, reg_l1=2e-2, reg_l2=6e-2)
    got, coef = swd.decon(mig, psf, *geo, 5e-4, workspace=ws, **kw)
    ref, ref_coef = orc.decon(nx, nz, mig, psf, *geo, 5e-4, **kw)
    direct, _ = swd.decon(mig, psf, *geo, 5e-4)
    assert np.array_equal(coef, ref_coef)
    assert rel_l2(got, ref) < TOL_DECON
    assert rel_l2(got, direct) > 1e-2
    other, _ = swd.decon(mig, psf, *geo, 5e-4, workspace=1 - ws, **kw)
    assert np.array_equal(got, other)


def test_image_blocks_against_fp64_every_step(case, swd, orc):
    """FP32 block sums of the imaging condition (the default) against adding every step into
    FP64: the raw images agree to 1e-6 relative L2, receiver illumination included."""
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK | swd.RTM_ILLUM_RCV
    assert case.E.get_option(swd.OPT_IMAGE_BLOCKS) == 1
    case.E.rtm_shot(case.shot, case.rick, data, flags=flags, want=())
    blk = case.E.rtm_raw(rcv=True)
    case.E.set_option(swd.OPT_IMAGE_BLOCKS, 0)
    try:
        case.E.rtm_shot(case.shot, case.rick, data, flags=flags, want=())
        ref = case.E.rtm_raw(rcv=True)
    finally:
        case.E.set_option(swd.OPT_IMAGE_BLOCKS, 1)
    for a, b in zip(blk, ref):
        assert np.abs(b).max() > 0
        assert rel_l2(a, b) < 1e-6


def test_backward_pairing_by_kind_same_bits(case, swd, orc):
    """The backward step with its phases paired by kind (velocities of both wavefields in one
    launch, pressures and imaging in the other; the default) against the reference's pairing:
    the raw images I, S and R are identical bit for bit (same per-cell arithmetic)."""
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK | swd.RTM_ILLUM_RCV
    path = case.path
    case.E.set_kernel_path(0)
    try:
        assert case.E.get_option(swd.OPT_BWD_BY_KIND) == 1
        case.E.rtm_shot(case.shot, case.rick, data, flags=flags, want=())
        a = case.E.rtm_raw(rcv=True)
        case.E.set_option(swd.OPT_BWD_BY_KIND, 0)
        case.E.rtm_shot(case.shot, case.rick, data, flags=flags, want=())
        b = case.E.rtm_raw(rcv=True)
    finally:
        case.E.set_option(swd.OPT_BWD_BY_KIND, 1)
        case.E.set_kernel_path(path)
    for x, y in zip(a, b):
        assert np.abs(y).max() > 0
        assert np.array_equal(x, y)


@pytest.mark.parametrize("shape", [(100, 60, 10, 4), (53, 41, 7, 1), (90, 37, 4, 5), (70, 45, 6, 8), (130, 71, 30, 3)])
def test_tma_velocity_kernels_same_bits(swd, orc, shape):
    """The velocity kernels that read the pressure through TMA-staged shared-memory tiles
    (SWD_OPT_TMA = 1) against the per-thread loads (the default): forward seismograms and the raw RTM images are
    identical bit for bit, on grids that are not multiples of the tile and for stencil orders
    1 to 8 (one and two row chunks of the z window)."""
    nx, nz, pml, Lc = shape
    c = Case(swd, orc, nx=nx, nz=nz, pml=pml, Lc=Lc, nt=240, path=0)
    data = orc.forward(c.M, c.G, c.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK | swd.RTM_ILLUM_RCV
    c.E.set_option(swd.OPT_TMA, 1)
    seis_t = c.E.forward(c.shot, c.rick)
    c.E.rtm_shot(c.shot, c.rick, data, flags=flags, want=())
    img_t = c.E.rtm_raw(rcv=True)
    c.E.set_option(swd.OPT_TMA, 0)
    seis_p = c.E.forward(c.shot, c.rick)
    c.E.rtm_shot(c.shot, c.rick, data, flags=flags, want=())
    img_p = c.E.rtm_raw(rcv=True)
    assert np.abs(seis_p).max() > 0
    assert np.array_equal(seis_t, seis_p)
    for a, b in zip(img_t, img_p):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("shape", [(100, 60, 10, 4), (123, 97, 9, 4), (77, 141, 12, 1), (90, 75, 10, 7), (64, 48, 8, 8)],
                         ids=["100x60_Lc4", "123x97_Lc4", "77x141_Lc1", "90x75_Lc7", "64x48_Lc8"])
@pytest.mark.parametrize("strips", ["f32", "f16"])
def test_staged_pressure_kernel_same_bits(swd, orc, shape, strips):
    """The forward pressure kernel with every stencil operand staged by TMA (SWD_OPT_STAGED = 1)
    against the per-thread loads: forward seismograms, the strips (so the reconstruction) and
    the raw RTM images identical bit for bit, with FP32
    and scaled FP16 strips, on grids that are not multiples of the tile and for stencil orders
    1, 4, 7 and 8; also through the velocity kernel with TMA-staged pressure."""
    nx, nz, pml, Lc = shape
    c = Case(swd, orc, nx=nx, nz=nz, pml=pml, Lc=Lc, nt=240, path=0)
    data = orc.forward(c.M, c.G, c.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK | swd.RTM_ILLUM_RCV
    c.E.set_strip_precision({"f32": swd.STRIP_F32, "f16": swd.STRIP_F16}[strips])
    out = {}
    for staged, tma in ((0, 0), (1, 0), (1, 1)):
        c.E.set_option(swd.OPT_STAGED, staged)
        c.E.set_option(swd.OPT_TMA, tma)
        seis = c.E.forward(c.shot, c.rick)
        c.E.rtm_shot(c.shot, c.rick, data, flags=flags, want=())
        out[(staged, tma)] = (seis,) + tuple(c.E.rtm_raw(rcv=True))
    c.E.set_option(swd.OPT_STAGED, 0)
    c.E.set_option(swd.OPT_TMA, 0)
    ref = out[(0, 0)]
    assert np.abs(ref[0]).max() > 0 and np.abs(ref[1]).max() > 0
    for key, got in out.items():
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), key


def test_autotune_same_bits_and_settles(swd, orc):
    """SWD_OPT_AUTOTUNE tries the step-kernel variants of the forward pass (per-thread or TMA
    velocity x per-thread or staged pressure, the pressure kernel at 4 or 6 blocks per SM, the
    velocity kernel at 6) and of the backward pass (by-kind pairing with per-thread or TMA
    velocities, reference pairing, the pressure-and-imaging kernel at 4 or 6 blocks per SM, the
    velocity kernel at 6) on successive shots, times each over its graph replays and keeps the
    fastest: every shot's images are the untuned ones bit for bit, and after seven shots both
    choices are made and stay."""
    c = Case(swd, orc, nx=123, nz=97, pml=9, Lc=4, nt=300, path=0)
    data = orc.forward(c.M, c.G, c.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK | swd.RTM_ILLUM_RCV
    c.E.rtm_shot(c.shot, c.rick, data, flags=flags, want=())
    ref = c.E.rtm_raw(rcv=True)
    c.E.set_option(swd.OPT_AUTOTUNE, 1)
    try:
        assert c.E.get_option(swd.OPT_TUNED_FWD) == -1 and c.E.get_option(swd.OPT_TUNED_BWD) == -1
        for shot in range(9):
            c.E.rtm_shot(c.shot, c.rick, data, flags=flags, want=())
            got = c.E.rtm_raw(rcv=True)
            for a, b in zip(got, ref):
                assert np.array_equal(a, b), shot
            if shot == 6:
                fwd, bwd = c.E.get_option(swd.OPT_TUNED_FWD), c.E.get_option(swd.OPT_TUNED_BWD)
                assert fwd in (0, 1, 2, 3, 8, 16, 32) and bwd in (0, 1, 4, 8, 16, 32)
        assert (c.E.get_option(swd.OPT_TUNED_FWD), c.E.get_option(swd.OPT_TUNED_BWD)) == (fwd, bwd)
    finally:
        c.E.set_option(swd.OPT_AUTOTUNE, 0)
    assert c.E.get_option(swd.OPT_TUNED_FWD) == -1


def test_pdl_launches_same_bits(case, swd, orc):
    """RTM step kernels as programmatic dependent launches (SWD_OPT_PDL = 1) against plain
    stream order (the default), with CUDA graphs and with host launches, reconstructing and
    stored-source: the seismograms and raw images are identical bit for bit."""
    data = orc.forward(case.M, case.G, case.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK
    path = case.path
    case.E.set_kernel_path(0)
    out = {}
    try:
        for pdl in (1, 0):
            case.E.set_option(swd.OPT_PDL, pdl)
            for graphs in (1, 0):
                case.E.set_option(swd.OPT_GRAPHS, graphs)
                seis = case.E.forward(case.shot, case.rick)
                case.E.rtm_shot(case.shot, case.rick, data, flags=flags, want=())
                rec = case.E.rtm_raw()
                case.E.set_source_storage(1, swd.STRIP_I16)
                case.E.rtm_shot(case.shot, case.rick, data, flags=flags, want=())
                st = case.E.rtm_raw()
                case.E.set_source_storage(0)
                out[(pdl, graphs)] = (seis, rec[0], rec[1], st[0], st[1])
    finally:
        case.E.set_option(swd.OPT_PDL, 0)
        case.E.set_option(swd.OPT_GRAPHS, 1)
        case.E.set_kernel_path(path)
    ref = out[(0, 0)]
    assert np.abs(ref[0]).max() > 0
    for key, got in out.items():
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), key


@pytest.mark.parametrize("cfg", ["c2", "c5"])
def test_full_grid_images_vs_fp64_oracle(swd, orc, cfg):
    """The benchmark grids themselves (1601x801 and 4001x1601 with their CPML, stencil and
    models) on a short record (nt = 300, so the FP64 oracle finishes in seconds): raw images, illumination and the filtered image of an RTM shot against the FP64
    oracle of the reference's method, within the 1e-4 parity tolerance (the images' target is
    1e-3)."""
    from swd_b200 import configs
    w = configs.CONFIGS[cfg]()
    nt = 300
    p = w.pmlc
    vmig = swd.pad_model(w.vp_mig, p)
    vtrue = swd.pad_model(w.vp, p)
    rho = np.full_like(vmig, 1000.0)
    rick = swd.ricker_wave(nt, w.f0, w.dt)
    # a short record reaches only the shallow part of the grid: source at mid-surface, a
    # receiver line 20 cells away over the top 100 rows
    sx, sz = p + w.nx // 2, p
    rx = np.full(100, sx + 20, np.int32)
    rz = (p + 2 + np.arange(100)).astype(np.int32)
    shot = swd.ShotSpec(sx, sz, rx, rz, nt)
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, nt)
    E.setup_default(vtrue, rho)
    data = E.forward(shot, rick)                    # observed data in the true model
    E.set_model(vmig, rho)
    out = E.rtm_shot(shot, rick, data, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK, want=("fimage",))
    I, S, _ = E.rtm_raw()
    cp = swd.get_absorbing_parameters(w.ntx, w.ntz, p, w.dx, w.dz, w.dt)
    M = orc.Model(vmig, rho, cp, swd.cal_xishu(w.Lc), p, w.Lc, nt, w.dx, w.dz, w.dt)
    G = orc.Geom(sx, sz, rx, rz)
    sh = orc.rtm_shot(M, G, rick, data, dtype=np.float64)
    _, fim = orc.rtm_post(M, sh["img"], sh["illum"], np.float64)
    eI, eS, eF = rel_l2(I, sh["img"]), rel_l2(S, sh["illum"]), rel_l2(out["fimage"], fim)
    print(f"{cfg} grid, nt={nt}: I {eI:.2e}  S {eS:.2e}  filtered image {eF:.2e} vs FP64")
    assert np.abs(sh["img"]).max() > 0
    assert eI < TOL and eS < TOL and eF < TOL


def _lean_blocks(c):
    """Blocks (8 columns x 128 rows) of the step kernels inside the lean box, computed from the
    case's CPML arrays the way the engine does; the lean-path test needs some."""
    def span(a, ah, n):
        lo, hi = c.pmlc + c.Lc, n - c.pmlc - c.Lc
        zero = (np.asarray(a) == 0) & (np.asarray(ah) == 0)
        while lo < hi and not zero[lo]:
            lo += 1
        while hi > lo and not zero[hi - 1]:
            hi -= 1
        return (lo, hi) if zero[lo:hi].all() else (0, 0)
    lx0, lx1 = span(c.cp["a_x"], c.cp["a_x_half"], c.ntx)
    lz0, lz1 = span(c.cp["a_z"], c.cp["a_z_half"], c.ntz)
    bx = sum(1 for b in range(c.ntx // 8 + 1) if 8 * b >= lx0 and 8 * b + 8 <= lx1)
    bz = sum(1 for b in range(c.ntz // 128 + 1) if 128 * b >= lz0 and 128 * b + 128 <= lz1)
    return bx * bz


@pytest.mark.parametrize("shape", [(101, 300, 10, 4), (77, 420, 12, 1), (90, 390, 10, 7), (64, 310, 8, 8)],
                         ids=["101x300_Lc4", "77x420_Lc1", "90x390_Lc7", "64x310_Lc8"])
@pytest.mark.parametrize("strips", ["f32", "f16"])
def test_lean_blocks_same_bits(swd, orc, shape, strips):
    """The step kernels' lean path (blocks inside the CPML-free, strip-free box: no update guards,
    CPML branches or strip code) against the general path for every block (SWD_OPT_LEAN = 0): the
    forward record, the raw RTM images (by-kind and reference pairing), the stored-source images and
    the twin record with its up/down split are identical bit for bit, with FP32 and FP16 strips, on
    grids that are not multiples of the block and for stencil orders 1, 4, 7 and 8."""
    nx, nz, pml, Lc = shape
    c = Case(swd, orc, nx=nx, nz=nz, pml=pml, Lc=Lc, nt=200, path=0)
    assert _lean_blocks(c) > 0
    data = orc.forward(c.M, c.G, c.rick)["seis"]
    flags = swd.RTM_PREPROCESS | swd.RTM_NO_STACK | swd.RTM_ILLUM_RCV
    c.E.set_strip_precision({"f32": swd.STRIP_F32, "f16": swd.STRIP_F16}[strips])
    hr = c.E.hilbert(c.rick)
    coef, _ = swd.kz_taper(swd.pow2(c.ntz), c.dz)
    out = {}
    for lean in (1, 0):
        c.E.set_option(swd.OPT_LEAN, lean)
        assert c.E.get_option(swd.OPT_LEAN) == lean
        r = [c.E.forward(c.shot, c.rick)]
        c.E.rtm_shot(c.shot, c.rick, data, flags=flags, want=())
        r += list(c.E.rtm_raw(rcv=True))
        c.E.set_option(swd.OPT_BWD_BY_KIND, 0)
        c.E.rtm_shot(c.shot, c.rick, data, flags=flags, want=())
        r += list(c.E.rtm_raw(rcv=True))
        c.E.set_option(swd.OPT_BWD_BY_KIND, 1)
        c.E.set_source_storage(1, swd.STRIP_I16)
        c.E.rtm_shot(c.shot, c.rick, data, flags=flags, want=())
        r += list(c.E.rtm_raw(rcv=True))
        c.E.set_source_storage(0)
        r += list(c.E.forward(c.shot, c.rick, hrick=hr, kz_coef=coef))
        out[lean] = r
    c.E.set_option(swd.OPT_LEAN, 1)
    assert np.abs(out[1][0]).max() > 0 and np.abs(out[1][1]).max() > 0
    for i, (a, b) in enumerate(zip(out[1], out[0])):
        assert np.array_equal(a, b), i
