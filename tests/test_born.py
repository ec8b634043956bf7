"""Born modelling and its exact adjoint (LSRTM / velocity gradients) through the C ABI,
against the CPU oracle and against the identities that define an adjoint.

Tolerances: Born data and adjoint gradients 1e-4 relative L2 against the FP64 oracle (FP32
engine); dot-product identity 1e-5 relative (FP32 wavefields, FP64 imaging); FP32
checkpoints reproduce full storage exactly; 16-bit checkpoints within the bounds stated in
CKPT_TOL against the FP32 full-storage gradient.
"""
import numpy as np
import pytest

from conftest import rel_l2
from test_gpu_parity import Case

pytestmark = pytest.mark.gpu

TOL = 1e-4
TOL_DOT = 1e-5
CKPT_TOL = {"f16": 2e-3, "bf16": 2e-2, "i16": 1e-3}   # gradient rel-L2 vs FP32 full storage


def _dk(case, seed=3, density=None):
    """bulk-modulus perturbation on the interior: dense Gaussian, or sparse spikes"""
    rng = np.random.default_rng(seed)
    kap = case.rho.astype(np.float64) * case.vp.astype(np.float64) ** 2
    r = np.zeros_like(kap)
    p = case.pmlc
    inner = rng.standard_normal((case.nx, case.nz))
    if density:
        inner *= rng.random((case.nx, case.nz)) < density
    r[p:-p, p:-p] = 0.05 * inner
    return (2 * kap * r).astype(np.float32)


@pytest.fixture(scope="module")
def bcase(swd, orc):
    return Case(swd, orc, path=0, nt=400)


@pytest.fixture(scope="module")
def bcase_scattered(swd, orc):
    return Case(swd, orc, path=0, nt=300, geometry="scattered")


@pytest.mark.parametrize("which", ["wells", "scattered"])
def test_born_data_matches_oracle(bcase, bcase_scattered, orc, which):
    c = bcase if which == "wells" else bcase_scattered
    dk = _dk(c)
    d = c.E.born(c.shot, c.rick, dk)
    ref = orc.born(c.M, c.G, c.rick, dk, np.float64)
    assert rel_l2(d, ref) < TOL


@pytest.mark.parametrize("which", ["wells", "scattered"])
def test_born_adjoint_matches_oracle(bcase, bcase_scattered, orc, which, swd):
    c = bcase if which == "wells" else bcase_scattered
    rng = np.random.default_rng(11)
    resid = rng.standard_normal((len(c.rix), c.nt)).astype(np.float32)
    c.E.set_checkpointing(0)
    g = c.E.born_adjoint(c.shot, c.rick, resid)
    ref = orc.born_adjoint(c.M, c.G, c.rick, resid, np.float64)
    assert rel_l2(g, ref) < TOL
    c.E.set_checkpointing(50, swd.STRIP_BF16)


@pytest.mark.parametrize("every", [0, 50])
def test_dot_product(bcase, swd, every):
    """<r, L dk> = <L^T r, dk> with both sides from the engine."""
    c = bcase
    c.E.set_checkpointing(every, swd.STRIP_F32)
    rng = np.random.default_rng(5)
    for trial in range(3):
        dk = _dk(c, seed=100 + trial)
        resid = rng.standard_normal((len(c.rix), c.nt)).astype(np.float32)
        d = c.E.born(c.shot, c.rick, dk)
        g = c.E.born_adjoint(c.shot, c.rick, resid)
        lhs = float(np.dot(resid.astype(np.float64).ravel(), d.astype(np.float64).ravel()))
        rhs = float(np.dot(g.ravel(), dk.astype(np.float64).ravel()))
        assert abs(lhs - rhs) <= TOL_DOT * abs(lhs), (lhs, rhs)
    c.E.set_checkpointing(50, swd.STRIP_BF16)


@pytest.mark.parametrize("every", [50, 64, 7, 400, 1000])
def test_fp32_checkpoints_equal_full_storage(bcase, swd, every):
    """Recomputing segments from FP32 snapshots replays the same kernels on the same state:
    the gradient equals the full-storage one (intervals that divide nt, leave a short last
    segment, are longer than the shot)."""
    c = bcase
    resid = np.random.default_rng(2).standard_normal((len(c.rix), c.nt)).astype(np.float32)
    c.E.set_checkpointing(0)
    full = c.E.born_adjoint(c.shot, c.rick, resid)
    c.E.set_checkpointing(every, swd.STRIP_F32)
    ck = c.E.born_adjoint(c.shot, c.rick, resid)
    assert rel_l2(ck, full) < 1e-6
    c.E.set_checkpointing(50, swd.STRIP_BF16)


@pytest.mark.parametrize("prec", ["f16", "bf16", "i16"])
def test_16bit_checkpoints_error(bcase, swd, prec):
    c = bcase
    resid = np.random.default_rng(4).standard_normal((len(c.rix), c.nt)).astype(np.float32)
    c.E.set_checkpointing(0)
    full = c.E.born_adjoint(c.shot, c.rick, resid)
    c.E.set_checkpointing(50, {"f16": swd.STRIP_F16, "bf16": swd.STRIP_BF16, "i16": swd.STRIP_I16}[prec])
    ck = c.E.born_adjoint(c.shot, c.rick, resid)
    err = rel_l2(ck, full)
    print(f"{prec} checkpoint gradient rel-L2 vs FP32 full storage: {err:.3e}")
    assert err < CKPT_TOL[prec]
    c.E.set_checkpointing(50, swd.STRIP_BF16)


def test_born_checkpoints_reused_by_adjoint(bcase, swd):
    """swd_born leaves the background snapshots in a caller buffer; the adjoint given that
    buffer skips its own background pass and gives the same gradient."""
    import torch
    c = bcase
    c.E.set_checkpointing(50, swd.STRIP_F32)
    resid = np.random.default_rng(6).standard_normal((len(c.rix), c.nt)).astype(np.float32)
    own = c.E.born_adjoint(c.shot, c.rick, resid)
    buf = torch.empty(c.E.checkpoint_bytes(c.nt), dtype=torch.uint8, device="cuda")
    c.E.born(c.shot, c.rick, _dk(c), ckpt=buf)
    reused = c.E.born_adjoint(c.shot, c.rick, resid, ckpt=buf)
    assert rel_l2(reused, own) < 1e-6
    c.E.set_checkpointing(50, swd.STRIP_BF16)


def _ops(swd, case, nshots=2):
    from swd_b200 import lsrtm
    ops = []
    for k in range(nshots):
        sx = case.pmlc + 10 + k * (case.nx - 20) // max(nshots - 1, 1)
        shot = swd.ShotSpec(sx, case.pmlc, case.rix, case.riz, case.nt)
        ops.append(lsrtm.BornOperator(case.E, shot, case.rick, case.vp, case.rho))
    return ops


def test_lsrtm_autograd_finite_differences(bcase, swd):
    """J(r) = 1/2 sum ||L r - d||^2 over 2 shots: autograd gradient against central
    differences along 32 random directions (J is quadratic, so the difference is exact up to
    rounding), and against the FP32 full-storage gradient."""
    import torch
    from swd_b200 import lsrtm
    c = bcase
    c.E.set_checkpointing(50, swd.STRIP_BF16)
    ops = _ops(swd, c)
    rng = np.random.default_rng(20261207)
    r_true = torch.tensor(0.05 * rng.standard_normal((c.nx, c.nz)) * (rng.random((c.nx, c.nz)) < 0.01),
                          dtype=torch.float32, device="cuda")
    with torch.no_grad():
        data = [lsrtm.born(r_true, op) for op in ops]
    r = torch.zeros((c.nx, c.nz), dtype=torch.float32, device="cuda", requires_grad=True)
    J = lsrtm.lsrtm_objective(r, ops, data)
    J.backward()
    g = r.grad.double().clone()
    # FP32 full-storage gradient
    c.E.set_checkpointing(0)
    r2 = torch.zeros_like(r, requires_grad=True)
    lsrtm.lsrtm_objective(r2, ops, data).backward()
    g_full = r2.grad.double()
    err_full = float((g - g_full).norm() / g_full.norm())
    print(f"BF16-checkpoint LSRTM gradient vs FP32 full storage: {err_full:.3e}")
    assert err_full < CKPT_TOL["bf16"]
    # finite differences with the exact (full-storage) gradient
    worst = 0.0
    for k in range(32):
        h = torch.tensor(rng.standard_normal((c.nx, c.nz)), dtype=torch.float32, device="cuda")
        eps = 0.05
        with torch.no_grad():
            jp = lsrtm.lsrtm_objective(eps * h, ops, data).item()
            jm = lsrtm.lsrtm_objective(-eps * h, ops, data).item()
        fd = (jp - jm) / (2 * eps)
        an = float((g_full * h.double()).sum())
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-30))
    print(f"worst FD mismatch over 32 directions: {worst:.3e}")
    assert worst < 1e-3
    c.E.set_checkpointing(50, swd.STRIP_BF16)


def test_velocity_gradient_finite_differences(bcase, swd):
    """Nonlinear modelling d = F(vp): autograd velocity gradient against central differences
    of J(vp) = 1/2 ||F(vp) - d_obs||^2 along random smooth directions."""
    import torch
    from swd_b200 import lsrtm
    c = bcase
    c.E.set_checkpointing(0)
    vp0 = torch.tensor(c.vp, device="cuda")
    rho = torch.tensor(c.rho, device="cuda")
    p = c.pmlc
    obs = lsrtm.modelling(vp0 * 1.0, c.E, c.shot, c.rick, rho).detach()
    # start from a model 2% slower in a central block, so the residual is non-zero
    pert = torch.zeros_like(vp0)
    pert[p + 30:p + 70, p + 20:p + 45] = -0.02
    v = (vp0 * (1 + pert)).requires_grad_(True)
    J = 0.5 * ((lsrtm.modelling(v, c.E, c.shot, c.rick, rho) - obs).double() ** 2).sum()
    J.backward()
    g = v.grad.double()
    rng = np.random.default_rng(9)
    for k in range(4):
        h = torch.zeros_like(vp0)
        xs, zs = rng.integers(p + 10, p + c.nx - 30), rng.integers(p + 10, p + c.nz - 25)
        h[xs:xs + 20, zs:zs + 15] = float(rng.choice([-1.0, 1.0])) * 5.0
        eps = 1.0
        with torch.no_grad():
            jp = 0.5 * ((lsrtm.modelling(v + eps * h, c.E, c.shot, c.rick, rho) - obs).double() ** 2).sum().item()
            jm = 0.5 * ((lsrtm.modelling(v - eps * h, c.E, c.shot, c.rick, rho) - obs).double() ** 2).sum().item()
        fd = (jp - jm) / (2 * eps)
        an = float((g * h.double()).sum())
        assert abs(fd - an) < 2e-2 * abs(an), (k, fd, an)
    c.E.set_model(c.vp, c.rho)
    c.E.set_checkpointing(50, swd.STRIP_BF16)


def test_gradient_resembles_rtm_image(swd, orc):
    """At r = 0 the LSRTM gradient is the migration -L^T d of the scattered data; it must
    image the same reflectors as the reference's RTM (cross-correlation imaging of the
    back-propagated data): correlation coefficient on the interior."""
    import torch
    from swd_b200 import lsrtm
    c = Case(swd, orc, path=0, nt=600, nx=120, nz=80, smooth=3)
    c.E.set_checkpointing(0)
    op = lsrtm.BornOperator(c.E, c.shot, c.rick, c.vp, c.rho)
    rng = np.random.default_rng(1)
    r_true = np.zeros((c.nx, c.nz))
    r_true[20:100:16, 15:70:11] = 0.05
    rt = torch.tensor(r_true, dtype=torch.float32, device="cuda")
    with torch.no_grad():
        d = lsrtm.born(rt, op)
    g = op.adjoint(d).cpu().numpy()
    img = c.E.rtm_shot(c.shot, c.rick, d.cpu().numpy(), flags=0, want=("image_pp",))["image_pp"]
    I, S, _ = c.E.rtm_raw()
    raw = I[c.pmlc:-c.pmlc, c.pmlc:-c.pmlc]
    sl = (slice(10, c.nx - 10), slice(8, c.nz - 8))
    a, b = g[sl].ravel(), raw[sl].ravel()
    corr = float(np.corrcoef(a, b)[0, 1])
    print(f"corr(gradient, RTM cross-correlation image) = {corr:.3f}")
    assert abs(corr) > 0.8
    del rng, img, S


def test_born_survey_on_engine_pool_equals_sequential(bcase, swd):
    """The survey-level Born function over a pool of three engines (shots run concurrently
    from three host threads) gives the per-shot data bit for bit and the sequential autograd
    gradient to FP32 summation order (1e-6)."""
    import torch
    from swd_b200 import lsrtm
    c = bcase
    c.E.set_checkpointing(50, swd.STRIP_BF16)
    ops = _ops(swd, c, nshots=5)
    engines = []
    for _ in range(3):
        E = swd.Engine(c.nx, c.nz, c.pml, c.Lc, c.dx, c.dz, c.dt, c.nt)
        E.set_stencil(c.rc)
        E.set_cpml(c.cp)
        E.set_model(c.vp, c.rho)
        E.set_kernel_path(0)
        E.set_checkpointing(50, swd.STRIP_BF16)
        engines.append(E)
    pool = lsrtm.EnginePool(engines)
    try:
        rng = np.random.default_rng(5)
        r_true = torch.tensor(0.05 * rng.standard_normal((c.nx, c.nz)), dtype=torch.float32, device="cuda")
        with torch.no_grad():
            seq = [lsrtm.born(r_true, op) for op in ops]
            par = lsrtm.born_survey(r_true, ops, pool)
        for a, b in zip(seq, par):
            assert torch.equal(a, b)
        data = [0.7 * d for d in seq]
        r1 = torch.zeros((c.nx, c.nz), dtype=torch.float32, device="cuda", requires_grad=True)
        lsrtm.lsrtm_objective(r1, ops, data).backward()
        r2 = torch.zeros_like(r1, requires_grad=True)
        lsrtm.lsrtm_objective(r2, ops, data, pool=pool).backward()
        err = float((r1.grad.double() - r2.grad.double()).norm() / r1.grad.double().norm())
        assert err < 1e-6
    finally:
        pool.close()


def test_born_on_the_lsrtm_grid_vs_fp64_oracle(swd, orc):
    """Born data and the checkpointed (BF16, every 50 steps) and full-storage adjoint gradients
    on the LSRTM benchmark grid itself (801x401 with its CPML, stencil and migration model; a
    300-step record with a shallow receiver line) against the FP64 oracle."""
    from swd_b200 import configs
    w = configs.c4()
    nt, p = 300, w.pmlc
    vp = swd.pad_model(w.vp_mig, p)
    rho = np.full_like(vp, 1000.0)
    rick = swd.ricker_wave(nt, w.f0, w.dt)
    sx, sz = p + w.nx // 2, p
    rx = np.full(80, sx + 15, np.int32)
    rz = (p + 2 + np.arange(80)).astype(np.int32)
    shot = swd.ShotSpec(sx, sz, rx, rz, nt)
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, nt)
    E.setup_default(vp, rho)
    dk = np.zeros_like(vp)
    dk[p:-p, p:-p] = 2 * 1000.0 * w.vp_mig ** 2 * w.extra["reflectivity"]
    dk = dk.astype(np.float32)
    cp = swd.get_absorbing_parameters(w.ntx, w.ntz, p, w.dx, w.dz, w.dt)
    M = orc.Model(vp, rho, cp, swd.cal_xishu(w.Lc), p, w.Lc, nt, w.dx, w.dz, w.dt)
    G = orc.Geom(sx, sz, rx, rz)
    d = E.born(shot, rick, dk)
    ref = orc.born(M, G, rick, dk, np.float64)
    resid = (0.5 * ref).astype(np.float32)
    gref = orc.born_adjoint(M, G, rick, resid, np.float64)
    E.set_checkpointing(0)
    g_full = E.born_adjoint(shot, rick, resid)
    E.set_checkpointing(50, swd.STRIP_BF16)
    g_ck = E.born_adjoint(shot, rick, resid)
    e_d, e_full, e_ck = rel_l2(d, ref), rel_l2(g_full, gref), rel_l2(g_ck, gref)
    print(f"LSRTM grid, nt={nt}: Born data {e_d:.2e}, gradient {e_full:.2e} (full), {e_ck:.2e} (BF16 checkpoints)")
    assert np.abs(ref).max() > 0 and np.abs(gref).max() > 0
    assert e_d < TOL and e_full < TOL and e_ck < CKPT_TOL["bf16"]
