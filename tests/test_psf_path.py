"""The PSF path against FP64: scatter records and PSF images.

The PSF data of the reference's scatter mode (forward/acoustic_hilbert_fftkz_HLForC.cpp:
620-795) are the difference of two FP32 records, with and without density scatter points
(rho += 1e-3 vp on a lattice, :697-705).  On the golden case (tests/golden/ref_gpu_small.npz)
that difference is about 2e-4 of the record, so FP32 rounding of either record becomes a
relative error of about 1e-3 of the difference.  These tests put both programs next to the FP64
oracle's difference of two double-precision records on the same inputs: the reference's own
record (CPU test, from the golden file), the engine's difference of two records, and the
engine's scattered-field mode, which propagates the difference itself (GPU tests).
"""
import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

GOLD = GOLDEN / "ref_gpu_small.npz"
pytestmark = pytest.mark.skipif(not GOLD.exists(), reason="reference-GPU golden not generated")


class PsfCase:
    """The golden case's scatter-mode inputs, built with the oracle's host preparation."""

    def __init__(self, orc):
        g = self.g = np.load(GOLD)
        nx, nz, pml, Lc, nt, swin, window = [int(v) for v in g["case"]]
        self.nx, self.nz, self.pml, self.Lc, self.nt = nx, nz, pml, Lc, nt
        self.pmlc = p = pml + Lc
        self.dx = self.dz = 5.0
        self.dt, self.f0 = 5e-4, 25.0
        vp = orc.pad_model(g["acc_vp"], p)
        self.vs = orc.smooth(vp, p, window)
        self.rho = np.full_like(self.vs, 1000.0)
        # density scatter points on the smoothed model, the reference's lattice rule
        rs = self.rho.copy()
        ntx, ntz = self.vs.shape
        for ix in range(p + swin // 2, ntx - p - swin // 2):
            for iz in range(p + swin // 2, ntz - p - 5):
                if (ix - (p + swin // 2)) % swin == 0 and (iz - (p + swin // 2)) % swin == 0:
                    rs[ix, iz] += self.vs[ix, iz] * np.float32(1.0e-3)
        assert np.array_equal(rs[p:-p, p:-p], g["rho_scatter"])
        self.rho_s = rs
        self.cp = orc.cpml(ntx, ntz, p, self.dx, self.dz, self.dt)
        self.rc = orc.cal_xishu(Lc)
        self.rick = orc.ricker(nt, self.f0, self.dt)
        self.rix, self.riz = orc.well_geometry(nx, nz, p, self.dz, 0.0, 100.0)
        self.sx, self.sz = p + 20, p
        self.G = orc.Geom(self.sx, self.sz, self.rix, self.riz)

    def model(self, orc, rho):
        return orc.Model(self.vs, rho, self.cp, self.rc, self.pmlc, self.Lc, self.nt, self.dx, self.dz, self.dt)

    def fp64_scatter(self, orc):
        """FP64 oracle: difference of the perturbed and background records."""
        d1 = orc.forward(self.model(orc, self.rho_s), self.G, self.rick, dtype=np.float64)["seis"]
        d0 = orc.forward(self.model(orc, self.rho), self.G, self.rick, dtype=np.float64)["seis"]
        return d1 - d0


@pytest.fixture(scope="module")
def psf(orc):
    c = PsfCase(orc)
    c.d64 = c.fp64_scatter(orc)
    return c


def test_reference_scatter_record_vs_fp64(psf):
    """The reference's own FP32 scatter record (its CUDA AFor, run on a B200) against the FP64
    difference: its error is the FP32 cancellation of two records, about 1e-3 of the difference."""
    err = rel_l2(psf.g["scatter"], psf.d64)
    print(f"reference AFor scatter record vs FP64 difference: {err:.2e}")
    assert np.abs(psf.d64).max() < 1e-3 * np.abs(psf.g["obs"]).max()
    assert err < 1e-2


@pytest.mark.gpu
def test_engine_scatter_record_vs_fp64(swd, orc, psf):
    """The engine's two FP32 records (background, perturbed) and their difference, as the reference
    forms it, and the PSF image migrated from it, against FP64: the records within 1e-4 of FP64,
    the difference within the reference's own cancellation bound."""
    c = psf
    E = swd.Engine(c.nx, c.nz, c.pml, c.Lc, c.dx, c.dz, c.dt, c.nt)
    E.setup_default(c.vs, c.rho)
    shot = swd.ShotSpec(c.sx, c.sz, c.rix, c.riz, c.nt)
    s0 = E.forward(shot, c.rick)
    E.set_model(c.vs, c.rho_s)
    s1 = E.forward(shot, c.rick)
    d1 = orc.forward(c.model(orc, c.rho_s), c.G, c.rick, dtype=np.float64)["seis"]
    e_rec = rel_l2(s1, d1)
    e_ref = rel_l2(c.g["scatter"], c.d64)
    e_diff = rel_l2(s1 - s0, c.d64)
    print(f"engine perturbed record {e_rec:.2e}; difference of records vs FP64 {e_diff:.2e} "
          f"(reference {e_ref:.2e})")
    assert e_rec < 1e-4
    assert e_diff < max(2 * e_ref, 1e-3)
    E.close()


def _fp64_up(orc, c, rho):
    """FP64 oracle up-going record of one model (Hilbert twin + kz split of the well columns)."""
    hr = c.g["rick_hilbert"]
    ntx, ntz = c.vs.shape
    nfftz = orc.pow2_len(ntz)
    coef, _ = orc.kz_taper(nfftz, c.dz)
    fw = orc.forward(c.model(orc, rho), c.G, c.rick, hrick=hr, col_ix=[c.pmlc, ntx - c.pmlc - 1], dtype=np.float64)
    rec_col = (c.rix != c.pmlc).astype(np.int32)
    up, _ = orc.kzsep(fw["cols"], ntz, nfftz, coef, rec_col, c.riz, np.float64)
    return up, coef


@pytest.mark.gpu
def test_exact_scattered_field_vs_fp64(swd, orc, psf):
    """swd_forward_scatter propagates the difference field itself (the perturbed model's
    coefficients, secondary sources from FP64 coefficient differences): its scatter record and
    its up-going scatter record are within 1e-4 of the FP64 differences on the difference's own
    scale, and the PSF image migrated from the up-going record within 1e-4 of the FP64 oracle's
    PSF image of the FP64 record."""
    c = psf
    E = swd.Engine(c.nx, c.nz, c.pml, c.Lc, c.dx, c.dz, c.dt, c.nt)
    E.setup_default(c.vs, c.rho)
    E.set_scatter_model(c.vs, c.rho_s)
    shot = swd.ShotSpec(c.sx, c.sz, c.rix, c.riz, c.nt)
    d = E.forward_scatter(shot, c.rick)
    e_rec = rel_l2(d, c.d64)
    up1, coef = _fp64_up(orc, c, c.rho_s)
    up0, _ = _fp64_up(orc, c, c.rho)
    up64 = up1 - up0
    d2, up, dn = E.forward_scatter(shot, c.rick, hrick=c.g["rick_hilbert"], kz_coef=coef)
    assert np.array_equal(d2, d)
    e_up = rel_l2(up, up64)
    # PSF image: the engine's RTM of its up-going scatter record vs FP64 RTM of the FP64 record
    out = E.rtm_shot(shot, c.rick, up, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK, want=("image_pp", "fimage"))
    sh = orc.rtm_shot(c.model(orc, c.rho), c.G, c.rick, up64.astype(np.float32), dtype=np.float64)
    norm, fim = orc.rtm_post(c.model(orc, c.rho), sh["img"], sh["illum"], np.float64)
    p = c.pmlc
    e_img = rel_l2(out["image_pp"], norm[p:-p, p:-p])
    e_fim = rel_l2(out["fimage"], fim)
    e_ref = rel_l2(c.g["scatter"], c.d64)
    print(f"exact scattered field vs FP64: record {e_rec:.2e}, up-going {e_up:.2e}, PSF image {e_img:.2e}, "
          f"filtered PSF image {e_fim:.2e} (reference's difference of records: {e_ref:.2e})")
    assert e_rec < 1e-4 and e_up < 1e-4
    assert e_img < 1e-4 and e_fim < 1e-4
    # clearing the perturbed model turns the mode off
    E.set_scatter_model(None, None)
    with pytest.raises(swd.SwdError):
        E.forward_scatter(shot, c.rick)
    E.close()
