"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: every model, wavelet and geometry is generated here with
numpy.random.default_rng(20261203 + index).  Grids, spacings, record lengths, CPML width
and stencil order are the configurations' own; the layered / random-field velocity models,
interface depths and receiver placement are this project's concrete choices for the
configurations' descriptions.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SEED0 = 20261203


@dataclass
class Workload:
    name: str
    nx: int
    nz: int
    dx: float
    dz: float
    nt: int
    dt: float
    pml: int
    Lc: int
    f0: float
    vp: np.ndarray                 # true model, (nx, nz)
    vp_mig: np.ndarray             # migration model, (nx, nz)
    sx: list = field(default_factory=list)      # source cells (interior coords)
    sz: int = 0
    rec_x: np.ndarray = None       # receiver cells (interior coords)
    rec_z: np.ndarray = None
    scatter_x: np.ndarray = None   # scatter-point lattice (interior coords)
    scatter_z: np.ndarray = None
    extra: dict = field(default_factory=dict)

    @property
    def pmlc(self):
        return self.pml + self.Lc

    @property
    def ntx(self):
        return self.nx + 2 * self.pmlc

    @property
    def ntz(self):
        return self.nz + 2 * self.pmlc

    def receivers_padded(self):
        return (np.asarray(self.rec_x, np.int32) + self.pmlc, np.asarray(self.rec_z, np.int32) + self.pmlc)

    def source_padded(self, i=0):
        return self.sx[i] + self.pmlc, self.sz + self.pmlc


def box_smooth(v, npts):
    """npts x npts mean filter with edge clamping (the configurations' 15-point box)."""
    h = npts // 2
    a = np.pad(np.asarray(v, np.float64), h, mode="edge")
    c = np.cumsum(np.cumsum(a, 0), 1)
    c = np.pad(c, ((1, 0), (1, 0)))
    nx, nz = v.shape
    s = c[npts:npts + nx, npts:npts + nz] - c[:nx, npts:npts + nz] - c[npts:npts + nx, :nz] + c[:nx, :nz]
    return (s / (npts * npts)).astype(np.float32)


def layered(nx, nz, rng, vmin=1500.0, vmax=4000.0, nlayers=6, zlo=20, zhi=190, gap=10):
    """Flat layers increasing with depth; interfaces at sorted seeded depths >= gap apart."""
    while True:
        z = np.sort(rng.integers(zlo, zhi + 1, nlayers - 1))
        if np.all(np.diff(z) >= gap):
            break
    vels = np.linspace(vmin, vmax, nlayers).astype(np.float32)
    v = np.empty((nx, nz), np.float32)
    edges = [0] + list(z) + [nz]
    for k in range(nlayers):
        v[:, edges[k]:edges[k + 1]] = vels[k]
    return v, z


def random_field(nx, nz, rng, corr=50.0, vmin=1800.0, vmax=4500.0, ndip=3, dipmax=15.0):
    """Gaussian random field (FFT-filtered white noise) mapped to [vmin, vmax] plus dipping
    planar interfaces adding +200..+400 m/s steps."""
    w = rng.standard_normal((nx, nz))
    kx = np.fft.fftfreq(nx)[:, None]
    kz = np.fft.fftfreq(nz)[None, :]
    filt = np.exp(-2.0 * (np.pi * corr) ** 2 * (kx ** 2 + kz ** 2) / 4.0)
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    f = (f - f.min()) / (f.max() - f.min())
    v = vmin + (vmax - vmin - 400.0 * ndip * 0.75) * f
    xs = np.arange(nx)[:, None]
    zs = np.arange(nz)[None, :]
    for _ in range(ndip):
        z0 = rng.uniform(0.2, 0.85) * nz
        dip = np.deg2rad(rng.uniform(-dipmax, dipmax))
        step = rng.uniform(200.0, 400.0)
        v = v + step * (zs > z0 + np.tan(dip) * (xs - nx / 2))
    return np.clip(v, vmin, vmax).astype(np.float32)


def c1(parity=False):
    """401x201 at 5 m, nt=2000, dt=0.5 ms, 30-cell CPML, 8th order; 6 flat layers;
    source x=50 m at the surface, 25 Hz; 181 receivers at x=1000 m, z=50..950 m."""
    rng = np.random.default_rng(SEED0 + 1)
    nx, nz = 401, 201
    v, z = layered(nx, nz, rng)
    w = Workload("c1_401x201_nt2000", nx, nz, 5.0, 5.0, 2000, 5.0e-4, 30, 4, 25.0, v, box_smooth(v, 15),
                 sx=[10], sz=0, rec_x=np.full(181, 200, np.int32), rec_z=np.arange(10, 191, dtype=np.int32))
    w.extra["interfaces"] = z
    return w


def c2():
    """1601x801 at 5 m, nt=6000, dt=0.4 ms, 30 Hz; random-field model 1800-4500 m/s with
    3 dipping interfaces; 641 receivers in one well; 20x10 scatter lattice."""
    rng = np.random.default_rng(SEED0 + 2)
    nx, nz = 1601, 801
    v = random_field(nx, nz, rng)
    w = Workload("c2_1601x801_nt6000", nx, nz, 5.0, 5.0, 6000, 4.0e-4, 30, 4, 30.0, v, box_smooth(v, 15),
                 sx=[100], sz=0, rec_x=np.full(641, 800, np.int32), rec_z=np.arange(80, 721, dtype=np.int32))
    # 20 x 10 scatter points, spacing 79 cells from 39 (odd spacing keeps a decon PSF lattice)
    w.scatter_x = 39 + 79 * np.arange(20)
    w.scatter_z = 39 + 79 * np.arange(10)
    return w


def c3(nshots=96):
    """96 walkaway-VSP shots on 1201x601 at 5 m; nt ~ U[3000, 6000], 200-600 receivers,
    f0 ~ U[20, 35] Hz, dt = 0.4 ms."""
    rng = np.random.default_rng(SEED0 + 3)
    nx, nz = 1201, 601
    v = random_field(nx, nz, rng)
    w = Workload("c3_1201x601_96shots", nx, nz, 5.0, 5.0, 6000, 4.0e-4, 30, 4, 30.0, v, box_smooth(v, 15))
    shots = []
    for s in range(nshots):
        nt = int(rng.integers(3000, 6001))
        nr = int(rng.integers(200, 601))
        f0 = float(rng.uniform(20.0, 35.0))
        sx = int(round(10 + s * (nx - 20) / max(1, nshots - 1)))
        z0 = int(rng.integers(0, nz - nr)) if nr < nz else 0
        shots.append(dict(nt=nt, f0=f0, sx=sx, sz=0, rec_x=np.full(nr, 600, np.int32),
                          rec_z=np.arange(z0, z0 + nr, dtype=np.int32)))
    w.extra["shots"] = shots
    return w


def c4(nshots=16):
    """Differentiable LSRTM gradient: 801x401 at 5 m, nt=4000, dt=0.4 ms, 16 surface shots
    (25 Hz) recorded by 321 receivers in a central well; reflectivity dv/v = sparse spikes
    N(0, 0.05) at 1% density on the interior; background = the 15-point box-smoothed
    random-field model."""
    rng = np.random.default_rng(SEED0 + 4)
    nx, nz = 801, 401
    v = random_field(nx, nz, rng)
    w = Workload("c4_801x401_nt4000_16shots", nx, nz, 5.0, 5.0, 4000, 4.0e-4, 30, 4, 25.0, v, box_smooth(v, 15),
                 sx=[int(round(10 + s * (nx - 20) / max(1, nshots - 1))) for s in range(nshots)], sz=0,
                 rec_x=np.full(321, 400, np.int32), rec_z=np.arange(40, 361, dtype=np.int32))
    w.extra["reflectivity"] = (0.05 * rng.standard_normal((nx, nz)) * (rng.random((nx, nz)) < 0.01)).astype(np.float32)
    return w


def c5():
    """Large imaging: 4001x1601 at 4 m, nt=8000, dt=0.35 ms, 25 Hz; random-field model
    1800-4500 m/s with 3 dipping interfaces; 24 surface shots; 1201 receivers in a central
    well (z = 200..1400 cells); scatter points on a 40x16 lattice (spacing 99 cells, offset 49);
    FP16-scaled boundary strips."""
    rng = np.random.default_rng(SEED0 + 5)
    nx, nz = 4001, 1601
    v = random_field(nx, nz, rng, corr=80.0)
    w = Workload("c5_4001x1601_nt8000", nx, nz, 4.0, 4.0, 8000, 3.5e-4, 30, 4, 25.0, v, box_smooth(v, 15),
                 sx=[int(round(50 + s * (nx - 100) / 23)) for s in range(24)], sz=0,
                 rec_x=np.full(1201, 2000, np.int32), rec_z=np.arange(200, 1401, dtype=np.int32))
    # 40 x 16 scatter points, spacing 99 cells from 49 (odd spacing keeps a decon PSF lattice)
    w.scatter_x = 49 + 99 * np.arange(40)
    w.scatter_z = 49 + 99 * np.arange(16)
    w.extra["strips"] = "f16"
    return w


def small(nx=100, nz=60, nt=400, pml=10, Lc=4, dx=5.0, dz=5.0, dt=5.0e-4, f0=25.0, seed=7):
    """Small two-well parity case; nx + 2*pmlc is a multiple of 16 for nx=100, pml=10, Lc=4
    (the reference CUDA build indexes past the grid otherwise)."""
    rng = np.random.default_rng(seed)
    v, _ = layered(nx, nz, rng, nlayers=3, zlo=15, zhi=nz - 15, gap=8)
    v = v + rng.uniform(-50, 50, v.shape).astype(np.float32)
    return Workload(f"small_{nx}x{nz}_nt{nt}", nx, nz, dx, dz, nt, dt, pml, Lc, f0, v.astype(np.float32),
                    box_smooth(v, 5), sx=[nx // 4], sz=0)


CONFIGS = {"c1": c1, "c2": c2, "c3": c3, "c4": c4, "c5": c5}


@dataclass
class DeconCase:
    """One windowed PSF deconvolution: image size, PSF lattice spacing (= PSF patch size),
    filter window and taper width, damping."""
    name: str
    nx: int
    nz: int
    psfwin: tuple
    filterwin: tuple
    snapwin: tuple
    epsilon: float
    seed: int


def decon_case(cfg):
    """The deconvolution of the c2 / c5 images (PSFs on the configuration's scatter lattice;
    output windows of about 64^2 and 128^2) and the reference's own window geometry."""
    if cfg == "c2":
        return DeconCase("c2 decon: 1601x801 image, PSFs on the 79-cell scatter lattice, 63^2 output windows, "
                         "157^2 transforms", 1601, 801, (79, 79), (79, 79), (24, 24), 5e-4, SEED0 + 2)
    if cfg == "c5":
        return DeconCase("c5 decon: 4001x1601 image, PSFs on the 99-cell scatter lattice, 127^2 output windows, "
                         "227^2 transforms", 4001, 1601, (99, 99), (129, 129), (54, 54), 5e-4, SEED0 + 5)
    if cfg == "shipped":
        return DeconCase("reference window geometry: 845x702 image, 31^2 PSFs, 71^2 filter, 101^2 transforms",
                         845, 702, (31, 31), (71, 71), (11, 11), 5e-4, SEED0)
    raise KeyError(cfg)


def decon_inputs(case):
    """Seeded migration image (box-smoothed white reflectivity) and PSF image (a separable
    Ricker blob of random amplitude at every lattice point halfpsfwin + k*psfwin)."""
    rng = np.random.default_rng(case.seed)
    mig = box_smooth(rng.standard_normal((case.nx, case.nz)).astype(np.float32), 3)
    t = np.arange(-7, 8, dtype=np.float64) * 0.3
    r = ((1 - 2 * t * t) * np.exp(-t * t)).astype(np.float32)
    blob = np.outer(r, r)
    psf = np.zeros((case.nx, case.nz), np.float32)
    hx, hz = case.psfwin[0] // 2, case.psfwin[1] // 2
    for ix in range(hx, case.nx, case.psfwin[0]):
        for iz in range(hz, case.nz, case.psfwin[1]):
            x0, z0 = max(ix - 7, 0), max(iz - 7, 0)
            x1, z1 = min(ix + 8, case.nx), min(iz + 8, case.nz)
            psf[x0:x1, z0:z1] += np.float32(rng.uniform(0.5, 1.5)) * blob[x0 - ix + 7:x1 - ix + 7, z0 - iz + 7:z1 - iz + 7]
    return mig, psf


def decon_layout(case):
    """Window lattice of a deconvolution (the reference's formulas): windows, transform size,
    output window, padded image size."""
    out = {}
    for a, k in (("x", 0), ("z", 1)):
        full = case.filterwin[k] + case.psfwin[k] - 1
        outwin = 2 * (case.psfwin[k] // 10) + 2 * case.snapwin[k] + 1
        step = outwin - case.snapwin[k]
        n = -(-(getattr(case, "n" + a) + full) // step) + 1
        out.update({f"full{a}": full, f"outwin{a}": outwin, f"stepnum{a}": n, f"n{a}p": n * step})
    out["windows"] = out["stepnumx"] * out["stepnumz"]
    return out
