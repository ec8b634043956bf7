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
    well (z = 200..1400 cells); scatter points on a 40x16 lattice (spacing 100 cells, offset 50);
    FP16-scaled boundary strips."""
    rng = np.random.default_rng(SEED0 + 5)
    nx, nz = 4001, 1601
    v = random_field(nx, nz, rng, corr=80.0)
    w = Workload("c5_4001x1601_nt8000", nx, nz, 4.0, 4.0, 8000, 3.5e-4, 30, 4, 25.0, v, box_smooth(v, 15),
                 sx=[int(round(50 + s * (nx - 100) / 23)) for s in range(24)], sz=0,
                 rec_x=np.full(1201, 2000, np.int32), rec_z=np.arange(200, 1401, dtype=np.int32))
    w.scatter_x = 50 + 100 * np.arange(40)
    w.scatter_z = 50 + 100 * np.arange(16)
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
