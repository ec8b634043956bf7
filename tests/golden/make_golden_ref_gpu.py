"""Runs the reference's own CUDA programs (AFor and AVSPRTM, built from its sources for
sm_100a by oracle/Makefile into oracle/_ref) on a small seeded model and saves their outputs
as tests/golden/ref_gpu_small.npz.  Needs a GPU; run on the B200 box:

    python tests/golden/make_golden_ref_gpu.py <output dir>/ref_gpu_small.npz

Geometry is chosen so the reference kernels stay inside their arrays: the padded width
ntx = 100 + 2*14 = 128 is a multiple of 16 (the RTM kernels' block) and of 8 (AFor's), so
fft_kz_sep_kernel's `ix <= ntx` guard and the `mx[ix]` source test never index past ntx.

The case: 100 x 60 interior, pml 10, Lc 4, dx = dz = 5 m, 400 steps of 0.5 ms, 25 Hz Ricker,
one shot at x = 100 m on the surface, offsetz = 100 m (21 depths in each of the two edge
wells, r_n = 42), smoothing window 5, scatter lattice 11.  Both scatter_flag = 0 (observed
data + RTM image) and scatter_flag = 1 (PSF data + PSF image) are run.
"""
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REFBIN = ROOT / "oracle" / "_ref"

CASE = dict(nx=100, nz=60, pml=10, Lc=4, dx=5.0, dz=5.0, itmax=400, dt=5.0e-4, f0=25.0, ns=1, sx0=100.0,
            shotdx=0.0, shotdep=0.0, recdix=0.0, offsetz=100.0, swin=11, window=5)


def model(nx=100, nz=60, seed=4242):
    rng = np.random.default_rng(seed)
    v = np.full((nx, nz), 1800.0, np.float32)
    v[:, 25:] = 2300.0
    v[:, 45:] = 2800.0
    v += rng.uniform(-40.0, 40.0, v.shape).astype(np.float32)
    return v


def write_params(path, c, scatter_flag):
    """parameter.txt layout read by input_parameters (acoustic_HLVSPRTMC.cpp:1931-2035)."""
    rows = [("--x grid number: nx", c["nx"]), ("--z grid number: nz", c["nz"]), ("--PML numbers: pml", c["pml"]),
            ("--FD order: Lc", c["Lc"]), ("--x grid interval (m): dx", c["dx"]), ("--z grid interval (m): dz", c["dz"]),
            ("--recording time: rectime-float//itmax-int//", c["itmax"]), ("--time sample (s): dt", c["dt"]),
            ("--Riker wavelet dominant frequency (Hz): f0", c["f0"]), ("--shot numbers: ns", c["ns"]),
            ("--the distance of the first shot at the left boundary (m): sx0", c["sx0"]),
            ("--shot interval X (m): shotdx", c["shotdx"]), ("--the depth of shots (m): shotdep", c["shotdep"]),
            ("--the distance of receivers (m): recdix=nx/2", c["recdix"]), ("--maximum offset", c["offsetz"]),
            ("--scatter_flag", scatter_flag), ("--scatter window  - 31", c["swin"]),
            ("--velocity smooth window", c["window"])]
    with open(path, "w") as f:
        for lab, v in rows:
            f.write(f"{lab}\n  {v}\n")


def run_case(work, scatter_flag, env):
    write_params(work / "parameter.txt", CASE, scatter_flag)
    subprocess.run([str(REFBIN / "AFor")], cwd=work / "forward", check=True, env=env, stdout=subprocess.DEVNULL)
    subprocess.run([str(REFBIN / "AVSPRTM")], cwd=work, check=True, env=env, stdout=subprocess.DEVNULL)


def main(out_path):
    c = CASE
    nx, nz, nt = c["nx"], c["nz"], c["itmax"]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
    res = {"acc_vp": model()}
    with tempfile.TemporaryDirectory() as d:
        work = Path(d)
        for sub in ("input", "output", "forward"):
            (work / sub).mkdir()
        res["acc_vp"].tofile(work / "input" / "acc_vp.bin")
        rd = lambda name: np.fromfile(work / "output" / name, np.float32)
        run_case(work, 0, env)
        r_n = rd("1source_seismogram_obs.bin").size // nt
        for k in ("obs", "obsup", "obsdown", "syn"):
            res[k] = rd(f"1source_seismogram_{k}.bin").reshape(r_n, nt)
        res["rick_hilbert"] = rd("rick_hilbert.bin")
        res["image_pp"] = rd("image_pp1.bin").reshape(nx, nz)
        res["image_sources"] = rd("image_sources1.bin").reshape(nx, nz)
        res["fimage_pp"] = rd("fimage_pp1.bin").reshape(nx, nz)
        res["migration_pp"] = rd("migration_pp.bin").reshape(nx, nz)
        res["ini_vp"] = rd("ini_vp.bin").reshape(nx, nz)
        run_case(work, 1, env)
        res["scatterup"] = rd("1source_seismogram_scatterup.bin").reshape(r_n, nt)
        res["scatter"] = rd("1source_seismogram_scatter.bin").reshape(r_n, nt)
        res["rho_scatter"] = rd("rho_scatter.bin").reshape(nx, nz)
        res["image_psf"] = rd("image_psf1.bin").reshape(nx, nz)
        res["fimage_psf"] = rd("fimage_psf1.bin").reshape(nx, nz)
        res["migration_psf"] = rd("migration_psf.bin").reshape(nx, nz)
    res["case"] = np.array([nx, nz, c["pml"], c["Lc"], nt, c["swin"], c["window"]], np.int32)
    np.savez_compressed(out_path, **res)
    print("wrote", out_path, "r_n =", r_n)


if __name__ == "__main__":
    sys.exit(main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).parent / "ref_gpu_small.npz")))
