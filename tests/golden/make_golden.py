"""Generates the CPU-side golden fixtures in tests/golden/ from the reference itself.

  ini_vp_kat.npz   crops of the reference's shipped input/acc_vp.bin and
                   kkdecon_acoustic/input/ini_vp.bin (ini_vp = ini_model_mine(acc_vp, 5),
                   a known-answer test of the smoothing) with enough halo to recompute them
  decon_ref.npz    inputs and outputs of the reference decon2d_mine built from its own
                   source (oracle/Makefile -> oracle/_ref/decon2d_mine) on seeded synthetic
                   images, two window geometries (square and non-square)

Run from the repository root in a container where the reference tree is mounted
(its location in the SWD_REFERENCE environment variable) after `make -C oracle ref`.
"""
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF = Path(os.environ["SWD_REFERENCE"]) if os.environ.get("SWD_REFERENCE") else None
OUT = Path(__file__).resolve().parent


def write_decon_params(path, nx, nz, psf, flt, snap, eps, mig="./input/mig.bin", psfimg="./input/psf.bin"):
    """kkdecon_acoustic/parameter.txt layout: label line, value line (read by
    kk_decon_interp_psf_minewindow.cpp:1527-1629)."""
    rows = [("--x grid number: nx", nx), ("--z grid number: nz", nz), ("--PSF x number: psfwinx", psf[0]),
            ("--PSF z number: psfwinz", psf[1]), ("--Filter x number: filterwinx", flt[0]),
            ("--Filter z number: filterwinz", flt[1]), ("--Snap x number: snapwinx", snap[0]),
            ("--Snap z number: snapwinz", snap[1]), ("--FFT epsilon", eps),
            ("--Accurate p-Velocity File----", "./input/acc_vp.bin"),
            ("--Migration p-Velocity File----", "./input/ini_vp.bin"), ("--Density File----", "./input/ini_rho.bin"),
            ("--Real Migration p-Image File----", mig), ("--pp-PSF Migration File----", psfimg),
            ("--P-Deconvolution Result-----", "./output/dec.bin"), ("--Inv PSF File-----", "./output/inv_psf.bin"),
            ("--Phase Shift FLag", 0), ("--Regularization coefficient: reg_eps L1-1e-1", 2e-2)]
    with open(path, "w") as f:
        for lab, v in rows:
            f.write(f"{lab}\n  {v}\n")


def synthetic_decon_inputs(nx, nz, psf, seed):
    rng = np.random.default_rng(seed)
    mig = rng.standard_normal((nx, nz)).astype(np.float32)
    p = np.zeros((nx, nz), np.float32)
    for ix in range(psf[0] // 2, nx, psf[0]):
        for iz in range(psf[1] // 2, nz, psf[1]):
            x0, x1, z0, z1 = max(ix - 2, 0), min(ix + 3, nx), max(iz - 2, 0), min(iz + 3, nz)
            p[x0:x1, z0:z1] += rng.standard_normal((x1 - x0, z1 - z0)).astype(np.float32)
    vp = rng.uniform(1500, 3000, (nx, nz)).astype(np.float32)
    return mig, p, vp


def run_ref_decon(nx, nz, mig, psfimg, vp, psf, flt, snap, eps):
    exe = ROOT / "oracle" / "_ref" / "decon2d_mine"
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(f"{d}/input")
        os.makedirs(f"{d}/output")
        write_decon_params(f"{d}/parameter.txt", nx, nz, psf, flt, snap, eps)
        vp.tofile(f"{d}/input/acc_vp.bin")
        vp.tofile(f"{d}/input/ini_vp.bin")
        mig.tofile(f"{d}/input/mig.bin")
        psfimg.tofile(f"{d}/input/psf.bin")
        subprocess.run([str(exe)], cwd=d, check=True, capture_output=True)
        dec = np.fromfile(f"{d}/output/dec.bin", np.float32).reshape(nx, nz)
        coef = np.fromfile(f"{d}/output/migration_coef.bin", np.float32).reshape(nx, nz)
    return dec, coef


DECON_CASES = [  # (nx, nz, psfwin, filterwin, snapwin, epsilon, seed)
    (120, 100, (11, 11), (21, 21), (5, 5), 5e-4, 11),
    (130, 97, (11, 9), (25, 21), (5, 4), 1e-3, 12),
]


def main():
    if REF is None:
        raise SystemExit("set SWD_REFERENCE to the reference tree")
    # smoothing known-answer test: crops with a 5-cell halo
    acc = np.fromfile(REF / "input" / "acc_vp.bin", np.float32).reshape(845, 702)
    ini = np.fromfile(REF / "kkdecon_acoustic" / "input" / "ini_vp.bin", np.float32).reshape(845, 702)
    crops = {}
    # interior crop: ini[400:440, 300:340] needs acc[395:445, 295:345]; the crop starts 10 rows
    # higher because ini_model_mine leaves the first 8 rows of whatever grid it smooths unchanged
    crops["acc_int"], crops["ini_int"] = acc[395:445, 290:345].copy(), ini[400:440, 300:340].copy()
    # corner crop touching the top/left edges (edge replication + the unsmoothed top 8 rows)
    crops["acc_corner"], crops["ini_corner"] = acc[0:45, 0:45].copy(), ini[0:40, 0:40].copy()
    np.savez_compressed(OUT / "ini_vp_kat.npz", **crops)
    # reference decon on synthetic inputs
    out = {}
    for k, (nx, nz, psf, flt, snap, eps, seed) in enumerate(DECON_CASES):
        mig, p, vp = synthetic_decon_inputs(nx, nz, psf, seed)
        dec, coef = run_ref_decon(nx, nz, mig, p, vp, psf, flt, snap, eps)
        out[f"mig{k}"], out[f"psf{k}"], out[f"dec{k}"], out[f"coef{k}"] = mig, p, dec, coef
    np.savez_compressed(OUT / "decon_ref.npz", **out)
    print("wrote", OUT / "ini_vp_kat.npz", OUT / "decon_ref.npz")


if __name__ == "__main__":
    sys.exit(main())
