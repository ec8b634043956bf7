"""Which side carries the difference between the reference's AVSPRTM and this engine's at scale.

TEST INFRASTRUCTURE, run on a B200 machine (needs the reference's programs built for sm_100a
by oracle/Makefile into oracle/_ref, and the drop-in programs next to libswd):

    python tests/golden/attribute_avsprtm_gap.py <out.json>

Case: 1612 x 801 at 5 m (ntx = 1680, a multiple of 16, so the reference's kernels stay in
their arrays), pml 30, Lc 4, nt = 6000, dt = 0.4 ms, 30 Hz, one surface shot at x = 4000 m,
two edge wells of 321 receivers (offsetz = 1600 m), smoothing window 10; true model the
c2-type random field at that size.  The reference's own AFor writes the up-going data, then
the reference's AVSPRTM and this engine's drop-in AVSPRTM migrate the same file in the same
tree.  The FP64 CPU oracle (the reference's reconstruction, imaging, normalisation and
Laplacian in double) migrates the same data on the same smoothed model.  The script reports
each program's normalised image, source illumination and filtered image against FP64, and the
two programs against each other.
"""
import importlib.util
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REFBIN = ROOT / "oracle" / "_ref"
PKG = ROOT / "simple-wavenumber-deconvolution_b200"
sys.path.insert(0, str(ROOT / "oracle"))

CASE = dict(nx=1612, nz=801, pml=30, Lc=4, dx=5.0, dz=5.0, itmax=6000, dt=4.0e-4, f0=30.0, ns=1, sx0=4000.0,
            shotdx=0.0, shotdep=0.0, recdix=0.0, offsetz=1600.0, swin=31, window=10)


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod   # dataclasses look their module up while the class is built
    spec.loader.exec_module(mod)
    return mod


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main(out_path):
    import pyoracle as orc
    mk = _load("make_golden_ref_gpu", HERE / "make_golden_ref_gpu.py")
    cfg = _load("swd_configs", PKG / "configs.py")
    c = CASE
    nx, nz, nt, p = c["nx"], c["nz"], c["itmax"], c["pml"] + c["Lc"]
    v = cfg.random_field(nx, nz, np.random.default_rng(cfg.SEED0 + 2))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
    res = {"case": c}
    with tempfile.TemporaryDirectory() as d:
        work = Path(d)
        for sub in ("input", "output", "forward"):
            (work / sub).mkdir()
        v.tofile(work / "input" / "acc_vp.bin")
        mk.write_params(work / "parameter.txt", c, 0)
        rd = lambda name: np.fromfile(work / "output" / name, np.float32)
        t = time.perf_counter()
        subprocess.run([str(REFBIN / "AFor")], cwd=work / "forward", check=True, env=env, stdout=subprocess.DEVNULL)
        subprocess.run([str(REFBIN / "AVSPRTM")], cwd=work, check=True, env=env, stdout=subprocess.DEVNULL)
        res["reference_programs_s"] = time.perf_counter() - t
        ref = {k: rd(f"{k}1.bin").reshape(nx, nz) for k in ("image_pp", "image_sources", "fimage_pp")}
        obsup = rd("1source_seismogram_obsup.bin")
        r_n = obsup.size // nt
        obsup = obsup.reshape(r_n, nt)
        subprocess.run([str(PKG / "AVSPRTM")], cwd=work, check=True, env=env, stdout=subprocess.DEVNULL)
        ours = {k: rd(f"{k}1.bin").reshape(nx, nz) for k in ("image_pp", "image_sources", "fimage_pp")}
    # the FP64 oracle on the same data and the same smoothed model
    t = time.perf_counter()
    vpad = orc.pad_model(v, p)
    vs = orc.smooth(vpad, p, c["window"])
    rho = np.full_like(vs, 1000.0)
    ntx, ntz = vs.shape
    M = orc.Model(vs, rho, orc.cpml(ntx, ntz, p, c["dx"], c["dz"], c["dt"]), orc.cal_xishu(c["Lc"]), p, c["Lc"], nt,
                  c["dx"], c["dz"], c["dt"])
    rix, riz = orc.well_geometry(nx, nz, p, c["dz"], c["shotdep"], c["offsetz"])
    assert len(rix) == r_n, (len(rix), r_n)
    G = orc.Geom(p + int(c["sx0"] / c["dx"]), p + int(c["shotdep"] / c["dz"]), rix, riz)
    sh = orc.rtm_shot(M, G, orc.ricker(nt, c["f0"], c["dt"]), obsup, dtype=np.float64)
    norm, fim = orc.rtm_post(M, sh["img"], sh["illum"], np.float64)
    res["oracle_s"] = time.perf_counter() - t
    fp64 = {"image_pp": norm[p:-p, p:-p], "image_sources": sh["illum"][p:-p, p:-p], "fimage_pp": fim}
    res["r_n"] = int(r_n)
    for k in fp64:
        res[k] = {"reference_vs_fp64": rel(ref[k], fp64[k]), "engine_vs_fp64": rel(ours[k], fp64[k]),
                  "engine_vs_reference": rel(ours[k], ref[k])}
    Path(out_path).write_text(json.dumps(res, indent=1))
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    sys.exit(main(sys.argv[1] if len(sys.argv) > 1 else "attribute_avsprtm_gap.json"))
