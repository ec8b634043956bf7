"""The drop-in programs AFor, AVSPRTM and decon2d_mine run in a project tree laid out like the
reference's (parameter.txt, input/, output/, forward/, kkdecon_acoustic/) and must write the
reference's files with the reference's results.  GPU tests compare against the outputs of
the reference's own programs (tests/golden/*.npz); CPU tests cover the error paths, which
return before any device work."""
import importlib.util
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, PKG_DIR, ROOT, rel_l2

TOL = 1e-4


def _mkg(name):
    spec = importlib.util.spec_from_file_location(name, GOLDEN / f"{name}.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _tree(d):
    for sub in ("input", "output", "forward"):
        (d / sub).mkdir(exist_ok=True)
    return d


def test_missing_parameter_file_is_an_error():
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        r = subprocess.run([str(PKG_DIR / "AVSPRTM")], cwd=d, capture_output=True, text=True)
        assert r.returncode != 0 and "Cannot open the parameters" in r.stdout
        r = subprocess.run([str(PKG_DIR / "AFor")], cwd=d / "forward", capture_output=True, text=True)
        assert r.returncode != 0


def test_truncated_parameter_file_is_an_error():
    mk = _mkg("make_golden_ref_gpu")
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        mk.write_params(d / "parameter.txt", mk.CASE, 0)
        lines = (d / "parameter.txt").read_text().splitlines()[:20]
        (d / "parameter.txt").write_text("\n".join(lines) + "\n")
        r = subprocess.run([str(PKG_DIR / "AVSPRTM")], cwd=d, capture_output=True, text=True)
        assert r.returncode != 0


@pytest.mark.parametrize("prog,line,msg", [
    ("AVSPRTM", "swd.data = sideways", "swd.data = sideways: expected up|full|down"),
    ("AVSPRTM", "swd.strip_precision = fp16", "swd.strip_precision = fp16: expected f32|f16|bf16|i16"),
    ("AFor", "swd.perturb = pressure", "swd.perturb = pressure: expected density|velocity"),
    ("AFor", "swd.scatter_field = born", "swd.scatter_field = born: expected difference|exact"),
])
def test_unknown_extension_value_is_an_error(prog, line, msg):
    """An extension value the program does not know stops it before any device work, instead
    of running with the default."""
    mk = _mkg("make_golden_ref_gpu")
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        mk.write_params(d / "parameter.txt", mk.CASE, 0)
        with open(d / "parameter.txt", "a") as f:
            f.write(line + "\n")
        cwd = d / "forward" if prog == "AFor" else d
        r = subprocess.run([str(PKG_DIR / prog)], cwd=cwd, capture_output=True, text=True)
        assert r.returncode != 0
        assert msg in r.stdout


def test_record_of_another_size_is_an_error():
    """A record whose size is not r_n x itmax of its shot stops AVSPRTM before any device work,
    with both shapes in the message (the reference would fread it without looking)."""
    mk = _mkg("make_golden_ref_gpu")
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        mk.write_params(d / "parameter.txt", mk.CASE, 0)
        mk.model().tofile(d / "input" / "acc_vp.bin")
        np.zeros((41, mk.CASE["itmax"]), np.float32).tofile(d / "output" / "1source_seismogram_obsup.bin")
        r = subprocess.run([str(PKG_DIR / "AVSPRTM")], cwd=d, capture_output=True, text=True)
        assert r.returncode != 0
        assert "holds 16400 floats; r_n x itmax = 42 x 400 = 16800 expected" in r.stdout
        (d / "output" / "1source_seismogram_obsup.bin").unlink()
        r = subprocess.run([str(PKG_DIR / "AVSPRTM")], cwd=d, capture_output=True, text=True)
        assert r.returncode != 0 and "Cannot Open the File: ./output/1source_seismogram_obsup.bin" in r.stdout


@pytest.mark.parametrize("prog", ["AFor", "AVSPRTM"])
@pytest.mark.parametrize("text,msg", [
    ("3\n10 5\n10 6\n", "3 receivers announced, 2 read"),
    ("2\n10 5\n100 6\n", "receiver 1 at (100, 6) lies outside the 100 x 60 model"),
    ("none\n", "no receiver count"),
])
def test_malformed_receivers_file_is_an_error(prog, text, msg):
    """A shot's own receiver list (input/<shot>source_receivers.txt) that is short, outside the
    model or without a count stops either program before any device work."""
    mk = _mkg("make_golden_ref_gpu")
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        mk.write_params(d / "parameter.txt", mk.CASE, 0)
        mk.model().tofile(d / "input" / "acc_vp.bin")
        (d / "input" / "1source_receivers.txt").write_text(text)
        cwd = d / "forward" if prog == "AFor" else d
        r = subprocess.run([str(PKG_DIR / prog)], cwd=cwd, capture_output=True, text=True)
        assert r.returncode != 0
        assert msg in r.stdout


@pytest.mark.gpu
def test_per_shot_receivers_and_record_selection(swd):
    """Two shots, the second with its own receiver list (30 receivers on one line, not the two
    edge wells): AFor writes each shot's records with its own trace count, and AVSPRTM migrates
    the full, down-going or up-going record (swd.data) of each shot with that shot's receivers,
    giving the images of swd_rtm_shot on the same arrays."""
    mk = _mkg("make_golden_ref_gpu")
    c = dict(mk.CASE, ns=2, shotdx=150.0)
    nx, nz, nt, pml, Lc = c["nx"], c["nz"], c["itmax"], c["pml"], c["Lc"]
    p = pml + Lc
    rx2, rz2 = np.full(30, 60), np.arange(5, 35)
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        v = mk.model()
        v.tofile(d / "input" / "acc_vp.bin")
        (d / "input" / "2source_receivers.txt").write_text("30\n" + "".join(f"{a} {b}\n" for a, b in zip(rx2, rz2)))
        mk.write_params(d / "parameter.txt", c, 0)
        subprocess.run([str(PKG_DIR / "AFor")], cwd=d / "forward", check=True, capture_output=True)
        rd = lambda name: np.fromfile(d / "output" / name, np.float32)
        r_n1 = rd("1source_seismogram_obs.bin").size // nt
        assert r_n1 == 42 and rd("2source_seismogram_obs.bin").size == 30 * nt
        E = swd.Engine(nx, nz, pml, Lc, c["dx"], c["dz"], c["dt"], nt)
        vp = swd.pad_model(v, p)
        rho = np.full_like(vp, 1000.0)
        E.setup_default(vp, rho)
        E.set_model(E.smooth(vp, p, c["window"]), rho)
        rick = swd.ricker_wave(nt, c["f0"], c["dt"])
        shot2 = swd.ShotSpec(p + int(c["sx0"] / c["dx"]) + int(c["shotdx"] / c["dx"]), p, rx2 + p, rz2 + p, nt)
        for which, suffix in (("full", ""), ("down", "down"), ("up", "up")):
            mk.write_params(d / "parameter.txt", c, 0)
            with open(d / "parameter.txt", "a") as f:
                f.write(f"swd.data = {which}\n")
            subprocess.run([str(PKG_DIR / "AVSPRTM")], cwd=d, check=True, capture_output=True)
            data2 = rd(f"2source_seismogram_obs{suffix}.bin").reshape(30, nt)
            assert np.abs(data2).max() > 0
            out = E.rtm_shot(shot2, rick, data2, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK,
                             want=("image_pp", "fimage"))
            assert rel_l2(rd("image_pp2.bin").reshape(nx, nz), out["image_pp"]) < 1e-6, which
            assert rel_l2(rd("fimage_pp2.bin").reshape(nx, nz), out["fimage"]) < 1e-6, which
        E.close()


@pytest.mark.gpu
def test_afor_exact_scatter_field_option(swd):
    """`swd.scatter_field = exact` writes the scatter records of swd_forward_scatter; they agree
    with the default difference of records to that difference's FP32 cancellation error."""
    g = np.load(GOLDEN / "ref_gpu_small.npz")
    mk = _mkg("make_golden_ref_gpu")
    nt = int(g["case"][4])
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        g["acc_vp"].tofile(d / "input" / "acc_vp.bin")
        rd = lambda name: np.fromfile(d / "output" / name, np.float32).reshape(-1, nt)
        mk.write_params(d / "parameter.txt", mk.CASE, 1)
        subprocess.run([str(PKG_DIR / "AFor")], cwd=d / "forward", check=True, capture_output=True)
        diff = {k: rd(f"1source_seismogram_{k}.bin") for k in ("scatter", "scatterup", "scatterdown")}
        with open(d / "parameter.txt", "a") as f:
            f.write("swd.scatter_field = exact\n")
        subprocess.run([str(PKG_DIR / "AFor")], cwd=d / "forward", check=True, capture_output=True)
        for k, a in diff.items():
            b = rd(f"1source_seismogram_{k}.bin")
            assert b.shape == a.shape and np.abs(b).max() > 0
            assert rel_l2(b, a) < 1e-2, k


def test_decon_rejects_even_windows():
    mk = _mkg("make_golden")
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        (d / "output").mkdir()
        mk.write_decon_params(d / "parameter.txt", 100, 90, (10, 11), (21, 21), (5, 5), 1e-3)
        r = subprocess.run([str(PKG_DIR / "decon2d_mine")], cwd=d, capture_output=True, text=True)
        assert "Should Be Odd" in r.stdout


@pytest.mark.gpu
def test_afor_and_avsprtm_reproduce_the_reference_programs():
    g = np.load(GOLDEN / "ref_gpu_small.npz")
    mk = _mkg("make_golden_ref_gpu")
    nx, nz, pml, Lc, nt, swin, window = [int(v) for v in g["case"]]
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        g["acc_vp"].tofile(d / "input" / "acc_vp.bin")
        rd = lambda name, shape: np.fromfile(d / "output" / name, np.float32).reshape(shape)
        for flag in (0, 1):
            mk.write_params(d / "parameter.txt", mk.CASE, flag)
            subprocess.run([str(PKG_DIR / "AFor")], cwd=d / "forward", check=True, capture_output=True)
            subprocess.run([str(PKG_DIR / "AVSPRTM")], cwd=d, check=True, capture_output=True)
        r_n = g["obs"].shape[0]
        assert rel_l2(rd("1source_seismogram_obs.bin", (r_n, nt)), g["obs"]) < TOL
        assert rel_l2(rd("1source_seismogram_obsup.bin", (r_n, nt)), g["obsup"]) < TOL
        assert rel_l2(rd("1source_seismogram_obsdown.bin", (r_n, nt)), g["obsdown"]) < TOL
        assert rel_l2(rd("rick_hilbert.bin", (nt,)), g["rick_hilbert"]) < 1e-5
        assert np.array_equal(rd("ini_vp.bin", (nx, nz)), g["ini_vp"])
        assert np.array_equal(rd("rho_scatter.bin", (nx, nz)), g["rho_scatter"])
        assert rel_l2(rd("image_pp1.bin", (nx, nz)), g["image_pp"]) < TOL
        assert rel_l2(rd("fimage_pp1.bin", (nx, nz)), g["fimage_pp"]) < TOL
        assert rel_l2(rd("migration_pp.bin", (nx, nz)), g["migration_pp"]) < TOL
        # PSF data are differences of two records; compare them on their own scale
        assert rel_l2(rd("1source_seismogram_scatterup.bin", (r_n, nt)), g["scatterup"]) < 1e-2
        assert rel_l2(rd("image_psf1.bin", (nx, nz)), g["image_psf"]) < 1e-2
        assert rel_l2(rd("migration_psf.bin", (nx, nz)), g["migration_psf"]) < 1e-2


@pytest.mark.gpu
def test_decon2d_mine_reproduces_the_reference_program():
    mk = _mkg("make_golden")
    g = np.load(GOLDEN / "decon_ref.npz")
    for k, (nx, nz, psf, flt, snap, eps, seed) in enumerate(mk.DECON_CASES):
        _, _, vp = mk.synthetic_decon_inputs(nx, nz, psf, seed)
        with tempfile.TemporaryDirectory() as d:
            d = Path(d)
            (d / "input").mkdir()
            (d / "output").mkdir()
            mk.write_decon_params(d / "parameter.txt", nx, nz, psf, flt, snap, eps)
            vp.tofile(d / "input" / "acc_vp.bin")
            vp.tofile(d / "input" / "ini_vp.bin")
            g[f"mig{k}"].tofile(d / "input" / "mig.bin")
            g[f"psf{k}"].tofile(d / "input" / "psf.bin")
            subprocess.run([str(PKG_DIR / "decon2d_mine")], cwd=d, check=True, capture_output=True)
            dec = np.fromfile(d / "output" / "dec.bin", np.float32).reshape(nx, nz)
            coef = np.fromfile(d / "output" / "migration_coef.bin", np.float32).reshape(nx, nz)
            assert (d / "output" / "start.flag").exists() and (d / "output" / "end.flag").exists()
            txt = (d / "output" / "migration_coef.txt").read_bytes().split(b"\r\t\n")
            assert len(txt) == nz + 1
        assert np.array_equal(coef, g[f"coef{k}"])
        assert rel_l2(dec, g[f"dec{k}"]) < 1e-3


@pytest.mark.gpu
def test_decon2d_mine_iterative_option(orc):
    """`swd.iterative = 1` runs the regularised deconvolution with the parameter file's own
    reg_eps (L1), L2 coefficient and iteration count, the entries the reference lists after
    reg_eps; checked against the oracle."""
    mk = _mkg("make_golden")
    nx, nz, psf, flt, snap, eps, seed = mk.DECON_CASES[0]
    mig, psfimg, vp = mk.synthetic_decon_inputs(nx, nz, psf, seed)
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        (d / "input").mkdir()
        (d / "output").mkdir()
        mk.write_decon_params(d / "parameter.txt", nx, nz, psf, flt, snap, eps)
        with open(d / "parameter.txt", "a") as f:
            f.write("--Regularization coefficient: reg_eps L2-5e-3\n  6.0e-2\n-- total iteration number: itn\n  30\n"
                    "swd.iterative = 1\n")
        vp.tofile(d / "input" / "acc_vp.bin")
        vp.tofile(d / "input" / "ini_vp.bin")
        mig.tofile(d / "input" / "mig.bin")
        psfimg.tofile(d / "input" / "psf.bin")
        r = subprocess.run([str(PKG_DIR / "decon2d_mine")], cwd=d, check=True, capture_output=True, text=True)
        assert "30 iterations" in r.stdout
        dec = np.fromfile(d / "output" / "dec.bin", np.float32).reshape(nx, nz)
    ref, _ = orc.decon(nx, nz, mig, psfimg, psf, flt, snap, eps, iters=30, reg_l1=2e-2, reg_l2=6e-2)
    assert rel_l2(dec, ref) < 1e-3


REF_ON_SWD = ROOT / "oracle" / "_ref"


@pytest.mark.parametrize("which,nrows", [("rtm", 33), ("fwd", 46)])
def test_compat_layouts_match_the_reference_structs(which, nrows):
    """The compat libraries read the reference's struct Source and struct MultiGPU through
    their own restatement of the layouts; every named member sits at the reference's offset
    and both structs have the reference's size (checker compiled from the reference's own
    headers by oracle/Makefile)."""
    exe = REF_ON_SWD / f"layout_{which}"
    if not exe.exists():
        pytest.skip("layout checker not built (reference sources absent)")
    rows = [line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                    check=True).stdout.splitlines()]
    assert len(rows) == nrows
    bad = [r for r in rows if r[2] != r[3]]
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.skipif(not (REF_ON_SWD / "AVSPRTM_on_swd").exists(), reason="reference hosts on libswd not built")
def test_reference_host_programs_on_libswd():
    """The reference's own, unmodified host programs (AFor, AVSPRTM) linked against the compat
    libraries (libswd_reffwd.so / libswd_refrtm.so) in place of their CUDA files reproduce the
    files of the reference's complete CUDA programs."""
    g = np.load(GOLDEN / "ref_gpu_small.npz")
    mk = _mkg("make_golden_ref_gpu")
    nx, nz, pml, Lc, nt, swin, window = [int(v) for v in g["case"]]
    with tempfile.TemporaryDirectory() as d:
        d = _tree(Path(d))
        g["acc_vp"].tofile(d / "input" / "acc_vp.bin")
        rd = lambda name, shape: np.fromfile(d / "output" / name, np.float32).reshape(shape)
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
        for flag in (0, 1):
            mk.write_params(d / "parameter.txt", mk.CASE, flag)
            subprocess.run([str(REF_ON_SWD / "AFor_on_swd")], cwd=d / "forward", check=True, capture_output=True, env=env)
            subprocess.run([str(REF_ON_SWD / "AVSPRTM_on_swd")], cwd=d, check=True, capture_output=True, env=env)
        r_n = g["obs"].shape[0]
        assert rel_l2(rd("1source_seismogram_obs.bin", (r_n, nt)), g["obs"]) < TOL
        assert rel_l2(rd("1source_seismogram_obsup.bin", (r_n, nt)), g["obsup"]) < TOL
        assert rel_l2(rd("1source_seismogram_obsdown.bin", (r_n, nt)), g["obsdown"]) < TOL
        assert rel_l2(rd("image_pp1.bin", (nx, nz)), g["image_pp"]) < TOL
        assert rel_l2(rd("fimage_pp1.bin", (nx, nz)), g["fimage_pp"]) < TOL
        assert rel_l2(rd("migration_pp.bin", (nx, nz)), g["migration_pp"]) < TOL
        assert rel_l2(rd("1source_seismogram_scatterup.bin", (r_n, nt)), g["scatterup"]) < 1e-2
        assert rel_l2(rd("migration_psf.bin", (nx, nz)), g["migration_psf"]) < 1e-2
