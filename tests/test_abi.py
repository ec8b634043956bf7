"""CPU tests of the C ABI boundary: libswd loads, exports every entry point that
include/swd.h declares, and its host preparation equals the oracle's (and therefore the
reference's) bit for bit.  No kernels run here."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT, PKG_DIR


def declared_functions():
    src = (ROOT / "include" / "swd.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(swd_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(swd):
    L = C.CDLL(str(PKG_DIR / "libswd.so"))
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_error_paths(swd):
    L = swd.lib()
    assert L.swd_version() >= 10000
    # argument validation happens before any device work
    h = C.c_void_p()
    assert L.swd_create(C.byref(h), None) == swd.SWD_ERR_ARG
    bad = swd.Grid(0, 10, 5, 4, 5.0, 5.0, 1e-3, 100, 0)
    assert L.swd_create(C.byref(h), C.byref(bad)) == swd.SWD_ERR_ARG
    assert L.swd_destroy(None) == swd.SWD_OK
    assert L.swd_last_error(None) == b"null context"


def test_python_constants_match_the_header(swd):
    """Every SWD_* integer constant of include/swd.h that the Python mirror names carries the
    header's value (options, strip precisions, RTM flags, kernel paths, status codes)."""
    src = (ROOT / "include" / "swd.h").read_text()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define SWD_([A-Z0-9_]+)\s+(-?\d+)\b", src)}
    checked = 0
    for name, value in defs.items():
        for py in (name, name.replace("ERR_", "SWD_ERR_") if name.startswith("ERR_") else None,
                   "SWD_" + name):
            if py and hasattr(swd, py):
                assert getattr(swd, py) == value, (name, getattr(swd, py), value)
                checked += 1
                break
    opts = [n for n in defs if n.startswith("OPT_")]
    assert len(opts) >= 12 and all(hasattr(swd, n) for n in opts), [n for n in opts if not hasattr(swd, n)]
    assert checked >= 20


def declared_arity():
    """{function: number of parameters} of every prototype in include/swd.h."""
    src = (ROOT / "include" / "swd.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|long long|const char|unsigned|size_t|void)\s*\**\s*(swd_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_python_signatures_match_the_header(swd):
    """Every ctypes signature the Python view declares has the header's parameter count."""
    arity = declared_arity()
    assert sorted(arity) == declared_functions()
    L = swd.lib()
    checked = 0
    for name, n in arity.items():
        f = getattr(L, name)
        if f.argtypes is not None:
            assert len(f.argtypes) == n, (name, len(f.argtypes), n)
            checked += 1
    assert checked >= 30


def test_python_structures_have_the_c_layout(swd, tmp_path):
    """The ctypes structures of the Python view (Grid, Shot, DeconParams) have the size and
    field offsets that a C compiler gives swd_grid, swd_shot and swd_decon_params."""
    import subprocess
    structs = {"swd_grid": swd.Grid, "swd_shot": swd.Shot, "swd_decon_params": swd.DeconParams}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "swd.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, field, value = line.split()
        got[(cname, field)] = int(value)
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_python_constants_equal_the_header(swd):
    """The Python view's status codes, strip precisions, RTM flags, kernel paths and option ids
    are the values include/swd.h defines."""
    defs = {m.group(1): int(m.group(2)) for m in
            re.finditer(r"^#define (SWD_\w+) (\d+)u?\b", (ROOT / "include" / "swd.h").read_text(), re.M)}
    pairs = {k: getattr(swd, k) for k in dir(swd) if k.startswith("SWD_")}
    pairs.update({"SWD_" + k: getattr(swd, k) for k in dir(swd)
                  if k.split("_")[0] in ("STRIP", "RTM", "PATH", "OPT") and isinstance(getattr(swd, k), int)})
    assert len(pairs) >= 24
    for name, value in pairs.items():
        assert name in defs, name
        assert defs[name] == value, (name, defs[name], value)
    assert len(swd.Engine.PROFILE_NAMES) == defs["SWD_NKERNELS"]


def test_decon_geometry(swd, orc):
    for args in [((845, 702), (31, 31), (71, 71), (11, 11)), ((120, 100), (11, 11), (21, 21), (5, 5)),
                 ((130, 97), (11, 9), (25, 21), (5, 4))]:
        (nx, nz), psf, flt, snap = args
        w, fx, fz = swd.decon_geometry(nx, nz, psf, flt, snap)
        g = orc.decon_geometry(nx, nz, psf, flt, snap)
        assert (w, fx, fz) == (g["totalnum"], g["FX"], g["FZ"])
    w, fx, fz = swd.decon_geometry(845, 702, (31, 31), (71, 71), (11, 11))
    assert (w, fx, fz) == (2484, 101, 101)     # the shipped parameters: 54 x 46 windows of 101^2
    with pytest.raises(swd.SwdError):
        swd.decon_geometry(100, 100, (10, 11), (21, 21), (5, 5))   # even PSF window


def test_decon_layout_of_the_bench_cases(swd, orc):
    """The benchmark's window lattice (configs.decon_layout, from which its byte and FLOP counts
    come) equals the oracle's and the engine's for the three decon workloads."""
    from swd_b200 import configs
    expect = {"shipped": 2484, "c2": 1222, "c5": 1593}
    for name, windows in expect.items():
        case = configs.decon_case(name)
        lay = configs.decon_layout(case)
        g = orc.decon_geometry(case.nx, case.nz, case.psfwin, case.filterwin, case.snapwin)
        assert lay["windows"] == g["totalnum"] == windows
        assert (lay["fullx"], lay["fullz"]) == (g["fullwx"], g["fullwz"])
        assert (lay["outwinx"], lay["outwinz"]) == (g["outwinx"], g["outwinz"])
        assert (lay["nxp"], lay["nzp"]) == (g["nxp"], g["nzp"])
        assert swd.decon_geometry(case.nx, case.nz, case.psfwin, case.filterwin, case.snapwin)[0] == windows


def test_decon_geometry_random_cases(swd, orc):
    """Window lattices of random images and window sizes: wherever the engine accepts the
    geometry, the oracle accepts it too and gives the same window count and transform size
    (integer work: exact)."""
    from hypothesis import given, settings, strategies as st

    odd = lambda lo, hi: st.integers(lo // 2, hi // 2).map(lambda k: 2 * k + 1)
    accepted = []

    @settings(max_examples=300, derandomize=True, deadline=None)
    @given(nx=st.integers(40, 1400), nz=st.integers(40, 1400), px=odd(5, 41), pz=odd(5, 41),
           fx_extra=st.integers(0, 30), fz_extra=st.integers(0, 30), sx=st.integers(2, 15), sz=st.integers(2, 15))
    def check(nx, nz, px, pz, fx_extra, fz_extra, sx, sz):
        psf, flt, snap = (px, pz), (px + 2 * fx_extra, pz + 2 * fz_extra), (sx, sz)
        try:
            w, fx, fz = swd.decon_geometry(nx, nz, psf, flt, snap)
        except swd.SwdError:
            return                      # outside the engine's limits (e.g. transform > 512)
        g = orc.decon_geometry(nx, nz, psf, flt, snap)
        assert (w, fx, fz) == (g["totalnum"], g["FX"], g["FZ"])
        accepted.append(w)

    check()
    assert len(accepted) > 100          # most draws are valid geometries


def test_host_prep_equals_oracle(swd, orc):
    for Lc in range(1, 9):
        assert np.array_equal(swd.cal_xishu(Lc).view(np.uint32), orc.cal_xishu(Lc).view(np.uint32))
    for args in [(469, 269, 34, 5.0, 5.0, 5e-4), (917, 766, 21, 10.0, 10.0, 1e-3), (4069, 1669, 34, 4.0, 4.0, 3.5e-4)]:
        a, b = swd.get_absorbing_parameters(*args), orc.cpml(*args)
        for k in a:
            assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k
    for nt, f0, dt in [(2000, 25.0, 5e-4), (6000, 30.0, 4e-4), (7000, 20.0, 1e-3)]:
        assert np.array_equal(swd.ricker_wave(nt, f0, dt).view(np.uint32), orc.ricker(nt, f0, dt).view(np.uint32))
    v = np.random.default_rng(1).uniform(1000, 5000, (37, 29)).astype(np.float32)
    assert np.array_equal(swd.pad_model(v, 9), orc.pad_model(v, 9))
    for n in [88, 128, 269, 469, 669, 869, 1669, 2000, 2048, 4096, 6000, 8000]:
        assert swd.pow2(n) == orc.pow2_len(n)
    for nf, dz in [(128, 5.0), (512, 5.0), (1024, 5.0), (2048, 4.0), (1024, 10.0)]:
        a, la = swd.kz_taper(nf, dz)
        b, lb = orc.kz_taper(nf, dz)
        assert la == lb
        if la >= 0:
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    for args in [(845, 702, 21, 10.0, 0.0, 5000.0), (100, 60, 14, 5.0, 0.0, 100.0), (401, 201, 34, 5.0, 50.0, 300.0)]:
        ra, za = swd.well_geometry(*args)
        rb, zb = orc.well_geometry(*args)
        assert np.array_equal(ra, rb) and np.array_equal(za, zb)


def test_host_prep_random_cases_equal_oracle(swd, orc):
    """The host preparation on random grids, spacings, time steps and acquisitions: CPML
    profiles, Ricker wavelets, kz tapers and well geometries equal the oracle's bit for bit."""
    from hypothesis import given, settings, strategies as st

    bits = lambda a: np.asarray(a, np.float32).view(np.uint32)

    @settings(max_examples=120, derandomize=True, deadline=None)
    @given(nx=st.integers(20, 900), nz=st.integers(20, 900), pml=st.integers(5, 40), Lc=st.integers(1, 8),
           dx=st.sampled_from([2.0, 2.5, 4.0, 5.0, 10.0, 12.5]), dt=st.floats(2.0 ** -13, 2.0 ** -10, width=32),
           nt=st.integers(16, 9000), f0=st.floats(5.0, 60.0, width=32),
           shotdep=st.floats(0.0, 200.0, width=32), offsetz=st.floats(1.0, 6000.0, width=32))
    def check(nx, nz, pml, Lc, dx, dt, nt, f0, shotdep, offsetz):
        pmlc = pml + Lc
        ntx, ntz = nx + 2 * pmlc, nz + 2 * pmlc
        a, b = swd.get_absorbing_parameters(ntx, ntz, pmlc, dx, dx, dt), orc.cpml(ntx, ntz, pmlc, dx, dx, dt)
        for k in a:
            assert np.array_equal(bits(a[k]), bits(b[k])), k
        assert np.array_equal(bits(swd.ricker_wave(nt, f0, dt)), bits(orc.ricker(nt, f0, dt)))
        nf = swd.pow2(ntz)
        assert nf == orc.pow2_len(ntz)
        ta, la = swd.kz_taper(nf, dx)
        tb, lb = orc.kz_taper(nf, dx)
        assert la == lb
        if la >= 0:
            assert np.array_equal(bits(ta), bits(tb))
        ra, za = swd.well_geometry(nx, nz, pmlc, dx, shotdep, offsetz)
        rb, zb = orc.well_geometry(nx, nz, pmlc, dx, shotdep, offsetz)
        assert np.array_equal(ra, rb) and np.array_equal(za, zb)

    check()


def test_synthetic_configs_are_seeded(swd):
    from swd_b200 import configs
    a, b = configs.c1(), configs.c1()
    assert np.array_equal(a.vp, b.vp)
    assert a.vp.shape == (401, 201) and a.ntx == 469 and a.ntz == 269
    assert np.all(np.diff(a.vp[200, :]) >= 0)           # layers increase with depth
    assert len(a.rec_z) == 181 and a.rec_z[0] == 10 and a.rec_z[-1] == 190
