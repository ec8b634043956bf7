"""The byte accounting behind bench.py's roofline lines, on the CPU: the per-launch algorithmic
bytes of the two backward pairings, the forward split against the one-launch step, the twin
kernels against two single wavefields, and the lookup of the ncu-measured traffic."""
import json

import numpy as np
import pytest


@pytest.fixture(scope="module")
def acct(swd):
    import bench
    from swd_b200 import configs
    w = configs.c2()
    cp = swd.get_absorbing_parameters(w.ntx, w.ntz, w.pmlc, w.dx, w.dz, w.dt)
    return bench, w, cp


def test_backward_pairings_differ_by_the_dpdt_round_trip(acct):
    # the by-kind pairing keeps dp/dt in registers: 20 bytes less per interior cell and step
    bench, w, cp = acct
    S, r_n = 19152, 641
    ab = lambda k: bench.algorithmic_bytes(k, w, cp, S, r_n)
    ref = ab("bwd_1") + ab("bwd_2")
    by_kind = ab("bwd_v") + ab("bwd_p")
    assert ref - by_kind == 20 * w.nx * w.nz


def test_forward_split_against_the_one_launch_step(acct):
    # two launches re-read p (velocity launch) and vx, vz (pressure launch) once more than one
    # fused launch, and each counts its own material: 16 bytes per cell between them
    bench, w, cp = acct
    S, r_n = 19152, 641
    ab = lambda k: bench.algorithmic_bytes(k, w, cp, S, r_n)
    assert ab("fwd_v") + ab("fwd_p") - ab("fwd_step") == 16 * w.ntx * w.ntz


def test_twin_kernels_share_the_material(acct):
    # the twin launch moves two wavefields but the coefficients once: 8 (v) / 4 (p) bytes per cell
    # fewer than two single-wavefield launches, plus the twin's well-column gather (8 bytes a row)
    bench, w, cp = acct
    w.extra["well_columns"] = 1
    N = w.ntx * w.ntz
    assert 2 * bench.algorithmic_bytes("fwd_v", w, cp, 0, 0) - bench.algorithmic_bytes("fwd_v2", w, cp, 0, 0) == 8 * N
    p2 = bench.algorithmic_bytes("fwd_p2", w, cp, 0, 641)
    assert 2 * bench.algorithmic_bytes("fwd_p", w, cp, 0, 641) - p2 == 4 * N - 8 * w.ntz


def test_cpml_cells_are_only_the_frame(acct):
    # the CPML memory is counted where a != 0 only: a thin frame against the grid
    bench, w, cp = acct
    N = w.ntx * w.ntz
    extra_v = bench.algorithmic_bytes("fwd_v", w, cp, 0, 0) - 28 * N
    assert 0 < extra_v < 8 * N // 4
    with pytest.raises(KeyError):
        bench.algorithmic_bytes("no_such_kernel", w, cp, 0, 0)


def test_measured_traffic_lookup(acct, tmp_path, monkeypatch):
    bench, _, _ = acct
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.measured_traffic("bwd_p", "c2", 100) is None          # no captures at all
    (tmp_path / "profiles").mkdir()
    (tmp_path / "profiles" / "traffic.json").write_text(json.dumps({
        "bwd_p": {"bytes_per_cell": 40.0, "by_config": {"c5": {"bytes_per_cell": 50.0}}},
        "fwd_v": {"source": "no figure"}}))
    assert bench.measured_traffic("bwd_p", "c2", 100) == pytest.approx(4000.0)
    assert bench.measured_traffic("bwd_p", "c5", 100) == pytest.approx(5000.0)   # a capture on that grid
    assert bench.measured_traffic("fwd_v", "c2", 100) is None
    assert bench.measured_traffic("adj_p", "c4", 100) is None


def test_committed_traffic_has_no_rereads(acct):
    # the DRAM bytes per cell of every committed capture on this grid stay at or below the
    # kernel's algorithmic bytes: no re-reads
    bench, w, cp = acct
    t = json.loads((bench.ROOT / "profiles" / "traffic.json").read_text())
    N = w.ntx * w.ntz
    w.extra["well_columns"] = 1
    for k in ("fwd_p", "bwd_v", "bwd_p", "fwd_v2", "fwd_p2"):
        alg = bench.algorithmic_bytes(k, w, cp, 19152, 641) / N
        assert t[k]["bytes_per_cell"] <= alg * 1.02, (k, t[k]["bytes_per_cell"], alg)
    # every figure, on this grid or another (an entry may hold captures of other grids only)
    vals = [v["bytes_per_cell"] for v in t.values() if "bytes_per_cell" in v]
    vals += [c["bytes_per_cell"] for v in t.values() for c in v.get("by_config", {}).values()]
    assert vals and np.isfinite(vals).all()


def test_workload_subrecords_keep_the_measured_figures(acct, monkeypatch):
    # the default line's sub-records keep each workload's own value, e2e, clocks, parity and
    # per-kernel roofline, and a workload that fails leaves its error in place of the figures
    bench, _, _ = acct
    rec = {"metric": "RTM shots/s", "value": 0.62, "unit": "shots/s", "steps": 2, "warmup": 3, "ms_per_step": 1600.0,
           "gpu_launches": 64002, "clocks": {"sm_mhz": 1965.0}, "parity": None, "cpu_baseline": {"value": 1e-3},
           "config": {"workload": "c5 PSF-RTM shot"}, "e2e": {"value": 0.61, "unit": "shots/s"},
           "roofline": {"bound": "hbm", "kernel": "bwd_p", "frac": 0.77, "kernels_frac": {"bwd_p": 0.77},
                        "timing": "events", "algorithmic_bytes_per_launch": 1}}
    c = bench.compact(rec)
    assert c["value"] == 0.62 and c["e2e"] == 0.61 and c["workload"] == "c5 PSF-RTM shot"
    assert c["roofline"] == {"bound": "hbm", "kernel": "bwd_p", "frac": 0.77, "kernels_frac": {"bwd_p": 0.77}}
    assert "cpu_baseline" not in c and c["warmup"] == 3 and c["clocks"] == {"sm_mhz": 1965.0}

    def ok(args, rank, world, dist):
        assert (rank, world, dist) == (0, 1, None) and args.warmup >= 3
        return dict(rec, value=float(args.steps))

    def bad(args, rank, world, dist):
        raise RuntimeError("no device")

    monkeypatch.setattr(bench, "run_ours", ok)
    monkeypatch.setattr(bench, "run_afor", ok)
    monkeypatch.setattr(bench, "run_decon", bad)
    import argparse
    subs = bench.extra_workloads(argparse.Namespace(config="c2", steps=20, warmup=5))
    assert subs["rtm_c5"]["value"] == 2.0 and subs["afor"]["value"] == 5.0
    assert subs["decon_c5"] == {"error": "RuntimeError: no device"}
