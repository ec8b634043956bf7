#!/usr/bin/env python3
"""Benchmark: RTM shots/s (and Gcell-updates/s) of one PSF-RTM shot on the 1601 x 801
configuration (5 m grid, nt = 6000, dt = 0.4 ms, 30 Hz Ricker, 641 well receivers, 30-cell
CPML, 8th-order stencil), with the roofline of the dominant kernel and a CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one RTM shot: forward modelling with boundary-strip saving, -int int preprocessing
of the receiver data, source-wavefield reconstruction + receiver back-propagation + FP64
imaging, illumination normalisation, -vp^2 Laplacian and stacking.
  value  shots/s with the inputs already in HBM (device pointers into the C ABI);
  e2e    the same through the C ABI with pinned host buffers: the H2D copy of the data and
         the D2H copy of the normalised and filtered images are inside the timed region.
L2 is flushed (a 256 MiB write) before every timed step; steps are timed with CUDA events
on the stream the library launches on.  Multi-GPU runs are replicas (one shot per rank per
step, no collective in the data path): value = all ranks' shots / the slowest rank's time.

--impl reference times the CPU implementation of the same shot on the host cores: the
reference has no CPU propagator, so this is the project's OpenMP restatement of the
reference's stencil, imaging and preprocessing loops (oracle/, kind "port"), run for a
bounded number of time steps per sample and extrapolated to the full record.  With
--workload / --config it times that workload's CPU restatement instead, with the same
metric and unit.  The cpu_baseline of our own lines is timed on rank 0 of a one-GPU run.

--profile-kernels [--workload afor|lsrtm|batch] [--config c5] --nt N runs one short shot of
the workload with kernels launched directly (no graphs), for ncu captures.

--workload batch measures batched multi-shot RTM on the 96-shot walkaway survey (1201 x 601,
nt ~ U[3000, 6000], 200-600 receivers, 20-35 Hz): a step is the whole survey migrated and
stacked by swd_rtm_batch (autotuned batch size, CUDA graphs, FP32 strips); the same survey
through the plain engine (one shot per launch sequence, host launches, FP32 strips) is timed
beside it, and the stacks are compared (also for int16 strips, which halve the strip memory).

--workload decon measures the windowed wavenumber PSF deconvolution (swd_decon) of the c2 or
c5 image (--config): a step deconvolves the whole image, every window of the lattice; value
is windows/s with image, PSF image and outputs in HBM, e2e the same call on pinned host
arrays.  The oracle's restatement of the reference's window loop (OpenMP over windows, FP64
FFTs) on the host cores is the CPU baseline, and its output the parity check.

--workload afor measures the PSF-data modelling stage (AFor) on the same 1601 x 801 shot: a step
is one forward modelling shot with the Hilbert twin wavefield and the kz up/down split of the
well column (swd_forward with the Hilbert wavelet and the kz taper), three trace sets out.

--workload lsrtm measures the differentiable LSRTM gradient instead (801 x 401, nt = 4000,
16 shots, reflectivity spikes at 1 % density): a step is one evaluation of
J(r) = 1/2 sum_s ||L_s r - d_s||^2 and its gradient through the torch autograd path (Born
forward with background checkpoints every 50 steps, checkpointed exact adjoint per shot).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "simple-wavenumber-deconvolution_b200"


def load_pkg():
    spec = importlib.util.spec_from_file_location("swd_b200", PKG / "__init__.py", submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["swd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_configs():
    """The seeded workload definitions (configs.py).  Taken from the package when it is loaded;
    otherwise configs.py is loaded on its own (it needs only numpy), so the reference arm runs
    without mapping libswd."""
    if "swd_b200" in sys.modules:
        return sys.modules["swd_b200"].configs
    if "swd_configs" not in sys.modules:
        spec = importlib.util.spec_from_file_location("swd_configs", PKG / "configs.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules["swd_configs"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["swd_configs"]


def load_oracle():
    """The CPU oracle (oracle/pyoracle.py), the checker and the CPU baseline; nothing of the
    product path goes through it."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    return pyoracle


def oracle_model(orc, w, vp_int, nsteps):
    """An oracle model of workload w on the migration or true velocity vp_int (interior), set up
    with the oracle's own restatement of the reference's host preparation (padding, CPML
    profiles, stencil coefficients), so the CPU legs use nothing of libswd."""
    vp = orc.pad_model(vp_int, w.pmlc)
    rho = np.full_like(vp, 1000.0)
    cp = orc.cpml(w.ntx, w.ntz, w.pmlc, w.dx, w.dz, w.dt)
    return orc.Model(vp, rho, cp, orc.cal_xishu(w.Lc), w.pmlc, w.Lc, nsteps, w.dx, w.dz, w.dt), vp


def max_over_ranks(dist, values, device):
    """Element-wise max over ranks of per-rank device timings: the slowest rank sets the job
    time of a replica run.  dist is torch.distributed (or None for one process)."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_throughput(units_per_rank, world, t_ms):
    """Whole-job units per second: every rank processed units_per_rank units in at most t_ms."""
    return units_per_rank * world / (t_ms / 1e3)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------------------------------
# workload
# ------------------------------------------------------------------------------------------
WORKLOADS = {
    "c2": "c2 PSF-RTM shot: 1601x801 @5 m, nt=6000, dt=0.4 ms, 30 Hz, 641 well receivers, pml 30, 8th order",
    "c5": "c5 PSF-RTM shot: 4001x1601 @4 m, nt=8000, dt=0.35 ms, 25 Hz, 1201 well receivers, pml 30, 8th order, "
          "FP16-scaled strips",
}
WORKLOAD = WORKLOADS["c2"]


def algorithmic_bytes(kernel, w, cp, strip_len, r_n, strip_esz=4):
    """Minimum bytes one launch of each kernel must move (each array touched once); strips
    cost strip_esz bytes per value (4 for FP32, 2 for 16-bit)."""
    N = w.ntx * w.ntz
    Ni = w.nx * w.nz
    nzc = lambda a: int(np.count_nonzero(a))
    x_v = nzc(cp["a_x_half"]) * w.ntz + nzc(cp["a_z_half"]) * w.ntx     # CPML cells of the v update
    x_p = nzc(cp["a_x"]) * w.ntz + nzc(cp["a_z"]) * w.ntx               # CPML cells of the p update
    if kernel == "fwd_v":      # p; vx, vz r/w; cbx, cbz; psi r/w in the frame
        return 28 * N + 8 * x_v
    if kernel == "fwd_p":      # vx, vz; p r/w; ck; phi r/w in the frame; strip save; traces
        return 20 * N + 8 * x_p + strip_esz * strip_len + 4 * r_n
    if kernel == "bwd_1":      # receiver p, v r/w, cbx, cbz (all cells) + psi in the frame;
        #                        source v, p r/w, ck, kap, dp/dt (interior); strips
        return 28 * N + 28 * Ni + 8 * x_v + strip_esz * strip_len
    if kernel == "bwd_2":      # receiver v, p r/w, ck (all cells) + phi in the frame; source p, v r/w,
        #                        cbx, cbz (interior); imaging (interior): dp/dt, the FP32 block sums of
        #                        I and S r/w every step, the FP64 I and S r/w on one step in 64; traces
        return 20 * N + 28 * Ni + 20 * Ni + Ni // 2 + 8 * x_p + 4 * r_n
    if kernel == "bwd_v":      # velocities of both wavefields: receiver p, v r/w, cbx, cbz (all cells) + psi
        #                        in the frame; source p, v r/w (interior; the same cbx, cbz)
        return 28 * N + 20 * Ni + 8 * x_v
    if kernel == "bwd_p":      # pressures of both wavefields + imaging: receiver v, p r/w, ck (all cells) +
        #                        phi in the frame; source v, p r/w, kap (interior); strips; FP32 block sums
        #                        of I and S r/w, the FP64 fold on one step in 64; traces
        return 20 * N + 20 * Ni + 16 * Ni + Ni // 2 + 8 * x_p + strip_esz * strip_len + 4 * r_n
    if kernel == "fwd_v2":     # velocities of the wavefield and its Hilbert twin (shared cbx, cbz)
        return 48 * N + 16 * x_v
    if kernel == "fwd_p2":     # pressures of both (shared ck); both fields' traces; the well columns of both
        return 36 * N + 16 * x_p + 8 * r_n + 8 * w.extra.get("well_columns", 1) * w.ntz
    if kernel == "fwd_step":   # one fused launch per forward step: p, vx, vz r/w, vp, rho, CPML, strips
        return 32 * N + 8 * (x_v + x_p) + strip_esz * strip_len + 4 * r_n
    if kernel == "bwd_step":   # one fused launch per backward step: receiver 24N, material 8N, source 24Ni, FP64 image 32Ni
        return 32 * N + 56 * Ni + 8 * (x_v + x_p) + strip_esz * strip_len + 4 * r_n
    raise KeyError(kernel)


def measured_traffic(kernel, config, cells):
    """DRAM bytes (read + written) of one launch of `kernel` on a grid of `cells` cells, from the
    ncu captures summarised in profiles/traffic.json (a capture on this grid when there is one);
    None without a capture."""
    tj = ROOT / "profiles" / "traffic.json"
    if not tj.exists():
        return None
    t = json.loads(tj.read_text()).get(kernel)
    if t:
        t = t.get("by_config", {}).get(config, t)
    return t["bytes_per_cell"] * cells if t and "bytes_per_cell" in t else None


def setup(swd, w, device):
    import torch
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, w.nt, device=device)
    pmlc = w.pmlc
    vp_true = swd.pad_model(w.vp, pmlc)
    vmig = swd.pad_model(w.vp_mig, pmlc)
    rho = np.full_like(vmig, 1000.0)
    E.setup_default(vmig, rho)
    rick = swd.ricker_wave(w.nt, w.f0, w.dt)
    rx, rz = w.receivers_padded()
    sx, sz = w.source_padded()
    shot = swd.ShotSpec(sx, sz, rx, rz, w.nt)
    # PSF data: +1 % velocity scatter points on the migration model, minus the background
    vs = vmig.copy()
    for ix in w.scatter_x:
        for iz in w.scatter_z:
            vs[ix + pmlc, iz + pmlc] *= np.float32(1.01)
    E.set_model(vs, rho)
    d1 = E.forward(shot, rick)
    E.set_model(vmig, rho)
    d0 = E.forward(shot, rick)
    data = (d1 - d0).astype(np.float32)
    return E, shot, rick, data, swd.get_absorbing_parameters(w.ntx, w.ntz, pmlc, w.dx, w.dz, w.dt)


def run_ours(args, rank, world, dist):
    import torch
    swd = load_pkg()
    from swd_b200 import configs
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    w = configs.CONFIGS[args.config]()
    E, shot, rick, data, cp = setup(swd, w, dev)
    if args.tma:
        E.set_option(swd.OPT_TMA, 1)
    if args.pdl:
        E.set_option(swd.OPT_PDL, 1)
    if args.staged:
        E.set_option(swd.OPT_STAGED, 1)
    if args.autotune:
        E.set_option(swd.OPT_AUTOTUNE, 1)
    if args.path is not None:
        E.set_kernel_path(args.path)
    strips = w.extra.get("strips", "f32")
    E.set_strip_precision({"f32": swd.STRIP_F32, "f16": swd.STRIP_F16}[strips])
    # a dedicated stream: the library captures its time loops into CUDA graphs, which the
    # legacy default stream does not allow
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    E.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    r_n, nt = data.shape
    # device-resident inputs / outputs for `value`
    d_data = torch.from_numpy(data).cuda()
    d_rick = torch.from_numpy(rick).cuda()
    d_img = torch.empty((w.nx, w.nz), dtype=torch.float32, device="cuda")
    d_fim = torch.empty((w.nx, w.nz), dtype=torch.float32, device="cuda")
    # pinned host buffers for `e2e`
    h_data = torch.from_numpy(data).pin_memory()
    h_rick = torch.from_numpy(rick).pin_memory()
    h_img = torch.empty((w.nx, w.nz), dtype=torch.float32).pin_memory()
    h_fim = torch.empty((w.nx, w.nz), dtype=torch.float32).pin_memory()

    import ctypes as C
    sh, keep = E._shot(shot)

    def step(dd, rk, img, fim):
        rc = swd.lib().swd_rtm_shot(E._h, C.byref(sh), swd._ptr(rk), swd._ptr(dd), swd.RTM_PREPROCESS, None,
                                    swd._ptr(img), None, swd._ptr(fim))
        E._ck(rc)

    def timed(dd, rk, img, fim, K, W, profile=False):
        for _ in range(W):
            step(dd, rk, img, fim)
        # with the autotuner on, its tries all happen before the timed shots
        for _ in range(8):
            if not args.autotune or min(E.get_option(swd.OPT_TUNED_FWD), E.get_option(swd.OPT_TUNED_BWD)) >= 0:
                break
            step(dd, rk, img, fim)
        if profile:
            E.profile(8)
            E.profile_read()
        n0 = E.launch_count()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(K):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(dd, rk, img, fim)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        launches = E.launch_count() - n0
        prof = E.profile_read() if profile else None
        E.profile(0)
        return total, launches, prof

    with ClockSampler(dev) as clk:
        t_val, launches, _ = timed(d_data, d_rick, d_img, d_fim, args.steps, args.warmup)
        t_e2e, _, _ = timed(h_data, h_rick, h_img, h_fim, args.steps, max(1, args.warmup // 3))
        # the per-kernel split of the roofline from a separate, shorter profiled pass, so that the
        # probe events it records are not inside the timed `value`
        _, _, prof = timed(d_data, d_rick, d_img, d_fim, max(2, args.steps // 5), 1, profile=True)
    stored = None
    if not args.no_stored:
        # the stored-source option: dp/dt kept at 16 bits by the forward pass, receiver-only
        # backward; its speed, and its raw image against the reconstruction away from the
        # Lc band at the interior edge (where the reconstruction reads a frozen frame)
        I0, S0, _ = E.rtm_raw()
        need = 2 * w.nt * w.nx * (w.nz + 8)
        free = torch.cuda.mem_get_info()[0]
        if need < 0.8 * free:
            E.set_source_storage(1, swd.STRIP_I16)
            ks = max(2, args.steps // 2)
            t_st, _, prof_st = timed(d_data, d_rick, d_img, d_fim, ks, 2, profile=True)
            I1, S1, _ = E.rtm_raw()
            E.set_source_storage(0)
            m = w.pmlc + w.Lc
            sl = (slice(m, -m), slice(m, -m))
            rel = lambda a, b: float(np.linalg.norm(a[sl] - b[sl]) / np.linalg.norm(b[sl]))
            t_st, = max_over_ranks(dist, [t_st], "cuda")
            stored = {"value": replica_throughput(ks, world, t_st), "unit": "shots/s", "precision": "i16",
                      "store_bytes_per_shot": int(need), "image_rel_l2_vs_reconstruction": rel(I1, I0),
                      "illumination_rel_l2_vs_reconstruction": rel(S1, S0),
                      "compared_on": "raw I and S, interior without the Lc band at its edge",
                      "step_us": {k: ms / n * 1e3 for k, (ms, n) in prof_st.items() if n and k in
                                  ("fwd_v", "fwd_p", "bwd_1", "bwd_2", "fwd_pass_step", "bwd_pass_step")}}
        else:
            stored = {"skipped": f"store of {need / 1e9:.1f} GB exceeds 80% of free device memory"}
    t_val, t_e2e = max_over_ranks(dist, [t_val, t_e2e], "cuda")
    if rank != 0:
        return None
    value = replica_throughput(args.steps, world, t_val)
    e2e = replica_throughput(args.steps, world, t_e2e)
    N, Ni = w.ntx * w.ntz, w.nx * w.nz
    cells_per_shot = nt * (N + Ni + N)
    slen = 2 * w.Lc * w.nx + 2 * w.Lc * (w.nz - 2 * w.Lc)
    # roofline of the dominant kernel (largest total time per step)
    per_launch = {k: ms / n for k, (ms, n) in prof.items() if n}
    if E.get_option(swd.OPT_BWD_BY_KIND):   # profile slots 2, 3 hold k_bwd_v, k_bwd_p
        per_launch = {{"bwd_1": "bwd_v", "bwd_2": "bwd_p"}.get(k, k): v for k, v in per_launch.items()}
    # Kernel durations: the whole-pass events (around the graph replays, nothing inside the
    # captured steps) give the time of one forward / backward time step; a probe copy of one
    # chunk brackets the kernels of its middle step, which inflates each by the event-node
    # overhead, so it is only used to split a step's time between its two launches.
    pairs = {"fwd_pass_step": ("fwd_v", "fwd_p"), "bwd_pass_step": ("bwd_1", "bwd_2") if "bwd_1" in per_launch
             else ("bwd_v", "bwd_p")}
    live = {}
    for ps, (k1, k2) in pairs.items():
        if ps in per_launch and k1 in per_launch and k2 in per_launch:
            t, a1, a2 = per_launch[ps], per_launch[k1], per_launch[k2]
            live[k1], live[k2] = t * a1 / (a1 + a2), t * a2 / (a1 + a2)
    for k in ("fwd_step", "bwd_step"):   # fused path: one launch per step
        ps = k.replace("_step", "_pass_step")
        if ps in per_launch and k in per_launch:
            live[k] = per_launch[ps]
    launches_per_shot = {"fwd_v": nt, "fwd_p": nt, "bwd_1": nt - 1, "bwd_2": nt - 1, "bwd_v": nt - 1, "bwd_p": nt - 1,
                         "fwd_step": nt, "bwd_step": nt - 1}
    dom = max(live, key=lambda k: live[k] * launches_per_shot[k])
    peak, src = peaks()
    ab = algorithmic_bytes(dom, w, cp, slen, r_n, 4 if strips == "f32" else 2)
    achieved = ab / (live[dom] * 1e-3) / 1e9
    traffic = measured_traffic(dom, args.config, N)
    # the CPU sample: --cpu-steps steps on the 1601x801 grid, fewer on larger grids (same work)
    cpu = rank0_single(rank, world, lambda: cpu_baseline(w, samples=1, nsteps=rtm_cpu_steps(args, w)))
    # the batched-survey target on a subset of its survey, after the timed region (one-GPU runs)
    batch = None
    if not args.no_batch and args.config == "c2":
        batch = rank0_single(rank, world, lambda: batch_subrecord(swd, dev))
    # the accuracy condition of the metric, once, after every timed region (one-GPU runs)
    parity = None
    if not args.no_parity:
        pnt = args.parity_nt or None   # the whole record (c5: about 9 minutes of host time)
        parity = rank0_single(rank, world, lambda: fp64_parity(swd, E, w, shot, rick, data, nt=pnt))
    options = {"staged_p": int(E.get_option(swd.OPT_STAGED)), "tma_v": int(E.get_option(swd.OPT_TMA)),
               "autotune": int(E.get_option(swd.OPT_AUTOTUNE)), "tuned_fwd": int(E.get_option(swd.OPT_TUNED_FWD)),
               "tuned_bwd": int(E.get_option(swd.OPT_TUNED_BWD))}
    E.close()
    return {
        "metric": "RTM shots/s", "value": value, "unit": "shots/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_val / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP64 imaging)", "data": "synthetic (seeded random-field model, PSF data)",
        "config": {"workload": WORKLOADS[args.config], "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MiB write) before every timed step", "strips": strips,
                   "options": options},
        "gcell_updates_per_s": value * cells_per_shot / 1e9,
        "e2e": {"value": e2e, "unit": "shots/s", "h2d_bytes_per_step": int(data.nbytes + rick.nbytes),
                "d2h_bytes_per_step": int(2 * w.nx * w.nz * 4)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_source": src,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": ab, "avg_launch_us": live[dom] * 1e3,
                     "kernels_us": {k: v * 1e3 for k, v in live.items()},
                     "kernels_frac": {k: algorithmic_bytes(k, w, cp, slen, r_n, 4 if strips == "f32" else 2) / v / 1e6 / peak
                                      for k, v in live.items()},
                     "step_us": {k: per_launch[k] * 1e3 for k in ("fwd_pass_step", "bwd_pass_step") if k in per_launch},
                     "timing": "CUDA events around each whole forward / backward pass of the shots of a separate "
                               "profiled pass after the timed ones (per step = "
                               "pass / steps), split between a step's two launches by the ratio of events around one "
                               "mid-chunk step of the captured time loop"},
        "gpu_launches": launches,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "stored_source": stored,
        "parity": parity,
        "batch": batch,
    }


PARITY_TOL = 1e-3   # the metric's accuracy condition: image rel-L2 against FP64


def oracle_rtm(w, shot, rick, data, nt):
    """The FP64 oracle's RTM of a shot's first nt steps (the reference's strip reconstruction,
    imaging, normalisation and -vp^2 Laplacian in double): raw image, illumination, filtered
    image and the host seconds it took."""
    orc = load_oracle()
    t = time.perf_counter()
    M, _ = oracle_model(orc, w, w.vp_mig, nt)
    G = orc.Geom(shot.s_ix, shot.s_iz, shot.r_ix, shot.r_iz)
    ref = orc.rtm_shot(M, G, np.ascontiguousarray(rick[:nt]), np.ascontiguousarray(data[:, :nt]), dtype=np.float64)
    _, fim = orc.rtm_post(M, ref["img"], ref["illum"], np.float64)
    return ref["img"], ref["illum"], fim, time.perf_counter() - t


def engine_vs_oracle(swd, E, shot, rick, data, nt, ref):
    """Relative L2 of the engine's raw image, illumination and filtered image of the same shot,
    record and inputs against oracle_rtm's; None where the FP64 image is zero (no signal yet)."""
    sh = swd.ShotSpec(shot.s_ix, shot.s_iz, shot.r_ix, shot.r_iz, nt)
    out = E.rtm_shot(sh, np.ascontiguousarray(rick[:nt]), np.ascontiguousarray(data[:, :nt]),
                     flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK, want=("fimage",))
    I, S, _ = E.rtm_raw()

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / nb) if nb > 0 else None
    res = {"image_rel_l2": rel(I, ref[0]), "illum_rel_l2": rel(S, ref[1]), "fimage_rel_l2": rel(out["fimage"], ref[2]),
           "tolerance": PARITY_TOL}
    errs = [res["image_rel_l2"], res["illum_rel_l2"], res["fimage_rel_l2"]]
    # a record too short for the data to reach the receivers leaves the image zero: no pass or fail
    res["pass"] = None if None in errs else max(errs) <= PARITY_TOL
    return res


def fp64_parity(swd, E, w, shot, rick, data, nt=None):
    """The metric's accuracy condition, checked outside every timed region: one more RTM shot of
    the benchmark (same engine, options and inputs; imaging without stacking) against the FP64
    CPU oracle's restatement of the reference's method (strip reconstruction, imaging,
    illumination normalisation and -vp^2 Laplacian, all in double) on the host cores.  Relative
    L2 errors of the raw image I, the source illumination S and the filtered image.  nt < the
    shot's record runs both on the first nt steps (stated in the result)."""
    nt = shot.nt if nt is None else min(nt, shot.nt)
    ref = oracle_rtm(w, shot, rick, data, nt)
    res = {"reference": "FP64 CPU oracle (oracle/), the reference's reconstruction and imaging in double",
           "nt": nt, "record": "full" if nt == shot.nt else f"first {nt} of {shot.nt} steps",
           "receivers": len(shot.r_ix)}
    res.update(engine_vs_oracle(swd, E, shot, rick, data, nt, ref))
    res["oracle_s"] = round(ref[3], 1)
    res["oracle_threads"] = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return res


def rank0_single(rank, world, sample):
    """The CPU baseline is timed on rank 0 of a one-GPU run only (None otherwise), so that
    ranks of a multi-GPU run do not time the host cores against one another."""
    return sample() if rank == 0 and world == 1 else None


def rtm_cpu_steps(args, w):
    """Time steps of the RTM CPU sample: --cpu-steps on the 1601x801 grid, fewer on larger
    grids (the same host work)."""
    return max(32, int(args.cpu_steps * 1669 * 869 / (w.ntx * w.ntz)))


def cpu_baseline(w, samples=1, nsteps=24):
    """OpenMP FP32 restatement of the reference loops (oracle/) on the host cores, for a
    bounded number of time steps of the same shot, extrapolated to nt."""
    orc = load_oracle()
    M, _ = oracle_model(orc, w, w.vp_mig, nsteps)
    rx, rz = w.receivers_padded()
    sx, sz = w.source_padded()
    G = orc.Geom(sx, sz, rx, rz)
    rick = orc.ricker(nsteps, w.f0, w.dt)
    data = np.random.default_rng(0).standard_normal((len(rx), nsteps)).astype(np.float32)
    best = None
    for _ in range(samples):
        t = time.perf_counter()
        orc.rtm_shot(M, G, rick, data)
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    per_shot = best * w.nt / nsteps
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": 1.0 / per_shot, "unit": "shots/s", "cores": cores, "kind": "port", "sample_s": best,
            "sample": f"{nsteps} of {w.nt} time steps (forward + backward) of the same shot on the full grid, "
                      f"extrapolated linearly; {best:.2f} s measured"}


AFOR_WORKLOAD = ("c2 PSF-data modelling shot (AFor): 1601x801 @5 m, nt=6000, dt=0.4 ms, 30 Hz, 641 well receivers, "
                 "pml 30, 8th order, with the Hilbert twin wavefield and the kz up/down split of the well column")


def afor_cpu_baseline(w, nsteps):
    """The oracle's FP32 OpenMP forward with the Hilbert twin and the well-column record on the
    host cores for nsteps steps of the same shot, extrapolated to nt (the kz split is a per-shot
    post-process, not included)."""
    orc = load_oracle()
    M, _ = oracle_model(orc, w, w.vp, nsteps)
    rx, rz = w.receivers_padded()
    sx, sz = w.source_padded()
    G = orc.Geom(sx, sz, rx, rz)
    rick = orc.ricker(nsteps, w.f0, w.dt)
    t = time.perf_counter()
    orc.forward(M, G, rick, hrick=rick[::-1].copy(), col_ix=sorted(set(int(x) for x in rx)))
    dt = time.perf_counter() - t
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": 1.0 / (dt * w.nt / nsteps), "unit": "shots/s", "cores": cores, "kind": "port", "sample_s": dt,
            "sample": f"{nsteps} of {w.nt} time steps of the twin forward on the full grid, extrapolated linearly; "
                      f"{dt:.2f} s measured"}


def run_afor(args, rank, world, dist):
    import ctypes as C
    import torch
    swd = load_pkg()
    from swd_b200 import configs
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    w = configs.c2()
    w.extra["well_columns"] = len(set(int(x) for x in w.rec_x))
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, w.nt, device=dev)
    vtrue = swd.pad_model(w.vp, w.pmlc)
    E.setup_default(vtrue, np.full_like(vtrue, 1000.0))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    E.set_stream(stream.cuda_stream)
    rick = swd.ricker_wave(w.nt, w.f0, w.dt)
    hrick = E.hilbert(rick)
    coef, _ = swd.kz_taper(swd.pow2(w.ntz), w.dz)
    rx, rz = w.receivers_padded()
    sx, sz = w.source_padded()
    shot = swd.ShotSpec(sx, sz, rx, rz, w.nt)
    sh, keep = E._shot(shot)
    r_n = len(rx)
    dev_in = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() for a in (rick, hrick, coef)]
    host_in = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory() for a in (rick, hrick, coef)]
    dev_out = [torch.empty((r_n, w.nt), dtype=torch.float32, device="cuda") for _ in range(3)]
    host_out = [torch.empty((r_n, w.nt), dtype=torch.float32).pin_memory() for _ in range(3)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step(ins, outs):
        E._ck(swd.lib().swd_forward(E._h, C.byref(sh), *[swd._ptr(t) for t in ins], *[swd._ptr(t) for t in outs]))

    def timed(ins, outs, K, W, profile=False):
        for _ in range(W):
            step(ins, outs)
        if profile:
            E.profile(8)
            E.profile_read()
        n0 = E.launch_count()
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(K):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(ins, outs)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        launches = E.launch_count() - n0
        prof = E.profile_read() if profile else None
        E.profile(0)
        return total, launches, prof

    with ClockSampler(dev) as clk:
        t_val, launches, prof = timed(dev_in, dev_out, args.steps, args.warmup, profile=True)
        t_e2e, _, _ = timed(host_in, host_out, args.steps, 1)
    t_val, t_e2e = max_over_ranks(dist, [t_val, t_e2e], "cuda")
    value = replica_throughput(args.steps, world, t_val)
    e2e = replica_throughput(args.steps, world, t_e2e)
    per_launch = {k: ms / n for k, (ms, n) in prof.items() if n}
    live = {}
    if all(k in per_launch for k in ("fwd_pass_step", "fwd_v", "fwd_p")):
        t, a1, a2 = per_launch["fwd_pass_step"], per_launch["fwd_v"], per_launch["fwd_p"]
        live = {"fwd_v2": t * a1 / (a1 + a2), "fwd_p2": t * a2 / (a1 + a2)}
    dom = max(live, key=live.get)
    peak, src = peaks()
    cp = swd.get_absorbing_parameters(w.ntx, w.ntz, w.pmlc, w.dx, w.dz, w.dt)
    ab = algorithmic_bytes(dom, w, cp, 0, r_n)
    achieved = ab / (live[dom] * 1e-3) / 1e9
    cpu = rank0_single(rank, world, lambda: afor_cpu_baseline(w, max(16, args.cpu_steps // 3)))
    return {
        "metric": "modelling shots/s", "value": value, "unit": "shots/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_val / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random-field model)",
        "config": {"workload": AFOR_WORKLOAD, "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MiB write) before every timed step"},
        "gcell_updates_per_s": value * 2 * w.nt * w.ntx * w.ntz / 1e9,   # the wavefield and its twin
        "e2e": {"value": e2e, "unit": "shots/s", "h2d_bytes_per_step": int(sum(t.numel() * 4 for t in host_in)),
                "d2h_bytes_per_step": int(3 * r_n * w.nt * 4)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_source": src,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": measured_traffic(dom, "c2", w.ntx * w.ntz),
                     "algorithmic_bytes_per_launch": ab,
                     "avg_launch_us": live[dom] * 1e3, "kernels_us": {k: v * 1e3 for k, v in live.items()},
                     "step_us": {"fwd_pass_step": per_launch.get("fwd_pass_step", 0.0) * 1e3}},
        "gpu_launches": launches,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }


LSRTM_WORKLOAD = ("c4 LSRTM gradient: 801x401 @5 m, nt=4000, dt=0.4 ms, 16 shots, 321 well receivers, "
                  "reflectivity spikes N(0,0.05) at 1% density, pml 30, 8th order")


def adjoint_bytes(kernel, w, cp, r_n):
    """Minimum bytes of one launch of each adjoint kernel (each array touched once)."""
    N = w.ntx * w.ntz
    nzc = lambda a: int(np.count_nonzero(a))
    x_v = nzc(cp["a_x_half"]) * w.ntz + nzc(cp["a_z_half"]) * w.ntx
    x_p = nzc(cp["a_x"]) * w.ntz + nzc(cp["a_z"]) * w.ntx
    if kernel == "adj_v":   # Qx, Qz in; v^x, v^z r/w; rho; Rx, Rz out; psi^ r/w in the frame
        return 36 * N + 8 * x_v
    if kernel == "adj_p":   # Rx, Rz in; p^ r/w; S0; FP64 grad r/w; ck; Qx, Qz out; phi^ in the frame; traces
        return 48 * N + 8 * x_p + 4 * r_n
    raise KeyError(kernel)


def run_lsrtm(args, rank, world, dist):
    import torch
    swd = load_pkg()
    from swd_b200 import configs, lsrtm
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    w = configs.c4()
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, w.nt, device=dev)
    pmlc = w.pmlc
    vmig = swd.pad_model(w.vp_mig, pmlc)
    rho = np.full_like(vmig, 1000.0)
    E.setup_default(vmig, rho)
    cp = swd.get_absorbing_parameters(w.ntx, w.ntz, pmlc, w.dx, w.dz, w.dt)
    rick = swd.ricker_wave(w.nt, w.f0, w.dt)
    rx, rz = w.receivers_padded()
    ops = [lsrtm.BornOperator(E, swd.ShotSpec(sx + pmlc, pmlc, rx, rz, w.nt), rick, vmig, rho, device=f"cuda:{dev}")
           for sx in w.sx]
    nshots, r_n = len(ops), len(rx)
    prec = {"f32": swd.STRIP_F32, "f16": swd.STRIP_F16, "bf16": swd.STRIP_BF16, "i16": swd.STRIP_I16}[args.ckpt_prec]
    r_true = torch.tensor(w.extra["reflectivity"], device="cuda")
    with torch.no_grad():
        data = [lsrtm.born(r_true, op) for op in ops]       # observed data: Born data of the true reflectivity
    r0 = 0.5 * r_true                                        # current model: residual = data of 0.5 r_true
    h_data = [d.cpu().pin_memory() for d in data]
    h_grad = torch.empty((w.nx, w.nz), dtype=torch.float32).pin_memory()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def gradient(dd, pool=None):
        r = r0.clone().requires_grad_(True)
        lsrtm.lsrtm_objective(r, ops, dd, pool=pool).backward()
        return r.grad

    engines = [E]

    def timed(K, W, e2e=False, profile=False, pool=None):
        for _ in range(W):
            gradient(data, pool)
        if profile:
            E.profile(8)
            E.profile_read()
        n0 = sum(e.launch_count() for e in engines)
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(K):
            flush.zero_()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            if e2e:
                dd = [hd.to("cuda", non_blocking=True) for hd in h_data]
                h_grad.copy_(gradient(dd, pool), non_blocking=True)
            else:
                g = gradient(data, pool)
            b.record()
            b.synchronize()
            total += a.elapsed_time(b)
        launches = sum(e.launch_count() for e in engines) - n0
        prof = E.profile_read() if profile else None
        E.profile(0)
        return total, launches, prof

    # accuracy of the checkpointed gradient against FP32 full storage (outside the timing)
    E.set_checkpointing(0)
    g_full = gradient(data).double()
    t0 = time.perf_counter()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    gradient(data)
    b.record()
    b.synchronize()
    t_full = a.elapsed_time(b)
    E.set_checkpointing(50, prec)
    g_ck = gradient(data).double()
    err = float((g_ck - g_full).norm() / g_full.norm())
    ck_bytes = E.checkpoint_bytes(w.nt)
    full_bytes = w.nt * w.ntx * ((w.ntz + 31) // 32 * 32) * 4
    with ClockSampler(dev) as clk:
        t_seq, launches, prof = timed(args.steps, args.warmup, profile=True)
        t_val, t_e2e = t_seq, None
        pool = None
        if args.streams > 1:
            # engines configured like E; shots spread over them from one host thread each
            for _ in range(args.streams - 1):
                Ek = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, w.nt, device=dev)
                Ek.setup_default(vmig, rho)
                Ek.set_checkpointing(50, prec)
                engines.append(Ek)
            pool = lsrtm.EnginePool(engines)
            t_val, launches, _ = timed(args.steps, args.warmup, pool=pool)
        t_e2e, _, _ = timed(args.steps, 1, e2e=True, pool=pool)
        if pool is not None:
            pool.close()
    t_val, t_e2e, t_seq = max_over_ranks(dist, [t_val, t_e2e, t_seq], "cuda")
    value = replica_throughput(nshots * args.steps, world, t_val)
    e2e = replica_throughput(nshots * args.steps, world, t_e2e)
    per_launch = {k: ms / n for k, (ms, n) in prof.items() if n}
    live = {}
    if all(k in per_launch for k in ("adj_pass_step", "adj_v", "adj_p")):
        t, a1, a2 = per_launch["adj_pass_step"], per_launch["adj_v"], per_launch["adj_p"]
        live = {"adj_v": t * a1 / (a1 + a2), "adj_p": t * a2 / (a1 + a2)}
    dom = max(live, key=live.get)
    peak, src = peaks()
    ab = adjoint_bytes(dom, w, cp, r_n)
    achieved = ab / (live[dom] * 1e-3) / 1e9
    N, Ni = w.ntx * w.ntz, w.nx * w.nz
    cpu = rank0_single(rank, world, lambda: lsrtm_cpu_baseline(w, nsteps=args.cpu_steps // 3))
    return {
        "metric": "LSRTM gradient shots/s", "value": value, "unit": "shots/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_val / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": f"f32 (FP64 gradient accumulation, {args.ckpt_prec} checkpoints)",
        "data": "synthetic (seeded random-field model, Born data of seeded reflectivity spikes)",
        "config": {"workload": LSRTM_WORKLOAD, "parallelism": f"replicas x{world}", "shots_per_step": nshots,
                   "checkpoints": f"every 50 steps, {args.ckpt_prec}", "l2": "flushed (256 MiB write) before every timed step",
                   "engines": args.streams},
        "sequential": {"value": replica_throughput(nshots * args.steps, world, t_seq), "unit": "shots/s",
                       "ms_per_step": t_seq / args.steps,
                       "what": "one engine, shots one after another (the kernel timings below are from this run)"},
        "gcell_updates_per_s": value * w.nt * 2 * N / 1e9,
        "executed_gcell_updates_per_s": value * w.nt * 4 * N / 1e9,
        "e2e": {"value": e2e, "unit": "shots/s", "h2d_bytes_per_step": int(nshots * r_n * w.nt * 4),
                "d2h_bytes_per_step": int(w.nx * w.nz * 4)},
        "gradient_vs_fp32_full_storage": {"rel_l2": err, "full_storage_ms_per_step": t_full,
                                          "checkpoint_bytes_per_shot": ck_bytes, "full_storage_bytes_per_shot": full_bytes},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_source": src, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": measured_traffic(dom, "c4", w.ntx * w.ntz),
                     "algorithmic_bytes_per_launch": ab,
                     "avg_launch_us": live[dom] * 1e3, "kernels_us": {k: v * 1e3 for k, v in live.items()},
                     "step_us": {k: per_launch[k] * 1e3 for k in ("fwd_pass_step", "adj_pass_step") if k in per_launch}},
        "gpu_launches": launches,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "wall_s": time.perf_counter() - t0,
    }


BATCH_WORKLOAD = ("c3 batched RTM: 96 walkaway-VSP shots, 1201x601 @5 m, nt ~ U[3000,6000], dt=0.4 ms, "
                  "200-600 well receivers, 20-35 Hz, pml 30, 8th order")


def batch_subrecord(swd, dev, nshots=24):
    """The batched-survey target beside the headline: the first nshots of the 96-shot walkaway
    survey (1201x601, nt ~ U[3000, 6000], 200-600 receivers) migrated and stacked by the plain engine
    (one shot per launch sequence, host launches, FP32 strips) and by swd_rtm_batch (autotuned batch,
    CUDA graphs, FP32 strips) on one engine, one pass each after a warm-up pass of the batched one,
    with the two stacks compared."""
    import torch
    from swd_b200 import configs
    w = configs.c3()
    cfg = w.extra["shots"][:nshots]
    ntmax = max(s["nt"] for s in cfg)
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, ntmax, device=dev)
    p = w.pmlc
    vtrue, vmig = swd.pad_model(w.vp, p), swd.pad_model(w.vp_mig, p)
    rho = np.full_like(vmig, 1000.0)
    E.setup_default(vtrue, rho)
    stream = torch.cuda.Stream()
    E.set_stream(stream.cuda_stream)
    shots = [swd.ShotSpec(c["sx"] + p, c["sz"] + p, c["rec_x"] + p, c["rec_z"] + p, c["nt"]) for c in cfg]
    ricks = [swd.ricker_wave(c["nt"], c["f0"], w.dt) for c in cfg]
    data = [E.forward(sh, rk) for sh, rk in zip(shots, ricks)]
    E.set_model(vmig, rho)

    def timed(fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    def plain():
        E.stack_reset()
        for sh, rk, d in zip(shots, ricks, data):
            E.rtm_shot(sh, rk, d, want=())

    def batched():
        E.stack_reset()
        E.rtm_batch(shots, ricks, data)

    E.set_option(swd.OPT_GRAPHS, 0)
    t_plain = timed(plain)
    st_plain = E.stack(edge_zero=False).astype(np.float64)
    E.set_option(swd.OPT_GRAPHS, 1)
    E.set_option(swd.OPT_BATCH, 0)
    batched()                                     # warm-up, and the batch-size probes
    t_bat = timed(batched)
    st_bat = E.stack(edge_zero=False).astype(np.float64)
    bsize = E.get_option(swd.OPT_BATCH_TUNED)
    E.close()
    return {"workload": f"the first {nshots} shots of the c3 walkaway survey (1201x601, nt ~ U[3000,6000])",
            "plain_shots_per_s": nshots / (t_plain / 1e3), "batched_shots_per_s": nshots / (t_bat / 1e3),
            "speedup": t_plain / t_bat, "batch_size": bsize,
            "stack_rel_l2_batched_vs_plain": float(np.linalg.norm(st_bat - st_plain) / np.linalg.norm(st_plain)),
            "target": "3x (bounded at about 2x by the survey's algorithmic bytes at the HBM rate)"}


def run_batch(args, rank, world, dist):
    import torch
    swd = load_pkg()
    from swd_b200 import configs
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    w = configs.c3()
    shots_cfg = w.extra["shots"]
    ntmax = max(s["nt"] for s in shots_cfg)
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, ntmax, device=dev)
    pmlc = w.pmlc
    vtrue, vmig = swd.pad_model(w.vp, pmlc), swd.pad_model(w.vp_mig, pmlc)
    rho = np.full_like(vmig, 1000.0)
    E.setup_default(vtrue, rho)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    E.set_stream(stream.cuda_stream)
    shots, ricks, data = [], [], []
    for s in shots_cfg:
        sh = swd.ShotSpec(s["sx"] + pmlc, s["sz"] + pmlc, s["rec_x"] + pmlc, s["rec_z"] + pmlc, s["nt"])
        rk = swd.ricker_wave(s["nt"], s["f0"], w.dt)
        shots.append(sh)
        ricks.append(rk)
        data.append(E.forward(sh, rk))           # observed data in the true model
    E.set_model(vmig, rho)
    cells = sum(s["nt"] * (2 * w.ntx * w.ntz + w.nx * w.nz) for s in shots_cfg)

    engines = [E]

    def timed(fn, K, W):
        for _ in range(W):
            fn()
        torch.cuda.synchronize()
        n0 = sum(e.launch_count() for e in engines)
        total = 0.0
        for _ in range(K):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total, sum(e.launch_count() for e in engines) - n0

    def plain():
        E.stack_reset()
        for sh, rk, d in zip(shots, ricks, data):
            E.rtm_shot(sh, rk, d, want=())

    def batched():
        E.stack_reset()
        E.rtm_batch(shots, ricks, data)

    # plain engine: one shot per launch sequence, host launches, FP32 strips
    E.set_option(swd.OPT_GRAPHS, 0)
    E.set_strip_precision(swd.STRIP_F32)
    t_plain, _ = timed(plain, args.steps, 1)
    st_plain = E.stack(edge_zero=False).astype(np.float64)
    # batched engine: autotuned batch, CUDA graphs, FP32 strips
    E.set_option(swd.OPT_GRAPHS, 1)
    E.set_option(swd.OPT_BATCH, 0)
    with ClockSampler(dev) as clk:
        t_bat, launches_bat = timed(batched, args.steps, args.warmup)
        st_bat = E.stack(edge_zero=False).astype(np.float64)
        # engine pool: the survey's shots spread over args.streams engines (own streams, one
        # host thread each), each migrating its share with swd_rtm_batch
        from swd_b200 import survey
        for _ in range(args.streams - 1):
            Ek = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, ntmax, device=dev)
            Ek.setup_default(vmig, rho)
            engines.append(Ek)
        pool = survey.EnginePool(engines)
        st_pool = []
        t_pool, launches = timed(lambda: st_pool.append(survey.rtm_survey(pool, shots, ricks, data, edge_zero=False)),
                                 args.steps, args.warmup)
        # the same pool in stored-source mode (int16 dp/dt; each engine one shot at a time)
        for Ek in engines:
            Ek.set_source_storage(1, swd.STRIP_I16)
        st_stored = []
        t_stored, _ = timed(lambda: st_stored.append(survey.rtm_survey(pool, shots, ricks, data, batched=False,
                                                                       edge_zero=False)), args.steps, args.warmup)
        for Ek in engines:
            Ek.set_source_storage(0)
        pool.close()
    st_pool = st_pool[-1].astype(np.float64)
    st_stored = st_stored[-1].astype(np.float64)
    # int16 strips: the image error of halving the strip memory
    E.set_strip_precision(swd.STRIP_I16)
    batched()
    st_bat16 = E.stack(edge_zero=False).astype(np.float64)
    E.set_strip_precision(swd.STRIP_F32)
    t_bat, t_plain, t_pool, t_stored = max_over_ranks(dist, [t_bat, t_plain, t_pool, t_stored], "cuda")
    stored_v = replica_throughput(len(shots) * args.steps, world, t_stored)
    band = (slice(w.Lc, -w.Lc), slice(w.Lc, -w.Lc))   # the stored mode differs from the reconstruction there
    value = replica_throughput(len(shots) * args.steps, world, t_bat)
    pool_v = replica_throughput(len(shots) * args.steps, world, t_pool)
    plain_v = replica_throughput(len(shots) * args.steps, world, t_plain)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return {
        "metric": "RTM shots/s", "value": value, "unit": "shots/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_bat / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP64 imaging)", "data": "synthetic (seeded random-field model)",
        "config": {"workload": BATCH_WORKLOAD, "parallelism": f"replicas x{world}", "shots_per_step": len(shots),
                   "batch_size": E.get_option(swd.OPT_BATCH_TUNED),
                   "what": "swd_rtm_batch on one engine (autotuned batch, CUDA graphs, FP32 strips)",
                   "l2": "inputs of one batch exceed L2"},
        "gcell_updates_per_s": cells * args.steps / (t_bat / 1e3) / 1e9,
        "plain_engine": {"value": plain_v, "unit": "shots/s", "ms_per_step": t_plain / args.steps,
                         "what": "swd_rtm_shot per shot, host launches (no graphs), FP32 strips"},
        "engine_pool": {"value": pool_v, "unit": "shots/s", "ms_per_step": t_pool / args.steps, "engines": args.streams,
                        "what": "rtm_survey: the shots over an engine pool, each engine through swd_rtm_batch",
                        "stack_rel_l2_vs_plain": rel(st_pool, st_plain)},
        "engine_pool_stored_source": {
            "value": stored_v, "unit": "shots/s", "ms_per_step": t_stored / args.steps, "engines": args.streams,
            "speedup_vs_plain": stored_v / plain_v,
            "what": "rtm_survey over the engine pool in stored-source mode (int16 dp/dt, receiver-only backward)",
            "stack_rel_l2_vs_plain": rel(st_stored, st_plain),
            "stack_correlation_vs_plain_without_edge_band": float(np.corrcoef(st_stored[band].ravel(),
                                                                              st_plain[band].ravel())[0, 1]),
            "note": "not a drop-in for the reference's stack: each shot's image is divided by its maximum "
                    "illumination, which the reference's reconstruction inflates in the Lc-wide band at the "
                    "interior edge by an amount that depends on the shot; the stored mode keeps the forward dp/dt "
                    "there, so the shots are stacked with other weights, while the raw images agree to 1e-4 away "
                    "from the band"},
        "speedup_vs_plain": value / plain_v,
        "stack_rel_l2_vs_plain": rel(st_bat, st_plain),
        "stack_rel_l2_int16_strips_vs_plain": rel(st_bat16, st_plain),
        "gpu_launches": launches,
        "cpu_baseline": rank0_single(rank, world, lambda: survey_cpu_baseline(w, max(8, args.cpu_steps // 3))),
        "clocks": clk.summary(),
    }


def decon_bytes(case, lay):
    """Algorithmic bytes of one deconvolution: image and PSF reads, the two padded float
    accumulators (mig_dec, mig_coef) written once."""
    return 4 * case.nx * case.nz * 2 + 8 * lay["nxp"] * lay["nzp"]


def decon_table_len(lay):
    """float2 entries of the window kernels' FFT tables (chirp, chirp transform, twiddles) for the
    window geometry's two transform lengths (one table when they are equal)."""
    def one(L):
        if L >= 32 and L & (L - 1) == 0:
            M = L
        else:
            M = 32
            while M < 2 * L - 1:
                M <<= 1
        return L + M + M // 2
    return one(lay["fullz"]) + (one(lay["fullx"]) if lay["fullx"] != lay["fullz"] else 0)


def decon_flops(lay):
    """FFT-equivalent flops of one deconvolution: 3 complex 2D transforms per window."""
    n = lay["fullx"] * lay["fullz"]
    return lay["windows"] * 3 * 5 * n * np.log2(n)


def decon_cpu(case, mig, psf):
    """The oracle's restatement of the reference's window loop on all host cores."""
    orc = load_oracle()
    cores = os.cpu_count() or 1
    t = time.perf_counter()
    dec, coef = orc.decon(case.nx, case.nz, mig, psf, case.psfwin, case.filterwin, case.snapwin, case.epsilon,
                          nthreads=cores)
    return time.perf_counter() - t, cores, dec, coef


def run_decon(args, rank, world, dist):
    import ctypes as C
    import torch
    swd = load_pkg()
    from swd_b200 import configs
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    case = configs.decon_case(args.config)
    lay = configs.decon_layout(case)
    mig, psf = configs.decon_inputs(case)
    E = swd.Engine(case.nx, case.nz, 30, 4, 5.0, 5.0, 4e-4, 2, device=dev)   # owns the stream and decon scratch
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    E.set_stream(stream.cuda_stream)
    L = swd.lib()
    p = swd.DeconParams(case.nx, case.nz, case.psfwin[0], case.psfwin[1], case.filterwin[0], case.filterwin[1],
                        case.snapwin[0], case.snapwin[1], case.epsilon, 0, 0, 0, 0, args.decon_iters, 2e-2, 6e-2)
    d_mig, d_psf = torch.from_numpy(mig).cuda(), torch.from_numpy(psf).cuda()
    d_dec, d_coef = torch.empty_like(d_mig), torch.empty_like(d_mig)
    h_mig, h_psf = torch.from_numpy(mig).pin_memory(), torch.from_numpy(psf).pin_memory()
    h_dec, h_coef = torch.empty(mig.shape).pin_memory(), torch.empty(mig.shape).pin_memory()
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")

    def call(a, b, c, d):
        rc = L.swd_decon(E._h, C.byref(p), a, b, c, d)
        if rc != swd.SWD_OK:
            raise swd.SwdError(rc, L.swd_last_error(E._h).decode())

    dev_args = (d_mig.data_ptr(), d_psf.data_ptr(), d_dec.data_ptr(), d_coef.data_ptr())
    host_args = (h_mig.data_ptr(), h_psf.data_ptr(), h_dec.data_ptr(), h_coef.data_ptr())

    def timed(args_, K, W):
        for _ in range(W):
            call(*args_)
        torch.cuda.synchronize()
        n0 = E.launch_count()
        total = 0.0
        for _ in range(K):
            flush.add_(1.0)                       # 256 MiB write: inputs out of L2
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            call(*args_)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total, E.launch_count() - n0

    with ClockSampler(dev) as clk:
        t_dev, launches = timed(dev_args, args.steps, args.warmup)
    t_e2e, _ = timed(host_args, args.steps, 1)
    t_dev, t_e2e = max_over_ranks(dist, [t_dev, t_e2e], "cuda")
    value = replica_throughput(lay["windows"] * args.steps, world, t_dev)
    e2e = replica_throughput(lay["windows"] * args.steps, world, t_e2e)
    ms = t_dev / args.steps
    hbm, src = peaks()
    nbytes = decon_bytes(case, lay)
    out = {
        "metric": "decon windows/s", "value": value, "unit": "windows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (FP64 spectral division)", "data": "synthetic (seeded image and PSF lattice)",
        "config": {"workload": case.name, "parallelism": f"replicas x{world}", "windows": lay["windows"],
                   "transform": [lay["fullx"], lay["fullz"]],
                   "variant": "shared memory" if (lay["fullx"] * lay["fullz"] + decon_table_len(lay)) * 8 <= 220 * 1024
                   else "global workspace",
                   "l2": "flushed (256 MiB write) before every timed step",
                   "iterations": args.decon_iters, "reg_l1": 2e-2 if args.decon_iters else 0.0,
                   "reg_l2": 6e-2 if args.decon_iters else 0.0},
        "e2e": {"value": e2e, "unit": "windows/s", "h2d_bytes_per_step": 2 * mig.nbytes,
                "d2h_bytes_per_step": 2 * mig.nbytes},
        "roofline": {"bound": "hbm", "kernel": "decon_window + decon_gather", "achieved": nbytes / (ms * 1e6),
                     "peak": hbm, "peak_source": src, "unit": "GB/s", "frac": nbytes / (ms * 1e6) / hbm,
                     "traffic": None, "algorithmic_bytes_per_launch": nbytes,
                     "note": "the window transforms are one-warp FP32 FFTs in registers and shared memory (Bluestein's "
                             "chirp-z through a power-of-two FFT for the odd lengths); HBM is not the bound",
                     "fft_equivalent_gflops": decon_flops(lay) / (ms * 1e6)},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.decon_iters:
        cpu_s, cores, odec, ocoef = decon_cpu(case, mig, psf)
        gdec = d_dec.cpu().numpy()
        out["cpu_baseline"] = {"value": lay["windows"] / cpu_s, "unit": "windows/s", "cores": cores, "kind": "port",
                               "sample": f"the whole image ({lay['windows']} windows), {cpu_s:.2f} s"}
        out["parity"] = {"dec_rel_l2_vs_oracle": float(np.linalg.norm(gdec - odec) / np.linalg.norm(odec)),
                         "coef_equal": bool(np.array_equal(d_coef.cpu().numpy(), ocoef))}
    return out


def survey_cpu_baseline(w, nsteps):
    """The oracle's FP32 OpenMP RTM of the survey's first shot for nsteps steps on the full grid;
    its time per step, times the survey's total steps (every shot's nt), gives the survey's
    shots/s."""
    orc = load_oracle()
    pmlc = w.pmlc
    M, _ = oracle_model(orc, w, w.vp_mig, nsteps)
    shots = w.extra["shots"]
    s = shots[0]
    G = orc.Geom(int(s["sx"]) + pmlc, int(s["sz"]) + pmlc, s["rec_x"] + pmlc, s["rec_z"] + pmlc)
    rick = orc.ricker(nsteps, s["f0"], w.dt)
    data = np.random.default_rng(0).standard_normal((len(s["rec_x"]), nsteps)).astype(np.float32)
    t = time.perf_counter()
    orc.rtm_shot(M, G, rick, data)
    dt = time.perf_counter() - t
    total = dt / nsteps * sum(int(x["nt"]) for x in shots)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": len(shots) / total, "unit": "shots/s", "cores": cores, "kind": "port", "sample_s": dt,
            "sample": f"{nsteps} steps (forward + backward) of the survey's first shot on the full grid; the time "
                      f"per step times the survey's {sum(int(x['nt']) for x in shots)} steps; {dt:.2f} s measured"}


def lsrtm_cpu_baseline(w, nsteps=100):
    """The oracle's Born modelling + adjoint (FP32, OpenMP stencils, serial adjoint scatters)
    for one shot over nsteps steps on the full grid, extrapolated to nt."""
    orc = load_oracle()
    pmlc = w.pmlc
    M, vp = oracle_model(orc, w, w.vp_mig, nsteps)
    rx, rz = w.receivers_padded()
    G = orc.Geom(w.sx[0] + pmlc, pmlc, rx, rz)
    rick = orc.ricker(nsteps, w.f0, w.dt)
    dk = np.zeros_like(vp)
    dk[pmlc:-pmlc, pmlc:-pmlc] = 2 * 1000.0 * w.vp_mig ** 2 * w.extra["reflectivity"]
    t = time.perf_counter()
    d = orc.born(M, G, rick, dk.astype(np.float32), np.float32)
    orc.born_adjoint(M, G, rick, d.astype(np.float32), np.float32)
    dt = time.perf_counter() - t
    per_shot = dt * w.nt / nsteps
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": 1.0 / per_shot, "unit": "shots/s", "cores": cores, "kind": "port", "sample_s": dt,
            "sample": f"Born + adjoint of 1 shot, {nsteps} of {w.nt} steps on the full grid, extrapolated; "
                      f"{dt:.2f} s measured"}


C5FLOW_WORKLOAD = ("c5 imaging + PSF + deconvolution flow: 4001x1601 @4 m, nt=8000, dt=0.35 ms, 25 Hz, 24 surface shots, "
                   "1201 well receivers, FP16-scaled strips; PSF data of a 40x16 lattice of +1% velocity points on the "
                   "migration model (exact scattered field); both images stacked over the shots; windowed "
                   "deconvolution with 127^2 output windows at the lattice's 99-cell PSF spacing")


def run_c5flow(args, rank, world, dist):
    """The large-survey flow of the reference's three programs on the 4001x1601 configuration: per
    shot, the PSF data of the scatter lattice (AFor's scatter mode, as an exact scattered field),
    the RTM of the observed data and the RTM of the PSF data (AVSPRTM, stacked), then the windowed
    deconvolution of the stacked image by the stacked PSF image (decon2d_mine).  A step is the whole
    flow; the observed data (the survey's input) are modelled once beforehand.  Per-image errors
    against FP64 come from the oracle on the shot nearest the well over the first --parity-nt steps
    (2000 by default; the full FP64 survey is days of host time) and from the oracle's window loop
    on the engine's own stacked images."""
    import ctypes as C
    import torch
    swd = load_pkg()
    from swd_b200 import configs
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    w = configs.c5()
    ns = args.c5_shots
    p = w.pmlc
    vtrue, vmig = swd.pad_model(w.vp, p), swd.pad_model(w.vp_mig, p)
    rho = np.full_like(vmig, 1000.0)
    vs = vmig.copy()
    for ix in w.scatter_x:
        for iz in w.scatter_z:
            vs[ix + p, iz + p] *= np.float32(1.01)
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, w.nt, device=dev)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    E.set_stream(stream.cuda_stream)
    E.set_strip_precision(swd.STRIP_F16)
    rick = swd.ricker_wave(w.nt, w.f0, w.dt)
    rx, rz = w.receivers_padded()
    shots = [swd.ShotSpec(w.sx[i] + p, p, rx, rz, w.nt) for i in range(ns)]
    E.setup_default(vtrue, rho)
    obs = [E.forward(s, rick) for s in shots]           # the survey's observed records (input)
    E.set_model(vmig, rho)
    E.set_scatter_model(vs, rho)
    case = configs.decon_case("c5")
    lay = configs.decon_layout(case)
    dp = swd.DeconParams(w.nx, w.nz, case.psfwin[0], case.psfwin[1], case.filterwin[0], case.filterwin[1],
                         case.snapwin[0], case.snapwin[1], case.epsilon, 0, 0, 0, 0, 0, 0.0, 0.0)
    d_mig = torch.empty((w.nx, w.nz), dtype=torch.float32, device="cuda")
    d_psf, d_dec, d_coef = torch.empty_like(d_mig), torch.empty_like(d_mig), torch.empty_like(d_mig)
    L = swd.lib()

    def flow():
        psf_data = []
        E.stack_reset()
        for s, d in zip(shots, obs):
            psf_data.append(E.forward_scatter(s, rick))
            E.rtm_shot(s, rick, d, want=())
        E._ck(L.swd_stack_get(E._h, 1, swd._ptr(d_mig)))
        E.stack_reset()
        for s, d in zip(shots, psf_data):
            E.rtm_shot(s, rick, d, want=())
        E._ck(L.swd_stack_get(E._h, 1, swd._ptr(d_psf)))
        E._ck(L.swd_decon(E._h, C.byref(dp), swd._ptr(d_mig), swd._ptr(d_psf), swd._ptr(d_dec), swd._ptr(d_coef)))
        return psf_data

    for _ in range(args.warmup):
        flow()
    torch.cuda.synchronize()
    n0 = E.launch_count()
    with ClockSampler(dev) as clk:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total = 0.0
        for _ in range(args.steps):
            a.record(stream)
            psf_data = flow()
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
    launches = E.launch_count() - n0
    t_ms, = max_over_ranks(dist, [total], "cuda")
    if rank != 0:
        return None
    per = t_ms / args.steps
    out = {"metric": "RTM shots/s", "value": 2 * ns * args.steps * world / (t_ms / 1e3), "unit": "shots/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": per, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 imaging, FP16 strips, FP64 spectral division)",
           "data": "synthetic (seeded random-field model)",
           "config": {"workload": C5FLOW_WORKLOAD, "shots": ns, "migrations_per_step": 2 * ns,
                      "parallelism": f"replicas x{world}", "windows": lay["windows"]},
           "flow_s": per / 1e3, "survey_images_per_s": 1e3 / per, "gpu_launches": launches, "clocks": clk.summary()}
    if not args.no_parity:
        orc = load_oracle()
        pnt = args.parity_nt or 2000
        # the shot nearest the well, whose first pnt steps already reach the receivers
        i0 = int(np.argmin([abs(s.s_ix - int(rx[0])) for s in shots]))
        mig, psf = d_mig.cpu().numpy(), d_psf.cpu().numpy()
        dec = d_dec.cpu().numpy()
        t = time.perf_counter()
        odec, _ = orc.decon(w.nx, w.nz, mig, psf, case.psfwin, case.filterwin, case.snapwin, case.epsilon,
                            nthreads=os.cpu_count() or 1)
        e_dec = float(np.linalg.norm(dec - odec) / np.linalg.norm(odec))
        # shot 1 over the first pnt steps: its RTM image (observed data) and PSF image (PSF data)
        par = {"deconvolved_image_vs_oracle_decon_of_the_same_images": e_dec, "shot": i0 + 1}
        # the shot's images with the flow's FP16 strips, and with int16 and FP32 strips for scale,
        # against one FP64 oracle run per record
        precs = {"f16": swd.STRIP_F16, "i16": swd.STRIP_I16, "f32": swd.STRIP_F32}
        for name, rec in (("image", obs[i0]), ("psf_image", psf_data[i0])):
            ref = oracle_rtm(w, shots[i0], rick, rec, pnt)
            par[name] = {}
            for pname, pv in precs.items():
                E.set_strip_precision(pv)
                par[name][pname + "_strips"] = engine_vs_oracle(swd, E, shots[i0], rick, rec, pnt, ref)
            E.set_strip_precision(swd.STRIP_F16)
        # the PSF data themselves: the exact scattered field against the FP64 difference of two records
        M0, _ = oracle_model(orc, w, w.vp_mig, pnt)
        M1 = orc.Model(vs, rho, orc.cpml(w.ntx, w.ntz, p, w.dx, w.dz, w.dt), orc.cal_xishu(w.Lc), p, w.Lc, pnt,
                       w.dx, w.dz, w.dt)
        G = orc.Geom(shots[i0].s_ix, shots[i0].s_iz, rx, rz)
        rk = np.ascontiguousarray(rick[:pnt])
        d64 = orc.forward(M1, G, rk, dtype=np.float64)["seis"] - orc.forward(M0, G, rk, dtype=np.float64)["seis"]
        E.set_scatter_model(vs, rho)
        sh = swd.ShotSpec(shots[i0].s_ix, shots[i0].s_iz, rx, rz, pnt)
        par["psf_data_vs_fp64_difference"] = float(np.linalg.norm(E.forward_scatter(sh, rk) - d64) / np.linalg.norm(d64))
        par["note"] = (f"shot {i0 + 1} (nearest the well), first {pnt} of {w.nt} steps, against the FP64 oracle; the "
                       "deconvolution against the oracle's FP64 window loop on the engine's stacked images")
        par["oracle_s"] = round(time.perf_counter() - t, 1)
        out["parity"] = par
    E.close()
    return out


def run_profile_kernels(args):
    """One RTM shot on the benchmark grid with a short record (--nt) and seeded random data,
    no warm-up shots and no data generation: the command the ncu captures run, so that few
    launches precede the captured ones.  Kernels are launched directly (no CUDA graphs; the
    kernels are the same ones the graphs replay), which keeps ncu's per-launch handling fast.
    Prints per-kernel event timings."""
    import ctypes as C
    if args.workload == "afor":
        return run_profile_afor(args)
    if args.workload == "lsrtm":
        return run_profile_lsrtm(args)
    if args.workload == "batch":
        return run_profile_batch(args)
    swd = load_pkg()
    from swd_b200 import configs
    w = configs.CONFIGS[args.config]()
    w.nt = args.nt
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, w.nt)
    vmig = swd.pad_model(w.vp_mig, w.pmlc)
    E.setup_default(vmig, np.full_like(vmig, 1000.0))
    E.set_option(swd.OPT_GRAPHS, 0)
    if args.ref_pairing:
        E.set_option(swd.OPT_BWD_BY_KIND, 0)
    if args.stored:
        E.set_source_storage(1, swd.STRIP_I16)
    if args.staged:
        E.set_option(swd.OPT_STAGED, 1)
    if args.path is not None:
        E.set_kernel_path(args.path)
    E.set_strip_precision({"f32": swd.STRIP_F32, "f16": swd.STRIP_F16}[w.extra.get("strips", "f32")])
    rick = swd.ricker_wave(w.nt, w.f0, w.dt)
    rx, rz = w.receivers_padded()
    sx, sz = w.source_padded()
    shot = swd.ShotSpec(sx, sz, rx, rz, w.nt)
    data = np.random.default_rng(0).standard_normal((len(rx), w.nt)).astype(np.float32) * 1e-6
    E.profile(1)
    E.rtm_shot(shot, rick, data, want=())
    prof = E.profile_read()
    print(json.dumps({"mode": "profile-kernels", "grid": [w.ntx, w.ntz], "nt": w.nt, "launches": E.launch_count(),
                      "kernels_us": {k: ms / n * 1e3 for k, (ms, n) in prof.items() if n}}))


def run_profile_afor(args):
    """--profile-kernels of the modelling workload: one forward of the 1601x801 shot with the
    Hilbert twin and the kz split of the well column, --nt steps, kernels launched directly."""
    import ctypes as C
    import torch
    swd = load_pkg()
    from swd_b200 import configs
    w = configs.c2()
    w.nt = args.nt
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, w.nt)
    vtrue = swd.pad_model(w.vp, w.pmlc)
    E.setup_default(vtrue, np.full_like(vtrue, 1000.0))
    E.set_option(swd.OPT_GRAPHS, 0)
    rick = swd.ricker_wave(w.nt, w.f0, w.dt)
    coef, _ = swd.kz_taper(swd.pow2(w.ntz), w.dz)
    rx, rz = w.receivers_padded()
    sx, sz = w.source_padded()
    sh, keep = E._shot(swd.ShotSpec(sx, sz, rx, rz, w.nt))
    ins = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() for a in (rick, E.hilbert(rick), coef)]
    outs = [torch.empty((len(rx), w.nt), dtype=torch.float32, device="cuda") for _ in range(3)]
    torch.cuda.synchronize()
    E.profile(1)
    E._ck(swd.lib().swd_forward(E._h, C.byref(sh), *[swd._ptr(t) for t in ins], *[swd._ptr(t) for t in outs]))
    torch.cuda.synchronize()
    prof = E.profile_read()
    print(json.dumps({"mode": "profile-kernels", "workload": "afor", "grid": [w.ntx, w.ntz], "nt": w.nt,
                      "launches": E.launch_count(),
                      "kernels_us": {k: ms / n * 1e3 for k, (ms, n) in prof.items() if n}}))


def run_profile_lsrtm(args):
    """--profile-kernels of the LSRTM workload: the Born data and the gradient of one 801x401
    shot (BF16 checkpoints every 50 steps), --nt steps, kernels launched directly."""
    import torch
    swd = load_pkg()
    from swd_b200 import configs, lsrtm
    w = configs.c4()
    w.nt = args.nt
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, w.nt)
    vmig = swd.pad_model(w.vp_mig, w.pmlc)
    rho = np.full_like(vmig, 1000.0)
    E.setup_default(vmig, rho)
    E.set_option(swd.OPT_GRAPHS, 0)
    E.set_checkpointing(50, swd.STRIP_BF16)
    rick = swd.ricker_wave(w.nt, w.f0, w.dt)
    rx, rz = w.receivers_padded()
    op = lsrtm.BornOperator(E, swd.ShotSpec(w.sx[0] + w.pmlc, w.pmlc, rx, rz, w.nt), rick, vmig, rho)
    r = torch.tensor(w.extra["reflectivity"], device="cuda").requires_grad_(True)
    torch.cuda.synchronize()
    E.profile(1)
    d = lsrtm.born(r, op)
    (0.5 * (d.double() ** 2).sum()).backward()
    torch.cuda.synchronize()
    prof = E.profile_read()
    print(json.dumps({"mode": "profile-kernels", "workload": "lsrtm", "grid": [w.ntx, w.ntz], "nt": w.nt,
                      "launches": E.launch_count(),
                      "kernels_us": {k: ms / n * 1e3 for k, (ms, n) in prof.items() if n}}))


def run_profile_batch(args):
    """--profile-kernels of the batched RTM: the first two shots of the 1201x601 survey as one
    batch (B = 2), --nt steps each, seeded random data, kernels launched directly."""
    swd = load_pkg()
    from swd_b200 import configs
    w = configs.c3()
    E = swd.Engine(w.nx, w.nz, w.pml, w.Lc, w.dx, w.dz, w.dt, args.nt)
    vmig = swd.pad_model(w.vp_mig, w.pmlc)
    E.setup_default(vmig, np.full_like(vmig, 1000.0))
    E.set_option(swd.OPT_GRAPHS, 0)
    E.set_option(swd.OPT_BATCH, 2)
    rng = np.random.default_rng(0)
    shots, ricks, data = [], [], []
    for s in w.extra["shots"][:2]:
        shots.append(swd.ShotSpec(s["sx"] + w.pmlc, s["sz"] + w.pmlc, s["rec_x"] + w.pmlc, s["rec_z"] + w.pmlc, args.nt))
        ricks.append(swd.ricker_wave(args.nt, s["f0"], w.dt))
        data.append(rng.standard_normal((len(s["rec_x"]), args.nt)).astype(np.float32) * 1e-6)
    E.profile(1)
    E.rtm_batch(shots, ricks, data)
    prof = E.profile_read()
    print(json.dumps({"mode": "profile-kernels", "workload": "batch", "grid": [w.ntx, w.ntz], "nt": args.nt,
                      "batch": E.get_option(swd.OPT_BATCH_TUNED), "launches": E.launch_count(),
                      "kernels_us": {k: ms / n * 1e3 for k, (ms, n) in prof.items() if n}}))


def run_reference_decon(args):
    configs = load_configs()
    case = configs.decon_case(args.config)
    lay = configs.decon_layout(case)
    mig, psf = configs.decon_inputs(case)
    t0 = time.perf_counter()
    times, cores = [], 1
    for i in range(args.warmup + args.steps):
        dt, cores, _, _ = decon_cpu(case, mig, psf)
        if i >= args.warmup:
            times.append(dt)
    mean = float(np.mean(times))
    value = lay["windows"] / mean
    return {"metric": "decon windows/s", "value": value, "unit": "windows/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 FFTs", "data": "synthetic", "impl": "reference",
            "config": {"workload": case.name, "parallelism": "host OpenMP"},
            "step": f"the whole image ({lay['windows']} windows)",
            "cpu_baseline": {"value": value, "unit": "windows/s", "cores": cores, "kind": "port",
                             "sample": f"the whole image ({lay['windows']} windows) per step"},
            "e2e": {"value": value, "unit": "windows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}


def run_reference(args):
    """The reference arm: the oracle's restatement of the reference's loops on the host cores,
    for the metric, unit and workload of our arm (--workload, --config).  Each step is one
    bounded sample of that workload (a few hundred time steps of the shot on the full grid, the
    oracle's own host preparation, nothing of libswd); `steps` and `ms_per_step` are those
    samples as timed, and `value` is the shot rate they extrapolate to."""
    if args.workload == "decon":
        return run_reference_decon(args)
    configs = load_configs()
    if args.workload == "afor":
        w = configs.c2()
        metric, workload = "modelling shots/s", AFOR_WORKLOAD
        sample = lambda: afor_cpu_baseline(w, max(16, args.cpu_steps // 3))
    elif args.workload == "lsrtm":
        w = configs.c4()
        metric, workload = "LSRTM gradient shots/s", LSRTM_WORKLOAD
        sample = lambda: lsrtm_cpu_baseline(w, nsteps=max(8, args.cpu_steps // 3))
    elif args.workload == "batch":
        w = configs.c3()
        metric, workload = "RTM shots/s", BATCH_WORKLOAD
        sample = lambda: survey_cpu_baseline(w, max(8, args.cpu_steps))
    elif args.workload == "c5flow":
        w = configs.c5()
        metric, workload = "RTM shots/s", C5FLOW_WORKLOAD
        sample = lambda: cpu_baseline(w, samples=1, nsteps=rtm_cpu_steps(args, w))
    else:
        w = configs.CONFIGS[args.config]()
        metric, workload = "RTM shots/s", WORKLOADS[args.config]
        sample = lambda: cpu_baseline(w, samples=1, nsteps=rtm_cpu_steps(args, w))
    t0 = time.perf_counter()
    per_unit, sample_s = [], []
    for i in range(args.warmup + args.steps):
        cb = sample()
        if i >= args.warmup:
            per_unit.append(1.0 / cb["value"])
            sample_s.append(cb["sample_s"])
    value = 1.0 / float(np.mean(per_unit))
    cb["value"] = value
    return {"metric": metric, "value": value, "unit": "shots/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(sample_s)) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload, "parallelism": "host OpenMP"},
            "step": "one bounded sample of the workload: " + cb["sample"].split(";")[0]
                    + "; value extrapolates the samples to whole shots",
            "cpu_baseline": cb, "e2e": {"value": value, "unit": "shots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}


def compact(rec):
    """The figures of a workload's own line that its sub-record in the default line keeps."""
    keep = ("metric", "value", "unit", "steps", "warmup", "ms_per_step", "dtype", "gpu_launches", "clocks", "parity")
    out = {k: rec[k] for k in keep if k in rec}
    out["workload"] = rec.get("config", {}).get("workload")
    if rec.get("e2e"):
        out["e2e"] = rec["e2e"].get("value")
    r = rec.get("roofline") or {}
    out["roofline"] = {k: r[k] for k in ("bound", "kernel", "achieved", "peak", "unit", "frac", "traffic",
                                         "kernels_us", "kernels_frac", "fft_equivalent_gflops", "note") if k in r}
    return out


def extra_workloads(args):
    """Sub-records of the default line (one-GPU runs, after its own timed regions): one shot of the
    4001x1601 RTM (FP16 strips, per-kernel roofline), the AFor modelling shot and the 4001x1601
    image's windowed deconvolution, each with its own warm-up and timed steps, L2 flush and clocks,
    so that these workloads are measured by every default run too.  A failure is recorded in
    place of the sub-record and leaves the headline line intact."""
    import copy
    subs = {}
    jobs = (("rtm_c5", run_ours, dict(config="c5", steps=2, warmup=3, no_parity=True, no_batch=True, no_stored=True,
                                      autotune=False, tma=False, staged=False, pdl=False, path=None)),
            ("afor", run_afor, dict(steps=5, warmup=3)),
            ("decon_c5", run_decon, dict(config="c5", steps=5, warmup=3)))
    for name, fn, over in jobs:
        a = copy.copy(args)
        for k, v in over.items():
            setattr(a, k, v)
        try:
            subs[name] = compact(fn(a, 0, 1, None))
        except Exception as e:   # recorded, not hidden: the sub-record carries the error
            subs[name] = {"error": f"{type(e).__name__}: {e}"}
    return subs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-steps", type=int, default=300, help="time steps per CPU-baseline sample")
    ap.add_argument("--profile-kernels", action="store_true", help="one short shot for ncu captures")
    ap.add_argument("--nt", type=int, default=30, help="record length of --profile-kernels")
    ap.add_argument("--path", type=int, default=None, help="kernel path: 0 plain (two launches per step), 1 fused")
    ap.add_argument("--stored", action="store_true", help="--profile-kernels: stored-source RTM (int16 dp/dt)")
    ap.add_argument("--ref-pairing", action="store_true",
                    help="--profile-kernels: the reference's pairing of the backward phases (k_bwd_1, k_bwd_2)")
    ap.add_argument("--workload", choices=["rtm", "lsrtm", "batch", "decon", "afor", "c5flow"], default="rtm")
    ap.add_argument("--c5-shots", type=int, default=24, help="--workload c5flow: shots of the survey")
    ap.add_argument("--config", choices=["c2", "c5", "shipped"], default="c2",
                    help="grid of --workload rtm (c2, c5) or decon (c2, c5, shipped: the reference's window geometry)")
    ap.add_argument("--no-stored", action="store_true", help="skip the stored-source measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-survey sub-record")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the sub-records of the other workloads (c5 shot, AFor modelling, c5 decon)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the image-error check against the FP64 oracle (a few minutes of host time)")
    ap.add_argument("--parity-nt", type=int, default=0,
                    help="record length of the FP64 check (0: the whole record; --workload c5flow: 2000 steps)")
    ap.add_argument("--tma", action="store_true", help="velocity kernels with TMA-staged pressure tiles (SWD_OPT_TMA)")
    ap.add_argument("--pdl", action="store_true", help="step kernels as programmatic dependent launches (SWD_OPT_PDL)")
    ap.add_argument("--autotune", action="store_true",
                    help="the passes choose their step-kernel variants by timing (SWD_OPT_AUTOTUNE)")
    ap.add_argument("--staged", action="store_true",
                    help="forward pressure kernel with every stencil operand staged by TMA (SWD_OPT_STAGED)")
    ap.add_argument("--streams", type=int, default=3,
                    help="--workload lsrtm: engines (streams and host threads) the survey's shots are spread over")
    ap.add_argument("--decon-iters", type=int, default=0,
                    help="--workload decon: FISTA iterations of the regularised option (L1 0.02, L2 0.06)")
    ap.add_argument("--ckpt-prec", choices=["f32", "f16", "bf16", "i16"], default="bf16",
                    help="checkpoint precision of --workload lsrtm")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        # the CPU restatement only: the package (and with it libswd) is not loaded
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    load_pkg()
    if args.profile_kernels:
        run_profile_kernels(args)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = td
    runner = {"rtm": run_ours, "lsrtm": run_lsrtm, "batch": run_batch, "decon": run_decon, "afor": run_afor,
              "c5flow": run_c5flow}[args.workload]
    out = runner(args, rank, world, dist)
    if rank == 0 and world == 1 and args.workload == "rtm" and args.config == "c2" and not args.no_extra:
        out["workloads"] = extra_workloads(args)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
