"""Differentiable modelling over libswd: torch.autograd.Function wrappers of the Born
operator (LSRTM, gradient with respect to reflectivity) and of the nonlinear forward
modelling (gradient with respect to velocity).

Both backward passes call swd_born_adjoint, the exact discrete adjoint of the engine's
forward step (CPML included), so autograd gradients satisfy the dot-product identity to
rounding.  Tensors stay on the GPU: pointers go straight to the C ABI.  The engine keeps its
own stream (so its time loops run as CUDA graphs); each call first waits for torch's current
stream and returns with its own stream drained, so inputs are complete before the engine
reads them and outputs are complete before torch reads them.

Parameterisation.  kappa = rho * vp^2 is the modulus the pressure update uses.  The Born
input is a reflectivity r = dvp / vp on the interior (nx, nz) grid, i.e. dkappa = 2 kappa r;
its gradient is 2 kappa * dJ/dkappa restricted to the interior.  The velocity gradient of the
nonlinear modelling is 2 rho vp * dJ/dkappa on the padded grid.

Background checkpoints.  With the engine's checkpointing on (Engine.set_checkpointing,
default every 50 steps in BF16), the Born forward leaves the background state snapshots in
a device buffer owned by the autograd graph (saved for backward), and the adjoint recomputes
each 50-step segment from them instead of storing the wavefield of every step.

Concurrent shots.  On grids where one shot's launches do not fill the GPU, an EnginePool of
identically configured engines (each with its own stream and buffers) runs the shots of a
survey from one host thread per engine; libswd calls release the GIL, so the engines' kernels
overlap on the device.  born_survey is the survey-level autograd function over such a pool.
"""
from __future__ import annotations

import numpy as np
import torch

from . import Engine, ShotSpec
from .survey import EnginePool


def _dev(t: torch.Tensor) -> torch.Tensor:
    return t.detach().contiguous()


def _sync(device):
    """Wait for the calling thread's current stream on `device` (nothing to wait for on the CPU)."""
    if torch.device(device).type == "cuda":
        torch.cuda.current_stream(device).synchronize()


class BornOperator:
    """Born modelling of one shot on an engine whose model (vp, rho) is already set.

    vp, rho: padded (ntx, ntz) models (numpy or torch); the operator keeps device copies of
    kappa = rho vp^2 for the reflectivity parameterisation."""

    def __init__(self, engine: Engine, shot: ShotSpec, rick, vp, rho, device="cuda"):
        self.E, self.shot = engine, shot
        self.device = torch.device(device)
        self.rick = np.ascontiguousarray(rick, np.float32)
        vp_t = torch.as_tensor(np.asarray(vp, np.float32), device=self.device)
        rho_t = torch.as_tensor(np.asarray(rho, np.float32), device=self.device)
        self.kappa = (rho_t * vp_t * vp_t).contiguous()
        p = engine.pmlc
        self.inner = (slice(p, p + engine.nx), slice(p, p + engine.nz))

    def dkappa(self, r: torch.Tensor) -> torch.Tensor:
        """2 kappa r on the padded grid (zero in the absorbing frame)."""
        dk = torch.zeros_like(self.kappa)
        dk[self.inner] = 2.0 * self.kappa[self.inner] * r
        return dk

    def ckpt_buffer(self, engine: Engine = None):
        n = (engine or self.E).checkpoint_bytes(self.shot.nt)
        return torch.empty(n, dtype=torch.uint8, device=self.device) if n else None

    def forward(self, r: torch.Tensor, ckpt=None, engine: Engine = None) -> torch.Tensor:
        """Born data of reflectivity r; `engine` (default: the operator's own) runs it."""
        E = engine or self.E
        d = torch.empty((len(self.shot.r_ix), self.shot.nt), dtype=torch.float32, device=self.device)
        dk = _dev(self.dkappa(r))
        _sync(self.device)
        E.born(self.shot, self.rick, dk, out=d, ckpt=ckpt)
        return d

    def adjoint_kappa(self, resid: torch.Tensor, ckpt=None, engine: Engine = None) -> torch.Tensor:
        """dJ/dkappa on the padded grid, float64."""
        E = engine or self.E
        g = torch.empty((E.ntx, E.ntz), dtype=torch.float64, device=self.device)
        res = _dev(resid.float())
        _sync(self.device)
        E.born_adjoint(self.shot, self.rick, res, out=g, ckpt=ckpt)
        return g

    def adjoint(self, resid: torch.Tensor, ckpt=None, engine: Engine = None) -> torch.Tensor:
        """Adjoint with respect to the interior reflectivity, float64."""
        g = self.adjoint_kappa(resid, ckpt, engine)
        return 2.0 * self.kappa[self.inner].double() * g[self.inner]


class BornModelling(torch.autograd.Function):
    """d = L r for one shot; backward applies L^T through the engine's exact adjoint."""

    @staticmethod
    def forward(ctx, r: torch.Tensor, op: BornOperator):
        ckpt = op.ckpt_buffer()
        d = op.forward(r.float(), ckpt)
        ctx.op = op
        ctx.ckpt = ckpt
        ctx.dtype = r.dtype
        return d

    @staticmethod
    def backward(ctx, grad_d):
        g = ctx.op.adjoint(grad_d, ctx.ckpt)
        return g.to(ctx.dtype), None


def born(r: torch.Tensor, op: BornOperator) -> torch.Tensor:
    return BornModelling.apply(r, op)


class ForwardModelling(torch.autograd.Function):
    """d = F(vp) (pressure at the receivers) for one shot; the gradient with respect to the
    padded velocity is 2 rho vp * (J^T grad_d) in kappa, J the Born operator at vp."""

    @staticmethod
    def forward(ctx, vp_pad: torch.Tensor, engine: Engine, shot: ShotSpec, rick, rho_pad: torch.Tensor):
        vp_c, rho_c = _dev(vp_pad.float()), _dev(rho_pad.float())
        _sync(vp_c.device)
        engine.set_model(vp_c, rho_c)
        d = torch.empty((len(shot.r_ix), shot.nt), dtype=torch.float32, device=vp_c.device)
        engine.forward(shot, rick, out=d)
        ctx.save_for_backward(vp_c, rho_c)
        ctx.engine, ctx.shot, ctx.rick, ctx.dtype = engine, shot, rick, vp_pad.dtype
        return d

    @staticmethod
    def backward(ctx, grad_d):
        vp_c, rho_c = ctx.saved_tensors
        E = ctx.engine
        res = _dev(grad_d.float())
        g = torch.empty((E.ntx, E.ntz), dtype=torch.float64, device=vp_c.device)
        _sync(vp_c.device)
        E.set_model(vp_c, rho_c)
        E.born_adjoint(ctx.shot, np.ascontiguousarray(ctx.rick, np.float32), res, out=g)
        gv = 2.0 * rho_c.double() * vp_c.double() * g
        return gv.to(ctx.dtype), None, None, None, None


def modelling(vp_pad: torch.Tensor, engine: Engine, shot: ShotSpec, rick, rho_pad: torch.Tensor) -> torch.Tensor:
    return ForwardModelling.apply(vp_pad, engine, shot, rick, rho_pad)


class BornSurvey(torch.autograd.Function):
    """(L_1 r, ..., L_S r) for the shots of a survey, the shots spread over an EnginePool;
    backward sums the shots' adjoints (each from the checkpoints its forward left) in float64."""

    @staticmethod
    def forward(ctx, r: torch.Tensor, ops, pool: EnginePool):
        r32 = _dev(r.float())
        # the pool's threads wait on their own (default) streams: finish this thread's work first
        _sync(r32.device)

        def fwd(E, op):
            ck = op.ckpt_buffer(E)
            return op.forward(r32, ck, engine=E), ck

        res = pool.map(fwd, ops)
        ctx.ops, ctx.pool, ctx.ckpts, ctx.dtype = ops, pool, [c for _, c in res], r.dtype
        return tuple(d for d, _ in res)

    @staticmethod
    def backward(ctx, *grads):
        items = [(op, g, ck) for op, g, ck in zip(ctx.ops, grads, ctx.ckpts) if g is not None]
        if items:
            _sync(items[0][1].device)   # the incoming gradients are complete before other threads read them
        parts = ctx.pool.map(lambda E, it: it[0].adjoint(it[1], it[2], engine=E), items)
        g = parts[0].clone()
        for q in parts[1:]:
            g += q
        return g.to(ctx.dtype), None, None


def born_survey(r: torch.Tensor, ops, pool: EnginePool):
    return BornSurvey.apply(r, ops, pool)


def lsrtm_objective(r: torch.Tensor, ops, data, pool: EnginePool = None) -> torch.Tensor:
    """J(r) = 1/2 sum_shots ||L_s r - d_s||^2, accumulated in float64; with a pool the shots
    run concurrently on its engines."""
    J = torch.zeros((), dtype=torch.float64, device=r.device)
    preds = born_survey(r, ops, pool) if pool is not None else [born(r, op) for op in ops]
    for p, d in zip(preds, data):
        res = p - d
        J = J + 0.5 * (res.double() ** 2).sum()
    return J
