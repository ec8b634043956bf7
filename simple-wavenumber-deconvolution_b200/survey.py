"""Surveys of many shots on one GPU: an EnginePool of identically configured engines, each
with its own CUDA stream, buffers and captured time loops, driven from one host thread per
engine.  libswd calls release the GIL, so the engines' kernels overlap on the device; this fills
the GPU on grids where one shot's launches are latency-bound (a few hundred thousand to a few
million cells), and it composes with swd_rtm_batch, which each engine may use for its share.

The reference migrates its shots one after another on each GPU (acoustic_HLVSPRTMC.cpp:576-745)
and sums the images with MPI_Allreduce (:750-752); rtm_survey reads each engine's stack (FP64 on
the device, float32 out, like the reference's image) and sums the parts in float64.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import RTM_PREPROCESS


class EnginePool:
    """n engines configured alike (same grid, model, stencil, CPML, checkpointing) and one host
    thread per engine.  map(fn, items) calls fn(engine, item) with item i on engine i % n, each
    engine working through its items in order; results come back in item order."""

    def __init__(self, engines):
        self.engines = list(engines)
        self._exec = ThreadPoolExecutor(max_workers=len(self.engines))

    def __len__(self):
        return len(self.engines)

    def map(self, fn, items):
        items = list(items)
        n = len(self.engines)

        def work(k):
            return [(i, fn(self.engines[k], items[i])) for i in range(k, len(items), n)]

        out = [None] * len(items)
        for part in self._exec.map(work, range(min(n, len(items)))):
            for i, v in part:
                out[i] = v
        return out

    def close(self):
        self._exec.shutdown()


def rtm_survey(pool: EnginePool, shots, ricks, datas, flags=RTM_PREPROCESS, batched=True, edge_zero=True):
    """Migrate and stack the shots over the pool: shot i on engine i % n, each engine through
    swd_rtm_batch (batched=True) or one swd_rtm_shot per shot; returns the stacked image
    (nx, nz) float32, the sum of the engines' stacks (edge zeroing is a mask, so zeroing each
    engine's stack equals zeroing the sum)."""
    n = len(pool.engines)
    for E in pool.engines:
        E.stack_reset()

    def work(E, k):
        idx = list(range(k, len(shots), n))
        if not idx:
            return None
        if batched:
            E.rtm_batch([shots[i] for i in idx], [ricks[i] for i in idx], [datas[i] for i in idx], flags=flags)
        else:
            for i in idx:
                E.rtm_shot(shots[i], ricks[i], datas[i], flags=flags, want=())
        return E.stack(edge_zero=edge_zero).astype(np.float64)

    parts = [p for p in pool.map(work, range(n)) if p is not None]
    return np.sum(parts, axis=0).astype(np.float32)
