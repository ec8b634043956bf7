"""Host logic of the survey-level Born autograd function (lsrtm.BornSurvey) on the CPU, with
stand-in operators and engines: shot i runs its forward on engine i % n and leaves its own
checkpoint buffer, the adjoint of each shot gets the buffer of its own forward, and the
gradient is the sum of the shots' adjoints in float64."""
import threading

import pytest
import torch


class FakeEngine:
    def __init__(self, k):
        self.k = k


class FakeOp:
    """d_i = a_i * (r * m_i) summed along z (a linear map), adjoint exact; records which
    engine and host thread ran each call and which checkpoint the adjoint received."""

    def __init__(self, i, shape):
        g = torch.Generator().manual_seed(100 + i)
        self.i = i
        self.m = torch.randn(shape, generator=g, dtype=torch.float64)
        self.a = 0.5 + i
        self.log = []

    def ckpt_buffer(self, engine):
        return ("ckpt", self.i, engine.k)

    def forward(self, r, ckpt, engine):
        self.log.append(("fwd", engine.k, ckpt, threading.get_ident()))
        return (self.a * (r.double() * self.m).sum(dim=1)).float()

    def adjoint(self, g, ckpt, engine):
        self.log.append(("adj", engine.k, ckpt, threading.get_ident()))
        return self.a * g.double()[:, None] * self.m


@pytest.fixture
def lsrtm(swd):
    from swd_b200 import lsrtm
    return lsrtm


def test_born_survey_forward_backward(lsrtm):
    from swd_b200 import survey
    shape = (6, 4)
    ops = [FakeOp(i, shape) for i in range(5)]
    pool = survey.EnginePool([FakeEngine(k) for k in range(2)])
    try:
        r = torch.randn(shape, dtype=torch.float64, requires_grad=True)
        outs = lsrtm.born_survey(r, ops, pool)
        weights = [torch.randn(shape[0], dtype=torch.float64) for _ in ops]
        J = sum((o.double() * w).sum() for o, w in zip(outs, weights))
        J.backward()
    finally:
        pool.close()
    assert len(outs) == len(ops)
    for op, o in zip(ops, outs):
        assert torch.allclose(o.double(), op.a * (r.detach() * op.m).sum(dim=1), rtol=1e-5, atol=1e-6)
    want = sum(op.a * w[:, None] * op.m for op, w in zip(ops, weights))
    assert r.grad.dtype == torch.float64
    # the shots' data are float32, so their incoming gradients are too: agreement to float32
    assert torch.allclose(r.grad, want, rtol=1e-6, atol=1e-6)
    for op in ops:
        (f, fk, fck, _), (a, ak, ack, _) = op.log
        assert (f, a) == ("fwd", "adj")
        assert fk == op.i % 2 and ak == op.i % 2       # shot i on engine i % n both ways
        assert ack == fck == ("ckpt", op.i, op.i % 2)  # the adjoint gets its own forward's buffer
    threads = {op.log[0][3] for op in ops}
    assert len(threads) == 2                            # one host thread per engine


def test_lsrtm_objective_with_and_without_pool(lsrtm, monkeypatch):
    """J(r) = 1/2 sum ||L_s r - d_s||^2 and its gradient agree between the sequential path
    (one autograd node per shot) and the pool path."""
    from swd_b200 import survey

    class SeqOp(FakeOp):
        E = None

        def __init__(self, i, shape):
            super().__init__(i, shape)
            self.E = FakeEngine(0)

        def ckpt_buffer(self, engine=None):
            return FakeOp.ckpt_buffer(self, engine or self.E)

        def forward(self, r, ckpt=None, engine=None):
            return FakeOp.forward(self, r, ckpt, engine or self.E)

        def adjoint(self, g, ckpt=None, engine=None):
            return FakeOp.adjoint(self, g, ckpt, engine or self.E)

    shape = (5, 3)
    ops = [SeqOp(i, shape) for i in range(4)]
    data = [torch.randn(shape[0], dtype=torch.float32) for _ in ops]
    r0 = torch.randn(shape, dtype=torch.float64)
    r1 = r0.clone().requires_grad_(True)
    J1 = lsrtm.lsrtm_objective(r1, ops, data)
    J1.backward()
    pool = survey.EnginePool([FakeEngine(k) for k in range(3)])
    try:
        r2 = r0.clone().requires_grad_(True)
        J2 = lsrtm.lsrtm_objective(r2, ops, data, pool=pool)
        J2.backward()
    finally:
        pool.close()
    assert torch.allclose(J1, J2, rtol=1e-12)
    assert torch.allclose(r1.grad, r2.grad, rtol=1e-10, atol=1e-12)
