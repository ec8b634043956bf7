"""Host logic of the engine pool (survey.py) on the CPU, with stand-in engines that record
what they are asked to do: shots go round-robin over the engines, each engine works through
its own shots in order on its own host thread, results come back in shot order, and
rtm_survey sums the engines' stacks after resetting them."""
import threading
import time

import numpy as np


class FakeEngine:
    def __init__(self, k, shape=(6, 5)):
        self.k = k
        self.calls = []
        self.threads = set()
        self.stack_img = np.zeros(shape)
        self.resets = 0

    def stack_reset(self):
        self.resets += 1
        self.stack_img[:] = 0.0

    def rtm_shot(self, shot, rick, data, flags=0, want=()):
        self.calls.append(("shot", shot))
        self.threads.add(threading.get_ident())
        time.sleep(0.01)
        self.stack_img += shot

    def rtm_batch(self, shots, ricks, datas, flags=0):
        self.calls.append(("batch", tuple(shots)))
        self.threads.add(threading.get_ident())
        for s in shots:
            self.stack_img += s

    def stack(self, edge_zero=True):
        img = self.stack_img.astype(np.float32).copy()
        if edge_zero:
            img[0, :] = 0.0
        return img


def test_pool_map_round_robin_and_order(swd):
    from swd_b200 import survey
    engines = [FakeEngine(k) for k in range(3)]
    pool = survey.EnginePool(engines)
    try:
        def work(E, i):
            time.sleep(0.02)   # like a shot: long enough that the engines' shares overlap
            return E.k, i, threading.get_ident()

        out = pool.map(work, range(8))
    finally:
        pool.close()
    assert [o[1] for o in out] == list(range(8))            # results in item order
    assert [o[0] for o in out] == [i % 3 for i in range(8)]  # item i on engine i % 3
    # each engine's items ran on one host thread, and the engines used different threads
    by_engine = {}
    for k, _, t in out:
        by_engine.setdefault(k, set()).add(t)
    assert all(len(v) == 1 for v in by_engine.values())
    assert len({next(iter(v)) for v in by_engine.values()}) == 3


def test_rtm_survey_sums_engine_stacks(swd):
    from swd_b200 import survey
    rng = np.random.default_rng(3)
    shots = [rng.standard_normal((6, 5)) for _ in range(7)]
    for batched in (True, False):
        engines = [FakeEngine(k) for k in range(3)]
        for E in engines:
            E.stack_img += 100.0                    # left over from an earlier survey
        pool = survey.EnginePool(engines)
        try:
            got = survey.rtm_survey(pool, shots, [None] * 7, [None] * 7, batched=batched, edge_zero=False)
            gotz = survey.rtm_survey(pool, shots, [None] * 7, [None] * 7, batched=batched, edge_zero=True)
        finally:
            pool.close()
        ref = np.sum([s.astype(np.float32) for s in shots], axis=0)
        assert np.allclose(got, ref, rtol=1e-5, atol=1e-5)
        refz = ref.copy()
        refz[0, :] = 0.0
        assert np.allclose(gotz, refz, rtol=1e-5, atol=1e-5)
        assert all(E.resets == 2 for E in engines)
        if batched:   # one batch per engine, holding its shots in order
            assert [E.calls[0][0] for E in engines] == ["batch"] * 3
            assert len(engines[0].calls[0][1]) == 3 and len(engines[2].calls[0][1]) == 2
        else:
            assert [len(E.calls) for E in engines] == [6, 4, 4]   # 3, 2, 2 shots per survey, two surveys


def test_pool_with_fewer_items_than_engines(swd):
    from swd_b200 import survey
    engines = [FakeEngine(k) for k in range(4)]
    pool = survey.EnginePool(engines)
    try:
        out = pool.map(lambda E, i: E.k * 10 + i, [0, 1])
        img = survey.rtm_survey(pool, [np.ones((6, 5))], [None], [None], batched=False, edge_zero=False)
    finally:
        pool.close()
    assert out == [0, 11]
    assert np.allclose(img, 1.0)
