"""Batched multi-shot RTM (swd_rtm_batch) through the C ABI: shots of uneven record length
and receiver aperture run together in batched launches must stack to the same image as the
same shots migrated one at a time with swd_rtm_shot, for every batch size, with and without
CUDA graphs, and with compressed strips.  The per-cell arithmetic is the same, so the stacks
agree to rounding (tolerance 1e-6 relative L2)."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6


class Survey:
    """A small model with 5 shots of different nt, source position and receiver set."""

    def __init__(self, swd, orc, nx=100, nz=60, pml=10, Lc=4, dt=5e-4, seed=11):
        rng = np.random.default_rng(seed)
        v = np.full((nx, nz), 1900.0, np.float32)
        v[:, nz // 3:] = 2500.0
        v += rng.uniform(-50, 50, v.shape).astype(np.float32)
        self.pmlc = p = pml + Lc
        self.nx, self.nz = nx, nz
        self.vp = orc.pad_model(v, p)
        self.rho = np.full_like(self.vp, 1000.0)
        self.nts = [400, 330, 290, 401, 350]
        self.nt_max = max(self.nts)
        self.E = swd.Engine(nx, nz, pml, Lc, 5.0, 5.0, dt, self.nt_max)
        self.E.setup_default(self.vp, self.rho)
        self.shots, self.ricks, self.data = [], [], []
        for k, nt in enumerate(self.nts):
            nr = 20 + 9 * k
            rx = np.full(nr, p + 60 + 5 * k, np.int32)
            rz = (p + 3 + np.arange(nr) * (nz - 6) // nr).astype(np.int32)
            if k == 2:                      # a duplicated receiver cell
                rz[5] = rz[4]
            shot = swd.ShotSpec(p + 10 + 17 * k, p, rx, rz, nt)
            rick = swd.ricker_wave(nt, 20.0 + 3 * k, dt)
            self.shots.append(shot)
            self.ricks.append(rick)
            self.data.append(self.E.forward(shot, rick))

    def sequential(self):
        self.E.stack_reset()
        for s, r, d in zip(self.shots, self.ricks, self.data):
            self.E.rtm_shot(s, r, d, want=())
        return self.E.stack(edge_zero=False)

    def batched(self, B):
        self.E.stack_reset()
        self.E.set_option(1, 1)
        self.E.set_option(2, B)
        self.E.rtm_batch(self.shots, self.ricks, self.data)
        return self.E.stack(edge_zero=False)


@pytest.fixture(scope="module")
def survey(swd, orc):
    return Survey(swd, orc)


@pytest.fixture(scope="module")
def reference(survey):
    return survey.sequential()


@pytest.mark.parametrize("B", [1, 2, 3, 5, 8])
def test_batch_stack_equals_sequential_shots(survey, reference, B):
    got = survey.batched(B)
    assert np.abs(reference).max() > 0
    assert rel_l2(got, reference) < TOL


def test_batch_without_graphs(survey, reference, swd):
    survey.E.stack_reset()
    survey.E.set_option(swd.OPT_BATCH, 3)
    survey.E.set_option(swd.OPT_GRAPHS, 0)
    survey.E.rtm_batch(survey.shots, survey.ricks, survey.data)
    got = survey.E.stack(edge_zero=False)
    survey.E.set_option(swd.OPT_GRAPHS, 1)
    assert rel_l2(got, reference) < TOL


def test_batch_autotune_picks_a_size(survey, reference, swd):
    survey.E.stack_reset()
    survey.E.set_option(swd.OPT_BATCH, 0)
    survey.E.rtm_batch(survey.shots, survey.ricks, survey.data)
    tuned = survey.E.get_option(swd.OPT_BATCH_TUNED)
    assert tuned in (1, 2, 4, 8)
    assert rel_l2(survey.E.stack(edge_zero=False), reference) < TOL


@pytest.mark.parametrize("prec", [1, 3], ids=["f16", "i16"])
def test_batch_compressed_strips(survey, swd, prec):
    survey.E.set_strip_precision(prec)
    ref = survey.sequential()
    got = survey.batched(4)
    survey.E.set_strip_precision(0)
    assert rel_l2(got, ref) < TOL


def test_batch_rejects_unsupported_flags(survey, swd):
    with pytest.raises(swd.SwdError):
        survey.E.rtm_batch(survey.shots, survey.ricks, survey.data, flags=swd.RTM_PREPROCESS | swd.RTM_NO_STACK)


def test_batch_checks_every_shot_before_migrating(survey, reference, swd):
    """A shot with its source outside the grid, behind shots that would batch first: the call
    fails on the host and the stack is left as it was (no shot of the call is stacked)."""
    E = survey.E
    E.set_option(swd.OPT_GRAPHS, 1)
    E.set_option(swd.OPT_BATCH, 1)
    E.stack_reset()
    E.rtm_batch(survey.shots[:1], survey.ricks[:1], survey.data[:1])
    before = E.stack(edge_zero=False)
    bad = survey.shots[1]
    bad = swd.ShotSpec(E.ntx + 5, bad.s_iz, bad.r_ix, bad.r_iz, bad.nt)
    shots = survey.shots[2:] + [bad]
    with pytest.raises(swd.SwdError, match="source cell"):
        E.rtm_batch(shots, survey.ricks[2:] + [survey.ricks[1]], survey.data[2:] + [survey.data[1]])
    assert np.array_equal(E.stack(edge_zero=False), before)


def test_survey_on_engine_pool(survey, reference, swd):
    """rtm_survey over three engines (concurrent host threads and streams, each through
    swd_rtm_batch) stacks to the sequential image up to the float32 rounding of the per-engine
    stacks."""
    from swd_b200 import survey as sv
    engines = []
    for _ in range(3):
        E = swd.Engine(survey.nx, survey.nz, 10, 4, 5.0, 5.0, 5e-4, survey.nt_max)
        E.setup_default(survey.vp, survey.rho)
        engines.append(E)
    pool = sv.EnginePool(engines)
    try:
        got = sv.rtm_survey(pool, survey.shots, survey.ricks, survey.data, edge_zero=False)
        again = sv.rtm_survey(pool, survey.shots, survey.ricks, survey.data, batched=False, edge_zero=False)
    finally:
        pool.close()
    assert rel_l2(got, reference) < 1e-6
    assert rel_l2(again, reference) < 1e-6


def test_batch_pairing_by_kind_same_bits(survey, swd):
    """Batched launches with the backward phases paired by kind (default) and with the
    reference's pairing stack to the same image bit for bit."""
    a = survey.batched(3)
    survey.E.set_option(swd.OPT_BWD_BY_KIND, 0)
    try:
        b = survey.batched(3)
    finally:
        survey.E.set_option(swd.OPT_BWD_BY_KIND, 1)
    assert np.array_equal(a, b)
