"""The serving loop's scheduling on the host, with a stand-in for the device context: admission in
arrival order within the HBM budget, continuous batching (a request that arrives while others
render joins once memory frees up), per-job frame steps, and the two stopping rules (fixed spp,
relative noise of the mean luminance). No GPU: the stand-in records what the loop asks of it."""
import numpy as np
import pytest

from snelly_b200 import serving


class FakeScene:
    def __init__(self, width, height):
        self.width, self.height = width, height


class FakeContext:
    def __init__(self, luminance=None):
        self.next_id = 1
        self.live = {}           # job id -> frames advanced
        self.max_live = 0
        self.ticks = []          # the {job: frames} of every advance_batch call
        self.destroyed = []
        self.luminance = luminance or (lambda jid, frame: 1.0)

    def new_job(self, snelly):
        jid = self.next_id
        self.next_id += 1
        self.live[jid] = 0
        self.max_live = max(self.max_live, len(self.live))
        return jid

    def advance_batch(self, step):
        assert set(step) <= set(self.live)
        self.ticks.append(dict(step))
        for jid, n in step.items():
            self.live[jid] += n

    def sync(self):
        pass

    def image_stats(self, jid):
        # running mean luminance after the job's frames so far, summed over its pixels
        frames = self.live[jid]
        mean = np.mean([self.luminance(jid, f) for f in range(frames)])
        return [0.0, mean * self.npx[jid], 0.0, 0.0, float(frames)]

    def destroy_job(self, jid):
        self.destroyed.append(jid)
        del self.live[jid]


class FakeSnelly:
    ctx = None

    def __init__(self, scene, context):
        self.width, self.height = scene.width, scene.height
        self.ctx = context
        self.seed = 1
        self._jid = None

    def render(self, frames):
        assert frames == 0
        self._jid = self.ctx.new_job(self)
        self.ctx.npx = getattr(self.ctx, "npx", {})
        self.ctx.npx[self._jid] = self.width * self.height

    def job_id(self):
        return self._jid

    def readback(self):
        return np.zeros((self.height, self.width, 4), np.float32)


class FakeClock:
    """Advances by `dt` seconds on every reading, so the loop sees time pass between ticks."""

    def __init__(self, dt=0.01):
        self.t, self.dt = 0.0, dt

    def __call__(self):
        self.t += self.dt
        return self.t


@pytest.fixture
def fake_api(monkeypatch):
    monkeypatch.setattr(serving.api, "Snelly", FakeSnelly)


def _req(rid, arrival, w=64, h=64, spp=8, noise=0.0, max_spp=1024):
    return serving.Request(rid, arrival, FakeScene(w, h), target_spp=spp, noise_target=noise, max_spp=max_spp)


def test_admission_stays_within_the_budget_and_keeps_arrival_order(fake_api):
    """Three equal requests at t = 0 with room for two: two run at once, the third is admitted
    when the first one leaves, and admission follows arrival order."""
    ctx = FakeContext()
    reqs = [_req(k, 0.0, spp=8) for k in range(3)]
    srv = serving.Server(ctx, hbm_budget_bytes=2 * serving.Server.job_bytes(reqs[0]), frames_per_tick=4)
    done, samples, elapsed = srv.run(reqs, clock=FakeClock())
    assert ctx.max_live == 2
    by_id = {r.rid: r for r in done}
    assert sorted(by_id) == [0, 1, 2]
    assert by_id[0].admitted <= by_id[1].admitted < by_id[2].admitted
    assert by_id[2].admitted >= min(by_id[0].finished, by_id[1].finished)
    assert all(r.spp == 8 for r in done)
    assert samples == 3 * 64 * 64 * 8
    assert not ctx.live and sorted(ctx.destroyed) == [1, 2, 3]


def test_fixed_spp_jobs_advance_by_the_tick_and_stop_at_their_target(fake_api):
    """A fixed-spp job advances by frames_per_tick frames per tick and by what is left on its last
    tick, so it stops at exactly its target; jobs of different targets share the ticks."""
    ctx = FakeContext()
    reqs = [_req(0, 0.0, spp=10), _req(1, 0.0, spp=3)]
    srv = serving.Server(ctx, hbm_budget_bytes=10 * serving.Server.job_bytes(reqs[0]), frames_per_tick=4)
    done, _, _ = srv.run(reqs, clock=FakeClock())
    assert [t for t in ctx.ticks] == [{1: 4, 2: 3}, {1: 4}, {1: 2}]
    assert {r.rid: r.spp for r in done} == {0: 10, 1: 3}


def test_a_request_arriving_later_joins_the_running_batch(fake_api):
    """Continuous batching: a request that arrives while another job renders is admitted on a
    later tick and advanced in the same batched calls as the running job."""
    ctx = FakeContext()
    reqs = [_req(0, 0.0, spp=40), _req(1, 0.05, spp=4)]
    srv = serving.Server(ctx, hbm_budget_bytes=10 * serving.Server.job_bytes(reqs[0]), frames_per_tick=4)
    done, _, _ = srv.run(reqs, clock=FakeClock(dt=0.01))
    shared = [t for t in ctx.ticks if len(t) == 2]
    assert shared, ctx.ticks
    by_id = {r.rid: r for r in done}
    assert by_id[1].admitted > 0.05 and by_id[1].finished < by_id[0].finished


def test_noise_target_stops_once_the_mean_is_steady(fake_api):
    """A noise-target job advances one frame per tick and stops once the relative standard error
    of its mean luminance, estimated from at least 4 frames, is at or below the target: with a
    constant luminance after 4 frames; with alternating frame means (0.5, 1.5, ...) later."""
    ctx = FakeContext(luminance=lambda jid, f: 1.0 if jid == 1 else (0.5 if f % 2 == 0 else 1.5))
    reqs = [_req(0, 0.0, spp=0, noise=0.02), _req(1, 0.0, spp=0, noise=0.02)]
    srv = serving.Server(ctx, hbm_budget_bytes=10 * serving.Server.job_bytes(reqs[0]))
    done, _, _ = srv.run(reqs, clock=FakeClock())
    assert all(set(t.values()) == {1} for t in ctx.ticks)
    by_id = {r.rid: r for r in done}
    assert by_id[0].spp == 4 and by_id[0].noise == 0.0
    # frame means of +-0.5 around 1: the standard error 0.5 / sqrt(k) reaches 2% at k ~ 625
    assert 600 <= by_id[1].spp <= 700 and by_id[1].noise <= 0.02


def test_noise_target_job_stops_at_its_spp_cap(fake_api):
    ctx = FakeContext(luminance=lambda jid, f: 0.5 if f % 2 == 0 else 1.5)
    done, _, _ = serving.Server(ctx, 1 << 40).run([_req(0, 0.0, spp=0, noise=1e-6, max_spp=12)], clock=FakeClock())
    assert done[0].spp == 12


def test_a_request_larger_than_the_budget_is_refused(fake_api):
    ctx = FakeContext()
    req = _req(0, 0.0, w=256, h=256)
    with pytest.raises(RuntimeError, match="more memory than the whole budget"):
        serving.Server(ctx, serving.Server.job_bytes(req) - 1).run([req], clock=FakeClock())
