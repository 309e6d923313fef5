"""The continuous-batching server: requests arriving while others render are admitted within the
HBM budget, all finish, and every result equals the same request rendered alone."""
import numpy as np
import pytest

from helpers import gpu_render
from snelly_b200 import api, serving

pytestmark = pytest.mark.gpu


def test_server_results_equal_solo_renders(gpu_ctx):
    reqs = serving.serving_requests(rate=40.0, duration=0.5, seed=9, spp_range=(2, 5), res_range=(24, 72),
                                    scene_names=("c0", "c1", "hooks"))
    assert len(reqs) >= 8
    budget = 3 * max(serving.Server.job_bytes(r) for r in reqs)  # forces queueing for memory
    srv = serving.Server(gpu_ctx, budget, keep_images=True)
    srv.warm(reqs)
    done, samples, elapsed = srv.run(reqs)
    assert sorted(r.rid for r in done) == [r.rid for r in reqs]
    assert all(r.finished >= r.admitted >= r.arrival - 1e-3 for r in done)
    by_id = {r.rid: r for r in reqs}
    for res in done:
        req = by_id[res.rid]
        assert res.spp >= 4 if req.noise_target else res.spp == req.target_spp
        alone = gpu_render(gpu_ctx, req.scene, res.spp, seed=req.seed)[1]
        np.testing.assert_array_equal(res.image, alone)


def test_image_stats_match_readback(gpu_ctx):
    s, img = gpu_render(gpu_ctx, __import__("snelly_b200").scenes.PlainSphere(50, 30), 5)
    st = gpu_ctx.image_stats(s.job_id())
    m = img.reshape(-1, 4).astype(np.float64)
    assert abs(st[1] - m[:, 1].sum()) <= 1e-5 * abs(m[:, 1].sum())
    assert st[4] == 5 * 50 * 30
