"""snelly_image_stats_static, the image statistics entry point that allocates nothing, called
through the C ABI and compared with snelly_image_stats. Collected last so it also runs after every
other test has used the device; it passes alone as well."""
import ctypes

import numpy as np
import pytest

from snelly_b200 import _native as N
from snelly_b200 import api, scenes

pytestmark = pytest.mark.gpu
EINVAL = -1  # SNELLY_EINVAL


def _static_stats(ctx, jid):
    out = (ctypes.c_double * 5)()
    rc = N.lib().snelly_image_stats_static(ctx.handle, ctypes.c_uint64(jid), out)
    return rc, np.array(out[:])


def test_static_stats_match_allocating_entry_point_twice(gpu_ctx):
    """Two calls in a row (the second one after the completion counter was reset) agree with
    snelly_image_stats within 1e-12 relative; the sums differ only in summation order."""
    s = api.Snelly(scenes.DispersiveFractal(320, 180), context=gpu_ctx)
    s.render(3)
    jid = s.job_id()
    ref = np.array(gpu_ctx.image_stats(jid), np.float64)
    for _ in range(2):
        rc, got = _static_stats(gpu_ctx, jid)
        assert rc == N.SNELLY_OK, N.lib().snelly_last_error()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)
        assert got[4] == 320 * 180 * 3
    s.render(1)  # more frames change the image; the next call sees them
    ref2 = np.array(gpu_ctx.image_stats(jid), np.float64)
    rc, got2 = _static_stats(gpu_ctx, jid)
    assert rc == N.SNELLY_OK
    np.testing.assert_allclose(got2, ref2, rtol=1e-12, atol=0)
    gpu_ctx.destroy_job(jid)


def test_static_stats_reject_jobs_beyond_the_scratch(gpu_ctx):
    """A job of more than 4096 x 2048 pixels is refused with SNELLY_EINVAL and a message naming the
    limit (checked before any device work)."""
    s = api.Snelly(scenes.PlainSphere(2900, 2900), context=gpu_ctx)
    s.render(0)
    rc, _ = _static_stats(gpu_ctx, s.job_id())
    assert rc == EINVAL
    assert b"8388608" in N.lib().snelly_last_error()
    gpu_ctx.destroy_job(s.job_id())
