"""Exhaustive device check of the arithmetic replacement the scene kernels' random number
generator uses in place of conversion and division instructions: the integer-to-float conversion
and the correctly rounded quotients for every state of every lane."""
import pytest

pytestmark = pytest.mark.gpu


def test_rng_quotients_match_ieee_division_for_all_states(gpu_ctx):
    assert gpu_ctx.selftest(0) == 0
