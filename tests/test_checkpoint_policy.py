"""The GlideStep checkpointing policy's arithmetic, on the CPU: the interval
picked for a memory budget, and argument errors."""
from __future__ import annotations

import math

import pytest


def test_interval_fits_the_budget_and_is_the_smallest():
    from glide_b200.torch import Checkpointing
    state = 168e6  # u, v, H, mask, phi of a 2048^2 binary64 level
    for n_steps, budget in ((20, 20 * state), (20, 10 * state), (100, 25 * state), (1000, 70 * state)):
        k = Checkpointing.interval_for(budget, n_steps, state)
        assert (math.ceil(n_steps / k) + k) * state <= budget
        if k > 1:
            assert (math.ceil(n_steps / (k - 1)) + k - 1) * state > budget
    # keep-all fits when the budget holds every state and one more
    assert Checkpointing.interval_for(21 * state, 20, state) == 1
    # at best 2 sqrt(n) states
    with pytest.raises(ValueError):
        Checkpointing.interval_for(8 * state, 20, state)


def test_policy_arguments():
    from glide_b200.torch import Checkpointing, checkpointing
    with pytest.raises(ValueError):
        Checkpointing(0)

    class Model:
        pass
    m = Model()
    assert checkpointing(m).every == 1
    assert checkpointing(m, every=4).every == 4
    assert m._glide_checkpointing.every == 4
    with pytest.raises(ValueError):
        checkpointing(m, max_bytes=1e9)
