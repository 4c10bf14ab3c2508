"""The binomial checkpointing schedule of tw_adjoint_gradient_revolve (host logic, no GPU).

tw_revolve_plan builds the schedule and replays it on state labels: every adjoint step n must
meet the forward states n and n + 1, the final state must be announced once before the first
adjoint step, and the adjoint steps must run from nt - 1 down to 0 exactly once each. Its
forward-step count must be minimal (nt) with a slot per step, quadratic with one slot (every
state recomputed from the start), never above the binomial bound (repetition number + 1) x nt
with two slots or more, and must not grow as slots are added.
"""
from math import comb

import pytest

from cases import load_twave


def repetitions(n, c):
    """The smallest t with C(c + t, c) >= n (c >= 1 free slots)."""
    t = 0
    while comb(c + t, c) < n:
        t += 1
    return t


@pytest.mark.parametrize("nt", [1, 2, 3, 7, 50, 333, 2000])
def test_schedule_is_valid_and_within_the_binomial_bound(nt):
    tw = load_twave()
    prev = None
    for slots in (1, 2, 3, 4, 6, 10, 40, nt):
        f, n = tw.revolve_plan(nt, slots)
        assert n > 0
        if slots >= nt:
            assert f == nt                                   # one slot per step: no recomputation
        c = min(slots, nt) - 1
        if c == 0:
            assert f == nt * (nt + 1) // 2                   # recompute from the start for every step
        else:
            assert f <= (repetitions(nt, c) + 1) * nt, (slots, f)
        if prev is not None:
            assert f <= prev                                 # more memory never costs more steps
        prev = f


def test_schedule_rejects_bad_arguments():
    tw = load_twave()
    with pytest.raises(tw.TwError):
        tw.revolve_plan(0, 3)
    with pytest.raises(tw.TwError):
        tw.revolve_plan(10, 0)
