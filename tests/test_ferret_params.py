"""Ferret parameter sets and the session's data flow on the oracle (CPU)."""
import numpy as np
import pytest

from cuot_b200.ferret import FERRET_B11, FERRET_B12, FERRET_B13, PrimalLPNParameter
from tests.ferret_replay import SMALL, check_cot, oracle_session, session_delta


def test_b13_limits():
    # ot_limit = n - (k + t*h + 128) (ferret_cot.hpp:80-81)
    assert FERRET_B13.M == 452000 + 1280 * 13 + 128
    assert FERRET_B13.ot_limit == 10016992 == FERRET_B13.buf_sz()
    for p in (FERRET_B11, FERRET_B12, FERRET_B13):
        assert p.n_pre >= p.M


def test_parameter_check():
    with pytest.raises(ValueError):
        PrimalLPNParameter(n=1000, t=1, k=10, h=10, n_pre=256, t_pre=1, k_pre=10, h_pre=8)
    with pytest.raises(ValueError):  # n_pre too small for one extension's M
        PrimalLPNParameter(n=1 << 12, t=4, k=1000, h=10, n_pre=256, t_pre=1, k_pre=10, h_pre=8)


def test_oracle_replay_keeps_cot_correlation():
    seed = b"ferret-session-cpu"
    v, w = oracle_session(SMALL, seed, 3)
    x = check_cot(v, w, session_delta(seed))
    assert 0.45 < x.mean() < 0.55
