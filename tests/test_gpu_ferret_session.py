"""Ferret random-COT session (cuot_b200/ferret.py): bootstrap + extension
loop with device-resident pre-COT carry-over, checked bit-exactly against the
same session replayed with the oracle, and through the COT correlation at the
ferret_b13 size."""
import numpy as np
import pytest

from tests.ferret_replay import SMALL, check_cot, oracle_session, session_delta
from tests.util import to_host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from cuot_b200.ferret import FERRET_B13, FerretSession  # noqa: E402


def test_session_matches_oracle_replay(ctx):
    seed = b"ferret-session-01"
    s = FerretSession(ctx, ctx, SMALL, seed)
    v1, w1 = s.rcot(SMALL.ot_limit + 123)   # crosses one extension boundary
    v2, w2 = s.rcot(2 * SMALL.ot_limit)     # and two more
    assert s.extensions == 5   # the bootstrap and four extensions
    exp_v, exp_w = oracle_session(SMALL, seed, 5)
    assert np.array_equal(to_host(s.ot_s), exp_v)
    assert np.array_equal(to_host(s.ot_r), exp_w)
    delta = session_delta(seed)
    x = check_cot(np.concatenate([to_host(v1), to_host(v2)]), np.concatenate([to_host(w1), to_host(w2)]), delta)
    assert 0.45 < x.mean() < 0.55
    # the last 123 served COTs are the first outputs of the last extension
    assert np.array_equal(to_host(v2)[-123:], exp_v[:123])
    assert np.array_equal(to_host(w2)[-123:], exp_w[:123])


def test_session_b13_correlation(ctx):
    """ferret_b13 parameters (n = 10,485,760, ot_limit = 10,016,992):
    bootstrap, two extensions; every served COT satisfies w = v ^ x Delta."""
    seed = b"ferret-session-b13"
    s = FerretSession(ctx, ctx, FERRET_B13, seed)
    assert FERRET_B13.ot_limit == 10016992
    v, w = s.rcot(FERRET_B13.ot_limit + 1000)
    assert s.extensions == 3
    x = check_cot(to_host(v), to_host(w), session_delta(seed))
    assert 0.49 < x.mean() < 0.51
