"""The Ferret session's data flow (cuot_b200/ferret.py) replayed on the
oracle: the checker for the GPU session tests, and a CPU test of the flow
itself."""
import numpy as np

import oracle
from cuot_b200.ferret import CONSIST_CHECK_COT_NUM, PrimalLPNParameter, session_key

SMALL = PrimalLPNParameter(n=32 << 9, t=32, k=1000, h=9, n_pre=8 << 8, t_pre=8, k_pre=500, h_pre=8)


def oracle_session(p, seed, extensions):
    """The session's data flow restated on the oracle; returns the output
    buffers (v, w) of the last extension."""
    key = session_key(seed)
    scalar = lambda i: oracle.prg(key, 1, offset=i)[0]
    delta = scalar(0).copy()
    delta[0] |= 1
    c = CONSIST_CHECK_COT_NUM
    nb = p.t_pre * p.h_pre + p.k_pre + c
    v = oracle.prg(scalar(1), nb)
    x = oracle.prg(scalar(2), nb)
    v[:, 0] &= 0xFE
    w = np.where((x[:, :1] & 1).astype(bool), v ^ delta, v)

    def extend(idx, t, h, k, mp_r, kk_s, kk_r):
        roots = oracle.prg(scalar(17 + 2 * idx), t)
        lv, ls, rs, ss = oracle.ferret_pprf_sender(roots, h, delta, threads=4)
        ch = (mp_r[:, 0] & 1).astype(np.uint8)
        mc = np.where(ch[:, None].astype(bool), rs, ls)
        rl = oracle.ferret_pprf_recver(mc, ch, ss, h, threads=4)
        sd = scalar(16 + 2 * idx)
        return oracle.lpn_primal(sd, kk_s, lv, threads=4), oracle.lpn_primal(sd, kk_r, rl, threads=4)

    m = p.t_pre * p.h_pre
    os_, or_ = extend(0, p.t_pre, p.h_pre, p.k_pre, w[:m], v[m + c:m + c + p.k_pre], w[m + c:m + c + p.k_pre])
    pre_s, pre_r = os_[:p.M], or_[:p.M]
    th = p.t * p.h
    for i in range(1, extensions):
        os_, or_ = extend(i, p.t, p.h, p.k, pre_r[:th], pre_s[c:c + p.k], pre_r[c:c + p.k])
        pre_s, pre_r = os_[p.ot_limit:], or_[p.ot_limit:]
    return os_, or_


def session_delta(seed) -> np.ndarray:
    d = oracle.prg(session_key(seed), 1, offset=0)[0].copy()
    d[0] |= 1
    return d


def check_cot(v, w, delta):
    assert not (v[:, 0] & 1).any()
    x = (w[:, 0] & 1).astype(bool)
    diff = v ^ w
    assert not diff[~x].any()
    assert (diff[x] == delta).all()
    return x
