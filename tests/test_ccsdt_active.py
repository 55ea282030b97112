"""Active-space CCSDt on the CPU oracle: the limits pin the mask.

With every occupied and virtual orbital active the triples are unrestricted and
CCSDt is CCSDT (same iterations, same energy); with no active occupied orbital
(closed shell) every triple is zero and CCSDt is CCSD.  In between, the converged triples
vanish outside the active space and the energy lies between the two.
"""
import numpy as np
import pytest

from ccq_b200 import config, integrals as I
from oracle.densecc import DenseCC, active_mask
from tests.helpers import random_system


def _solve(s, method, active=None):
    cc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method, active=active)
    e, it, failed, hist, tvec = cc.solve(tol=1e-11, max_iter=200)
    assert not failed
    return e, it, tvec


@pytest.mark.parametrize('n,oa,ob,froz', [(6, 3, 3, 0), (7, 3, 2, 0), (7, 3, 3, 1)])
def test_ccsdt_limits(n, oa, ob, froz):
    s = random_system(n, oa, ob, seed=23, sigma=0.08, froz=froz)
    d = s['dims']
    e_t, it_t, tv_t = _solve(s, 'CCSDT')
    e_full, it_full, _ = _solve(s, 'CCSDT', active=(froz, n))
    assert it_full == it_t and abs(e_full - e_t) < 1e-13
    e_sd, it_sd, _ = _solve(s, 'CCSD')
    lay = I.TLayout(d)
    if oa == ob:
        # no active occupied orbital (for open shells the alpha orbitals above occ_b stay active,
        # as with ccq's act_occ_b <= occ_b)
        e_none, _, tv = _solve(s, 'CCSDT', active=(d.occ_b, n))
        assert abs(e_none - e_sd) < 1e-11
        for b in ('T3A', 'T3B', 'T3C', 'T3D'):
            assert not np.any(lay.view(tv, b))
    # one active occupied and two active virtual spatial orbitals
    act = (d.occ_b - 1, d.occ_a + 2)
    e_act, _, tv = _solve(s, 'CCSDT', active=act)
    for b in ('T3A', 'T3B', 'T3C', 'T3D'):
        v = lay.view(tv, b)
        assert not np.any(v[~active_mask(b, v.shape, d, act)])
        assert np.any(v) or not np.any(lay.view(tv_t, b))
    assert min(e_sd, e_t) - 1e-12 <= e_act <= max(e_sd, e_t) + 1e-12 or abs(e_act - e_t) < abs(e_sd - e_t)


def test_ccsdt_input_keys():
    cfg = config.parse_lines(['nel=8', 'nvirt=12', 'calc_type=CCSDt', 'act_occ=1', 'act_unocc=3']).calc_macros()
    # process_sys_data: act_occ_b = max(occ_b - act_occ, froz), act_unocc_a = min(occ_a + act_unocc, orbs)
    assert (cfg.act_occ_b, cfg.act_unocc_a, cfg.lvl_t) == (3, 7, True)
    with pytest.raises(ValueError, match='active space'):
        config.parse_lines(['nel=8', 'nvirt=12', 'calc_type=CCSDt']).calc_macros()
