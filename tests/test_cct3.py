"""CC(t;3) on the CPU: CR-CC(2,3) corrections over the triples outside the
CCSDt active space (calc_type=CC(t;3), src/parser.f90:400-411;
src/mm_correct.f90:61-62 and the skips at :131, :190, :244, :300).

The dense spin-orbital restatement applies crcc23's skip literally (an
occupied spatial orbital above act_occ_b and a virtual one up to act_unocc_a);
the numpy executor of the CR-CC(2,3) plan applies it per spin block.  Both
must give the same four corrections from a CCSDt solve, and the two limits
hold: an empty active space is CR-CC(2,3) on CCSD, a full one leaves nothing
to correct.
"""
import os

import numpy as np
import pytest

from ccq_b200 import config
from oracle.blockcc import BlockCRCC
from oracle.crcc import DenseCRCC
from oracle.densecc import DenseCC
from tests.helpers import random_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _plan(rhf=False):
    return open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CRCC23' + ('_rhf' if rhf else '') + '.plan')).read()


def _ccsdt(s, act, tol=1e-12):
    d = s['dims']
    cc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDT', active=act)
    e, it, failed, hist, tvec = cc.solve(tol=tol, max_iter=200)
    assert not failed
    return cc, e, tvec


@pytest.mark.parametrize('n,oa,ob,froz,act', [(6, 3, 3, 0, (2, 4)), (8, 4, 3, 1, (2, 6)), (7, 4, 2, 0, (1, 6))])
def test_block_executor_matches_dense_skip(n, oa, ob, froz, act):
    s = random_system(n, oa, ob, seed=17, sigma=0.08, froz=froz)
    d = s['dims']
    cc, e, tvec = _ccsdt(s, act)
    dc = DenseCRCC(cc, tvec, e)
    _, itl, fl, hl = dc.solve_left(tol=1e-12, max_iter=300)
    bc = BlockCRCC(_plan(), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, active=act)
    t12 = tvec[:bc.layout.vec_size('CCSD')]
    _, itl2, fl2, hl2 = bc.solve_left(t12, e, tol=1e-12, max_iter=300)
    assert not fl and not fl2 and itl == itl2
    np.testing.assert_allclose([h[0] for h in hl2], [h[0] for h in hl], atol=1e-12, rtol=0)
    masked = dc.energies(active=act)
    np.testing.assert_allclose(bc.crcc23(t12), masked, rtol=1e-10, atol=1e-16)
    # the skip removes a real part of the correction
    full = dc.energies()
    assert np.all(np.abs(full - masked) > 1e-8)


def test_limits_of_the_active_space():
    """Closed shell: act_occ = act_unocc = 0 (act_occ_b = occ, act_unocc_a = occ) keeps every triple;
    the whole space (act_occ_b = froz, act_unocc_a = orbs) leaves none."""
    s = random_system(6, 3, 3, seed=5, sigma=0.08, froz=0)
    d = s['dims']
    cc, e, tvec = _ccsdt(s, (d.froz, d.orbs))
    dc = DenseCRCC(cc, tvec, e)
    dc.solve_left(tol=1e-12, max_iter=300)
    assert np.all(dc.energies(active=(d.froz, d.orbs)) == 0.0)
    np.testing.assert_array_equal(dc.energies(active=(d.occ_b, d.occ_a)), dc.energies())
    bc = BlockCRCC(_plan(), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, active=(d.froz, d.orbs))
    t12 = tvec[:bc.layout.vec_size('CCSD')]
    bc.solve_left(t12, e, tol=1e-12, max_iter=300)
    assert np.all(bc.crcc23(t12) == 0.0)
    # the empty active space: CCSDt is CCSD
    cc0, e0, t0 = _ccsdt(s, (d.occ_b, d.occ_a))
    ccsd = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSD')
    e1, *_ = ccsd.solve(tol=1e-12, max_iter=200)
    assert abs(e0 - e1) < 1e-12


@pytest.mark.parametrize('name', ['CCT3', 'CCt3', 'CC(t;3)'])
def test_calc_type_names_and_active_space(name):
    cfg = config.parse_lines([f'nel=6\n', 'nvirt=8\n', f'calc_type={name}\n', 'act_occ=1\n', 'act_unocc=2\n'])
    cfg.calc_macros()
    assert cfg.calc_type == 'CC(t;3)' and cfg.lvl_t and not cfg.lvl_q
    assert (cfg.act_occ_b, cfg.act_unocc_a) == (2, 5)
    bare = config.parse_lines([f'nel=6\n', 'nvirt=8\n', f'calc_type={name}\n'])
    with pytest.raises(ValueError, match='active space'):
        bare.calc_macros()
