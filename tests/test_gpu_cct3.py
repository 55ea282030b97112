"""CC(t;3) on the GPU: a CCSDt solve (CCSDT context with the active space),
then a CR-CC(2,3) context holding its T1 and T2 with the same active space:
the left CCSD solve takes the iterations of the numpy executor, and the four
corrections over the triples outside the active space equal the executor's
from the device's T and lambda.  The input deck path lands on the two limits
(full active space: CCSDT, no correction; empty: CR-CC(2,3)) and on the dense
restatement for a partial active space."""
import os

import numpy as np
import pytest

from ccq_b200 import config, driver, integrals as I, lib
from oracle.blockcc import BlockCRCC
from oracle.crcc import DenseCRCC
from oracle.densecc import DenseCC
from tests.helpers import random_system

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ctx(s, ctype, rhf=False):
    d = s['dims']
    return lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, ctype, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'],
                       rhf=rhf)


@pytest.mark.parametrize('n,oa,ob,froz,act', [(8, 4, 4, 0, (3, 6)), (9, 4, 3, 1, (2, 7))])
def test_cct3_matches_plan_executor(n, oa, ob, froz, act):
    s = random_system(n, oa, ob, seed=23, sigma=0.08, froz=froz)
    d = s['dims']
    cfg = config.Config(calc_type='CCSDT', tol=1e-11, max_iter=200).calc_macros()
    ctx = _ctx(s, 'CCSDT')
    try:
        ctx.set_active(*act)
        r = driver.solve_cc(ctx, cfg, out=lambda x: None)
        t = ctx.get_t()
    finally:
        ctx.close()
    assert not r.failed
    cr = _ctx(s, 'CR-CC(2,3)')
    try:
        cr.set_active(*act)
        t12 = t[:cr.t_size]
        cr.set_t(t12)
        left = driver.solve_lcc(cr, cfg, r.e_cor, out=lambda x: None)
        e23 = cr.crcc23()
        text = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CRCC23.plan')).read()
        bc = BlockCRCC(text, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, active=act)
        _, itl, fl, hl = bc.solve_left(t12, r.e_cor, tol=cfg.tol, max_iter=cfg.max_iter)
        assert not left.failed and not fl and left.iterations == itl
        np.testing.assert_allclose([h['e'] for h in left.history], [h[0] for h in hl], atol=1e-10, rtol=0)
        bc.lvec[:cr.vec_size] = cr.get_l()
        ref = bc.crcc23(t12)
        assert np.all(np.abs(e23) > 1e-7)
        np.testing.assert_allclose(e23, ref, rtol=1e-11, atol=0)
        # without the active space the sums run over every triple
        bc.active = None
        assert np.all(np.abs(bc.crcc23(t12) - e23) > 1e-9)
    finally:
        cr.close()


def _deck(tmp_path, ints, nel, nvirt, body):
    tmp_path.mkdir(parents=True, exist_ok=True)
    I.write_onebody(str(tmp_path / 'onebody.inp'), ints['e1'])
    I.write_twobody(str(tmp_path / 'twobody.inp'), ints['e2'], ints['enuc'])
    (tmp_path / 'in.inp').write_text(f'nel={nel}\nnvirt={nvirt}\ntol=1.0e-11\nmax_iterations=200\n'
                                     'keep_bin=.false.\n' + body)
    lines = []
    r = driver.run(str(tmp_path / 'in.inp'), out=lines.append, base_dir=str(tmp_path))
    assert not r.failed
    return r, lines


def _random_ints():
    s = random_system(7, 3, 3, seed=31, sigma=0.08)
    return s, dict(e1=s['h'], e2=s['e2'], enuc=0.0)


def test_h4_known_answer(tmp_path, h4):
    """H4 (no triples contribute: CCSD = CCSDT there) through calc_type=CCT3 with the whole space active."""
    r, lines = _deck(tmp_path, h4, 4, 4, 'calc_type=CCT3\nact_occ=2\nact_unocc=2\n')
    assert np.all(r.e23 == 0.0)
    # known answer of the reference's tests/test_small.py for CCSDT on this system
    assert abs(r.e_total - (-1.978696408825)) < 1e-9
    assert any(l.strip().startswith('CC(t;3),A') for l in lines)


def test_limits_through_the_input_deck(tmp_path):
    s, ints = _random_ints()
    full, _ = _deck(tmp_path / 'full', ints, 6, 8, 'calc_type=CC(t;3)\nact_occ=3\nact_unocc=4\n')
    ccsdt, _ = _deck(tmp_path / 'ccsdt', ints, 6, 8, 'calc_type=CCSDT\n')
    assert np.all(full.e23 == 0.0)
    assert full.iterations == ccsdt.iterations and abs(full.e_total - ccsdt.e_total) < 1e-12
    empty, _ = _deck(tmp_path / 'empty', ints, 6, 8, 'calc_type=CC(t;3)\nact_occ=0\nact_unocc=0\n')
    crcc, _ = _deck(tmp_path / 'crcc', ints, 6, 8, 'calc_type=CR-CC(2,3)\n')
    assert np.all(np.abs(crcc.e23) > 1e-7)
    np.testing.assert_allclose(empty.e23, crcc.e23, rtol=1e-8, atol=0)
    assert abs(empty.e_total - crcc.e_total) < 1e-11


def test_partial_active_space_matches_dense(tmp_path):
    s, ints = _random_ints()
    r, _ = _deck(tmp_path, ints, 6, 8, 'calc_type=CCt3\nact_occ=1\nact_unocc=2\n')
    act = (2, 5)
    d = s['dims']
    cc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDT', active=act)
    e, it, failed, _, tvec = cc.solve(tol=1e-11, max_iter=200, compressed_diis=True)
    dc = DenseCRCC(cc, tvec, e)
    dc.solve_left(tol=1e-11, max_iter=200)
    ref = dc.energies(active=act)
    assert abs(r.e_ccsdt - e) < 1e-10 and r.iterations == it
    assert np.all(np.abs(ref) > 1e-7)
    np.testing.assert_allclose(r.e23, ref, rtol=1e-7, atol=0)
    assert abs(r.e_cor - (e + ref[3])) < 1e-10
