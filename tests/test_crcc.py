"""CR-CC(2,3): the derived equations, the reference restatement and the plan (CPU).

ExactCRCC (determinant space: Hbar applied to Fock-space vectors, the left
equations solved by dense algebra, Hbar diagonals from quasiparticle
expectation values) pins DenseCRCC (the reference's algorithm on dense
spin-orbital tensors with the equations of ccq_b200.eqgen.lagrange).  The
numpy executor of the committed CR-CC(2,3) plan must then reproduce DenseCRCC
iteration by iteration (left energies, lambda) and in the four corrections.
"""
import os

import numpy as np
import pytest

from ccq_b200 import synth
from ccq_b200.eqgen import lagrange
from oracle.blockcc import BlockCRCC
from oracle.crcc import DenseCRCC, ExactCRCC
from oracle.densecc import DenseCC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _system(norb, nel, seed=7, sigma=0.1):
    return synth.system(synth.SynthSpec(norb, nel, 2 * norb, sigma, seed))


def _ccsd(s, tol=1e-12):
    cc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], 'CCSD')
    e, it, failed, hist, tvec = cc.solve(tol=tol, max_iter=200)
    assert not failed
    return cc, e, tvec


def test_term_counts_are_stable():
    # the generated left residual, moment and left-projection term lists
    assert len(lagrange.left_residual_terms(1)) == 45
    assert len(lagrange.left_residual_terms(2)) == 69
    assert len(lagrange.triples_moment_terms()) == 81
    assert len(lagrange.triples_left_terms()) == 36


def test_dense_restatement_matches_determinant_space():
    """Hbar diagonals, lambda, M3, l3, D_D and the four energies from first principles."""
    s = _system(5, 4)
    cc, e, tvec = _ccsd(s)
    dc = DenseCRCC(cc, tvec, e, bbb_quirk=False)
    ex = ExactCRCC(dc.so.h, dc.so.v, dc.so.O, dc.t1, dc.t2).solve()
    for nm in ('h1o', 'h1v', 'h2vo'):
        np.testing.assert_allclose(getattr(dc, nm), getattr(ex, nm), atol=1e-12, rtol=0)
    off = ~np.eye(dc.so.O, dtype=bool)
    np.testing.assert_allclose(dc.h2oo[off], ex.h2oo[off], atol=1e-12, rtol=0)
    off = ~np.eye(dc.so.V, dtype=bool)
    np.testing.assert_allclose(dc.h2vv[off], ex.h2vv[off], atol=1e-12, rtol=0)
    _, it, failed, _ = dc.solve_left(tol=1e-12, max_iter=300)
    assert not failed
    np.testing.assert_allclose(dc.l1, ex.l1, atol=1e-11, rtol=0)
    np.testing.assert_allclose(dc.l2, ex.l2, atol=1e-11, rtol=0)
    e23 = dc.energies()
    for (o, v), m in ex.M3.items():
        assert abs(dc.M3[v + o] - m) < 1e-13
        assert abs(dc.L3[v + o] - ex.L3[(o, v)]) < 1e-12
        if abs(m) > 1e-12:
            assert abs(dc.denominators(o, v)[3] - ex.Dexact[(o, v)]) < 1e-12
    assert np.abs(e23).min() > 1e-6
    np.testing.assert_allclose(e23, ex.energies(np.diag(dc.so.f)), rtol=1e-10, atol=0)


@pytest.mark.parametrize('norb,nel,rhf', [(6, 6, False), (7, 6, True)])
def test_plan_executor_matches_dense_restatement(norb, nel, rhf):
    name = 'CRCC23' + ('_rhf' if rhf else '')
    text = open(os.path.join(ROOT, 'ccq_b200', 'plans', name + '.plan')).read()
    s = _system(norb, nel)
    d = s['dims']
    bc = BlockCRCC(text, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d)
    e, it, failed, hist, tvec = bc.solve(tol=1e-12, max_iter=200)
    cc, e2, tvec2 = _ccsd(s)
    assert abs(e - e2) < 1e-12
    dc = DenseCRCC(cc, tvec2, e2)
    _, itl, fl, hl = dc.solve_left(tol=1e-12, max_iter=300)
    _, itl2, fl2, hl2 = bc.solve_left(tvec, e, tol=1e-12, max_iter=300)
    assert not fl and not fl2 and itl == itl2
    np.testing.assert_allclose([h[0] for h in hl2], [h[0] for h in hl], atol=1e-12, rtol=0)
    e23 = bc.crcc23(tvec)
    np.testing.assert_allclose(e23, dc.energies(), rtol=1e-10, atol=0)


def test_plan_file_matches_generator():
    from ccq_b200.eqgen import plan as P
    text = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CRCC23.plan')).read()
    assert P.build_plan('CR-CC(2,3)').text() == text


@pytest.mark.parametrize('n,oa,ob,froz', [(7, 4, 3, 0), (8, 4, 4, 1), (8, 5, 3, 1)])
def test_open_shell_and_frozen_core_plan_matches_dense(n, oa, ob, froz):
    """Open shell (the beta-beta-beta cal_d3 bound then skips occ_a - occ_b + 1 virtuals) and frozen core."""
    from tests.helpers import random_system
    text = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CRCC23.plan')).read()
    s = random_system(n, oa, ob, seed=11, sigma=0.08, froz=froz)
    d = s['dims']
    bc = BlockCRCC(text, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d)
    e, it, failed, hist, tvec = bc.solve(tol=1e-12, max_iter=200)
    assert not failed
    cc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSD')
    e2, it2, f2, h2, tvec2 = cc.solve(tol=1e-12, max_iter=200)
    assert abs(e - e2) < 1e-12 and it == it2
    dc = DenseCRCC(cc, tvec2, e2)
    _, itl, _, hl = dc.solve_left(tol=1e-12, max_iter=300)
    _, itl2, _, hl2 = bc.solve_left(tvec, e, tol=1e-12, max_iter=300)
    assert itl == itl2
    np.testing.assert_allclose([h[0] for h in hl2], [h[0] for h in hl], atol=1e-12, rtol=0)
    np.testing.assert_allclose(bc.crcc23(tvec), dc.energies(), rtol=1e-10, atol=1e-16)
