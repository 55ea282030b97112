"""Symbolic CC residuals vs the equation-free determinant-space residual."""
import numpy as np
import pytest

from ccq_b200 import integrals as I
from ccq_b200.eqgen import wick
from oracle.detcc import DetCC
from oracle.spinorb import SpinOrbitalSystem
from tests.helpers import random_system, random_t


@pytest.mark.parametrize('method,n,oa,ob', [('CCSD', 4, 2, 2), ('CCSD', 4, 2, 1), ('CCSDT', 4, 2, 2),
                                            ('CCSDT', 4, 2, 1), ('CCSDTQ', 4, 2, 2)])
def test_residual_matches_exact_projection(method, n, oa, ob):
    s = random_system(n, oa, ob, seed=11)
    so = SpinOrbitalSystem(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], oa, ob)
    tranks = wick.METHOD_TRANKS[method]
    nmax = max(tranks)
    t, t4 = random_t(s['dims'], seed=3, scale=0.05, nmax=nmax)
    lay = I.TLayout(s['dims'])
    blocks = {b: lay.view(t, b) for b in I.T_VEC_ORDER if int(b[1]) <= nmax}
    blocks.update(t4)
    ts = so.from_blocks(blocks, nmax)
    dc = DetCC(so.h, so.v, so.O)
    w = dc.sim_vector(ts)
    for level in range(1, nmax + 1):
        R_exact = dc.residual(ts, level, w)
        R_gen = so.residual(ts, level, tranks)
        assert np.abs(R_exact).max() > 1e-3
        np.testing.assert_allclose(R_gen, R_exact, atol=1e-13, rtol=0)
    assert abs(dc.energy(ts) - so.energy(ts)) < 1e-14


def test_ccsd_term_structure():
    terms = wick.residual_terms(2, (2,))
    assert len(terms) == 18
    # <ab||ij> enters with coefficient 1, the vvvv ladder with 1/2
    d = {str(t): c for c, t in terms}
    assert d[str([('v', ('a0', 'a1', 'i0', 'i1'))])] == 1
    assert d[str([('v', ('a0', 'a1', 'v0', 'v1')), ('t2', ('v0', 'v1', 'i0', 'i1'))])] == wick.Fraction(1, 2)


def test_orbit_groups_reproduce_terms():
    terms = wick.residual_terms(3, (2, 3))
    groups = wick.orbit_groups(3, terms)
    assert sum(len(m) for _, m in groups) == len(terms)
    assert len(groups) < len(terms)
