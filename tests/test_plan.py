"""Spin-blocked plan (oracle/blockcc.py) vs dense spin-orbital oracle (no spin integration)."""
import numpy as np
import pytest

from ccq_b200 import integrals as I
from oracle.blockcc import BlockCC
from oracle.densecc import DenseCC
from tests.helpers import random_system, random_t

CASES = [('CCSD', False, 5, 2, 2), ('CCSD', True, 5, 2, 2), ('CCSD', False, 5, 3, 2),
         ('CCSDT', False, 5, 2, 2), ('CCSDT', True, 5, 2, 2), ('CCSDT', False, 5, 3, 2),
         ('CCSDTQ', False, 4, 2, 2)]


@pytest.mark.parametrize('method,rhf,n,oa,ob', CASES)
def test_sweeps_match_dense(method, rhf, n, oa, ob, plan_text):
    s = random_system(n, oa, ob, seed=5)
    txt = plan_text(method, rhf)
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method, rhf=rhf, shift=0.1)
    bc = BlockCC(txt, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method, shift=0.1)
    nmax = {'CCSD': 2, 'CCSDT': 3, 'CCSDTQ': 4}[method]
    t0, t4 = random_t(s['dims'], seed=9, scale=0.03, nmax=nmax)
    t1, t2 = t0.copy(), t0.copy()
    for b, v in t4.items():
        dc.t4[b] = v.copy()
        bc.buf[b][...] = v
    for _ in range(2):
        dc.update(t1)
        bc.update(t2)
    np.testing.assert_allclose(t2, t1, atol=1e-13, rtol=0)
    for b in t4:
        np.testing.assert_allclose(bc.buf[b], dc.t4[b], atol=1e-13, rtol=0)
    assert abs(dc.energy(t1) - bc.energy(t2)) < 1e-13


@pytest.mark.parametrize('method', ['CCSD', 'CCSDT'])
def test_rhf_plan_converges_to_uhf_energy(method, plan_text):
    s = random_system(6, 2, 2, seed=21)
    out = []
    for rhf in (False, True):
        bc = BlockCC(plan_text(method, rhf), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method)
        e, it, failed, _, _ = bc.solve(tol=1e-11, max_iter=100)
        assert not failed
        out.append(e)
    assert abs(out[0] - out[1]) < 1e-10
