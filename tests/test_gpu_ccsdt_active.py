"""Active-space CCSDt on the GPU (CCSDT plan, triples outside the active space
held at zero by the residual gather) against the CPU oracle with the same mask:
sweeps to 1e-12, converged solves with the same iteration count and energy."""
import numpy as np
import pytest

from ccq_b200 import config, driver, integrals as I, lib
from oracle.densecc import DenseCC
from tests.helpers import random_system, random_t

pytestmark = pytest.mark.gpu


def _ctx(s, act):
    d = s['dims']
    c = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDT', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'])
    c.set_active(*act)
    return c


@pytest.mark.parametrize('n,oa,ob,froz', [(6, 3, 3, 0), (7, 3, 2, 0), (8, 4, 3, 1)])
def test_ccsdt_sweeps_and_solve_match_oracle(n, oa, ob, froz):
    s = random_system(n, oa, ob, seed=29, sigma=0.08, froz=froz)
    d = s['dims']
    act = (d.occ_b - 1, d.occ_a + 2)
    # two sweeps from random amplitudes
    ctx = _ctx(s, act)
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDT', active=act)
    t, _ = random_t(d, seed=8, scale=0.03, nmax=3)
    ctx.set_t(t)
    tc = t.copy()
    for _ in range(2):
        ctx.update()
        dc.update(tc)
    np.testing.assert_allclose(ctx.get_t(), tc, atol=1e-12, rtol=0)
    ctx.close()
    # converged
    ctx = _ctx(s, act)
    cfg = config.Config(calc_type='CCSDT', tol=1e-10, max_iter=200).calc_macros()
    r = driver.solve_cc(ctx, cfg, out=lambda x: None)
    ctx.close()
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDT', active=act)
    e, it, failed, _, _ = dc.solve(tol=1e-10, max_iter=200)
    assert not r.failed and not failed
    assert r.iterations == it and abs(r.e_cor - e) < 1e-10


def test_ccsdt_input_deck(tmp_path, h4):
    I.write_onebody(str(tmp_path / 'onebody.inp'), h4['e1'])
    I.write_twobody(str(tmp_path / 'twobody.inp'), h4['e2'], h4['enuc'])
    (tmp_path / 'in.inp').write_text('nel=4\nnvirt=4\ncalc_type=CCSDt\nact_occ=1\nact_unocc=1\ntol=1.0e-11\n'
                                     'max_iterations=100\nkeep_bin=.false.\n')
    r = driver.run(str(tmp_path / 'in.inp'), out=lambda x: None, base_dir=str(tmp_path))
    dc = DenseCC(h4['f_a'], h4['f_b'], h4['v_aa'], h4['v_ab'], h4['v_bb'], h4['dims'], 'CCSDT', active=(1, 3))
    e, it, failed, _, _ = dc.solve(tol=1e-11, max_iter=100)
    assert not r.failed and r.iterations == it and abs(r.e_cor - e) < 1e-10
