"""GPU solver against the plan-independent dense oracle on mid-size open-shell systems.

The fixtures (tests/golden/make_dense.py) come from oracle/densecc.py, which
evaluates the generated equations on dense spin-orbital tensors: no spin
integration and no contraction plan, so these checks do not share the plan
text the GPU executes.  The systems have three or more alpha holes (the
alpha-alpha-alpha and beta-beta-beta triples are not empty, unlike the H4
fixture's), one has a frozen core, one is rhf, and the CCSDTQ one has
non-empty T4B, T4C and T4D blocks.
"""
import json
import os

import numpy as np
import pytest

from ccq_b200 import config, driver, integrals as I, lib
from oracle.densecc import DenseCC
from tests.conftest import GOLDEN
from tests.helpers import random_system, random_t

pytestmark = pytest.mark.gpu

CASES = ['ccsdt_open_n10', 'ccsdt_froz_n10', 'ccsdt_rhf_n10', 'ccsdtq_open_n7']


def _fixture(name):
    p = os.path.join(GOLDEN, 'dense_midsize.json')
    if not os.path.exists(p):
        pytest.skip('dense_midsize.json not generated')
    data = json.load(open(p))
    if name not in data:
        pytest.skip(f'{name} not in dense_midsize.json')
    return data[name]


def _ctx(s, method, rhf=False, shift=0.0):
    d = s['dims']
    return lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, method, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                       s['v_bb'], rhf=rhf, shift=shift, diis_space=5)


@pytest.mark.parametrize('name', CASES)
def test_converged_solve_matches_dense_oracle(name):
    g = _fixture(name)
    s = random_system(g['n'], g['occ_a'], g['occ_b'], seed=g['seed'], sigma=g['sigma'], froz=g['froz'])
    ctx = _ctx(s, g['method'], rhf=g['rhf'], shift=g['shift'])
    cfg = config.Config(calc_type=g['method'], tol=g['tol'], diis_space=5, rhf=g['rhf'], max_iter=100).calc_macros()
    r = driver.solve_cc(ctx, cfg, out=lambda x: None)
    ctx.close()
    assert not r.failed
    assert abs(r.e_cor - g['e_cor']) < 1e-10
    # the same algorithm (block order, DIIS schedule, convergence rule): the same iteration count,
    # and the energies of the early iterations agree to round-off
    assert r.iterations == g['iterations']
    for k, h in enumerate(r.history[:5]):
        assert abs(h['e'] - g['history'][k]) < 1e-11, k


@pytest.mark.parametrize('rhf,froz', [(False, 0), (False, 1), (True, 0)])
def test_ccsdt_sweep_matches_dense_oracle(rhf, froz):
    """One CCSDT sweep from random amplitudes, every block to 1e-12."""
    s = random_system(10, 4, 4 if (rhf or froz) else 3, seed=41, sigma=0.08, froz=froz)
    ctx = _ctx(s, 'CCSDT', rhf=rhf, shift=0.05)
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], 'CCSDT', shift=0.05, rhf=rhf)
    t, _ = random_t(s['dims'], seed=6, scale=0.03, nmax=3)
    if rhf:
        # closed-shell amplitudes: beta blocks are the rhf copies of the alpha ones
        from oracle import solver as S
        lay = I.TLayout(s['dims'])
        lay.view(t, 'T1B')[...] = lay.view(t, 'T1A')
        lay.view(t, 'T2C')[...] = lay.view(t, 'T2A')
        lay.view(t, 'T3D')[...] = lay.view(t, 'T3A')
        lay.view(t, 'T3C')[...] = S.tran3bto3c(lay.view(t, 'T3B'))
    ctx.set_t(t)
    ctx.update()
    tg = ctx.get_t()
    e_gpu = ctx.energy()
    ctx.close()
    tc = t.copy()
    dc.update(tc)
    lay = I.TLayout(s['dims'])
    for b in I.T_VEC_ORDER:
        np.testing.assert_allclose(lay.view(tg, b), lay.view(tc, b), atol=1e-12, rtol=0, err_msg=b)
    assert abs(e_gpu - dc.energy(tc)) < 1e-12


def test_ccsdtq_sweep_matches_dense_oracle():
    """One CCSDTQ sweep (7 orbitals, 4 alpha / 3 beta holes) against the dense oracle's stored sweep."""
    p = os.path.join(GOLDEN, 'dense_sweep_ccsdtq.npz')
    if not os.path.exists(p):
        pytest.skip('dense_sweep_ccsdtq.npz not generated')
    f = np.load(p)
    s = random_system(7, 4, 3, seed=35, sigma=0.08)
    ctx = _ctx(s, 'CCSDTQ', shift=0.05)
    ctx.set_t(f['t_in'])
    lay = I.TLayout(s['dims'])
    t4 = [b for b in lay.t4_shape if b + '_in' in f.files and f[b + '_in'].size]
    for b in t4:
        ctx.set_block(b, f[b + '_in'])
    ctx.update()
    tg = ctx.get_t()
    for b in I.T_VEC_ORDER:
        np.testing.assert_allclose(lay.view(tg, b), lay.view(f['t_out'], b), atol=1e-12, rtol=0, err_msg=b)
    for b in t4:
        out = f[b + '_out']
        np.testing.assert_allclose(ctx.get_block(b, out.shape), out, atol=1e-12, rtol=0, err_msg=b)
    assert abs(ctx.energy() - float(f['energy'])) < 1e-12
    ctx.close()
