"""Active-space CCSDt on the GPU (CCSDT plan, triples outside the active space
held at zero by the residual gather) against the CPU oracle with the same mask:
sweeps to 1e-12, converged solves with the same iteration count and energy."""
import numpy as np
import pytest

from ccq_b200 import config, driver, integrals as I, lib
from oracle.densecc import DenseCC, active_mask
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
    e, it, failed, _, _ = dc.solve(tol=1e-11, max_iter=100, compressed_diis=True)
    assert not r.failed and r.iterations == it and abs(r.e_cor - e) < 1e-10


def _ctx_restricted(s, act, rhf=False):
    d = s['dims']
    return lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDt', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'],
                       rhf=rhf, active=act)


@pytest.mark.parametrize('n,oa,ob,froz,act_d,seed', [(8, 4, 3, 0, (1, 2), 29), (8, 4, 4, 1, (1, 3), 37),
                                                      (9, 4, 3, 0, (2, 1), 29), (7, 3, 2, 0, (0, 2), 29)])
def test_restricted_ccsdt_matches_oracle(n, oa, ob, froz, act_d, seed):
    """calc_type CCSDt: the T3 residual contractions run over the active triples only, and DIIS runs over
    ccq's compressed T vector; sweeps, converged energies and iteration counts equal the dense oracle's
    with the same mask and the same DIIS vector, at a fraction of the FLOPs."""
    s = random_system(n, oa, ob, seed=seed, sigma=0.08, froz=froz)
    d = s['dims']
    act = (d.occ_b - act_d[0], d.occ_a + act_d[1])
    ctx = _ctx_restricted(s, act)
    full = _ctx(s, act)
    flops_r, flops_f = ctx.stats()['flops'], full.stats()['flops']
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDT', active=act)
    t, _ = random_t(d, seed=9, scale=0.03, nmax=3)
    lay = I.TLayout(d)
    for b in ('T3A', 'T3B', 'T3C', 'T3D'):
        v = lay.view(t, b)
        v[...] = np.where(active_mask(b, v.shape, d, act), v, 0)
    ctx.set_t(t)
    full.set_t(t)
    tc = t.copy()
    for _ in range(2):
        ctx.update()
        full.update()
        dc.update(tc)
    np.testing.assert_allclose(ctx.get_t(), tc, atol=1e-12, rtol=0)
    np.testing.assert_allclose(full.get_t(), tc, atol=1e-12, rtol=0)
    full.close()
    ctx.close()
    assert flops_r < flops_f
    ctx = _ctx_restricted(s, act)
    cfg = config.Config(calc_type='CCSDT', tol=1e-10, max_iter=200).calc_macros()
    r = driver.solve_cc(ctx, cfg, out=lambda x: None)
    assert ctx.vec_size == lib.t_size_act(d.froz, d.occ_a, d.occ_b, d.orbs, *act)
    ctx.close()
    e, it, failed, hist, _ = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDT',
                                     active=act).solve(tol=1e-10, max_iter=200, compressed_diis=True)
    assert not r.failed and not failed
    assert r.iterations == it and abs(r.e_cor - e) < 1e-10
    for k in range(min(8, it)):
        assert abs(r.history[k]['e'] - hist[k][0]) < 1e-11, k


def test_restricted_ccsdt_rhf_and_compressed_layout():
    """rhf CCSDt, and ccq's compressed T vector in and out of the context (set_t of the expanded vector)."""
    s = random_system(8, 4, 4, seed=37, sigma=0.08)
    d = s['dims']
    act = (d.occ_b - 1, d.occ_a + 2)
    ctx = _ctx_restricted(s, act, rhf=True)
    cfg = config.Config(calc_type='CCSDT', tol=1e-10, max_iter=200, rhf=True).calc_macros()
    r = driver.solve_cc(ctx, cfg, out=lambda x: None)
    t = ctx.get_t()
    ctx.close()
    e, it, failed, _, _ = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDT', rhf=True,
                                  active=act).solve(tol=1e-10, max_iter=200, compressed_diis=True)
    assert not r.failed and r.iterations == it and abs(r.e_cor - e) < 1e-10
    dims = (d.froz, d.occ_a, d.occ_b, d.orbs)
    c = lib.t_compress(dims, *act, t)
    assert c.size == lib.t_size_act(*dims, *act) < t.size
    ctx = _ctx_restricted(s, act, rhf=True)
    ctx.set_t(lib.t_expand(dims, *act, c, t.size))
    np.testing.assert_array_equal(ctx.get_t(), t)
    ctx.close()
