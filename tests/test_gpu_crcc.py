"""CR-CC(2,3) on the GPU against the numpy executor of the same plan.

The numpy executor is pinned to the dense spin-orbital restatement and to
determinant space by tests/test_crcc.py.  Here the device solve must take the
same CCSD and left iterations (energies per iteration to 1e-10 Eh) and give
the same four corrections when both start from the device's T and lambda.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _setup(norb, nel, rhf, seed=7):
    from ccq_b200 import config, lib, synth
    from oracle.blockcc import BlockCRCC
    s = synth.system(synth.SynthSpec(norb, nel, 2 * norb, 0.1, seed))
    d = s['dims']
    text = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CRCC23' + ('_rhf' if rhf else '') + '.plan')).read()
    bc = BlockCRCC(text, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d)
    ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CR-CC(2,3)', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                      s['v_bb'], rhf=rhf)
    cfg = config.Config(calc_type='CR-CC(2,3)', tol=1e-11, max_iter=200).calc_macros()
    return s, bc, ctx, cfg


@pytest.mark.parametrize('norb,nel,rhf', [(8, 6, False), (9, 8, True)])
def test_crcc23_matches_plan_executor(norb, nel, rhf):
    from ccq_b200 import driver
    s, bc, ctx, cfg = _setup(norb, nel, rhf)
    try:
        r = driver.solve_cc(ctx, cfg, out=lambda x: None)
        e, it, failed, hist, tvec = bc.solve(tol=cfg.tol, max_iter=cfg.max_iter)
        assert not r.failed and not failed and r.iterations == it
        assert abs(r.e_cor - e) < 1e-11
        left = driver.solve_lcc(ctx, cfg, r.e_cor, out=lambda x: None)
        _, itl, fl, hl = bc.solve_left(tvec, e, tol=cfg.tol, max_iter=cfg.max_iter)
        assert not left.failed and not fl and left.iterations == itl
        np.testing.assert_allclose([h['e'] for h in left.history], [h[0] for h in hl], atol=1e-10, rtol=0)
        e23 = ctx.crcc23()
        # the executor's corrections from the device's own T and lambda
        tdev = ctx.get_t()
        bc.lvec[:ctx.vec_size] = ctx.get_l()
        ref = bc.crcc23(tdev)
        assert np.all(np.abs(e23) > 1e-6)
        np.testing.assert_allclose(e23, ref, rtol=1e-11, atol=0)
        # and from its own converged solve, to the left tolerance
        ref2 = bc.crcc23(tvec)
        np.testing.assert_allclose(e23, ref2, rtol=1e-6, atol=0)
    finally:
        ctx.close()


def test_crcc23_matches_oracle_fixture():
    """12 orbitals (nel=8): iteration counts and the four corrections of tests/golden/synthetic.json."""
    import json
    from ccq_b200 import config, driver, lib, synth
    g = json.load(open(os.path.join(ROOT, 'tests', 'golden', 'synthetic.json')))['small_crcc23']
    spec = synth.SynthSpec(**g['spec'])
    s = synth.system(spec)
    d = s['dims']
    ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CR-CC(2,3)', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                      s['v_bb'])
    try:
        cfg = config.Config(calc_type='CR-CC(2,3)', tol=g['tol'], max_iter=200).calc_macros()
        r = driver.solve_cc(ctx, cfg, out=lambda x: None)
        left = driver.solve_lcc(ctx, cfg, r.e_cor, out=lambda x: None)
        e23 = ctx.crcc23()
    finally:
        ctx.close()
    assert r.iterations == g['iterations'] and left.iterations == g['left_iterations']
    assert abs(r.e_cor - g['e_cor']) < 1e-10
    np.testing.assert_allclose(e23, g['e23'], rtol=1e-7, atol=0)


def test_crcc23_repeatable_and_graph_free_agree():
    """The left iterations replayed from a CUDA graph and launched one by one agree."""
    from ccq_b200 import driver
    out = []
    for graph in (True, False):
        s, bc, ctx, cfg = _setup(8, 6, False, seed=3)
        cfg.gpu_graph = graph
        try:
            r = driver.solve_cc(ctx, cfg, out=lambda x: None)
            ctx.use_graph(graph)
            left = driver.solve_lcc(ctx, cfg, r.e_cor, out=lambda x: None)
            out.append((left.iterations, ctx.crcc23()))
        finally:
            ctx.close()
    assert out[0][0] == out[1][0]
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-12, atol=0)


def test_driver_runs_crcc23_input_deck(tmp_path):
    from ccq_b200 import driver, synth
    spec = synth.SynthSpec(8, 6, 16, 0.1, 5)
    inp = synth.write_inputs(spec, str(tmp_path), 'CR-CC(2,3)', tol=1e-10)
    lines = []
    r = driver.run(inp, out=lines.append)
    text = '\n'.join(lines)
    assert 'Left Coupled cluster' in text and 'CC(t;3)' in text
    assert not r.failed
    assert abs(r.e_cor - (r.e_ccsd + r.e23[3])) < 1e-14


def test_lambda_calls_need_a_crcc_context():
    from ccq_b200 import lib, synth
    s = synth.system(synth.SynthSpec(6, 4, 12, 0.1, 1))
    d = s['dims']
    ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSD', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'])
    try:
        with pytest.raises(lib.CCQB200Error):
            ctx.lambda_init(0.0)
        with pytest.raises(lib.CCQB200Error):
            ctx.crcc23()
    finally:
        ctx.close()


@pytest.mark.parametrize('n,oa,ob,froz', [(7, 4, 3, 0), (8, 5, 3, 1)])
def test_open_shell_and_frozen_core(n, oa, ob, froz):
    from ccq_b200 import config, driver, lib
    from oracle.blockcc import BlockCRCC
    from tests.helpers import random_system
    s = random_system(n, oa, ob, seed=11, sigma=0.08, froz=froz)
    d = s['dims']
    text = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CRCC23.plan')).read()
    bc = BlockCRCC(text, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d)
    ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CR-CC(2,3)', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                      s['v_bb'])
    try:
        cfg = config.Config(calc_type='CR-CC(2,3)', tol=1e-11, max_iter=200).calc_macros()
        r = driver.solve_cc(ctx, cfg, out=lambda x: None)
        e, it, failed, _, tvec = bc.solve(tol=cfg.tol, max_iter=200)
        assert r.iterations == it and abs(r.e_cor - e) < 1e-11
        left = driver.solve_lcc(ctx, cfg, r.e_cor, out=lambda x: None)
        _, itl, _, hl = bc.solve_left(tvec, e, tol=cfg.tol, max_iter=200)
        assert left.iterations == itl
        np.testing.assert_allclose([h['e'] for h in left.history], [h[0] for h in hl], atol=1e-10, rtol=0)
        e23 = ctx.crcc23()
        bc.lvec[:ctx.vec_size] = ctx.get_l()
        np.testing.assert_allclose(e23, bc.crcc23(ctx.get_t()), rtol=1e-11, atol=1e-16)
    finally:
        ctx.close()
