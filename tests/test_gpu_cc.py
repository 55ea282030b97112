"""Resident GPU solver through the C ABI vs the CPU oracle.

Sweep-level parity: one or two update sweeps from random amplitudes agree with
oracle/blockcc.py to 1e-12 (FP64, reordered sums only).  Converged parity:
energies agree with the committed oracle fixtures and with the H4 known
answers of the reference's tests to 1e-10 Eh (plus the fixture's 2.3e-10
rounding offset for H4).
"""
import json
import os

import numpy as np
import pytest

from ccq_b200 import config, driver, integrals as I, lib, synth
from oracle.blockcc import BlockCC
from tests.conftest import GOLDEN
from tests.helpers import random_system, random_t

pytestmark = pytest.mark.gpu


def make_ctx(s, method, rhf=False, shift=0.0, ds=5):
    d = s['dims']
    return lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, method, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                       s['v_bb'], rhf=rhf, shift=shift, diis_space=ds)


@pytest.mark.parametrize('method,rhf,n,oa,ob', [('CCSD', False, 6, 2, 2), ('CCSD', False, 7, 3, 2),
                                                ('CCSD', True, 6, 2, 2), ('CCSDT', False, 6, 2, 2),
                                                ('CCSDT', False, 7, 3, 2), ('CCSDT', True, 7, 3, 3)])
def test_sweep_parity(method, rhf, n, oa, ob, plan_text):
    s = random_system(n, oa, ob, seed=13)
    ctx = make_ctx(s, method, rhf, shift=0.05)
    bc = BlockCC(plan_text(method, rhf), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method,
                 shift=0.05)
    t, _ = random_t(s['dims'], seed=2, scale=0.03, nmax=3 if method != 'CCSD' else 2)
    ctx.set_t(t)
    tc = t.copy()
    for _ in range(2):
        ctx.update()
        bc.update(tc)
    tg = ctx.get_t()
    np.testing.assert_allclose(tg, tc, atol=1e-12, rtol=0)
    assert abs(ctx.energy() - bc.energy(tc)) < 1e-12
    ctx.close()


@pytest.mark.parametrize('method,froz', [('CCSD', 1), ('CCSDT', 1), ('CCSDT', 2)])
def test_sweep_parity_frozen_core(method, froz, plan_text):
    # froz inactive occupied orbitals (spatial): the active range starts at froz in every block
    s = random_system(8, 4, 3, seed=19, sigma=0.08, froz=froz)
    ctx = make_ctx(s, method, False, shift=0.02)
    bc = BlockCC(plan_text(method, False), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method,
                 shift=0.02)
    t, _ = random_t(s['dims'], seed=3, scale=0.03, nmax=3 if method != 'CCSD' else 2)
    ctx.set_t(t)
    tc = t.copy()
    for _ in range(2):
        ctx.update()
        bc.update(tc)
    np.testing.assert_allclose(ctx.get_t(), tc, atol=1e-12, rtol=0)
    assert abs(ctx.energy() - bc.energy(tc)) < 1e-12
    ctx.close()


@pytest.mark.parametrize('rhf', [False, True])
def test_sweep_parity_ccsdtq(plan_text, rhf):
    s = random_system(5, 2, 2, seed=17)
    ctx = make_ctx(s, 'CCSDTQ', rhf, shift=0.05)
    bc = BlockCC(plan_text('CCSDTQ', rhf), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'],
                 'CCSDTQ', shift=0.05)
    t, t4 = random_t(s['dims'], seed=4, scale=0.03, nmax=4)
    ctx.set_t(t)
    for b, v in t4.items():
        ctx.set_block(b, v)
        bc.buf[b][...] = v
    tc = t.copy()
    for sweep in range(2):
        ctx.update()
        bc.update(tc)
        tg = ctx.get_t()
        lay = I.TLayout(s['dims'])
        for b in I.T_VEC_ORDER:
            np.testing.assert_allclose(lay.view(tg, b), lay.view(tc, b), atol=1e-12, rtol=0, err_msg=f'{b} sweep {sweep}')
        for b in t4:
            np.testing.assert_allclose(ctx.get_block(b, t4[b].shape), bc.buf[b], atol=1e-12, rtol=0,
                                       err_msg=f'{b} sweep {sweep}')
    ctx.close()


def _cfg(method, tol=1e-10, ds=5, rhf=False, graph=True, max_iter=100):
    c = config.Config(calc_type=method, tol=tol, diis_space=ds, rhf=rhf, max_iter=max_iter, gpu_graph=graph)
    return c.calc_macros()


def test_h4_ccsdt_rhf_known_answer(h4):
    ctx = make_ctx(h4, 'CCSDT', rhf=True)
    r = driver.solve_cc(ctx, _cfg('CCSDT', tol=1e-11, rhf=True), out=lambda s: None)
    assert not r.failed
    assert abs(r.e_cor + h4['e_ref'] - (-1.978696408825)) < 2.3e-10 + 1e-11


def test_h4_ccsdtq_known_answer(h4, plan_text):
    plan_text('CCSDTQ', False)
    ctx = make_ctx(h4, 'CCSDTQ')
    r = driver.solve_cc(ctx, _cfg('CCSDTQ', tol=1e-11), out=lambda s: None)
    assert not r.failed
    assert abs(r.e_cor + h4['e_ref'] - (-1.975861644132)) < 2.3e-10 + 1e-11


def _golden(name):
    p = os.path.join(GOLDEN, 'synthetic.json')
    data = json.load(open(p))
    if name not in data:
        pytest.skip(f'{name} not in fixtures')
    return data[name]


@pytest.mark.parametrize('name', ['c0_ccsd', 'small_ccsdt', 'small_ccsdt_open', 'small_ccsdtq'])
def test_converged_energy_matches_oracle_fixture(name):
    g = _golden(name)
    spec = synth.SynthSpec(**g['spec'])
    s = synth.system(spec)
    if g['occ_b'] != g['occ_a']:
        fa, fb = I.fock(s['h'], s['e2'], g['occ_a'], g['occ_b'])
        s['f_a'], s['f_b'] = fa, fb
        s['dims'] = I.Dims(0, g['occ_a'], g['occ_b'], spec.norb)
    ctx = make_ctx(s, g['method'], rhf=g['rhf'])
    r = driver.solve_cc(ctx, _cfg(g['method'], tol=g['tol'], rhf=g['rhf'], max_iter=200), out=lambda s: None)
    assert not r.failed
    assert abs(r.e_cor - g['e_cor']) < 1e-10
    # same algorithm, same iteration count (Gauss-Seidel order, DIIS schedule)
    assert abs(r.iterations - g['iterations']) <= 1
    ctx.close()


def test_graph_and_eager_agree():
    s = synth.system(synth.SynthSpec(12, 6, 24, 0.03, 7))
    es = []
    for graph in (False, True):
        ctx = make_ctx(s, 'CCSDT')
        r = driver.solve_cc(ctx, _cfg('CCSDT', tol=1e-9, graph=graph), out=lambda s: None)
        es.append(r.e_cor)
        ctx.close()
    assert abs(es[0] - es[1]) < 1e-11


def test_driver_runs_input_deck(tmp_path):
    spec = synth.SynthSpec(10, 4, 20, 0.04, 5)
    inp = synth.write_inputs(spec, str(tmp_path), 'CCSD', tol=1e-9)
    lines = []
    r = driver.run(inp, out=lines.append)
    assert not r.failed
    assert any('Calculation Summary' in l for l in lines)
    assert lines[-1].split()[0] == 'CCSD'
    s = synth.system(spec)
    bc = BlockCC(open(os.path.join(os.path.dirname(lib.LIB_PATH), 'plans', 'CCSD.plan')).read(),
                 s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], 'CCSD')
    e, *_ = bc.solve(tol=1e-9, max_iter=100)
    assert abs(r.e_cor - e) < 1e-10


def test_bad_arguments_fail_loudly():
    s = random_system(5, 2, 2, seed=1)
    with pytest.raises(lib.CCQB200Error):
        make_ctx(s, 'CCSDTQQ')
    ctx = make_ctx(s, 'CCSD')
    with pytest.raises(lib.CCQB200Error):
        ctx._lib.ccq_b200_set_t(ctx.ptr, None, 3) and lib._err(-1)
        lib._err(ctx._lib.ccq_b200_set_t(ctx.ptr, lib._p(np.zeros(3)), 3))
    ctx.close()


@pytest.mark.parametrize('method', ['CCSD', 'CCSDT'])
def test_fortran_and_row_major_integrals_give_the_same_sweep(method):
    """ccq_b200_init (Fortran-ordered f and v, as ccq holds them) and ccq_b200_init_rowmajor (C order)
    build the same context: two sweeps agree bit for bit."""
    s = random_system(7, 3, 2, seed=23, froz=1)
    d = s['dims']
    t, _ = random_t(d, seed=8, scale=0.03, nmax=3 if method != 'CCSD' else 2)
    out = []
    for conv in (np.ascontiguousarray, np.asfortranarray):
        arrs = [conv(s[k]) for k in ('f_a', 'f_b', 'v_aa', 'v_ab', 'v_bb')]
        ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, method, *arrs, shift=0.05)
        ctx.set_t(t)
        ctx.update()
        ctx.update()
        out.append((ctx.get_t(), ctx.energy()))
        ctx.close()
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
