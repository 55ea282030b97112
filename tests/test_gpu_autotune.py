"""Autotuner: tuning leaves the solve unchanged and the tuned sweeps stay exact.

``ccq_b200_autotune`` times every contraction's candidate configurations
(64 x 64 or skinny tiles, split-K chunk, int8 slices or DMMA) in one eager
sweep and restores the amplitudes.  After tuning: the amplitudes are those of
before, the tuned FP64 sweeps agree with the numpy plan executor to 1e-12
(only the order of the sums changes), and a tuned solve reaches the untuned
solve's energy and iteration count.
"""
import numpy as np
import pytest

from ccq_b200 import config, driver, lib, synth
from oracle.blockcc import BlockCC
from tests.helpers import random_system, random_t

pytestmark = pytest.mark.gpu


def make_ctx(s, method, shift=0.0):
    d = s['dims']
    return lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, method, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                       s['v_bb'], shift=shift)


@pytest.mark.parametrize('method,n,oa,ob', [('CCSD', 7, 3, 2), ('CCSDT', 7, 3, 2), ('CCSDTQ', 5, 2, 2)])
def test_tuned_sweeps_match_oracle(method, n, oa, ob, plan_text):
    s = random_system(n, oa, ob, seed=13)
    ctx = make_ctx(s, method, shift=0.05)
    bc = BlockCC(plan_text(method, False), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method,
                 shift=0.05)
    t, t4 = random_t(s['dims'], seed=2, scale=0.03, nmax={'CCSD': 2, 'CCSDT': 3, 'CCSDTQ': 4}[method])
    ctx.set_t(t)
    for b, v in t4.items():
        ctx.set_block(b, v)
        bc.buf[b][...] = v
    before, after = ctx.autotune(2)
    assert 0.0 < after <= before
    # tuning is not an iteration: every amplitude block is as it was
    np.testing.assert_array_equal(ctx.get_t(), t)
    for b, v in t4.items():
        np.testing.assert_array_equal(ctx.get_block(b, v.shape), v)
    tc = t.copy()
    for _ in range(2):
        ctx.update()
        bc.update(tc)
    np.testing.assert_allclose(ctx.get_t(), tc, atol=1e-12, rtol=0)
    for b in t4:
        np.testing.assert_allclose(ctx.get_block(b, t4[b].shape), bc.buf[b], atol=1e-12, rtol=0)
    assert abs(ctx.energy() - bc.energy(tc)) < 1e-12
    ctx.close()


@pytest.mark.parametrize('prec', ['fp64', 'split'])
def test_tuned_solve_matches_untuned(prec):
    # 32 orbitals, 12 electrons: the ladder contractions are large enough for int8 slices
    s = synth.system(synth.SynthSpec(32, 12, 64, 0.03, 11))
    res = {}
    for tune in (False, True):
        ctx = make_ctx(s, 'CCSDT')
        ctx.set_precision(lib.PREC_SPLIT if prec == 'split' else lib.PREC_FP64, 4)
        if tune:
            before, after = ctx.autotune(2)
            assert after <= before
        cfg = config.Config(calc_type='CCSDT', tol=1e-10, max_iter=80, gpu_precision=prec, gpu_slices=4,
                            gpu_fp64_finish=1e-7).calc_macros()
        r = driver.solve_cc(ctx, cfg, out=lambda x: None)
        assert not r.failed
        res[tune] = r
        ctx.close()
    assert abs(res[True].e_cor - res[False].e_cor) < 1e-10
    assert abs(res[True].iterations - res[False].iterations) <= 1


@pytest.mark.parametrize('tile', [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize('method,n,oa,ob', [('CCSD', 7, 3, 2), ('CCSDT', 7, 3, 2)])
def test_forced_kernel_family_matches_oracle(tile, method, n, oa, ob, plan_text):
    """Every contraction on one GETT family (64 x 64 DMMA, skinny DMMA, small-K FMA, register-direct DMMA)."""
    s = random_system(n, oa, ob, seed=21)
    ctx = make_ctx(s, method, shift=0.05)
    ctx.force_tile(tile)
    bc = BlockCC(plan_text(method, False), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method,
                 shift=0.05)
    t, _ = random_t(s['dims'], seed=5, scale=0.03, nmax=3 if method == 'CCSDT' else 2)
    ctx.set_t(t)
    tc = t.copy()
    for _ in range(2):
        ctx.update()
        bc.update(tc)
    np.testing.assert_allclose(ctx.get_t(), tc, atol=1e-12, rtol=0)
    ctx.close()


def test_small_k_kernel_on_large_views():
    """20 orbitals: several 256-wide F tiles and 32-wide S tiles per contraction, grouped launches; the
    small-K FMA kernel and the register-direct DMMA kernel against the default families."""
    s = synth.system(synth.SynthSpec(20, 8, 40, 0.05, 3))
    d = s['dims']
    t, _ = random_t(d, seed=6, scale=0.02, nmax=3)
    out = {}
    for tile in (0, 3, 6):
        ctx = make_ctx(s, 'CCSDT')
        ctx.force_tile(tile)
        ctx.set_t(t)
        for _ in range(2):
            ctx.update()
        out[tile] = ctx.get_t()
        ctx.close()
    np.testing.assert_allclose(out[3], out[0], atol=1e-12, rtol=0)
    np.testing.assert_allclose(out[6], out[0], atol=1e-12, rtol=0)
