"""Externally corrected CC on the GPU: the CCSDTQ context with T3 / T4 held at the
exact cluster amplitudes of the FCI state (ccq_b200_set_external) iterates T1
and T2 to the FCI energy and the exact T1, T2, in the oracle's iteration count;
T3 / T4 stay as given."""
import numpy as np
import pytest

from ccq_b200 import config, driver, lib
from tests.test_extcor import ec_setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('n,oa,ob', [(5, 2, 2), (5, 3, 2)])
def test_external_correction_matches_fci_and_oracle(n, oa, ob):
    s, dc, t0, t4, blocks, e_fci = ec_setup(n, oa, ob)
    d = s['dims']
    ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDTQ', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                      s['v_bb'])
    ctx.set_t(t0)
    for b, v in t4.items():
        ctx.set_block(b, v)
    ctx.set_external(True)
    cfg = config.Config(calc_type='CCSDTQ', tol=1e-12, max_iter=200).calc_macros()
    r = driver.solve_cc(ctx, cfg, out=lambda x: None)
    tg = ctx.get_t()
    t4g = {b: ctx.get_block(b, v.shape) for b, v in t4.items()}
    ctx.close()
    assert not r.failed
    assert abs(r.e_cor - e_fci) < 1e-10
    lay = dc.layout
    for b in ('T1A', 'T1B', 'T2A', 'T2B', 'T2C'):
        np.testing.assert_allclose(lay.view(tg, b), blocks[b], atol=1e-9, rtol=0)
    for b in ('T3A', 'T3B', 'T3C', 'T3D'):
        np.testing.assert_array_equal(lay.view(tg, b), lay.view(t0, b))
    for b, v in t4.items():
        np.testing.assert_array_equal(t4g[b], v)
    dc.t4 = {b: v.copy() for b, v in t4.items()}
    e, it, failed, _, _ = dc.solve(tol=1e-12, max_iter=200, t0=t0)
    assert r.iterations == it and abs(r.e_cor - e) < 1e-11


def test_external_amplitudes_from_input_deck(tmp_path, h4):
    """gpu_external_t= names a .npz of T3 / T4 blocks: the H4 deck then gives its FCI energy."""
    from ccq_b200 import integrals as I
    from oracle.densecc import DenseCC
    from tests.helpers import fci_cluster_amplitudes
    dc = DenseCC(h4['f_a'], h4['f_b'], h4['v_aa'], h4['v_ab'], h4['v_bb'], h4['dims'], 'CCSDTQ', external=True)
    ts, e_fci = fci_cluster_amplitudes(dc.so, 4)
    names = [b for b in I.T_VEC_ORDER if b[1] == '3'] + sorted(dc.layout.t4_shape)
    np.savez(tmp_path / 'ext.npz', **dc.so.to_blocks(ts, names))
    I.write_onebody(str(tmp_path / 'onebody.inp'), h4['e1'])
    I.write_twobody(str(tmp_path / 'twobody.inp'), h4['e2'], h4['enuc'])
    (tmp_path / 'in.inp').write_text('nel=4\nnvirt=4\ncalc_type=CCSDTQ\ngpu_external_t=ext.npz\ntol=1.0e-12\n'
                                     'max_iterations=200\nkeep_bin=.false.\n')
    lines = []
    r = driver.run(str(tmp_path / 'in.inp'), out=lines.append, base_dir=str(tmp_path))
    assert not r.failed and any('External T3 and T4' in x for x in lines)
    assert abs(r.e_cor - e_fci) < 1e-10
