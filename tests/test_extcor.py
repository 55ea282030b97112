"""Externally corrected CC on the CPU oracle: with the exact T3 and T4 of the FCI
state (cluster analysis of the FCI vector in determinant space), iterating only
T1 and T2 lands on the FCI energy and on the exact T1, T2.  This is the
fixed-point property that makes externally corrected CC exact for exact
external amplitudes; the GPU path is checked against it in
tests/test_gpu_extcor.py."""
import numpy as np
import pytest

from ccq_b200 import integrals as I
from oracle.densecc import DenseCC
from tests.helpers import fci_cluster_amplitudes, random_system


def ec_setup(n, oa, ob, seed=31):
    s = random_system(n, oa, ob, seed=seed, sigma=0.09)
    d = s['dims']
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDTQ', external=True)
    ts, e_fci = fci_cluster_amplitudes(dc.so, 4)
    names = [b for b in I.T_VEC_ORDER] + sorted(dc.layout.t4_shape)
    blocks = dc.so.to_blocks(ts, names)
    lay = dc.layout
    t0 = np.zeros(lay.t_size)
    for b in I.T_VEC_ORDER:
        if b[1] == '3':
            lay.view(t0, b)[...] = blocks[b]
    t4 = {b: blocks[b] for b in lay.t4_shape}
    return s, dc, t0, t4, blocks, e_fci


@pytest.mark.parametrize('n,oa,ob', [(5, 2, 2), (5, 3, 2)])
def test_exact_external_triples_and_quadruples_give_fci(n, oa, ob):
    s, dc, t0, t4, blocks, e_fci = ec_setup(n, oa, ob)
    dc.t4 = {b: v.copy() for b, v in t4.items()}
    e, it, failed, hist, tvec = dc.solve(tol=1e-12, max_iter=200, t0=t0)
    assert not failed
    assert abs(e - e_fci) < 1e-10
    for b in ('T1A', 'T1B', 'T2A', 'T2B', 'T2C'):
        np.testing.assert_allclose(dc.layout.view(tvec, b), blocks[b], atol=1e-9, rtol=0)
    # the external amplitudes were not touched
    for b in ('T3A', 'T3B', 'T3C', 'T3D'):
        np.testing.assert_array_equal(dc.layout.view(tvec, b), dc.layout.view(t0, b))


def test_external_key():
    from ccq_b200 import config
    cfg = config.parse_lines(['nel=4', 'nvirt=4', 'calc_type=CCSDTQ', 'gpu_external_t=ext.npz']).calc_macros()
    assert cfg.gpu_external_t == 'ext.npz' and cfg.lvl_q
