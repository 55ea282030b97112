"""The runtime's reading of a plan (restricted tables, sorted Z reads) equals the full oracle."""
import numpy as np
import pytest

from oracle.blockcc import BlockCC
from tests.helpers import random_system, random_t
from tests.runtime_emul import emulate, parse_annotated


@pytest.mark.parametrize('method,rhf,n,oa,ob', [('CCSD', False, 5, 2, 2), ('CCSD', True, 5, 2, 2),
                                                ('CCSDT', False, 6, 3, 2), ('CCSDT', True, 6, 3, 3),
                                                ('CCSDTQ', False, 5, 2, 2)])
def test_emulated_runtime_matches_oracle(method, rhf, n, oa, ob, plan_text):
    txt = plan_text(method, rhf)
    s = random_system(n, oa, ob, seed=31)
    args = (s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method)
    ref = BlockCC(txt, *args, shift=0.02)
    emu = BlockCC(txt, *args, shift=0.02)
    emu.plan = dict(emu.plan)
    ann = parse_annotated(txt)
    emu.plan['buffers'] = ann['buffers']
    for name, (kind, dims, groups) in ann['buffers'].items():
        if kind == 'work':
            emu.buf[name][...] = np.nan
    nmax = {'CCSD': 2, 'CCSDT': 3, 'CCSDTQ': 4}[method]
    t, t4 = random_t(s['dims'], seed=6, scale=0.03, nmax=nmax)
    for b, v in t4.items():
        ref.buf[b][...] = v
        emu.buf[b][...] = v
    t1, t2 = t.copy(), t.copy()
    ops = ann['ops']
    k = [i for i, o in enumerate(ops) if o[0] == 'PHASE' and o[1] == 'energy'][0]
    ref.update(t1)
    emulate(emu, t2, ops[:k])
    assert np.all(np.isfinite(t2))
    np.testing.assert_allclose(t2, t1, atol=1e-14, rtol=0)
    for b in t4:
        assert np.all(np.isfinite(emu.buf[b]))
        np.testing.assert_allclose(emu.buf[b], ref.buf[b], atol=1e-14, rtol=0)
