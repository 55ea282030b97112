"""Checkpoint / restart on the GPU: a solve stopped at iteration k and resumed
from its checkpoint (t_vec, T4 blocks, DIIS ring, solver state) in a fresh
context follows the uninterrupted solve: same iteration count, energies per
iteration within 1e-10, final energy within 1e-12.  Checkpoints of another
system and truncated files are refused without touching device state."""
import os

import numpy as np
import pytest

from ccq_b200 import config, driver, lib
from tests.helpers import random_system

pytestmark = pytest.mark.gpu


def make_ctx(s, method, ds=5):
    d = s['dims']
    return lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, method, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                       s['v_bb'], diis_space=ds)


def _cfg(method, max_iter, **kw):
    return config.Config(calc_type=method, tol=1e-10, max_iter=max_iter, **kw).calc_macros()


@pytest.mark.parametrize('method,n,oa,ob,k', [('CCSD', 8, 3, 3, 7), ('CCSDT', 7, 3, 2, 8), ('CCSDTQ', 5, 2, 2, 5)])
def test_restart_follows_uninterrupted_solve(tmp_path, method, n, oa, ob, k):
    s = random_system(n, oa, ob, seed=9, sigma=0.08)
    path = str(tmp_path / 'ck.bin')
    ref = make_ctx(s, method)
    r_ref = driver.solve_cc(ref, _cfg(method, 200), out=lambda x: None)
    ref.close()
    # the resumed part runs at least one DIIS step (every 6th iteration) from the restored ring
    assert not r_ref.failed and r_ref.iterations >= (k // 6 + 1) * 6 + 1
    first = make_ctx(s, method)
    r1 = driver.solve_cc(first, _cfg(method, k), out=lambda x: None)
    first.save_checkpoint(path, r1.iterations, r1.state)
    first.close()
    info = lib.checkpoint_info(path)
    assert info['calc_type'] == method and info['iteration'] == k and info['with_ring']
    second = make_ctx(s, method)
    r2 = driver.solve_cc(second, _cfg(method, 200, restart=True, bin_file=path), out=lambda x: None)
    second.close()
    assert not r2.failed
    assert r2.iterations == r_ref.iterations
    np.testing.assert_allclose([h['e'] for h in r2.history], [h['e'] for h in r_ref.history[k:]], atol=1e-10, rtol=0)
    assert abs(r2.e_cor - r_ref.e_cor) < 1e-12


def test_checkpoint_of_another_system_or_truncated_is_refused(tmp_path):
    s = random_system(7, 3, 2, seed=4)
    a = make_ctx(s, 'CCSDT')
    driver.solve_cc(a, _cfg('CCSDT', 3), out=lambda x: None)
    path = str(tmp_path / 'a.bin')
    a.save_checkpoint(path, 3, [0.0] * 6)
    t_a = a.get_t()
    a.close()
    other = make_ctx(random_system(8, 3, 2, seed=4), 'CCSDT')
    with pytest.raises(lib.CCQB200Error, match='another system'):
        other.load_checkpoint(path)
    other.close()
    b = make_ctx(s, 'CCSDT')
    before = b.get_t()
    cut = str(tmp_path / 'cut.bin')
    data = open(path, 'rb').read()
    open(cut, 'wb').write(data[:len(data) - 100])
    with pytest.raises(lib.CCQB200Error, match='size'):
        b.load_checkpoint(cut)
    np.testing.assert_array_equal(b.get_t(), before)
    it, st, ring = b.load_checkpoint(path)
    assert it == 3 and ring
    np.testing.assert_array_equal(b.get_t(), t_a)
    b.close()


def test_input_deck_restart(tmp_path, h4):
    """keep_bin writes the checkpoint at the end of a run; restart= continues it to the same answer."""
    from ccq_b200 import integrals as I
    d = tmp_path
    I.write_onebody(str(d / 'onebody.inp'), h4['e1'])
    I.write_twobody(str(d / 'twobody.inp'), h4['e2'], h4['enuc'])
    base = 'nel=4\nnvirt=4\ncalc_type=CCSDT\ntol=1.0e-11\noutput_bin=h4.ck\n'
    (d / 'full.inp').write_text(base + 'max_iterations=100\nkeep_bin=.false.\n')
    (d / 'part.inp').write_text(base + 'max_iterations=5\n')
    (d / 'rest.inp').write_text(base + 'max_iterations=100\nrestart\n')
    full = driver.run(str(d / 'full.inp'), out=lambda x: None, base_dir=str(d))
    assert not os.path.exists(d / 'h4.ck')
    part = driver.run(str(d / 'part.inp'), out=lambda x: None, base_dir=str(d))
    assert part.failed and os.path.exists(d / 'h4.ck')
    lines = []
    rest = driver.run(str(d / 'rest.inp'), out=lines.append, base_dir=str(d))
    assert any('Restart correlation energy' in x for x in lines)
    assert not rest.failed and rest.iterations == full.iterations
    assert abs(rest.e_total - full.e_total) < 1e-12
