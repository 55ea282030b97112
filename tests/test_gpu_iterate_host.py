"""ccq_b200_iterate_host: one iteration from a host t_vec to a host t_vec with the
block copies overlapped with the sweep gives what iterate + get_t give, across
DIIS steps, in every graph mode, with pinned or pageable host memory."""
import numpy as np
import pytest

from ccq_b200 import lib
from tests.helpers import random_system

pytestmark = pytest.mark.gpu


def _ctx(s, method, graph):
    d = s['dims']
    c = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, method, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'])
    c.use_graph(graph)
    return c


@pytest.mark.parametrize('method,graph,pinned', [('CCSDT', 1, True), ('CCSDT', 2, False), ('CCSDT', 0, True),
                                                 ('CCSD', 1, True), ('CCSDTQ', 1, False), ('CCSDTQ', 1, True),
                                                 ('CCSDT', 1, 'two')])
def test_iterate_host_equals_iterate_and_get_t(method, graph, pinned):
    """pinned True: one pinned buffer in and out; 'two': separate pinned input and output buffers (the
    input read block by block inside the dependency-graph sweep); False: pageable memory."""
    import torch
    s = random_system(7, 3, 2, seed=12, sigma=0.08) if method != 'CCSDTQ' else random_system(5, 2, 2, seed=12)
    a = _ctx(s, method, graph)
    b = _ctx(s, method, graph)
    n = a.t_size
    if pinned == 'two':
        bin_ = torch.zeros(n, dtype=torch.float64, pin_memory=True)
        bout = torch.zeros(n, dtype=torch.float64, pin_memory=True)
        pin, pout = bin_.data_ptr(), bout.data_ptr()
        view = bout.numpy()
    elif pinned:
        buf = torch.zeros(n, dtype=torch.float64, pin_memory=True)
        pin, pout = buf.data_ptr(), buf.data_ptr()
        view = buf.numpy()
    else:
        tin = np.zeros(n)
        tout = np.zeros(n)
        pin, pout = tin.ctypes.data, tout.ctypes.data
    for it in range(1, 9):    # DIIS at iteration 6
        ea, ra, da = a.iterate(it)
        ta = a.get_t()
        eb, rb, db = b.iterate_host(it, pin, pout)
        tb = view.copy() if pinned else tout.copy()
        if pinned == 'two':
            bin_.numpy()[...] = view
        elif not pinned:
            tin[...] = tout
        assert da == db
        assert abs(ea - eb) < 1e-12 and abs(ra - rb) < 1e-12
        np.testing.assert_allclose(tb, ta, atol=1e-12, rtol=0)
        h2d, d2h = b.io_bytes()
        # the whole vector out once: block by block as the sweep finishes them, or after the extrapolation of
        # a DIIS step; the device holds the amplitude blocks of the method (t_vec may be longer)
        full = d2h
        assert 0 < full <= 8 * n
        if pinned and graph == 1 and method != 'CCSD':
            # the T3 blocks were read from the mapped host vector at their canonical elements only
            assert h2d < full
        else:
            assert h2d == full
    a.close()
    b.close()


def test_iterate_host_mid_size():
    """30 orbitals, 8 + 8 occupied (T3 blocks of 5.5 M elements, read at their canonical elements from the
    mapped host vector): the result equals iterate + get_t across a DIIS step, with separate pinned input and
    output buffers."""
    import torch
    from ccq_b200 import synth
    s = synth.system(synth.SynthSpec(30, 16, 60, 0.03, 7))
    d = s['dims']
    a = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDT', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'])
    b = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDT', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'])
    a.use_graph(1)
    b.use_graph(1)
    n = a.t_size
    bin_ = torch.zeros(n, dtype=torch.float64, pin_memory=True)
    bout = torch.zeros(n, dtype=torch.float64, pin_memory=True)
    try:
        for it in range(1, 8):
            ea, ra, da = a.iterate(it)
            eb, rb, db = b.iterate_host(it, bin_.data_ptr(), bout.data_ptr())
            assert da == db
            assert abs(ea - eb) < 1e-12 and abs(ra - rb) < 1e-12
            np.testing.assert_allclose(bout.numpy(), a.get_t(), atol=1e-12, rtol=0)
            bin_.numpy()[...] = bout.numpy()
    finally:
        a.close()
        b.close()
