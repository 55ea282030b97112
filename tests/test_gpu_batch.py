"""Batched CCSD: many contexts iterated concurrently on one GPU.

Each instance must reproduce its own serial solve (the numpy executor of the
CCSD plan): the same iteration count and the energy to 1e-10 Eh.
"""
import os

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_batch_matches_serial_oracle():
    from ccq_b200 import batch, synth
    from oracle.blockcc import BlockCC
    specs = [synth.SynthSpec(n, 2 * (n // 5), 2 * n, 0.03, 2000 + n) for n in (10, 13, 16, 11, 18, 12)]
    res, tim = batch.solve_batch(specs, tol=1e-9)
    plan = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CCSD.plan')).read()
    for spec, r in zip(specs, res):
        s = synth.system(spec)
        bc = BlockCC(plan, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], 'CCSD')
        e, it, failed, _, _ = bc.solve(tol=1e-9, max_iter=200)
        assert not r['failed'] and r['iterations'] == it
        assert abs(r['e_cor'] - e) < 1e-10


def test_async_iteration_needs_a_wait():
    from ccq_b200 import batch, lib, synth
    x = batch.Instance(synth.SynthSpec(10, 4, 20, 0.03, 5))
    try:
        x.ctx.iterate_async(1)
        with pytest.raises(lib.CCQB200Error):
            x.ctx.iterate_async(2)
        x.ctx.iterate_wait()
        with pytest.raises(lib.CCQB200Error):
            x.ctx.iterate_wait()
    finally:
        x.close()
