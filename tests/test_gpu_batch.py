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


def test_pipelined_batch_matches_serial_oracle():
    """Instances iterating while host threads still create the other contexts give their own serial solves."""
    from ccq_b200 import batch, synth
    from oracle.blockcc import BlockCC
    specs = [synth.SynthSpec(n, 2 * (n // 5), 2 * n, 0.03, 2000 + n) for n in (10, 13, 16, 11, 18, 12)]
    res, tim = batch.solve_pipelined(specs, tol=1e-9, threads=2)
    assert tim['total_s'] >= tim['setup_s']
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


def test_grouped_batch_matches_serial_oracle():
    """The same solves as one batch (ccq_b200_batch_*): each plan operation of all instances in one launch,
    instances of uneven size (their tiles and canonical elements in one grid), instances finishing at
    different iterations (the finished ones switched off)."""
    from ccq_b200 import batch, synth
    from oracle.blockcc import BlockCC
    specs = [synth.SynthSpec(n, 2 * (n // 5), 2 * n, 0.03, 2000 + n) for n in (10, 13, 16, 11, 18, 12)]
    res, tim = batch.solve_batch(specs, tol=1e-9, grouped=True)
    plan = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CCSD.plan')).read()
    its = set()
    for spec, r in zip(specs, res):
        s = synth.system(spec)
        bc = BlockCC(plan, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], 'CCSD')
        e, it, failed, _, _ = bc.solve(tol=1e-9, max_iter=200)
        assert not r['failed'] and r['iterations'] == it
        assert abs(r['e_cor'] - e) < 1e-10
        its.add(it)
    assert len(its) > 1


def test_grouped_batch_keeps_every_amplitude():
    """A grouped batch iteration leaves each context's amplitudes as its own iteration would (to round-off)."""
    import numpy as np
    from ccq_b200 import batch, lib, synth
    specs = [synth.SynthSpec(n, 2 * (n // 5), 2 * n, 0.03, 3000 + n) for n in (12, 15)]
    one = [batch.Instance(sp) for sp in specs]
    grp = [batch.Instance(sp) for sp in specs]
    bt = lib.Batch([x.ctx for x in grp])
    try:
        for it in (1, 2, 3):
            for x in one:
                x.ctx.iterate(it)
            bt.iterate(it, [1, 1])
        for a, b in zip(one, grp):
            np.testing.assert_allclose(b.ctx.get_t(), a.ctx.get_t(), atol=1e-13, rtol=0)
        # a switched-off context does not move
        t0 = grp[1].ctx.get_t()
        bt.iterate(4, [1, 0])
        assert np.array_equal(grp[1].ctx.get_t(), t0)
    finally:
        bt.close()
        for x in one + grp:
            x.close()


def test_grouped_batch_matches_fixture_c3():
    """All 64 instances of the batched workload as one batch, against the committed oracle energies and
    iteration counts."""
    import json
    from ccq_b200 import batch
    g = json.load(open(os.path.join(ROOT, 'tests', 'golden', 'synthetic.json')))['c3_batched_ccsd']
    res, tim = batch.solve_batch(batch.c3_specs(), tol=1e-8, grouped=True)
    for r, x in zip(res, g['instances']):
        assert not r['failed'] and r['iterations'] == x['iterations'] and abs(r['e_cor'] - x['e_cor']) < 1e-10
