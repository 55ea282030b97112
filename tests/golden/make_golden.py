"""Converged FP64 oracle energies for the synthetic workloads (writes synthetic.json).

    python tests/golden/make_golden.py [--c2] [--force]

The oracle is the numpy executor of the contraction plan (oracle/blockcc.py),
itself pinned against the determinant-space residuals and the H4 known answers.
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ccq_b200 import synth  # noqa: E402
from oracle.blockcc import BlockCC, BlockCRCC  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'synthetic.json')

CASES = {
    'c0_ccsd': (synth.C0, 'CCSD', False),
    'small_ccsdt': (synth.SynthSpec(12, 6, 24, 0.03, 7), 'CCSDT', False),
    'small_ccsdt_open': (synth.SynthSpec(10, 6, 20, 0.04, 8), 'CCSDT', False),
    'small_ccsdtq': (synth.SynthSpec(8, 4, 16, 0.05, 9), 'CCSDTQ', False),
}
C2_CASES = {'c2_ccsdt': (synth.C2, 'CCSDT', True)}
CRCC_CASES = {
    'small_crcc23': (synth.SynthSpec(12, 8, 24, 0.05, 11), False),
    'c1_crcc23': (synth.C1, False),
}


def run_crcc(name, spec, rhf, tol=1e-10):
    """CCSD, left CCSD and the four CR-CC(2,3) corrections with the plan's numpy executor."""
    s = synth.system(spec)
    plan = os.path.join(ROOT, 'ccq_b200', 'plans', 'CRCC23' + ('_rhf' if rhf else '') + '.plan')
    t0 = time.time()
    bc = BlockCRCC(open(plan).read(), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'])
    e, it, failed, hist, tvec = bc.solve(tol=tol, max_iter=200)
    assert not failed
    el, itl, fl, hl = bc.solve_left(tvec, e, tol=tol, max_iter=200)
    assert not fl
    e23 = bc.crcc23(tvec)
    d = s['dims']
    return dict(spec=spec.__dict__, method='CR-CC(2,3)', rhf=rhf, occ_a=d.occ_a, occ_b=d.occ_b, e_cor=e,
                e_ref=s['e_ref'], iterations=it, tol=tol, left_iterations=itl, e_left=el,
                e23=[float(x) for x in e23], seconds=time.time() - t0,
                history=[h[0] for h in hist], left_history=[h[0] for h in hl])


def run(name, spec, method, rhf, tol=1e-10):
    s = synth.system(spec)
    if name.endswith('_open'):
        # open-shell variant: one alpha electron more than beta
        from ccq_b200 import integrals as I
        occ = spec.nel // 2
        fa, fb = I.fock(s['h'], s['e2'], occ, occ - 1)
        s['f_a'], s['f_b'] = fa, fb
        s['dims'] = I.Dims(0, occ, occ - 1, spec.norb)
        s['e_ref'] = I.hf_energy(s['h'], s['e2'], occ, occ - 1)
    plan = os.path.join(ROOT, 'ccq_b200', 'plans', method + ('_rhf' if rhf else '') + '.plan')
    t0 = time.time()
    bc = BlockCC(open(plan).read(), s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method)
    e, it, failed, hist, _ = bc.solve(tol=tol, max_iter=200)
    assert not failed
    d = s['dims']
    return dict(spec=spec.__dict__, method=method, rhf=rhf, occ_a=d.occ_a, occ_b=d.occ_b, e_cor=e,
                e_ref=s['e_ref'], iterations=it, tol=tol, seconds=time.time() - t0,
                history=[h[0] for h in hist])


def run_c3(tol=1e-8):
    """The 64 batched CCSD instances (ccq_b200.batch.c3_specs), each solved on its own."""
    from ccq_b200 import batch
    out = []
    t0 = time.time()
    plan = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CCSD.plan')).read()
    for spec in batch.c3_specs():
        s = synth.system(spec)
        bc = BlockCC(plan, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], 'CCSD')
        e, it, failed, hist, _ = bc.solve(tol=tol, max_iter=200)
        assert not failed
        out.append(dict(spec=spec.__dict__, e_cor=e, iterations=it))
    return dict(method='CCSD', tol=tol, instances=out, seconds=time.time() - t0)


def main():
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    cases = dict(CASES)
    if '--c2' in sys.argv:
        cases.update(C2_CASES)
    for name, (spec, method, rhf) in cases.items():
        if name in data and '--force' not in sys.argv:
            continue
        data[name] = run(name, spec, method, rhf)
        print(name, data[name]['e_cor'], data[name]['iterations'], f"{data[name]['seconds']:.1f}s", flush=True)
        json.dump(data, open(OUT, 'w'), indent=1)
    if 'c3_batched_ccsd' not in data or '--force' in sys.argv:
        data['c3_batched_ccsd'] = run_c3()
        print('c3_batched_ccsd', f"{data['c3_batched_ccsd']['seconds']:.1f}s", flush=True)
        json.dump(data, open(OUT, 'w'), indent=1)
    for name, (spec, rhf) in CRCC_CASES.items():
        if name in data and '--force' not in sys.argv:
            continue
        data[name] = run_crcc(name, spec, rhf)
        print(name, data[name]['e_cor'], data[name]['e23'], data[name]['iterations'], data[name]['left_iterations'],
              f"{data[name]['seconds']:.1f}s", flush=True)
        json.dump(data, open(OUT, 'w'), indent=1)


if __name__ == '__main__':
    main()
