"""Mid-size open-shell, frozen-core and rhf solves with the plan-independent dense oracle.

    python tests/golden/make_dense.py [--force]

Writes dense_midsize.json (converged energies, iteration counts and the
iteration history) and dense_sweep_ccsdtq.npz (one CCSDTQ sweep from seeded
random amplitudes).  The oracle is oracle/densecc.py: the generated equations
evaluated on dense spin-orbital tensors (no spin integration, no contraction
plan) with ccq's block-sequential sweep, Jacobi rule, DIIS and convergence
test.  The systems have at least three alpha holes, so the alpha-alpha-alpha
triples (and for CCSDTQ the T4B/T4C/T4D quadruples) are not empty.
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.densecc import DenseCC  # noqa: E402
from tests.helpers import random_system, random_t  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, 'dense_midsize.json')
SWEEP = os.path.join(HERE, 'dense_sweep_ccsdtq.npz')

# name: (method, n, occ_a, occ_b, froz, rhf, seed, sigma, shift)
CASES = {
    'ccsdt_open_n10': ('CCSDT', 10, 4, 3, 0, False, 31, 0.08, 0.0),
    'ccsdt_froz_n10': ('CCSDT', 10, 4, 4, 1, False, 32, 0.08, 0.0),
    'ccsdt_rhf_n10': ('CCSDT', 10, 4, 4, 0, True, 33, 0.08, 0.0),
    'ccsdtq_open_n7': ('CCSDTQ', 7, 4, 3, 0, False, 34, 0.08, 0.0),
}
SWEEP_CASE = ('CCSDTQ', 7, 4, 3, 0, False, 35, 0.08, 0.05)


def system(case):
    method, n, oa, ob, froz, rhf, seed, sigma, shift = case
    return random_system(n, oa, ob, seed=seed, sigma=sigma, froz=froz)


def solve(case, tol=1e-10):
    method, n, oa, ob, froz, rhf, seed, sigma, shift = case
    s = system(case)
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method, shift=shift, rhf=rhf)
    t0 = time.time()
    e, it, failed, hist, _ = dc.solve(diis_space=5, max_iter=100, tol=tol)
    assert not failed
    return dict(method=method, n=n, occ_a=oa, occ_b=ob, froz=froz, rhf=rhf, seed=seed, sigma=sigma, shift=shift,
                tol=tol, e_cor=e, iterations=it, history=[h[0] for h in hist], seconds=time.time() - t0)


def sweep():
    method, n, oa, ob, froz, rhf, seed, sigma, shift = SWEEP_CASE
    s = system(SWEEP_CASE)
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], method, shift=shift, rhf=rhf)
    t, t4 = random_t(s['dims'], seed=5, scale=0.03, nmax=4)
    dc.t4 = {k: v.copy() for k, v in t4.items()}
    tv = t.copy()
    dc.update(tv)
    out = {'t_in': t, 't_out': tv, 'energy': np.array(dc.energy(tv))}
    for k in t4:
        out[k + '_in'] = t4[k]
        out[k + '_out'] = dc.t4[k]
    np.savez_compressed(SWEEP, **out)


def main():
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    only = [a for a in sys.argv[1:] if not a.startswith('--')]
    for name, case in CASES.items():
        if only and name not in only:
            continue
        if name in data and '--force' not in sys.argv:
            continue
        data[name] = solve(case)
        print(name, data[name]['e_cor'], data[name]['iterations'], f"{data[name]['seconds']:.0f}s", flush=True)
        cur = json.load(open(OUT)) if os.path.exists(OUT) else {}
        cur[name] = data[name]
        json.dump(cur, open(OUT, 'w'), indent=1)
    if (not only or 'sweep' in only) and (not os.path.exists(SWEEP) or '--force' in sys.argv):
        sweep()
        print('sweep written', flush=True)


if __name__ == '__main__':
    main()
