"""Single-kernel probes for profiling (one GETT launch of a fixed shape).

    python -m ccq_b200.probe egemm K1 K2 K3 [repeats]
    python -m ccq_b200.probe egemm_split K1 K2 K3 [slices] [tile|persistent]
    python -m ccq_b200.probe sweep fp64|split OUTFILE [warm-up iterations] [0|1|2|3|tune]
    python -m ccq_b200.probe warmstart CCSDT|CCSDTQ NORB NEL [COUNT TRAIN EPOCHS]

Runs ccq_b200_egemm (the FP64 GETT kernel) on random column-major operands;
the vvvv ladder of the CCSDT T3 update at 40 orbitals is (1024, 16384, 1024).
"""
import sys
import time

import numpy as np


def main(argv):
    from ccq_b200 import lib
    kind = argv[0]
    if kind == 'egemm':
        k1, k2, k3 = (int(x) for x in argv[1:4])
        rep = int(argv[4]) if len(argv) > 4 else 1
        rng = np.random.default_rng(0)
        A = np.asfortranarray(rng.normal(size=(k3, k1)))
        B = np.asfortranarray(rng.normal(size=(k3, k2)))
        for _ in range(rep):
            t0 = time.perf_counter()
            C = lib.egemm(k1, k2, k3, A, B)
            dt = time.perf_counter() - t0
        ref = B[:, :64].T @ A[:, :64]
        err = float(np.abs(C[:64, :64] - ref).max())
        print(f'egemm {k1}x{k2}x{k3}: wall {dt * 1e3:.2f} ms (incl. copies), max err {err:.2e}')
        assert err < 1e-9
    elif kind == 'egemm_split':
        k1, k2, k3 = (int(x) for x in argv[1:4])
        S = int(argv[4]) if len(argv) > 4 else 4
        persistent = (argv[5] == 'persistent') if len(argv) > 5 else None
        rng = np.random.default_rng(0)
        A = np.asfortranarray(rng.normal(size=(k3, k1)))
        B = np.asfortranarray(rng.normal(size=(k3, k2)))
        for _ in range(3 if persistent is not None else 1):
            C = lib.egemm_split(k1, k2, k3, A, B, S, persistent=persistent)
        ref = B[:, :64].T @ A[:, :64]
        err = float(np.abs(C[:64, :64] - ref).max())
        # the split bound: 2^(-7S+2) k3 max|A| max|B|
        bound = 2.0 ** (-7 * S + 2) * k3 * np.abs(A[:, :64]).max() * np.abs(B[:, :64]).max()
        print(f'egemm_split {k1}x{k2}x{k3} S={S}: max err {err:.2e} (bound {bound:.2e})')
        assert err <= bound
    elif kind == 'sweep':
        # per-operation device times of one CCSDT sweep on the 40-orbital workload
        import os
        from ccq_b200 import synth
        prec = argv[1] if len(argv) > 1 else 'fp64'
        out = argv[2] if len(argv) > 2 else 'ops_profile.txt'
        warm = int(argv[3]) if len(argv) > 3 else 3
        family = argv[4] if len(argv) > 4 else '0'   # kernel family to force (0..3) or 'tune'
        s = synth.system(synth.C2)
        d = s['dims']
        # a one-vector DIIS ring keeps the device footprint small for profiler captures
        ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDT', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                          s['v_bb'], diis_space=1)
        ctx.set_precision(lib.PREC_SPLIT if prec == 'split' else lib.PREC_FP64, 4)
        if family == 'tune':
            print('autotune (ms before, after):', ctx.autotune(3))
        elif family != '0':
            ctx.force_tile(int(family))
        for it in range(1, warm + 1):
            ctx.iterate(it)
        if os.path.exists(out):
            os.remove(out)
        os.environ['CCQ_B200_PROFILE_DUMP'] = out
        ctx.profile(True)
        ctx.iterate(warm + 1)
        print(ctx.profile_get())
        ctx.close()
    elif kind == 'warmstart':
        # the learned warm start on a lambda-swept family: METHOD NORB NEL [COUNT TRAIN EPOCHS]
        import json
        from ccq_b200 import warmstart
        method, norb, nel = argv[1], int(argv[2]), int(argv[3])
        count = int(argv[4]) if len(argv) > 4 else 200
        train = int(argv[5]) if len(argv) > 5 else 150
        epochs = int(argv[6]) if len(argv) > 6 else 600
        r = warmstart.study(method, norb, nel, count, train, epochs=epochs, log=print)
        print(json.dumps(r))
    else:
        raise SystemExit(f'unknown probe {kind}')


if __name__ == '__main__':
    main(sys.argv[1:])
