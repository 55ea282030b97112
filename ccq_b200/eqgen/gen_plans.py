"""Regenerate the committed contraction plans (``ccq_b200/plans/*.plan``).

    python -m ccq_b200.eqgen.gen_plans [CCSD CCSDT CCSDTQ CR-CC(2,3)]

CCSDTQ takes several minutes (the level-4 antisymmetriser search).
"""
import os
import sys

from .plan import build_plan, plan_flops

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FILE_NAME = {'CR-CC(2,3)': 'CRCC23'}   # plan file / embedded name of a calc_type


def main(methods):
    out = os.path.join(HERE, 'plans')
    os.makedirs(out, exist_ok=True)
    for m in methods:
        for rhf in (False, True):
            p = build_plan(m, rhf, workers=os.cpu_count())
            name = FILE_NAME.get(m, m) + ('_rhf' if rhf else '')
            with open(os.path.join(out, name + '.plan'), 'w') as fh:
                fh.write(p.text())
            print(name, len(p.ops), 'ops', f'{plan_flops(p):.3e} FLOP per sweep at 40 orbitals', flush=True)


if __name__ == '__main__':
    main(sys.argv[1:] or ['CCSD', 'CCSDT', 'CCSDTQ', 'CR-CC(2,3)'])
