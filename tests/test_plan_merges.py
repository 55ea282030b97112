"""The committed plans are what the plan compiler generates, with its two merges applied.

The shared-operand merge (one large product for the GETTs that add into one output with the same amplitude
operand) and the equal-view merge (one Z buffer per class of equal assemble view sets) are pinned
semantically by tests/test_plan.py and tests/test_runtime_semantics.py; this checks that the embedded CCSD and
CCSDT plans are the compiler's current output and keeps their sizes from drifting back.
"""
import os

from ccq_b200.eqgen.plan import build_plan, plan_flops

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _committed(name):
    return open(os.path.join(HERE, 'ccq_b200', 'plans', name + '.plan')).read()


def test_committed_plans_equal_the_compiler_output():
    for method in ('CCSD', 'CCSDT'):
        for rhf in (False, True):
            name = method + ('_rhf' if rhf else '')
            assert build_plan(method, rhf).text() == _committed(name), name


def test_ccsdt_plan_sizes():
    b = build_plan('CCSDT', False)
    assert plan_flops(b) < 1.95e11          # 2.71e11 before the shared-operand merge
    text = b.text()
    assert text.count('\nBUF Z') == 55      # 94 before the equal-view merge
    asm = {l.split()[1]: int(l.split()[3]) for l in text.split('\n') if l.startswith('ASSEMBLE')}
    assert asm['T3B'] == 14 and asm['T3C'] == 14   # 57 gathered views each before
