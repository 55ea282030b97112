import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200) and libccq_b200.so')
    config.addinivalue_line('markers', 'slow: long CPU oracle run')


@pytest.fixture(scope='session')
def h4():
    from ccq_b200 import integrals as I
    d = os.path.join(GOLDEN, 'h4_sto3g')
    e1 = I.read_onebody(os.path.join(d, 'onebody.inp'), 4)
    e2, enuc = I.read_twobody(os.path.join(d, 'twobody.inp'), 4)
    fa, fb = I.fock(e1, e2, 2, 2)
    vaa, vab, vbb = I.spin_blocks(e2, 0)
    return dict(e1=e1, e2=e2, enuc=enuc, f_a=fa, f_b=fb, v_aa=vaa, v_ab=vab, v_bb=vbb,
                dims=I.Dims(0, 2, 2, 4), e_ref=I.hf_energy(e1, e2, 2, 2) + enuc)


@pytest.fixture(scope='session')
def plan_text():
    def get(method, rhf):
        p = os.path.join(ROOT, 'ccq_b200', 'plans', method + ('_rhf' if rhf else '') + '.plan')
        if not os.path.exists(p):
            pytest.skip(f'{p} not generated')
        return open(p).read()
    return get
