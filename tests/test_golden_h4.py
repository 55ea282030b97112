"""H4/STO-3G known answers of the reference's own tests (tests/test_small.py:40-50).

The integral fixture (tools/ccq_py/{onebody,twobody}.inp) stores ERIs to 10
decimals, so every total energy sits 2.3e-10 Eh below the published one; the
offset is the same for the reference energy and cancels in E_corr.
"""
import numpy as np
import pytest

from oracle.blockcc import BlockCC
from oracle.densecc import DenseCC
from oracle.detcc import DetCC
from oracle.spinorb import SpinOrbitalSystem

E_REF = -1.858240957484
E_CCSDT = -1.978696408825
E_CCSDTQ = -1.975861644132
FIXTURE_OFFSET = 2.3e-10


def test_reference_energy(h4):
    assert abs(h4['e_ref'] - E_REF) < FIXTURE_OFFSET + 1e-11


def test_ccsdtq_is_fci(h4):
    # four electrons: CCSDTQ == FCI, computed here by diagonalisation
    so = SpinOrbitalSystem(h4['f_a'], h4['f_b'], h4['v_aa'], h4['v_ab'], h4['v_bb'], 2, 2)
    e_fci = DetCC(so.h, so.v, so.O).fci_energy() + h4['e_ref']
    assert abs(e_fci - E_CCSDTQ) < FIXTURE_OFFSET + 1e-11


@pytest.mark.parametrize('rhf', [True, False])
def test_ccsdt_dense_oracle(h4, rhf):
    cc = DenseCC(h4['f_a'], h4['f_b'], h4['v_aa'], h4['v_ab'], h4['v_bb'], h4['dims'], 'CCSDT', rhf=rhf)
    e, it, failed, hist, _ = cc.solve(tol=1e-11, max_iter=60)
    assert not failed
    assert abs(e + h4['e_ref'] - E_CCSDT) < FIXTURE_OFFSET + 1e-11


@pytest.mark.parametrize('method,gold', [('CCSDT', E_CCSDT), ('CCSDTQ', E_CCSDTQ)])
def test_block_plan_oracle(h4, method, gold, plan_text):
    txt = plan_text(method, False)
    bc = BlockCC(txt, h4['f_a'], h4['f_b'], h4['v_aa'], h4['v_ab'], h4['v_bb'], h4['dims'], method)
    e, it, failed, hist, _ = bc.solve(tol=1e-11, max_iter=80)
    assert not failed
    assert abs(e + h4['e_ref'] - gold) < FIXTURE_OFFSET + 1e-11
