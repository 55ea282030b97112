"""CAD-FCIQMC on the GPU: a walker file holding an exact FCI state, read and
cluster-analysed by the native reader, gives T3 and T4 that, held fixed while
T1 and T2 iterate on the CCSDTQ plan, reproduce the FCI energy; on H4 that is
the reference's known answer for calc_type=CADFCIQMC."""
import numpy as np
import pytest

from ccq_b200 import driver, integrals as I
from oracle import walkers as W
from oracle.spinorb import SpinOrbitalSystem
from tests.helpers import fci_state, random_system

pytestmark = pytest.mark.gpu


def _run(tmp_path, e1, e2, enuc, so, nel, nvirt, extra=''):
    psi, e_fci = fci_state(so)
    W.write(str(tmp_path / 'walkers.dat'), so, 1000.0 * psi)
    I.write_onebody(str(tmp_path / 'onebody.inp'), e1)
    I.write_twobody(str(tmp_path / 'twobody.inp'), e2, enuc)
    (tmp_path / 'in.inp').write_text(f'nel={nel}\nnvirt={nvirt}\ncalc_type=CADFCIQMC\next_cor_file=walkers.dat\n'
                                     'keep_bin=.false.\n' + extra)
    lines = []
    r = driver.run(str(tmp_path / 'in.inp'), out=lines.append, base_dir=str(tmp_path))
    assert not r.failed
    return r, e_fci, lines


def test_h4_known_answer(tmp_path, h4):
    # the reference's CADFCIQMC input for this system (tests/h4_sto3g/CADFCIQMC.inp)
    so = SpinOrbitalSystem(h4['f_a'], h4['f_b'], h4['v_aa'], h4['v_ab'], h4['v_bb'], 2, 2)
    r, e_fci, lines = _run(tmp_path, h4['e1'], h4['e2'], h4['enuc'], so, 4, 4,
                           'tol=1.0e-11\ndiis_space=8\nmax_iterations=80\nshift=0.12\n')
    assert abs(r.e_cor - e_fci) < 1e-9
    # known answer of the reference's tests/test_small.py (the fixture's 10-decimal ERIs: 2.3e-10 offset)
    assert abs(r.e_total - (-1.975861644132)) < 5e-10
    assert any('External correlation energy' in l for l in lines)


@pytest.mark.parametrize('n,oa,froz,sd', [(5, 2, 0, True), (6, 3, 1, False)])
def test_exact_state_gives_fci(tmp_path, n, oa, froz, sd):
    s = random_system(n, oa, oa, seed=41, sigma=0.12, froz=froz)
    d = s['dims']
    so = SpinOrbitalSystem(s['f_a'][froz:, froz:], s['f_b'][froz:, froz:], s['v_aa'], s['v_ab'], s['v_bb'],
                           d.oa, d.ob)
    extra = f'froz={2 * froz}\ntol=1.0e-11\nmax_iterations=100\n' + ('' if sd else 'ext_cor_sd=.false.\n')
    r, e_fci, _ = _run(tmp_path, s['h'], s['e2'], 0.0, so, 2 * oa, 2 * (n - oa), extra)
    assert abs(r.e_cor - e_fci) < 1e-9
