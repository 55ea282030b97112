"""Input deck, integral files and T-vector layout (parser.f90, integrals.f90, cc_utils.f90)."""
import numpy as np
import pytest

from ccq_b200 import config, integrals as I, synth


def test_parser_semantics(tmp_path):
    p = tmp_path / 'x.inp'
    p.write_text('# comment line\nfroz=2\nnel=10\nnvir=30  \n! other\nrhf=.true.\n'
                 'tol=-8\nshift=0.12\ncalc_type=CCSDT\nrestart\nkey=1 # inline comment skips the line\n')
    c = config.parse(str(p)).calc_macros()
    assert c.froz == 1 and c.occ_a == 5 and c.occ_b == 5 and c.orbs == 20
    assert c.rhf and c.tol == 1e-8 and c.shift == 0.12 and c.restart
    assert c.lvl_t and not c.lvl_q
    assert 'key' not in c.extra


def test_tol_real_and_multiplicity(tmp_path):
    p = tmp_path / 'x.inp'
    p.write_text('nel=6\nnvir=10\nmult=3\ntol=1.0e-7\ncalc_type=CCSD\n')
    c = config.parse(str(p))
    assert c.tol == 1e-7 and c.occ_a == 3 and c.occ_b == 2


def test_defaults():
    c = config.Config()
    assert c.diis_space == 5 and c.max_iter == 60 and c.tol == 1e-4 and c.shift == 0.0 and not c.rhf


def test_unknown_calc_type():
    # active-space CCSDt stays on the reference's CPU program
    c = config.Config(calc_type='CCSDt')
    with pytest.raises(ValueError):
        c.calc_macros()


def test_crcc23_macros():
    c = config.Config(calc_type='CR-CC(2,3)').calc_macros()
    assert not c.lvl_t and not c.lvl_q


def test_integral_round_trip(tmp_path):
    h, e2, enuc = synth.generate(synth.SynthSpec(6, 4, 12, 0.05, 3))
    I.write_onebody(str(tmp_path / 'one.inp'), h)
    I.write_twobody(str(tmp_path / 'two.inp'), e2, 0.5)
    h2 = I.read_onebody(str(tmp_path / 'one.inp'), 6)
    e22, en = I.read_twobody(str(tmp_path / 'two.inp'), 6)
    np.testing.assert_allclose(h2, h, atol=1e-15)
    np.testing.assert_allclose(e22, e2, atol=1e-15)
    assert en == 0.5


def test_onebody_count_check(tmp_path):
    h, e2, _ = synth.generate(synth.SynthSpec(6, 4, 12, 0.05, 3))
    I.write_onebody(str(tmp_path / 'one.inp'), h)
    with pytest.raises(ValueError):
        I.read_onebody(str(tmp_path / 'one.inp'), 5)


def test_synthetic_fock_is_diagonal():
    s = synth.SynthSpec(10, 4, 20, 0.05, 1)
    h, e2, _ = synth.generate(s)
    fa, fb = I.fock(h, e2, 2, 2)
    assert np.abs(fa - np.diag(np.diag(fa))).max() < 1e-14
    d = np.diag(fa)
    assert np.all(d[:2] < -0.4) and np.all(d[2:] > 0.1)


def test_t_layout_matches_get_t_sizes():
    dims = I.Dims(0, 8, 7, 40)
    lay = I.TLayout(dims)
    oa, ob, va, vb = 8, 7, 32, 33
    sizes = [oa * va, ob * vb, oa ** 2 * va ** 2, oa * ob * va * vb, ob ** 2 * vb ** 2,
             oa ** 3 * va ** 3, oa ** 2 * ob * va ** 2 * vb, oa * ob ** 2 * va * vb ** 2, ob ** 3 * vb ** 3]
    assert lay.pos == list(np.cumsum([1] + sizes))
    assert lay.vec_size('CCSD') == sum(sizes[:5])
    assert lay.vec_size('CCSDT') == lay.t_size


def test_spin_blocks_antisymmetric():
    h, e2, _ = synth.generate(synth.SynthSpec(6, 4, 12, 0.05, 3))
    vaa, vab, vbb = I.spin_blocks(e2, 0)
    np.testing.assert_allclose(vaa, -vaa.transpose(1, 0, 2, 3), atol=1e-15)
    np.testing.assert_allclose(vaa, -vaa.transpose(0, 1, 3, 2), atol=1e-15)
    np.testing.assert_allclose(vab, vab.transpose(2, 3, 0, 1), atol=1e-15)
