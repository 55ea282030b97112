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
    # CCSDt without an active space is a configuration error (src/parser.f90:251-254)
    c = config.Config(calc_type='CCSDt')
    with pytest.raises(ValueError):
        c.calc_macros()
    with pytest.raises(ValueError, match='not served'):
        config.Config(calc_type='stoch-CC').calc_macros()


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


def test_acc_keys_parsed(tmp_path):
    # get_acc_opts (src/parser.f90:527-542): list-directed reals, blanks or commas
    p = tmp_path / 'x.inp'
    p.write_text('nel=4\nnvir=4\ncalc_type=CCSD\nt2t2_t2=1.0, 0.0 0.5,0.5 0\nt3_t2=1d0 0.5D0\n')
    c = config.parse(str(p)).calc_macros()
    assert c.acc['t2t2_t2'] == [1.0, 0.0, 0.5, 0.5, 0.0]
    assert c.acc['t3_t2'] == [1.0, 0.5]
    assert c.acc['t1t3_t2'] == [1.0] * 4 and not c.acc_default()
    p.write_text('nel=4\nnvir=4\ncalc_type=CCSD\nt2t3_t3=1 1\n')
    with pytest.raises(ValueError):
        config.parse(str(p))


def test_acc_defaults_and_dcsd_macro():
    c = config.Config(calc_type='CCSD').calc_macros()
    assert c.acc_default()
    # DCSD-MC sets t2t2_t2 after the keys are read (src/parser.f90:350-358)
    c = config.Config(calc_type='DCSD-MC').calc_macros()
    assert c.acc['t2t2_t2'] == [1.0, 0.0, 0.5, 0.5, 0.0] and not c.acc_default()


def test_run_keys(tmp_path):
    p = tmp_path / 'x.inp'
    p.write_text('nel=4\nnvir=4\ncalc_type=CCSD\nlvl_t=.true.\nsorted_ints=.true.\necho\noutput_log=o.log\n')
    c = config.parse(str(p)).calc_macros()
    # lvl_t is read and checked, then get_calc_macros decides (src/parser.f90:360-366)
    assert c.lvl_t_key and not c.lvl_t and c.sorted_ints and c.echo and c.output_log == 'o.log'
    p.write_text('nel=4\nnvir=4\ncalc_type=CCSD\nlvl_q=maybe\n')
    with pytest.raises(ValueError, match='lvl_q must logical'):
        config.parse(str(p))


def test_acc_factors_refused_by_driver(tmp_path):
    # a deck whose ACC factors differ from 1.0 must not run as plain CC
    from ccq_b200 import driver
    p = tmp_path / 'x.inp'
    p.write_text('nel=4\nnvir=4\ncalc_type=CCSDT\nt3_t2=0.0 1.0\n')
    with pytest.raises(ValueError, match='ACC diagram factors'):
        driver.run(str(p), out=lambda x: None, base_dir=str(tmp_path))
    p.write_text('nel=4\nnvir=4\ncalc_type=DCSD-MC\next_cor_file=w\n')
    with pytest.raises(ValueError, match='ACC diagram factors'):
        driver.run(str(p), out=lambda x: None, base_dir=str(tmp_path))
