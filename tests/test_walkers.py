"""FCIQMC walker files (calc_type=CADFCIQMC) on the CPU: the native reader and
cluster analysis (C ABI, host path) against the exact cluster amplitudes of an
FCI state and against the Fock-space oracle, plus the file's edge cases.

The FCI state is written in the walker format by oracle.walkers; the native
reader applies the reference's excitation_sign_qmc parity and a cluster
formula, the oracle the inverse reordering and exp(T) in Fock space, and the
truth is tests.helpers.fci_cluster_amplitudes (no file at all)."""
import numpy as np
import pytest

from ccq_b200 import config, driver, integrals as I, lib
from oracle import walkers as W
from oracle.spinorb import SpinOrbitalSystem
from tests.helpers import fci_cluster_amplitudes, fci_state, random_system

ALL = I.T_VEC_ORDER + I.T4_ORDER


def _so(n, oa, ob, froz, seed=3):
    s = random_system(n, oa, ob, seed=seed, sigma=0.15, froz=froz)
    d = s['dims']
    fz = d.froz
    so = SpinOrbitalSystem(s['f_a'][fz:, fz:], s['f_b'][fz:, fz:], s['v_aa'], s['v_ab'], s['v_bb'], d.oa, d.ob)
    return s, d, so


def _native(path, d, **kw):
    t, t4, info = lib.walkers_read(path, d.froz, d.occ_a, d.occ_b, d.orbs, d.occ_a + d.occ_b, **kw)
    lay = I.TLayout(d)
    out = {b: lay.view(t, b) for b in I.T_VEC_ORDER}
    if t4:
        out.update(t4)
    return out, info


@pytest.mark.parametrize('n,oa,ob,froz', [(4, 2, 2, 0), (5, 3, 2, 0), (6, 3, 3, 1)])
def test_fci_state_gives_exact_cluster_amplitudes(tmp_path, n, oa, ob, froz):
    s, d, so = _so(n, oa, ob, froz)
    psi, _ = fci_state(so)
    p = str(tmp_path / 'walkers')
    W.write(p, so, -2.5 * psi)      # any normalisation and sign of the walker populations
    ts, _ = fci_cluster_amplitudes(so, 4)
    truth = so.to_blocks(ts, ALL)
    got, info = _native(p, d)
    assert abs(abs(info['c_hf']) - 2.5) < 1e-14
    for b in ALL:
        np.testing.assert_allclose(got[b], truth[b], atol=1e-14, rtol=0, err_msg=b)
    assert max(np.abs(truth[b]).max() for b in ('T3A', 'T3B', 'T3C', 'T3D')) > 1e-4
    if oa + ob - 2 * froz >= 4:
        assert max(np.abs(truth[b]).max() for b in I.T4_ORDER) > 1e-5
    orc = W.cluster_blocks(so, W.read(p, so, so.O))
    for b in ALL:
        np.testing.assert_allclose(orc[b], truth[b], atol=1e-14, rtol=0, err_msg=b)


def test_sparse_walker_list_matches_oracle(tmp_path):
    """A stochastic-looking list: a random subset of determinants, some repeated (triples keep the last
    value, quadruples add up), records split over two lines, quintuples and a trailing line that ends
    the read."""
    s, d, so = _so(6, 3, 2, 0, seed=9)
    rng = np.random.default_rng(4)
    ref = (1 << so.O) - 1
    # the Ms sector of the reference, about 60 % of it populated
    amask = sum(1 << P for P in range(so.N) if so.spin[P] == 0)
    states = np.arange(1 << so.N)
    sector = [x for x in states if bin(int(x)).count('1') == so.O and
              bin(int(x) & amask).count('1') == bin(ref & amask).count('1')]
    psi = np.zeros(1 << so.N)
    psi[sector] = 0.1 * rng.normal(size=len(sector))
    keep = np.zeros_like(psi)
    nz = np.array(sector)
    pick = nz[rng.random(nz.size) < 0.6]
    keep[pick] = psi[pick]
    keep[ref] = 7.0
    p = str(tmp_path / 'walkers')
    W.write(p, so, keep)
    lines = open(p).read().splitlines()
    # repeat two records with new populations, and split one record over two lines
    extra = []
    for x in (nz[nz != ref][:40]):
        lvl = bin(int(x) ^ ref).count('1') // 2
        if lvl in (3, 4) and len(extra) < 4:
            tmp = str(tmp_path / 'one')
            one = np.zeros_like(psi)
            one[x] = 0.25 * (1 + len(extra))
            W.write(tmp, so, one)
            extra.append(open(tmp).read().strip())
    head, tail = lines[5].split(' ', 2)[:2], lines[5].split(' ', 2)[2]
    lines[5] = ' '.join(head) + '\n   ' + tail
    lines += extra + ['99 1.0 1 2', 'not a record', '5 0.5 1 2 3 4 5 6']
    with open(p, 'w') as fh:
        fh.write('\n'.join(lines) + '\n')
    got, info = _native(p, d)
    assert info['records'] > 100 and info['quadruples'] > 0
    orc = W.cluster_blocks(so, W.read(p, so, so.O))
    for b in ALL:
        np.testing.assert_allclose(got[b], orc[b], atol=1e-13, rtol=0, err_msg=b)
    assert abs(info['c_hf']) == 7.0
    assert info['higher'] > 0


def test_without_singles_and_doubles(tmp_path):
    s, d, so = _so(5, 3, 2, 0)
    psi, _ = fci_state(so)
    p = str(tmp_path / 'walkers')
    W.write(p, so, psi)
    full, _ = _native(p, d)
    t3only, _ = _native(p, d, with_sd=False)
    for b in I.T_VEC_ORDER:
        if int(b[1]) < 3:
            assert not np.any(t3only[b])
        else:
            np.testing.assert_array_equal(t3only[b], full[b])


@pytest.mark.parametrize('body,msg', [
    ('1 0.5 1 2 3 6\n', 'Hartree-Fock'),
    ('1 1.0 1 2 3 4\n2 0.1 1 2 3 5\n', 'Ms'),
    ('1 1.0 1 2 3 4\n2 0.1 1 2 3 40\n', 'outside'),
    ('1 1.0 1 2 3 4\n2 0.1 1 2 3 3\n', 'twice'),
])
def test_errors(tmp_path, body, msg):
    p = str(tmp_path / 'walkers')
    with open(p, 'w') as fh:
        fh.write(body)
    d = I.Dims(0, 2, 2, 5)
    with pytest.raises(lib.CCQB200Error, match=msg):
        lib.walkers_read(p, d.froz, d.occ_a, d.occ_b, d.orbs, 4)
    with pytest.raises(lib.CCQB200Error, match='not found'):
        lib.walkers_read(str(tmp_path / 'nope'), 0, 2, 2, 5, 4)


def test_input_deck_keys(tmp_path):
    deck = ['nel=4\n', 'nvirt=6\n', 'calc_type=CADFCIQMC\n', 'ext_cor_file=w.dat\n', 'ext_cor_sd=.false.\n']
    cfg = config.parse_lines(deck)
    cfg.calc_macros()
    assert cfg.ext_cor_file == 'w.dat' and cfg.ext_cor_sd is False and not cfg.lvl_t
    # the walker file is checked before any device work (src/parser.f90:236-239)
    (tmp_path / 'in.inp').write_text(''.join(deck))
    I.write_onebody(str(tmp_path / 'onebody.inp'), np.eye(5))
    I.write_twobody(str(tmp_path / 'twobody.inp'), np.zeros((5, 5, 5, 5)), 0.0)
    with pytest.raises(ValueError, match='Walkers file not found'):
        driver.run(str(tmp_path / 'in.inp'), out=lambda x: None, base_dir=str(tmp_path))
    (tmp_path / 'w.dat').write_text('1 1.0 1 2 3 4\n')
    (tmp_path / 'in.inp').write_text(''.join(deck) + 'ext_cor_file_h5\n')
    with pytest.raises(ValueError, match='HDF5'):
        driver.run(str(tmp_path / 'in.inp'), out=lambda x: None, base_dir=str(tmp_path))


def test_reader_output_drives_external_cc_to_fci(tmp_path):
    """The reader's t_vec and T4 blocks, as the CADFCIQMC driver passes them to the context, make the
    oracle's externally corrected CCSDTQ (T3, T4 fixed) converge to the FCI energy."""
    from oracle.densecc import DenseCC
    s, d, so = _so(5, 2, 2, 0, seed=41)
    psi, e_fci = fci_state(so)
    p = str(tmp_path / 'walkers')
    W.write(p, so, psi)
    t, t4, _ = lib.walkers_read(p, d.froz, d.occ_a, d.occ_b, d.orbs, d.occ_a + d.occ_b)
    dc = DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDTQ', external=True)
    dc.t4 = {b: v.copy() for b, v in t4.items()}
    e, it, failed, _, _ = dc.solve(tol=1e-12, max_iter=200, t0=t)
    assert not failed and abs(e - e_fci) < 1e-10
