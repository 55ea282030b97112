"""FCIDUMP reader: the native reader (C ABI, host path) equals the oracle's
restatement of load_fcidump bit for bit, and reproduces the H4 fixture's
integrals from a FCIDUMP holding only its unique integrals with shuffled
orbital labels (no GPU needed)."""
import numpy as np
import pytest

from ccq_b200 import config, driver, integrals as I, lib
from oracle import fcidump as ofci


def _h4_fcidump(path, h4, order=(2, 0, 3, 1)):
    # orbital p is written as label order[p] + 1; its energy p + 1 restores the order on read
    I.write_fcidump(path, h4['e1'], h4['e2'], h4['enuc'], nelec=4, eps=np.arange(1.0, 5.0), order=order)


def test_h4_roundtrip_native_and_oracle(tmp_path, h4):
    p = str(tmp_path / 'FCIDUMP')
    _h4_fcidump(p, h4)
    assert lib.fcidump_header(p) == (4, 4)
    assert ofci.header(p) == (4, 4)
    e1, e2, en = lib.fcidump_read(p, 4)
    o1, o2, oen = ofci.load(p, 4)
    np.testing.assert_array_equal(e1, o1)
    np.testing.assert_array_equal(e2, o2)
    assert en == oen == h4['enuc']
    # the eight-fold expansion of the unique integrals gives back every element of the fixture
    np.testing.assert_array_equal(e1, h4['e1'])
    np.testing.assert_array_equal(e2, h4['e2'])


def _write(path, text):
    with open(path, 'w') as fh:
        fh.write(text)


EDGE = """ &FCI NORB=  3,NELEC= 2,MS2=0,
  ORBSYM=1,1,1,
  ISYM=1,
 &END
  0.5D+00   1   1   1   1
  0.25  2 1
     2   1
 -0.125  3 3 1 1   trailing words are skipped
  0.75   2   2   2   2

  0.0625 1 2 1 3
  0.3    1   1   1   1
  -0.5   2   0   0   0
  -0.7   3   0   0   0
  -0.9   1   0   0   0
  -0.2   1   1   0   0
  0.1    3   2   0   0
  1.5    0   0   0   0
  not a record
  9.9    1   1   1   1
"""


def test_edge_cases_match_oracle(tmp_path):
    """D exponents, a record over two lines, trailing tokens, a blank line, a later record overwriting
    an earlier one, orbital renumbering by energy, the read stopping at a line that does not parse."""
    p = str(tmp_path / 'FCIDUMP')
    _write(p, EDGE)
    assert lib.fcidump_header(p) == (3, 2)
    e1, e2, en = lib.fcidump_read(p, 3)
    o1, o2, oen = ofci.load(p, 3)
    np.testing.assert_array_equal(e1, o1)
    np.testing.assert_array_equal(e2, o2)
    assert en == oen == 1.5
    # energies -0.9 (orbital 1), -0.5 (2), -0.7 (3): new order 1, 3, 2
    assert e2[0, 0, 0, 0] == 0.3               # the later (11|11) record wins; 9.9 is never read
    # (21|21) -> new 0-based (20|20): e2int(i,j,a,b) = e2[2,2,0,0] and its permutations
    assert e2[2, 2, 0, 0] == 0.25 and e2[0, 2, 2, 0] == 0.25 and e2[0, 0, 2, 2] == 0.25
    assert e2[1, 0, 1, 0] == -0.125            # (33|11) -> new 0-based (11|00) = e2[1,0,1,0]
    assert e2[2, 2, 2, 2] == 0.75
    assert e1[1, 2] == e1[2, 1] == 0.1 and e1[0, 0] == -0.2


def test_ties_keep_file_order_and_missing_energies(tmp_path):
    body = " &FCI NORB=3,NELEC=2,\n &END\n 1.0 1 1 1 1\n 2.0 2 2 2 2\n 3.0 3 3 3 3\n -1.0 3 0 0 0\n 0.0 0 0 0 0\n"
    p = str(tmp_path / 'FCIDUMP')
    _write(p, body)
    e1, e2, en = lib.fcidump_read(p, 3)
    o1, o2, _ = ofci.load(p, 3)
    np.testing.assert_array_equal(e2, o2)
    # orbital 3 (energy -1) comes first, orbitals 1 and 2 (energy 0) keep their order
    assert (e2[0, 0, 0, 0], e2[1, 1, 1, 1], e2[2, 2, 2, 2]) == (3.0, 1.0, 2.0)


@pytest.mark.parametrize('body,msg', [
    (" &FCI NORB=2,NELEC=2,\n 1.0 1 1 1 1\n", 'END'),
    (" &FCI NORB=2,NELEC=2,\n &END\n 1.0 3 1 1 1\n", 'outside'),
])
def test_errors(tmp_path, body, msg):
    p = str(tmp_path / 'FCIDUMP')
    _write(p, body)
    with pytest.raises(lib.CCQB200Error, match=msg):
        lib.fcidump_read(p, 2)


def test_missing_file_and_norb_mismatch(tmp_path):
    with pytest.raises(lib.CCQB200Error, match='not found'):
        lib.fcidump_header(str(tmp_path / 'nope'))
    p = str(tmp_path / 'FCIDUMP')
    _write(p, " &FCI NORB=2,NELEC=2,\n &END\n")
    with pytest.raises(lib.CCQB200Error, match='NORB'):
        lib.fcidump_read(p, 3)


def test_input_deck_with_fcidump_key(tmp_path, h4):
    """fcidump= replaces nel/nvirt of the deck by the header's (parser.f90:168-169) and the integrals."""
    _h4_fcidump(str(tmp_path / 'h4.fcidump'), h4)
    deck = tmp_path / 'input.inp'
    deck.write_text('nel=99\nnvirt=99\ncalc_type=CCSDT\nfcidump=h4.fcidump\n')
    cfg = config.parse(str(deck))
    config.apply_fcidump(cfg, str(tmp_path / 'h4.fcidump'))
    assert (cfg.nel, cfg.nvirt, cfg.orbs, cfg.occ_a, cfg.occ_b) == (4, 4, 4, 2, 2)
    sysd = driver.load_system(cfg.calc_macros(), str(tmp_path))
    np.testing.assert_array_equal(sysd['v_ab'], h4['v_ab'])
    assert sysd['e_ref'] == h4['e_ref']


def test_colliding_records_match_oracle(tmp_path):
    """Random records with repeats in every index order: each element keeps the last record's value."""
    n = 7
    rng = np.random.default_rng(5)
    idx = rng.integers(1, n + 1, size=(5000, 4))
    vals = rng.normal(size=5000)
    lines = [' &FCI NORB=7,NELEC=4,', ' &END']
    lines += [f'{v: .17E} {i} {a} {j} {b}' for v, (i, a, j, b) in zip(vals, idx.tolist())]
    lines += [f'{float(-k): .3f} {k} 0 0 0' for k in rng.permutation(np.arange(1, n + 1)).tolist()]
    p = str(tmp_path / 'FCIDUMP')
    _write(p, '\n'.join(lines) + '\n')
    e1, e2, en = lib.fcidump_read(p, n)
    o1, o2, oen = ofci.load(p, n)
    np.testing.assert_array_equal(e2, o2)
    assert np.count_nonzero(e2) > 0.9 * n ** 4
