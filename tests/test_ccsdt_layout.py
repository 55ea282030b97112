"""ccq's compressed CCSDt T vector: the C ABI converters against the numpy restatement of
get_t_sizes_act and the sub-block declarations (no GPU needed)."""
import numpy as np
import pytest

from ccq_b200 import integrals as I, lib
from oracle import ccsdt_layout as L
from oracle.densecc import active_mask
from oracle import solver as S

CASES = [(0, 4, 3, 10, 2, 6), (1, 4, 4, 10, 2, 7), (0, 3, 3, 8, 1, 4), (0, 5, 4, 9, 3, 9), (0, 4, 2, 8, 0, 4)]


def _active_t(dims, m1, m2, seed):
    """A full T vector with the reference's antisymmetry, zero outside the active triples."""
    froz, occ_a, occ_b, orbs = dims
    d = I.Dims(froz, occ_a, occ_b, orbs)
    lay = I.TLayout(d)
    rng = np.random.default_rng(seed)
    t = np.zeros(lay.t_size)
    for b in I.T_VEC_ORDER:
        if not lay.size(b):
            continue
        v = S.antisym_fill(b, rng.normal(0, 0.1, lay.shape[b]))
        if b[1] == '3':
            v = np.where(active_mask(b, v.shape, d, (m1, m2)), v, 0.0)
        lay.view(t, b)[...] = v
    return t


@pytest.mark.parametrize('dims_act', CASES)
def test_sizes_follow_get_t_sizes_act(dims_act):
    dims, (m1, m2) = dims_act[:4], dims_act[4:]
    pos = L.pos_offsets(*dims, m1, m2)
    assert lib.t_size_act(*dims, m1, m2) == pos[-1] - 1
    # the sub-block sizes of the declarations match the pos() differences
    full, subs = L.ranges(*dims, m1, m2)
    sizes = [int(np.prod([L._n(r) for r in rr])) for _, rr in subs]
    assert sizes == [pos[k + 1] - pos[k] for k in range(5, 15)]


@pytest.mark.parametrize('dims_act', CASES)
def test_compress_expand_match_oracle_and_round_trip(dims_act):
    dims, (m1, m2) = dims_act[:4], dims_act[4:]
    t = _active_t(dims, m1, m2, seed=sum(dims_act))
    c = lib.t_compress(dims, m1, m2, t)
    np.testing.assert_array_equal(c, L.compress(t, dims, m1, m2))
    back = lib.t_expand(dims, m1, m2, c, t.size)
    np.testing.assert_array_equal(back, t)
    np.testing.assert_array_equal(L.expand(c, dims, m1, m2), t)


def test_compressed_element_positions():
    """Spot checks straight from the declarations: t3B1(c,b,a,k,j,i) with a active and i active."""
    dims, m1, m2 = (0, 4, 3, 10), 2, 6
    froz, N1, N2, N3 = dims
    t = _active_t(dims, m1, m2, seed=3)
    c = lib.t_compress(dims, m1, m2, t)
    pos = L.pos_offsets(*dims, m1, m2)
    lay = I.TLayout(I.Dims(*dims))
    t3b = lay.view(t, 'T3B')     # C-order [i][j][k][a][b][c] = Fortran t3b(c,b,a,k,j,i)
    shp = (N3 - N2, N3 - N1, m2 - N1, N2 - froz, N1 - froz, N1 - m1)   # t3B1's extents
    for (cc, b, a, k, j, i) in [(0, 0, 0, 0, 0, 0), (3, 2, 1, 2, 3, 1), (6, 5, 0, 1, 2, 0)]:
        off = cc + shp[0] * (b + shp[1] * (a + shp[2] * (k + shp[3] * (j + shp[4] * i))))
        # global Fortran indices: a from N1+1, i from M1+1
        assert c[pos[6] - 1 + off] == t3b[i + (m1 - froz), j, k, a, b, cc]


def test_bad_arguments():
    dims = (0, 4, 3, 10)
    with pytest.raises(lib.CCQB200Error):
        lib.t_size_act(*dims, 5, 6)      # act_occ_b above occ_b
    with pytest.raises(lib.CCQB200Error):
        lib.t_compress(dims, 2, 6, np.zeros(7))


def test_compressed_diis_of_the_oracle():
    """DIIS over ccq's compressed vector: with every orbital active the compressed vector is the full one
    (the same solve); with a partial active space the solve reaches the masked full-DIIS energy."""
    from oracle.densecc import DenseCC
    from tests.helpers import random_system
    s = random_system(5, 3, 2, seed=29, sigma=0.08)
    d = s['dims']
    cc = lambda act: DenseCC(s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d, 'CCSDT', active=act)  # noqa
    full = (d.froz, d.orbs)
    e1, it1, f1, _, _ = cc(full).solve(tol=1e-10, max_iter=100)
    e2, it2, f2, _, _ = cc(full).solve(tol=1e-10, max_iter=100, compressed_diis=True)
    assert not f1 and not f2 and it1 == it2 and abs(e1 - e2) < 1e-12
    act = (d.occ_b - 1, d.occ_a + 1)
    e3, _, f3, _, _ = cc(act).solve(tol=1e-10, max_iter=100)
    e4, _, f4, _, _ = cc(act).solve(tol=1e-10, max_iter=100, compressed_diis=True)
    assert not f3 and not f4 and abs(e3 - e4) < 1e-9
