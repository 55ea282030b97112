"""Warm-start network: CPU oracle self-check, features and sample assembly (no GPU)."""
import numpy as np

from ccq_b200 import synth, warmstart
from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    F = warmstart.NFEAT
    p = rng.normal(0, 0.3, 32 * F + 32 + 32 * 32 + 32 + 32 + 1)
    X = rng.normal(size=(40, F))
    T = rng.normal(size=40)
    loss, g = mlp.loss_and_grad(p, X, T)
    for k in rng.choice(p.size, 25, replace=False):
        d = np.zeros_like(p)
        d[k] = 1e-6
        fd = (mlp.loss_and_grad(p + d, X, T)[0] - mlp.loss_and_grad(p - d, X, T)[0]) / 2e-6
        assert abs(fd - g[k]) < 1e-7 + 1e-5 * abs(fd)


def test_mp2_start_is_the_first_sweeps_doubles():
    """T2 = -<ij||ab> / D, antisymmetric, T1 and T3 zero."""
    s = synth.system(synth.SynthSpec(8, 4, 16, 0.03, 4000, 1.3))
    lay = warmstart.tlayout(s)
    t = warmstart.mp2_t(s, lay)
    m = lay.view(t, 'T2A')
    assert np.allclose(m, -m.transpose(1, 0, 2, 3)) and np.abs(m).max() > 0
    assert not np.any(lay.view(t, 'T1A')) and not np.any(lay.view(t, 'T3B'))


def test_family_and_split():
    fam = warmstart.c4_family()
    assert len(fam) == 200 and fam[0].lam == 0.5 and fam[-1].lam == 2.0
    tr, ev = warmstart.c4_split()
    assert len(tr) == 150 and len(ev) == 50 and not set(tr) & set(ev)


def test_bracket_interpolates_between_neighbours():
    lams = [0.5, 0.8, 1.0, 1.4]
    (a, wa), (b, wb) = warmstart.bracket(lams, 0.9)
    assert {a, b} == {1, 2} and abs(wa - 0.5) < 1e-12 and abs(wb - 0.5) < 1e-12
    # the member itself left out (training): its two neighbours
    assert {k for k, w in warmstart.bracket(lams, 0.8, exclude=1)} == {0, 2}
    # beyond the last member: linear extrapolation from the two nearest
    br = warmstart.bracket(lams, 1.6)
    assert {k for k, w in br} == {2, 3}
    assert abs(sum(w * lams[k] for k, w in br) - 1.6) < 1e-12 and abs(sum(w for k, w in br) - 1.0) < 1e-12


def _antisym_t(lay, rng, names=('T1A', 'T1B', 'T2A', 'T2B', 'T2C', 'T3A', 'T3B', 'T3C', 'T3D')):
    from oracle import solver as S
    t = np.zeros(lay.t_size)
    for b in names:
        if lay.size(b):
            lay.view(t, b)[...] = S.antisym_fill(b, rng.normal(0, 0.01, lay.shape[b]))
    return t


def test_two_anchor_start_keeps_the_antisymmetry():
    """interpolated start and both feature sets: symmetric features, so base * (1 + r(x)) keeps the
    antisymmetry of every T2 and T3 block; at an anchor's own lambda the start is that anchor."""
    from oracle import solver as S
    specs = [synth.SynthSpec(8, 6, 16, 0.03, 4000, l) for l in (1.0, 1.2)]
    rng = np.random.default_rng(5)
    sols = []
    for sp in specs:
        s = synth.system(sp)
        lay = warmstart.tlayout(s)
        sols.append((sp, s, lay, _antisym_t(lay, rng)))
    members = [(w, None, sols[k][3], sols[k][0].lam) for k, w in warmstart.bracket([1.0, 1.2], 1.1)]
    s = synth.system(synth.SynthSpec(8, 6, 16, 0.03, 4000, 1.1))
    lay = warmstart.tlayout(s)
    t = warmstart.interp_start(s, 1.1, lay, members)
    for b in ('T2A', 'T3A', 'T3B'):
        v = lay.view(t, b)
        assert np.allclose(S.antisym_fill(b, v), v)
    for name, X, b, sel, shape in warmstart.interp_features(s, 1.1, members, lay, ('T2A',), cut=0.0):
        full = np.zeros((int(np.prod(shape)), warmstart.NFEAT))
        full[sel] = X
        Xr = full.reshape(shape + (warmstart.NFEAT,))
        nz = np.abs(lay.view(t, 'T2A')) > 0
        for perm in ((1, 0, 2, 3), (0, 1, 3, 2)):
            assert np.allclose(Xr[nz], Xr.transpose(perm + (4,))[nz])
    for name, X, b, sel, shape in warmstart.interp_features(s, 1.1, members, lay, ('T3A',), cut=0.0):
        full = np.zeros((int(np.prod(shape)), warmstart.NFEAT))
        full[sel] = X
        Xr = full.reshape(shape + (warmstart.NFEAT,))
        nz = np.abs(lay.view(t, 'T3A')) > 0
        for perm in ((1, 0, 2, 3, 4, 5), (0, 1, 2, 4, 3, 5), (2, 1, 0, 3, 4, 5)):
            P = Xr.transpose(perm + (6,))
            assert np.allclose(Xr[nz], P[nz])
    # at the anchor's own lambda the interpolation gives that anchor's amplitudes
    own = [(w, None, sols[k][3], sols[k][0].lam) for k, w in warmstart.bracket([1.0, 1.2], 1.0)]
    t0 = warmstart.interp_start(sols[0][1], 1.0, sols[0][2], own)
    for b in ('T1A', 'T3B'):
        np.testing.assert_allclose(sols[0][2].view(t0, b), sols[0][2].view(sols[0][3], b), atol=1e-15)
