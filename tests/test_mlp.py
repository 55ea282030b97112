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


def test_features_keep_the_amplitude_symmetry():
    s = synth.system(synth.SynthSpec(8, 4, 16, 0.03, 4000, 1.3))
    for name, X, mp2, shape in warmstart.system_blocks(s, 1.3):
        Xr = X.reshape(shape + (warmstart.NFEAT,))
        m = mp2.reshape(shape)
        if name in ('T2A', 'T2C'):
            # antisymmetric mp2, symmetric features: mp2 * (1 + r(x)) stays antisymmetric
            assert np.allclose(m, -m.transpose(1, 0, 2, 3))
            assert np.allclose(Xr, Xr.transpose(1, 0, 2, 3, 4))
            assert np.allclose(Xr, Xr.transpose(0, 1, 3, 2, 4))


def test_anchor_features_keep_the_symmetry():
    """The anchor's converged ratio t/mp2 - 1 is symmetric where mp2 is antisymmetric."""
    spec = synth.SynthSpec(8, 4, 16, 0.03, 4000, 1.1)
    s = synth.system(spec)
    lay = warmstart.tlayout(s)
    rng = np.random.default_rng(3)
    t = np.zeros(lay.t_size)
    for name, X, mp2, shape in warmstart.system_blocks(s, 1.1):
        # an antisymmetric stand-in for a converged T2: mp2 times a symmetric factor
        f = 1.0 + 0.1 * rng.normal(size=shape)
        if name in ('T2A', 'T2C'):
            f = 0.25 * (f + f.transpose(1, 0, 2, 3) + f.transpose(0, 1, 3, 2) + f.transpose(1, 0, 3, 2))
        lay.view(t, name)[...] = mp2.reshape(shape) * f
    anchor = warmstart.anchor_of(spec, t)
    s2 = synth.system(synth.SynthSpec(8, 4, 16, 0.03, 4000, 1.3))
    for name, X, mp2, shape in warmstart.system_blocks(s2, 1.3, anchor):
        Xr = X.reshape(shape + (warmstart.NFEAT,))
        assert np.allclose(Xr[..., 7], 1.3 - 1.1)
        if name in ('T2A', 'T2C'):
            assert np.allclose(Xr, Xr.transpose(1, 0, 2, 3, 4))
            assert np.allclose(Xr, Xr.transpose(0, 1, 3, 2, 4))


def test_family_and_split():
    fam = warmstart.c4_family()
    assert len(fam) == 200 and fam[0].lam == 0.5 and fam[-1].lam == 2.0
    tr, ev = warmstart.c4_split()
    assert len(tr) == 150 and len(ev) == 50 and not set(tr) & set(ev)
