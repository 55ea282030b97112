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
            assert np.allclose(Xr[..., [0, 1, 2, 3, 4, 5]], Xr.transpose(1, 0, 2, 3, 4))
            assert np.allclose(Xr, Xr.transpose(0, 1, 3, 2, 4))


def test_family_and_split():
    fam = warmstart.c4_family()
    assert len(fam) == 200 and fam[0].lam == 0.5 and fam[-1].lam == 2.0
    tr, ev = warmstart.c4_split()
    assert len(tr) == 150 and len(ev) == 50 and not set(tr) & set(ev)
