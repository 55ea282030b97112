"""Shared builders for the tests (random and synthetic systems)."""
import numpy as np

from ccq_b200 import integrals as I


def random_system(n, occ_a, occ_b, seed, sigma=0.1, froz=0):
    rng = np.random.default_rng(seed)
    L = 2 * n
    B = rng.normal(0, sigma, (L, n, n))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    chem = np.einsum('Lpq,Lrs->pqrs', B, B)
    e2 = chem.transpose(0, 2, 1, 3).copy()
    h = rng.normal(0, 0.05, (n, n))
    h = 0.5 * (h + h.T) + np.diag(np.linspace(-2.0, 1.0, n))
    fa, fb = I.fock(h, e2, occ_a, occ_b)
    vaa, vab, vbb = I.spin_blocks(e2, froz)
    return dict(h=h, e2=e2, f_a=fa, f_b=fb, v_aa=vaa, v_ab=vab, v_bb=vbb,
                dims=I.Dims(froz, occ_a, occ_b, n))


def random_t(dims, seed, scale=0.02, nmax=3):
    """Random amplitudes with the reference's antisymmetry (canonical + fill)."""
    from oracle import solver as S
    rng = np.random.default_rng(seed)
    lay = I.TLayout(dims)
    t = np.zeros(lay.t_size)
    for b in I.T_VEC_ORDER:
        if int(b[1]) > nmax:
            continue
        v = lay.view(t, b)
        v[...] = S.antisym_fill(b, rng.normal(0, scale, v.shape))
    t4 = {}
    if nmax >= 4:
        for b, shp in lay.t4_shape.items():
            t4[b] = S.antisym_fill(b, rng.normal(0, scale, shp))
    return t, t4
