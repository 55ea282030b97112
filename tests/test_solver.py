"""ccq's driver quirks as restated by the oracle (src/diis.F90, src/solve_cc.f90)."""
import numpy as np

from oracle import solver as S


def test_ring_slots_and_residuum():
    r = S.Ring(5, 3)
    assert [r.slot(i) for i in range(1, 13)] == [1, 2, 3, 4, 5, 6, 1, 2, 3, 4, 5, 6]
    r.write(1, np.array([3.0, 4.0, 0.0]))
    assert abs(r.residuum(1) - np.sqrt(5.0)) < 1e-15      # sqrt(sqrt(25))


def test_diis_uses_oldest_vectors_and_corner():
    ds = 3
    r = S.Ring(ds, 4)
    rng = np.random.default_rng(0)
    vecs = [rng.normal(size=4) for _ in range(ds + 1)]
    for i, v in enumerate(vecs, 1):
        r.write(i, v)
    out = r.diis()
    d = [vecs[i + 1] - vecs[i] for i in range(ds)]
    B = np.array([[di @ dj for dj in d] for di in d])
    B = np.block([[B, -np.ones((ds, 1))], [-np.ones((1, ds)), -np.ones((1, 1))]])
    c = np.linalg.solve(B, np.r_[np.zeros(ds), -1.0])
    np.testing.assert_allclose(out, sum(c[i] * vecs[i] for i in range(ds)), atol=1e-12)


def test_convergence_needs_three_small_changes():
    seq = iter([1.0, 0.5, 0.5 + 1e-9, 0.5 + 2e-9, 0.5 + 2e-9, 0.5 + 2e-9])
    t = np.zeros(2)
    e, it, failed, hist = S.jacobi_iter(lambda t: None, lambda t: next(seq), t, 2, diis_space=5, max_iter=6, tol=1e-8)
    assert it == 5 and not failed


def test_nan_stops():
    t = np.zeros(2)
    e, it, failed, _ = S.jacobi_iter(lambda t: None, lambda t: float('nan'), t, 2, max_iter=10, tol=1e-8)
    assert failed and it == 1


def test_canonical_fill_t3b():
    rng = np.random.default_rng(1)
    t = S.antisym_fill('T3B', rng.normal(size=(3, 3, 2, 4, 4, 5)))
    np.testing.assert_allclose(t, -t.transpose(1, 0, 2, 3, 4, 5))
    np.testing.assert_allclose(t, -t.transpose(0, 1, 2, 4, 3, 5))
    assert np.all(t[0, 0] == 0)


def test_tran3bto3c_is_spin_flip():
    rng = np.random.default_rng(2)
    t3b = S.antisym_fill('T3B', rng.normal(size=(3, 3, 3, 4, 4, 4)))
    t3c = S.tran3bto3c(t3b)
    np.testing.assert_allclose(t3c[0, 1, 2, 0, 1, 2], t3b[1, 2, 0, 1, 2, 0])
    np.testing.assert_allclose(t3c, -t3c.transpose(0, 2, 1, 3, 4, 5))
