"""Warm-start network kernels against the CPU oracle, and the warm start's effect."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand(seed, n=3000):
    from ccq_b200 import warmstart
    rng = np.random.default_rng(seed)
    ws = warmstart.WarmStart(seed=seed)
    ws.params = (ws.params + rng.normal(0, 0.05, ws.params.size)).astype(np.float32)
    X = rng.normal(size=(n, warmstart.NFEAT))
    T = rng.normal(size=n)
    return ws, X, T


def test_forward_and_gradient_kernels_match_oracle():
    import torch
    from ccq_b200 import warmstart
    from oracle import mlp
    ws, X, T = _rand(1)
    y = ws.predict_ratio(X)   # identity scaling: raw network output
    np.testing.assert_allclose(y, mlp.forward(ws.params.astype(np.float64), X.astype(np.float32)), rtol=1e-4,
                               atol=1e-5)
    dev = torch.device('cuda')
    P = torch.tensor(ws.params, device=dev)
    Xd = torch.tensor(X.astype(np.float32), device=dev)
    Td = torch.tensor(T.astype(np.float32), device=dev)
    G = torch.zeros_like(P)
    L = torch.zeros(1, device=dev)
    l = warmstart._bind()
    assert l.ccq_b200_mlp_grad(P.data_ptr(), warmstart.NFEAT, Xd.data_ptr(), Td.data_ptr(), X.shape[0], G.data_ptr(),
                               L.data_ptr(), torch.cuda.current_stream().cuda_stream) == 0
    loss, g = mlp.loss_and_grad(ws.params.astype(np.float64), X.astype(np.float32), T.astype(np.float32))
    assert abs(L.item() - loss) < 1e-4 * loss
    gd = G.cpu().numpy()
    assert np.abs(gd - g).max() < 2e-4 * np.abs(g).max()


def test_adam_step_matches_numpy():
    import torch
    from ccq_b200 import warmstart
    rng = np.random.default_rng(2)
    n = 777
    p, g = rng.normal(size=n).astype(np.float32), rng.normal(size=n).astype(np.float32)
    m, v = (0.1 * rng.normal(size=n)).astype(np.float32), np.abs(0.1 * rng.normal(size=n)).astype(np.float32)
    dev = torch.device('cuda')
    P, G, M, V = (torch.tensor(a, device=dev) for a in (p, g, m, v))
    l = warmstart._bind()
    assert l.ccq_b200_mlp_adam(P.data_ptr(), G.data_ptr(), M.data_ptr(), V.data_ptr(), n, 1e-2, 3,
                               torch.cuda.current_stream().cuda_stream) == 0
    m2 = 0.9 * m + 0.1 * g
    v2 = 0.999 * v + 0.001 * g * g
    p2 = p - 1e-2 * (m2 / (1 - 0.9 ** 3)) / (np.sqrt(v2 / (1 - 0.999 ** 3)) + 1e-8)
    np.testing.assert_allclose(P.cpu().numpy(), p2, rtol=1e-5, atol=1e-6)


def test_warm_start_converges_to_the_same_energy_in_fewer_iterations():
    """Every start reaches the plain start's energy within tol; the learned start needs fewer iterations
    than T = 0, and its networks do better than the same interpolation without them."""
    from ccq_b200 import warmstart
    res = warmstart.study('CCSDT', norb=12, nel=6, count=40, train=30, tol=1e-8, epochs=400)
    st = res['starts']
    assert res['max_dE'] < 1e-8 and all(v['max_dE'] < 1e-8 and not v['failed'] for v in st.values())
    assert res['warm_iterations_mean'] < res['plain_iterations_mean']
    assert st['warm']['iterations_mean'] <= st['interp']['iterations_mean']
