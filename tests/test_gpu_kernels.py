"""GETT kernel through the dgemm.f90 drop-in (egemm / egemm1 / egemm2) vs numpy FP64."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (7, 5, 3), (64, 64, 16), (100, 37, 513), (257, 3, 1000), (3, 300, 5000),
          (1000, 1000, 64), (1024, 64, 1024), (65, 129, 17),
          # skinny tiles (one side <= 32): split-K, transposed launch, 16- and 32-row tiles,
          # odd and even K (8- and 16-byte operand copies), long outputs without split-K
          (8, 2048, 8192), (2048, 8, 4096), (16, 100000, 8), (32, 5000, 300), (1, 70000, 256),
          (33, 40, 1000), (17, 3000, 64), (4000, 17, 130), (24, 24, 2001), (30, 1001, 7)]


@pytest.mark.parametrize('k1,k2,k3', SHAPES)
def test_egemm(k1, k2, k3):
    from ccq_b200 import lib
    rng = np.random.default_rng(k1 * 7 + k2 * 3 + k3)
    A = np.asfortranarray(rng.normal(size=(k3, k1)))
    B = np.asfortranarray(rng.normal(size=(k3, k2)))
    C = lib.egemm(k1, k2, k3, A, B)
    ref = B.T @ A
    tol = 1e-13 * max(1, np.sqrt(k3)) * 10
    np.testing.assert_allclose(C, ref, atol=tol, rtol=0)


def test_egemm_k0_gives_zero():
    from ccq_b200 import lib
    C = lib.egemm(5, 4, 0, np.zeros((0, 5)), np.zeros((0, 4)))
    assert np.all(C == 0)


def test_egemv_variants():
    from ccq_b200 import lib
    rng = np.random.default_rng(4)
    A = np.asfortranarray(rng.normal(size=(300, 70)))
    b = rng.normal(size=300)
    np.testing.assert_allclose(lib.egemm1(70, 300, A, b), A.T @ b, atol=1e-12)
    np.testing.assert_allclose(lib.egemm2(70, 300, b, A), A.T @ b, atol=1e-12)
