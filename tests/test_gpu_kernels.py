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


def _fortran_symbols():
    import ctypes
    from ccq_b200 import lib
    l = lib.load()
    dp = ctypes.POINTER(ctypes.c_double)
    i64p = ctypes.POINTER(ctypes.c_int64)
    e0, e1, e2 = l.egemm_, l.egemm1_, l.egemm2_
    e0.restype = e1.restype = e2.restype = None
    e0.argtypes = [i64p, i64p, i64p, dp, dp, dp]
    e1.argtypes = [i64p, i64p, dp, dp, dp]
    e2.argtypes = [i64p, i64p, dp, dp, dp]
    return e0, e1, e2


@pytest.mark.parametrize('k1,k2,k3', [(7, 5, 3), (100, 37, 513), (8, 2048, 300)])
def test_fortran_link_names_by_reference(k1, k2, k3):
    """egemm_/egemm1_/egemm2_ called as gfortran calls dgemm.f90's routines: every argument by
    reference, integers ILP64 (src/dgemm.f90:1-73), arrays column-major."""
    import ctypes
    e0, e1, e2 = _fortran_symbols()
    rng = np.random.default_rng(k1 + k2 + k3)
    A = np.asfortranarray(rng.normal(size=(k3, k1)))
    B = np.asfortranarray(rng.normal(size=(k3, k2)))
    C = np.asfortranarray(np.full((k2, k1), np.nan))
    i1, i2, i3 = ctypes.c_int64(k1), ctypes.c_int64(k2), ctypes.c_int64(k3)
    ptr = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    e0(ctypes.byref(i1), ctypes.byref(i2), ctypes.byref(i3), ptr(A), ptr(B), ptr(C))
    tol = 1e-13 * max(1, np.sqrt(k3)) * 10
    np.testing.assert_allclose(C, B.T @ A, atol=tol, rtol=0)
    b = rng.normal(size=k3)
    c1 = np.full(k1, np.nan)
    e1(ctypes.byref(i1), ctypes.byref(i3), ptr(A), ptr(b), ptr(c1))      # C(k1) = A(k3,k1)^T B(k3)
    np.testing.assert_allclose(c1, A.T @ b, atol=tol, rtol=0)
    c2 = np.full(k2, np.nan)
    e2(ctypes.byref(i2), ctypes.byref(i3), ptr(b), ptr(B), ptr(c2))      # C(k2) = B(k3,k2)^T A(k3)
    np.testing.assert_allclose(c2, B.T @ b, atol=tol, rtol=0)
