"""egemm on caller-owned device memory without any device allocation.

ccq_b200_egemm_dev_noalloc serves hosts that cannot let the library allocate
(their own pool owns the GPU's memory, or a cudaMalloc would stall a
time-critical loop).  Checked here through the C ABI against numpy's B^T A and
the allocating ccq_b200_egemm on several calls in a row (split-K, one K chunk,
skinny tiles, k3 = 0), plus the size limit of its fixed scratch array.  Collected last (file name) so that a
failure here stops a -x run only after every other test has run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fn():
    from ccq_b200 import lib
    l = lib.load()
    f = l.ccq_b200_egemm_dev_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int64] * 3 + [ctypes.c_void_p] * 4
    return f


# (k1, k2, k3) of the calls in a row, and what each exercises:
#   (300, 77, 1000)   64x64 tiles, split-K over 30 chunks (C zeroed, partial sums added atomically)
#   (64, 1024, 130)   64x64 tiles, split-K over 5 chunks
#   (1024, 1024, 64)  64x64 tiles, one K chunk (plain stores, no zeroing)
#   (8, 2048, 8192)   skinny 16-row tiles, split-K
#   (40, 30, 0)       k3 = 0: C = 0
CASES = [(300, 77, 1000), (64, 1024, 130), (1024, 1024, 64), (8, 2048, 8192), (40, 30, 0)]


def test_noalloc_matches_allocating_egemm_and_numpy():
    import torch
    from ccq_b200 import lib
    f = _fn()
    torch.cuda.init()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(123)
    for call, (k1, k2, k3) in enumerate(CASES):
        A = np.asfortranarray(rng.normal(size=(k3, k1)))
        B = np.asfortranarray(rng.normal(size=(k3, k2)))
        ref = B.T @ A
        alloc = lib.egemm(k1, k2, k3, A, B)
        dA = torch.from_numpy(A.ravel(order='F').copy()).cuda()
        dB = torch.from_numpy(B.ravel(order='F').copy()).cuda()
        dC = torch.full((k1 * k2,), float('nan'), dtype=torch.float64, device='cuda')
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = f(k1, k2, k3, dA.data_ptr() if k3 else None, dB.data_ptr() if k3 else None, dC.data_ptr(),
               stream.cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        if call > 0:
            # after the per-device set-up of the first call nothing is allocated
            assert torch.cuda.mem_get_info()[0] == free0
        C = dC.cpu().numpy().reshape((k2, k1), order='F')
        tol = 1e-13 * max(1, np.sqrt(k3)) * 10
        np.testing.assert_allclose(C, ref, atol=tol, rtol=0)
        np.testing.assert_allclose(C, alloc, atol=tol, rtol=0)
        if k3 == 0:
            assert np.all(C == 0)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    f = _fn()
    d = torch.zeros(4, dtype=torch.float64, device='cuda')
    assert f(65537, 1, 1, d.data_ptr(), d.data_ptr(), d.data_ptr(), None) == -7
    assert f(1, 1, 70000, d.data_ptr(), d.data_ptr(), d.data_ptr(), None) == -7
