"""Split-precision (int8 Ozaki slices on tcgen05) GETT vs FP64.

Bound per element: |C - C_ref| <= 2^(-7S+2) * k3 * max|A col| * max|B col|
(slice truncation plus dropped levels, with margin).  The converged test
checks that the split sweeps followed by FP64 iterations land on the FP64
energy to 1e-10 Eh.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bound(A, B, S, k3):
    ra = np.abs(A).max(axis=0)      # per output row m (column of Fortran A(k3,k1))
    rb = np.abs(B).max(axis=0)
    return 2.0 ** (-7 * S + 2) * k3 * np.outer(rb, ra)


@pytest.mark.parametrize('S', [2, 3, 4])
@pytest.mark.parametrize('k1,k2,k3', [(128, 128, 64), (300, 1000, 1000), (1024, 2048, 1024), (129, 257, 100)])
def test_egemm_split_error_bound(S, k1, k2, k3):
    from ccq_b200 import lib
    rng = np.random.default_rng(k1 + 7 * k2 + S)
    A = np.asfortranarray(rng.normal(size=(k3, k1)) * np.exp(rng.normal(size=(1, k1))))
    B = np.asfortranarray(rng.normal(size=(k3, k2)) * 1e-3)
    ref = B.T @ A
    C = lib.egemm_split(k1, k2, k3, A, B, S)
    err = np.abs(C - ref)
    assert np.all(err <= _bound(A, B, S, k3)), float((err / _bound(A, B, S, k3)).max())
    if S == 4:
        # columns of A span e^{+-3}: relative to the largest product scale
        assert (err / (k3 * np.outer(np.abs(B).max(axis=0), np.abs(A).max(axis=0)))).max() < 2 ** -26


@pytest.mark.parametrize('S', [2, 3, 4])
@pytest.mark.parametrize('k1,k2,k3', [(128, 128, 64), (129, 257, 100), (1024, 4096, 512), (2000, 3000, 320)])
def test_persistent_split_kernel_equals_per_tile_kernel(S, k1, k2, k3):
    """One CTA per SM over all tiles (two TMEM accumulator sets, overlapped epilogue) gives the per-tile
    kernel's result bit for bit: the int32 level sums are exact and recombined in the same order.  The
    1024 x 4096 and 2000 x 3000 cases give every CTA several tiles, so both accumulator sets are reused."""
    from ccq_b200 import lib
    rng = np.random.default_rng(k1 + k2 + S)
    A = np.asfortranarray(rng.normal(size=(k3, k1)))
    B = np.asfortranarray(rng.normal(size=(k3, k2)))
    c0 = lib.egemm_split(k1, k2, k3, A, B, S, persistent=False)
    c1 = lib.egemm_split(k1, k2, k3, A, B, S, persistent=True)
    np.testing.assert_array_equal(c1, c0)
    assert np.all(np.abs(c1 - B.T @ A) <= _bound(A, B, S, k3))


def test_egemm_split_zero_and_tiny_rows():
    from ccq_b200 import lib
    rng = np.random.default_rng(5)
    k1, k2, k3 = 256, 256, 192
    A = np.asfortranarray(rng.normal(size=(k3, k1)))
    A[:, 3] = 0.0
    A[:, 7] *= 1e-200
    B = np.asfortranarray(rng.normal(size=(k3, k2)))
    C = lib.egemm_split(k1, k2, k3, A, B, 4)
    ref = B.T @ A
    assert np.all(C[:, 3] == 0.0)
    # the 1e-200 row keeps its own scale: error bounded by that row's magnitude
    assert np.all(np.abs(C - ref) <= _bound(A, B, 4, k3))
    assert np.abs(C[:, 7] - ref[:, 7]).max() < 1e-190


def test_split_sweeps_then_fp64_converge_to_fp64_energy():
    from ccq_b200 import config, driver, lib, synth
    spec = synth.SynthSpec(32, 12, 64, 0.03, 11)
    s = synth.system(spec)
    d = s['dims']
    es = {}
    for prec in ('fp64', 'split'):
        ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDT', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                          s['v_bb'])
        cfg = config.Config(calc_type='CCSDT', tol=1e-10, max_iter=80, gpu_precision=prec, gpu_slices=4,
                            gpu_fp64_finish=1e-7).calc_macros()
        r = driver.solve_cc(ctx, cfg, out=lambda x: None)
        assert not r.failed
        if prec == 'split':
            assert sum(1 for h in r.history if h['split']) >= 3
            # the sliced kernels really ran on this system's ladder terms
            ctx.set_precision(lib.PREC_SPLIT, 4)
            ctx.profile(True)
            ctx.iterate(r.iterations + 1)
            prof = ctx.profile_get()
            ctx.profile(False)
            assert prof['gett_split']['launches'] > 0
        es[prec] = r.e_cor
        ctx.close()
    assert abs(es['split'] - es['fp64']) < 1e-10
