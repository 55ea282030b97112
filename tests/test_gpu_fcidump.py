"""FCIDUMP on the GPU: the device expansion of the two-body integrals equals the
host reader bit for bit (later records overwrite earlier ones, also when many
records collide), and a CCSDT run of an input deck pointing at a FCIDUMP of the
H4 fixture lands on the reference's known answer."""
import numpy as np
import pytest

from ccq_b200 import driver, integrals as I, lib

pytestmark = pytest.mark.gpu


def _device_e2(path, n):
    import torch
    e2 = torch.zeros(n ** 4, dtype=torch.float64, device='cuda')
    e1, en = lib.fcidump_read_device(path, n, e2.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return e1, e2.cpu().numpy().reshape((n, n, n, n), order='F'), en


def test_device_expansion_equals_host(tmp_path, h4):
    p = str(tmp_path / 'h4.fcidump')
    I.write_fcidump(p, h4['e1'], h4['e2'], h4['enuc'], nelec=4, eps=np.arange(1.0, 5.0), order=(2, 0, 3, 1))
    e1h, e2h, enh = lib.fcidump_read(p, 4)
    e1d, e2d, end = _device_e2(p, 4)
    np.testing.assert_array_equal(e1d, e1h)
    np.testing.assert_array_equal(e2d, e2h)
    assert end == enh


def test_device_last_record_wins_under_collisions(tmp_path):
    """14 orbitals, 60 000 records drawn with repeats in every index order: most elements are written by
    several records with different values; the device result keeps the last one, like the host."""
    n = 14
    rng = np.random.default_rng(3)
    idx = rng.integers(1, n + 1, size=(60000, 4))
    vals = rng.normal(size=60000)
    lines = [' &FCI NORB=14,NELEC=6,', ' &END']
    lines += [f'{v: .17E} {i} {a} {j} {b}' for v, (i, a, j, b) in zip(vals, idx.tolist())]
    lines += [f'{float(-k): .3f} {k} 0 0 0' for k in rng.permutation(np.arange(1, n + 1)).tolist()]
    lines.append(' 0.25 0 0 0 0')
    p = str(tmp_path / 'FCIDUMP')
    with open(p, 'w') as fh:
        fh.write('\n'.join(lines) + '\n')
    e1h, e2h, enh = lib.fcidump_read(p, n)
    e1d, e2d, end = _device_e2(p, n)
    np.testing.assert_array_equal(e2d, e2h)
    assert end == enh == 0.25


def test_h4_ccsdt_through_fcidump_deck(tmp_path, h4):
    I.write_fcidump(str(tmp_path / 'h4.fcidump'), h4['e1'], h4['e2'], h4['enuc'], nelec=4,
                    eps=np.arange(1.0, 5.0), order=(3, 1, 0, 2))
    (tmp_path / 'input.inp').write_text('calc_type=CCSDT\nfcidump=h4.fcidump\ntol=1.0e-11\nrhf=.true.\n'
                                        'max_iterations=100\n')
    r = driver.run(str(tmp_path / 'input.inp'), out=lambda s: None, base_dir=str(tmp_path))
    assert not r.failed
    # known answer of the reference's tests/test_small.py (the fixture's 10-decimal ERIs: 2.3e-10 offset)
    assert abs(r.e_total - (-1.978696408825)) < 2.3e-10 + 1e-11
