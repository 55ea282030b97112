"""Checkpoint files and restart keys without a GPU: the header reader refuses
missing and foreign files; the reference's restart / output_bin keys and the
gpu_checkpoint_every key parse."""
import pytest

from ccq_b200 import config, lib


def test_info_refuses_missing_and_foreign_files(tmp_path):
    with pytest.raises(lib.CCQB200Error, match='Restart file not found'):
        lib.checkpoint_info(str(tmp_path / 'none.bin'))
    p = tmp_path / 'x.bin'
    p.write_bytes(b'not a checkpoint at all, just bytes' * 10)
    with pytest.raises(lib.CCQB200Error, match='not a checkpoint'):
        lib.checkpoint_info(str(p))
    p.write_bytes(b'CCQB200C' + b'\0' * 12)
    with pytest.raises(lib.CCQB200Error, match='truncated'):
        lib.checkpoint_info(str(p))


def test_restart_keys():
    cfg = config.parse_lines(['nel=4', 'nvirt=4', 'calc_type=CCSD', 'restart', 'output_bin=run.ck',
                              'gpu_checkpoint_every=5'])
    assert cfg.restart and cfg.bin_path() == 'run.ck' and cfg.gpu_checkpoint_every == 5
    cfg = config.parse_lines(['nel=4', 'nvirt=4', 'label=h4'])
    assert not cfg.restart and cfg.bin_path() == 'tvec_h4.bin'
    assert config.parse_lines(['nel=4']).bin_path() == 'tvec.bin'
