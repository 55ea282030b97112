"""The C ABI library loads and exports every symbol of include/ccq_b200.h (no GPU needed)."""
import ctypes
import os

import pytest

from ccq_b200 import lib


def test_library_exports_header_symbols():
    if not os.path.exists(lib.LIB_PATH):
        from ccq_b200 import build
        build.build()
    so = ctypes.CDLL(lib.LIB_PATH)
    names = lib.header_symbols()
    assert 'ccq_b200_egemm' in names and 'egemm_' in names and 'ccq_b200_init' in names
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing
    assert set(lib.SIGNATURES) <= set(names)


def test_last_error_without_device():
    l = lib.load()
    buf = ctypes.create_string_buffer(64)
    assert l.ccq_b200_last_error(buf, 64) == 0


def test_plans_are_embedded():
    from ccq_b200 import build
    build.write_plans_header()
    text = open(os.path.join(os.path.dirname(lib.LIB_PATH), 'csrc', 'plans_embedded.h')).read()
    for name in ('CCSD', 'CCSD_rhf', 'CCSDT', 'CCSDT_rhf'):
        assert f'"{name}"' in text
