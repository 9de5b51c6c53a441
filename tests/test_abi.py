"""C-ABI checks that need no GPU: the library loads, exports every entry point that
include/tremor_b200.h declares, converts cc <-> ED bit-identically to the reference,
and fails with an error code (no crash, no CPU fallback) where there is no device."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import tremor_b200
from tests import oracle_bindings as ob

HEADER = Path(__file__).resolve().parents[1] / 'include' / 'tremor_b200.h'


def declared_symbols():
    text = re.sub(r'/\*.*?\*/', '', HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r'\b(tm_[a-z0-9_]+)\s*\(', text)))


def test_library_exports_every_declared_symbol():
    lib = tremor_b200.load_library()
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name


def test_conversions_bit_identical_to_reference():
    lib = tremor_b200.load_library()
    rng = np.random.default_rng(5)
    for _ in range(2000):
        m = int(rng.integers(1, 20000))
        cc = np.float32(rng.uniform(-1.2, 1.2))
        ed = np.float32(rng.uniform(0, 4 * m))
        a = np.float32(lib.tm_cc_to_ed(float(cc), m))
        b = np.float32(ob.oracle().tmo_cc_to_ed(float(cc), m))
        assert a.view(np.uint32) == b.view(np.uint32)
        a = np.float32(lib.tm_ed_to_cc(float(ed), m))
        b = np.float32(ob.oracle().tmo_ed_to_cc(float(ed), m))
        assert a.view(np.uint32) == b.view(np.uint32)


def test_argument_errors_are_codes():
    lib = tremor_b200.load_library()
    h = ctypes.c_void_p()
    x = np.zeros(16, np.float32)
    assert lib.tm_ctx_create(None, 16, 0, ctypes.byref(h)) == -1
    assert lib.tm_ctx_create(x.ctypes.data_as(ctypes.c_void_p), 0, 0, ctypes.byref(h)) == -1
    assert lib.tm_set_kernel(None, 1) == -1
    assert lib.tm_result_count(None, 0, None) == -1


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason='checks the no-device path')
def test_no_device_is_an_error_not_a_fallback():
    with pytest.raises(tremor_b200.TremorError) as e:
        tremor_b200.Context(np.zeros(1024, np.float32))
    assert e.value.code == -6
