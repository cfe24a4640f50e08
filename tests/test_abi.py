"""The C ABI boundary, checked without a GPU: the shared library loads, exports
every entry point include/wos_gpu.h declares, and reports the absence of a
device as an error (no CPU fallback)."""
import ctypes as C
import os
import re

import pytest

from gpu_util import wos

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"WOS_API\s+[\w\s\*]+?\b(wos_\w+)\s*\(", txt))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 35
    assert {"wos_propagate", "wos_splitstep", "wos_polychromatic", "wos_volume",
            "wos_partially_coherent", "wos_asm_loss_grad"} <= names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(wos.LIB_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(wos.EXPORTS) == declared_symbols()


def test_status_strings_and_backend_info():
    L = wos.lib()
    for s in range(8):
        assert L.wos_status_string(s)
    assert b"sm_100a" in L.wos_backend_info()


@pytest.mark.skipif(wos.device_count() > 0, reason="checks the no-device path")
def test_no_device_fails_loudly():
    with pytest.raises(wos.WosError) as e:
        wos.GPU(wos.FP32)
    assert e.value.status == 6   # WOS_NOT_INITIALISED


def test_invalid_arguments_rejected_before_any_device_work():
    L = wos.lib()
    h = C.c_void_p()
    assert L.wos_ctx_create(0, 7, C.byref(h)) == 1                  # bad precision
    assert L.wos_propagate(None, None, 1.0, 1, None, None) == 1     # null ctx
    assert L.wos_ctx_set_col_width(None, 3) == 1
