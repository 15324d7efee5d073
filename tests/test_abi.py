"""The C-ABI library loads, exports every symbol the header declares, and
fails loudly (no CPU fallback) where no device is usable."""
import ctypes
import subprocess

import pytest

from peridyn_b200 import _abi


def test_library_exports_header_symbols():
    L = _abi.lib()
    names = _abi.header_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(names) <= exported
    # everything exported is declared (no stray internals on the ABI)
    assert exported <= set(names)


def test_abi_version_and_status_strings():
    L = _abi.lib()
    assert L.pd_abi_version() == 2
    assert L.pd_status_string(0) == b"ok"
    assert L.pd_status_string(_abi.PD_ERR_FAMILY_OVERFLOW).startswith(b"family")


def test_null_handles_are_rejected():
    L = _abi.lib()
    assert L.pd_env_destroy(None) == 0
    assert L.pd_env_finalize(None) == _abi.PD_ERR_ARG
    assert b"NULL" in L.pd_last_error()
    assert L.pd_env_create(None, 0, 0, 1.0) == _abi.PD_ERR_ARG


def test_no_cpu_fallback_without_device():
    if _abi.device_count() > 0:
        pytest.skip("a CUDA device is visible")
    L = _abi.lib()
    h = ctypes.c_void_p()
    st = L.pd_env_create(ctypes.byref(h), 0, 0, 1e-8)
    assert st == _abi.PD_ERR_NO_DEVICE
    assert b"no CUDA device" in L.pd_last_error()
