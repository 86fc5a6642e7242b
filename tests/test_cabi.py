"""The C ABI library loads without a GPU and exports every symbol declared in
include/*.h (no compute calls)."""
import ctypes
import os
import re

import pytest

from taremincloth_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(tc_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared()
    assert len(declared) > 40
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert declared <= set(_lib.SIGNATURES), sorted(declared - set(_lib.SIGNATURES))


def test_loader_binds_and_reports_no_gpu_here():
    L = _lib.load()
    assert L.tc_last_error() is not None
    if not os.path.exists("/dev/nvidia0"):
        assert L.tc_gpu_available() == 0


def test_create_without_gpu_raises_runtime_error():
    if os.path.exists("/dev/nvidia0"):
        pytest.skip("a GPU is present")
    import numpy as np
    from taremincloth_b200 import ClothSimulator
    with pytest.raises(RuntimeError):
        ClothSimulator(np.zeros((3, 3), np.float32), np.array([[0, 1], [1, 2]], np.uint32))


def test_drop_in_module_imports():
    import taremin_cloth_core
    assert hasattr(taremin_cloth_core, "ClothSimulator")


def test_device_lost_flag_is_host_side():
    """Marking a device lost and reading its status need no GPU (no CUDA call)."""
    from taremincloth_b200 import _lib
    from taremincloth_b200.simulator import device_status, mark_device_lost
    lost, epoch = device_status(5)
    assert not lost and epoch >= 1
    mark_device_lost(5)
    assert device_status(5) == (True, epoch)
    with pytest.raises(RuntimeError):
        _lib.check(_lib.load().tc_mark_device_lost(64))
