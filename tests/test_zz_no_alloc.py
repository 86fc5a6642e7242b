"""The allocation-free hash build (tc_hash_build_static) against the
simulator's own hash build (tc_get_hash_state).

tc_hash_build_static exists for callers that cannot allocate device memory
(hosts that own all device buffers through their own allocator, threads that
must not call cudaMalloc / cudaFree, memory-capped services): it takes the
caller's device buffers and keeps its scratch in a fixed static array inside
libtcloth.so.  Here torch stands in for such a caller's allocator.  Outputs
are integer arrays, so they must match bit for bit; two calls in a row with
different sizes check that the shared scratch is reset between calls.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_build(L, positions, cell, table, torch):
    n = len(positions)
    pos = torch.zeros((max(n, 1), 4), dtype=torch.float32, device="cuda")
    pos[:n, :3] = torch.from_numpy(np.ascontiguousarray(positions)).cuda()
    cs = torch.full((table + 1,), -1, dtype=torch.int32, device="cuda")
    srt = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    status = L.tc_hash_build_static(C.c_void_p(pos.data_ptr()), n, float(cell), int(table), C.c_void_p(cs.data_ptr()),
                                    C.c_void_p(srt.data_ptr()), C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return status, cs.cpu().numpy().view(np.uint32), srt.cpu().numpy().view(np.uint32)[:n]


def test_static_hash_build_matches_simulator_build():
    import torch
    from taremincloth_b200 import ClothSimulator, _lib, scenes
    L = _lib.load()
    for sc in (scenes.config2(n=96, subdiv=3), scenes.config1()):
        g = scenes.build(ClothSimulator, sc)
        g.step(sc["dt"], sc["substeps"])
        cs_ref, srt_ref = g.get_hash_state(0)          # existing entry point
        _, p, _ = g.get_state()
        status, cs, srt = _static_build(L, p, g.get_cell_size(), g.get_counts()["table_size"], torch)
        _lib.check(status)
        np.testing.assert_array_equal(cs, cs_ref)
        np.testing.assert_array_equal(srt, srt_ref)


def test_static_hash_build_rejects_oversize():
    import torch
    from taremincloth_b200 import _lib
    L = _lib.load()
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    for n, table in ((262145, 1024), (16, 65537 * 2), (16, 512)):
        status = L.tc_hash_build_static(C.c_void_p(dummy.data_ptr()), n, 0.01, table, C.c_void_p(dummy.data_ptr()),
                                        C.c_void_p(dummy.data_ptr()), None)
        with pytest.raises(ValueError):
            _lib.check(status)


def test_static_hash_build_empty_and_invalid_arguments():
    import torch
    from taremincloth_b200 import _lib
    L = _lib.load()
    # n = 0: every bucket empty, twice in a row (the second call sees the first's scratch)
    for table in (1024, 4096):
        status, cs, _ = _static_build(L, np.zeros((0, 3), np.float32), 0.01, table, torch)
        _lib.check(status)
        assert cs.shape == (table + 1,) and not cs.any()
    buf = torch.zeros(64, dtype=torch.float32, device="cuda")
    base = buf.data_ptr()
    for cell in (0.0, -1.0, float("nan")):
        status = L.tc_hash_build_static(C.c_void_p(base), 4, cell, 1024, C.c_void_p(base), C.c_void_p(base), None)
        with pytest.raises(ValueError):
            _lib.check(status)
    # positions are read as float4 rows: a pointer off a 16-byte boundary is refused
    status = L.tc_hash_build_static(C.c_void_p(base + 4), 4, 0.01, 1024, C.c_void_p(base), C.c_void_p(base), None)
    with pytest.raises(ValueError):
        _lib.check(status)
    # a null sorted array with vertices to sort is refused
    status = L.tc_hash_build_static(C.c_void_p(base), 4, 0.01, 1024, C.c_void_p(base), None, None)
    with pytest.raises(ValueError):
        _lib.check(status)
    torch.cuda.synchronize()
