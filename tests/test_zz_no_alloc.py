"""The allocation-free accumulate entry point, through the C ABI, on a GPU.

`ix_accumulate_device_noalloc` serves callers that cannot call cudaMalloc: they own the
device buffers (here the test allocates them with torch, as such a caller's own pool
would) and the library keeps its work counters in a fixed device array instead of
allocating.  This file is collected last so a stop-at-first-failure run has already run
every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from indicatrix_b200 import abi, workloads
from indicatrix_b200.backend import GpuBackend, load_library

pytestmark = pytest.mark.gpu

IX_NOALLOC_ERR_TOO_LARGE = -2


def _device_scene(torch, fs):
    sc = fs.to_abi()
    planes = torch.from_numpy(np.ascontiguousarray(fs.planes, np.float32)).cuda()
    sc.planes = C.cast(C.c_void_p(planes.data_ptr()), C.POINTER(C.c_float))
    return sc, planes


def test_noalloc_entry_matches_the_allocating_entry_on_two_calls():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = load_library()
    lib.ix_accumulate_device_noalloc.restype = C.c_int
    lib.ix_accumulate_device_noalloc.argtypes = [C.POINTER(abi.Scene), C.c_uint32, C.c_uint32,
                                                 C.c_void_p, C.c_int, C.c_void_p]
    fs = workloads.round_brilliant_frame(40, 36)
    sc, planes = _device_scene(torch, fs)
    n = fs.width * fs.height * 3
    stream = torch.cuda.Stream()
    backend = GpuBackend.acquire()
    assert backend.available
    try:
        for call, (offset, spp) in enumerate([(0, 24), (24, 40)]):
            got = torch.full((n,), 0.5, dtype=torch.float64, device="cuda")
            want = torch.full((n,), 0.5, dtype=torch.float64, device="cuda")
            rc = lib.ix_accumulate_device_noalloc(C.byref(sc), offset, spp, C.c_void_p(got.data_ptr()), 1,
                                                  C.c_void_p(stream.cuda_stream))
            assert rc == abi.IX_DONE, f"call {call}: rc {rc}"
            assert backend.accumulate_device(sc, offset, spp, want.data_ptr(), True,
                                             stream.cuda_stream) == 0
            torch.cuda.synchronize()
            g, w = got.cpu().numpy(), want.cpu().numpy()
            # same kernel, same inputs: equal to the allocating entry (f64 sums, 1e-12)
            assert np.allclose(g, w, rtol=1e-12, atol=1e-12), f"call {call}"
            assert np.all(np.isfinite(g)) and g.sum() > 0.5 * n
    finally:
        backend.close()


def test_noalloc_entry_rejects_requests_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = load_library()
    lib.ix_accumulate_device_noalloc.restype = C.c_int
    lib.ix_accumulate_device_noalloc.argtypes = [C.POINTER(abi.Scene), C.c_uint32, C.c_uint32,
                                                 C.c_void_p, C.c_int, C.c_void_p]
    fs = workloads.round_brilliant_frame(8, 8)
    sc, planes = _device_scene(torch, fs)
    sc.width = 65535
    sc.height = 65535  # under 2^32 pixels (larger frames do not route), x 2 spp: beyond 64 launches of 2^26 paths
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = lib.ix_accumulate_device_noalloc(C.byref(sc), 0, 2, C.c_void_p(out.data_ptr()), 0, None)
    assert rc == IX_NOALLOC_ERR_TOO_LARGE
    torch.cuda.synchronize()
    assert float(out.abs().sum()) == 0.0
