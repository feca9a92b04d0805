"""pmb_cumsum_u8_to_u32_noalloc: the prefix sum for callers that must not allocate device memory
(their host framework already owns the device's memory pool, or a cudaMalloc would stall a
latency-critical loop by synchronising the device). It must match the allocating entry point
bit for bit, on consecutive calls that share its fixed scratch array.

This file is named so that pytest collects it last."""

import ctypes as C

import numpy as np
import pytest

from polars_b200 import _abi as A
from polars_b200._native import default_handle

pytestmark = pytest.mark.gpu


def _allocating_reference(a: np.ndarray) -> np.ndarray:
    h = default_handle()
    out = np.empty(a.size, dtype=np.uint32)
    h.check(h._lib.pmb_cumsum_u8_to_u32(h.raw, a.ctypes.data, out.ctypes.data, a.size, 0))
    return out


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls():
    import torch

    lib = A.lib()
    rng = np.random.default_rng(2024)
    # the second call is shorter, so stale look-back state of the first would break it
    for n in (3_000_017, 1_234_567):
        a = rng.integers(0, 256, n).astype(np.uint8)
        want = _allocating_reference(a)
        dev_in = torch.from_numpy(a).cuda()
        dev_out = torch.empty(n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = lib.pmb_cumsum_u8_to_u32_noalloc(C.c_void_p(dev_in.data_ptr()), C.c_void_p(dev_out.data_ptr()), n, None)
        assert rc == A.PMB_OK
        got = dev_out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = A.lib()
    rc = lib.pmb_cumsum_u8_to_u32_noalloc(C.c_void_p(1), C.c_void_p(1), A.NOALLOC_MAX_ROWS + 1, None)
    assert rc == A.PMB_E_INVALID
