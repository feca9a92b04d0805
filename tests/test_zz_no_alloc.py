"""pmb_cumsum_u8_to_u32_noalloc: the prefix sum for callers that must not allocate device memory
(their host framework already owns the device's memory pool, or a cudaMalloc would stall a
latency-critical loop by synchronising the device). It must match the allocating entry point
bit for bit, and the oracle's prefix sum, on consecutive calls that share its fixed scratch
array, on a non-default stream, and at its largest size.

This file is named so that pytest collects it last."""

import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle
from polars_b200 import _abi as A
from polars_b200._native import default_handle

pytestmark = pytest.mark.gpu


def _allocating_reference(a: np.ndarray) -> np.ndarray:
    h = default_handle()
    out = np.empty(a.size, dtype=np.uint32)
    h.check(h._lib.pmb_cumsum_u8_to_u32(h.raw, a.ctypes.data, out.ctypes.data, a.size, 0))
    return out


def _noalloc(a: np.ndarray, stream=None) -> np.ndarray:
    """The prefix sum through the no-allocation entry point, on `stream` (a torch stream; None is
    the legacy default stream)."""
    import torch

    lib = A.lib()
    n = a.size
    dev_in = torch.from_numpy(a).cuda()
    dev_out = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    handle = None if stream is None else C.c_void_p(stream.cuda_stream)
    rc = lib.pmb_cumsum_u8_to_u32_noalloc(C.c_void_p(dev_in.data_ptr()), C.c_void_p(dev_out.data_ptr()), n, handle)
    assert rc == A.PMB_OK
    if stream is not None:
        stream.synchronize()
    return dev_out.cpu().numpy().view(np.uint32)


def test_noalloc_matches_the_oracle_and_the_allocating_entry_point_on_consecutive_calls():
    rng = np.random.default_rng(2024)
    # the second call is shorter, so stale look-back state of the first would break it
    for n in (3_000_017, 1_234_567):
        a = rng.integers(0, 256, n).astype(np.uint8)
        got = _noalloc(a)
        assert np.array_equal(got, pyoracle.cumsum_u8_to_u32(a))
        assert np.array_equal(got, _allocating_reference(a))


def test_noalloc_on_a_non_default_stream():
    import torch

    rng = np.random.default_rng(7)
    a = rng.integers(0, 256, 777_777).astype(np.uint8)
    s = torch.cuda.Stream()
    got = _noalloc(a, stream=s)
    assert np.array_equal(got, pyoracle.cumsum_u8_to_u32(a))


def test_noalloc_at_its_maximum_size_fills_every_tile():
    # PMB_NOALLOC_MAX_ROWS rows use every tile state of the scratch array; values below 32 keep
    # the total under 2^32, so the last prefix is the plain sum
    rng = np.random.default_rng(11)
    n = A.NOALLOC_MAX_ROWS
    a = rng.integers(0, 32, n).astype(np.uint8)
    got = _noalloc(a)
    want = pyoracle.cumsum_u8_to_u32(a)
    assert np.array_equal(got, want)
    assert int(got[-1]) == int(a.sum(dtype=np.int64))
    # and a short call after it still starts from clean scratch
    b = rng.integers(0, 256, 4099).astype(np.uint8)
    assert np.array_equal(_noalloc(b), pyoracle.cumsum_u8_to_u32(b))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = A.lib()
    rc = lib.pmb_cumsum_u8_to_u32_noalloc(C.c_void_p(1), C.c_void_p(1), A.NOALLOC_MAX_ROWS + 1, None)
    assert rc == A.PMB_E_INVALID
