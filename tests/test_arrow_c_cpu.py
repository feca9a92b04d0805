"""Arrow C Data Interface ingest (pmb_column_from_arrow, pmb_column_from_arrow_device) without a
GPU: pyarrow arrays exported through the C (Device) Data Interface become libpmb columns that
point at the arrays' own buffers, with their offsets, validity and dtypes."""

import ctypes as C

import numpy as np
import pyarrow as pa
import pytest

from polars_b200 import _abi as A

TYPES = [(pa.bool_(), A.BOOL), (pa.int8(), A.I8), (pa.uint8(), A.U8), (pa.int16(), A.I16), (pa.uint16(), A.U16),
         (pa.int32(), A.I32), (pa.uint32(), A.U32), (pa.int64(), A.I64), (pa.uint64(), A.U64),
         (pa.float32(), A.F32), (pa.float64(), A.F64)]


def _release(obj):
    fn = C.CFUNCTYPE(None, C.c_void_p)(obj.release)
    fn(C.addressof(obj))


def _export(arr, device=False):
    schema = A.ArrowSchema()
    if device:
        out = A.ArrowDeviceArray()
        arr._export_to_c_device(C.addressof(out), C.addressof(schema))
    else:
        out = A.ArrowArray()
        arr._export_to_c(C.addressof(out), C.addressof(schema))
    return out, schema


@pytest.mark.parametrize("typ,dt", TYPES, ids=lambda x: str(x))
@pytest.mark.parametrize("device", [False, True])
def test_arrays_become_columns_over_their_buffers(typ, dt, device):
    lib = A.lib()
    rng = np.random.default_rng(1)
    n = 1000
    vals = rng.random(n) < 0.5 if typ == pa.bool_() else rng.integers(0, 100, n).astype(typ.to_pandas_dtype())
    arr = pa.array(vals, type=typ, mask=rng.random(n) < 0.1).slice(13, 900)
    out, schema = _export(arr, device)
    col = A.Column()
    fn = lib.pmb_column_from_arrow_device if device else lib.pmb_column_from_arrow
    assert fn(C.byref(out), C.byref(schema), C.byref(col)) == 0
    bufs = arr.buffers()
    assert col.dtype == dt and col.length == 900 and col.offset == arr.offset == 13
    assert col.data == bufs[1].address and col.validity == bufs[0].address  # no copy
    assert col.on_device == 0
    _release(out.array if device else out)
    _release(schema)


def test_no_nulls_means_no_bitmap_and_other_device_types_are_refused():
    lib = A.lib()
    arr = pa.array(np.arange(10, dtype=np.int64))
    out, schema = _export(arr, device=True)
    col = A.Column()
    assert lib.pmb_column_from_arrow_device(C.byref(out), C.byref(schema), C.byref(col)) == 0
    assert col.validity is None and col.on_device == 0
    out.device_type = 7  # another device type
    assert lib.pmb_column_from_arrow_device(C.byref(out), C.byref(schema), C.byref(col)) == 5  # PMB_E_UNSUPPORTED
    out.device_type = A.ARROW_DEVICE_CPU
    _release(out.array)
    _release(schema)


def test_dictionary_arrays_give_their_codes_and_other_types_are_refused():
    lib = A.lib()
    d = pa.array(["b", "a", None, "b"]).dictionary_encode()
    out, schema = _export(d)
    col = A.Column()
    assert lib.pmb_column_from_arrow(C.byref(out), C.byref(schema), C.byref(col)) == 0
    assert col.dtype == A.I32 and col.length == 4 and col.data == d.indices.buffers()[1].address
    _release(out)
    _release(schema)
    s = pa.array(["x", "y"])
    out, schema = _export(s)
    assert lib.pmb_column_from_arrow(C.byref(out), C.byref(schema), C.byref(col)) == 5  # strings: not a column
    _release(out)
    _release(schema)
    released = A.ArrowArray()
    assert lib.pmb_column_from_arrow(C.byref(released), C.byref(schema), C.byref(col)) == 1  # PMB_E_INVALID


def test_cuda_arrays_of_another_device_or_without_a_device_are_refused():
    # a CUDA array must live on the current device; in a process without a CUDA device (this
    # test's CPU run) every CUDA array is refused, whatever its device_id
    import torch

    lib = A.lib()
    arr = pa.array(np.arange(10, dtype=np.int64))
    out, schema = _export(arr, device=True)
    col = A.Column()
    out.device_type = A.ARROW_DEVICE_CUDA
    cur = torch.cuda.current_device() if torch.cuda.is_available() else None
    out.device_id = 5 if cur is None else cur + 1
    rc = lib.pmb_column_from_arrow_device(C.byref(out), C.byref(schema), C.byref(col))
    assert rc == (5 if cur is None else 1)  # PMB_E_UNSUPPORTED without a device, else PMB_E_INVALID
    if cur is not None:
        out.device_id = cur
        assert lib.pmb_column_from_arrow_device(C.byref(out), C.byref(schema), C.byref(col)) == 0
        assert col.on_device == 1
    out.device_type = A.ARROW_DEVICE_CPU
    _release(out.array)
    _release(schema)


def test_dictionary_schemas_are_told_apart():
    lib = A.lib()
    d = pa.array(["b", "a", None, "b"]).dictionary_encode()
    out, schema = _export(d)
    assert lib.pmb_column_is_dictionary(C.byref(schema)) == 1
    _release(out)
    _release(schema)
    out, schema = _export(pa.array([1, 2, 3]))
    assert lib.pmb_column_is_dictionary(C.byref(schema)) == 0
    _release(out)
    _release(schema)
    assert lib.pmb_column_is_dictionary(None) == 1  # PMB_E_INVALID
