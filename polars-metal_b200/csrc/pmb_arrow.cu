// pmb_arrow.cu — Arrow C Data Interface arrays as libpmb columns, without a copy.
//
// A producer that speaks the Arrow C (Device) Data Interface — polars-arrow's FFI, pyarrow,
// arrow-rs, a GPU dataframe library — hands over `struct ArrowArray` / `struct ArrowDeviceArray`
// plus `struct ArrowSchema`; the column here points at the array's own buffers. The reference
// bridges Arrow buffers to Metal in crates/polars-metal-buffer/src/bridge.rs:1-60, and its Python
// side first copies every column into `bytes` (python/polars_metal/_udf.py:1441-1456).
#include <cuda_runtime.h>

#include <cstring>

#include "pmb.h"

namespace {

// Arrow format string of a primitive type -> PMB dtype, or -1
int dtype_of_format(const char* f) {
  if (!f || !f[0] || f[1] != '\0') return -1;
  switch (f[0]) {
    case 'b': return PMB_BOOL;
    case 'c': return PMB_I8;
    case 'C': return PMB_U8;
    case 's': return PMB_I16;
    case 'S': return PMB_U16;
    case 'i': return PMB_I32;
    case 'I': return PMB_U32;
    case 'l': return PMB_I64;
    case 'L': return PMB_U64;
    case 'f': return PMB_F32;
    case 'g': return PMB_F64;
    default: return -1;
  }
}

int fill(const struct ArrowArray* a, const struct ArrowSchema* s, int32_t on_device, pmb_column* out) {
  if (!a || !s || !out) return PMB_E_INVALID;
  if (!a->release || !s->release) return PMB_E_INVALID;  // a released (moved-from) structure
  // a dictionary-encoded column: its indices are this array's buffers, in the schema's format
  const int dt = dtype_of_format(s->format);
  if (dt < 0 || (s->dictionary && (dt == PMB_BOOL || dt == PMB_F32 || dt == PMB_F64))) return PMB_E_UNSUPPORTED;
  if (a->n_buffers != 2 || !a->buffers || a->length < 0 || a->offset < 0) return PMB_E_INVALID;
  if (a->length > 0 && !a->buffers[1]) return PMB_E_INVALID;
  memset(out, 0, sizeof(*out));
  out->data = a->buffers[1];
  out->validity = a->null_count == 0 ? nullptr : (const uint8_t*)a->buffers[0];
  out->length = a->length;
  out->offset = a->offset;
  out->dtype = dt;
  out->on_device = on_device;
  return PMB_OK;
}

}  // namespace

extern "C" int pmb_column_from_arrow(const struct ArrowArray* array, const struct ArrowSchema* schema,
                                     pmb_column* out) {
  return fill(array, schema, 0, out);
}

extern "C" int pmb_column_from_arrow_device(const struct ArrowDeviceArray* array, const struct ArrowSchema* schema,
                                            pmb_column* out) {
  if (!array) return PMB_E_INVALID;
  switch (array->device_type) {
    case ARROW_DEVICE_CUDA: {
      // the kernels dereference the buffers on the current device: an array of another GPU
      // would be read through a peer mapping or fault, so it is refused here
      int cur = -1;
      if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        return PMB_E_UNSUPPORTED;  // no usable CUDA device in this process
      }
      if (array->device_id != (int64_t)cur) return PMB_E_INVALID;
      return fill(&array->array, schema, 1, out);
    }
    case ARROW_DEVICE_CPU:
    case ARROW_DEVICE_CUDA_HOST: return fill(&array->array, schema, 0, out);
    default: return PMB_E_UNSUPPORTED;
  }
}

extern "C" int pmb_column_is_dictionary(const struct ArrowSchema* schema) {
  if (!schema || !schema->release) return PMB_E_INVALID;
  return schema->dictionary ? 1 : 0;
}
