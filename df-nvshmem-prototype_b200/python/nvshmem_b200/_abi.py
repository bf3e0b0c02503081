"""Constants and record layouts of the library's C ABI (include/nvshmemx.h,
include/nvshmemx_ops.h), with no dependency on the shared library itself, so
that the traffic generators can be used where the library is not loaded
(e.g. by the CPU baseline)."""
from __future__ import annotations

import numpy as np

# status codes (include/nvshmemx.h)
SUCCESS, ERR_INVALID, ERR_NOMEM, ERR_CUDA, ERR_STATE, ERR_TIMEOUT, ERR_BOUNDS, ERR_COOP, ERR_UNSUPPORTED = range(9)
ERRORS_EXIT, ERRORS_RETURN = 0, 1
CMP_EQ, CMP_NE, CMP_GT, CMP_GE, CMP_LT, CMP_LE = range(6)

# requests (include/nvshmemx_ops.h)
REQ_PUT, REQ_GET, REQ_SIGNAL, REQ_P, REQ_G = range(5)
DT_INT, DT_FLOAT, DT_DOUBLE = range(3)
DT_WIDTH = {DT_INT: 4, DT_FLOAT: 4, DT_DOUBLE: 8}
MODE_THREAD, MODE_WARP, MODE_BLOCK, MODE_BULK = range(4)

REQUEST_DTYPE = np.dtype([
    ("src_off", "<u8"), ("dst_off", "<u8"), ("bytes", "<u4"),
    ("src_pe", "<u2"), ("dst_pe", "<u2"), ("op", "u1"), ("dtype", "u1"),
    ("flags", "<u2"), ("value", "<i4"),
])
assert REQUEST_DTYPE.itemsize == 32

# nvshmemx_request_compact: offsets / 4, PUT-GET bytes / 4 or SIGNAL value,
# meta = src_pe | dst_pe << 10 | op << 20 | dtype << 23
REQUEST_COMPACT_DTYPE = np.dtype([("src_off4", "<u4"), ("dst_off4", "<u4"), ("arg", "<u4"), ("meta", "<u4")])
assert REQUEST_COMPACT_DTYPE.itemsize == 16

TRACE_DTYPE = np.dtype([
    ("t_ns", "<i8"), ("spin_ns", "<i8"), ("local_addr", "<u8"), ("remote_addr", "<u8"),
    ("bytes", "<u4"), ("op", "<u2"), ("pe", "<u2"), ("peer", "<u2"), ("tid", "<u2"),
    ("block", "<u4"),
])
assert TRACE_DTYPE.itemsize == 48

# nvshmemx_picked_group (include/nvshmemx_picker.h)
PICKED_GROUP_DTYPE = np.dtype([("first", "<i4"), ("count", "<i4"), ("variant", "<i4"), ("source", "<i4"),
                               ("features", "<f4", (6,))])
assert PICKED_GROUP_DTYPE.itemsize == 40
PATTERN_PAIRS, PATTERN_ALLTOALL, PATTERN_NEIGHBOR, PATTERN_RANDOM = range(4)
