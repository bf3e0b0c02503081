"""The 16-byte compact request form (nvshmemx_request_compact in
include/nvshmemx_ops.h) on the host: the converter's output decodes, by the
layout the header documents, back to the same requests, and requests the
form cannot hold are refused."""
import numpy as np
import pytest

from nvshmem_b200 import (DT_DOUBLE, DT_FLOAT, DT_INT, REQ_G, REQ_GET, REQ_P, REQ_PUT, REQ_SIGNAL,
                          REQUEST_COMPACT_DTYPE, REQUEST_DTYPE, to_compact)
from nvshmem_b200.traffic import c4_batch
from _util import requests


def decode(c: np.ndarray) -> np.ndarray:
    """The header's layout, field by field."""
    out = np.zeros(len(c), dtype=REQUEST_DTYPE)
    meta = c["meta"].astype(np.uint64)
    op = (meta >> 20) & 7
    out["op"] = op
    out["dtype"] = (meta >> 23) & 3
    out["src_pe"] = meta & 1023
    out["dst_pe"] = (meta >> 10) & 1023
    is_p = op == REQ_P
    out["src_off"] = np.where(is_p, c["src_off4"].astype(np.uint64), c["src_off4"].astype(np.uint64) * 4)
    out["dst_off"] = c["dst_off4"].astype(np.uint64) * 4
    is_copy = (op == REQ_PUT) | (op == REQ_GET)
    out["bytes"] = np.where(is_copy, c["arg"].astype(np.uint64) * 4, 0)
    out["value"] = np.where(op == REQ_SIGNAL, c["arg"].view(np.int32), 0)
    assert not (meta >> 25).any()
    return out


def test_layout_is_sixteen_bytes():
    assert REQUEST_COMPACT_DTYPE.itemsize == 16


def test_c4_batch_round_trips():
    r = c4_batch(seed=4, n=20000, npes=64, heap=64 << 20)
    c = to_compact(r)
    assert c.nbytes * 2 == r.nbytes
    d = decode(c)
    keep = r.copy()
    keep["bytes"] = np.where((r["op"] == REQ_PUT) | (r["op"] == REQ_GET), r["bytes"], 0)
    keep["value"] = np.where(r["op"] == REQ_SIGNAL, r["value"], 0)
    assert np.array_equal(d, keep)


def test_every_op_round_trips():
    rows = [dict(src_off=64, dst_off=4096, bytes=12, src_pe=3, dst_pe=1023, op=REQ_PUT, dtype=DT_INT),
            dict(src_off=(16 << 30) - 4, dst_off=8, bytes=(1 << 32) - 4, src_pe=1023, dst_pe=0, op=REQ_GET,
                 dtype=DT_DOUBLE),
            dict(src_off=0, dst_off=128, bytes=0, src_pe=5, dst_pe=6, op=REQ_SIGNAL, dtype=DT_INT, value=-7),
            dict(src_off=0x3F800000, dst_off=256, bytes=0, src_pe=2, dst_pe=9, op=REQ_P, dtype=DT_FLOAT),
            dict(src_off=512, dst_off=1024, bytes=0, src_pe=7, dst_pe=8, op=REQ_G, dtype=DT_DOUBLE)]
    r = requests(rows)
    assert np.array_equal(decode(to_compact(r)), r)


@pytest.mark.parametrize("field,value", [("src_off", 66), ("dst_off", 16 << 30), ("src_pe", 1024),
                                         ("bytes", 6)])
def test_requests_without_a_compact_form_are_refused(field, value):
    r = requests([dict(src_off=64, dst_off=4096, bytes=12, src_pe=3, dst_pe=4, op=REQ_PUT, dtype=DT_INT)])
    r[0][field] = value
    with pytest.raises(ValueError):
        to_compact(r)


def test_p_of_a_double_is_refused():
    r = requests([dict(src_off=1, dst_off=8, bytes=0, src_pe=0, dst_pe=1, op=REQ_P, dtype=DT_DOUBLE)])
    with pytest.raises(ValueError):
        to_compact(r)
