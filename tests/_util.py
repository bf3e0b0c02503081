"""Shared helpers for the tests: request-list builders and heap comparison."""
import numpy as np

from nvshmem_b200 import (DT_DOUBLE, DT_FLOAT, DT_INT, REQ_G, REQ_GET, REQ_P,
                          REQ_PUT, REQ_SIGNAL, REQUEST_DTYPE)
from nvshmem_b200.traffic import Stream

WIDTH = {DT_INT: 4, DT_FLOAT: 4, DT_DOUBLE: 8}


def requests(rows):
    """rows: dicts with src_off, dst_off, bytes, src_pe, dst_pe, op, dtype, value."""
    r = np.zeros(len(rows), dtype=REQUEST_DTYPE)
    for i, d in enumerate(rows):
        for k, v in d.items():
            r[i][k] = v
    return r


def random_requests(seed, n, npes, heap, ops=(REQ_PUT, REQ_GET, REQ_SIGNAL, REQ_P, REQ_G),
                    max_bytes=65536, align=4, mixed_alignment=True):
    """n requests with disjoint destinations in the upper half of each heap and
    sources in the lower half.  Offsets are multiples of `align`, with a
    random 0..12 byte skew per request when mixed_alignment (so source and
    destination differ modulo 16)."""
    st = Stream(seed)
    half = heap // 2
    rows = []
    cursor = [half] * npes
    for i in range(n):
        op = ops[int(st.randint(1, len(ops))[0])]
        dt = int(st.randint(1, 3)[0])
        w = WIDTH[dt]
        src_pe = int(st.randint(1, npes)[0])
        dst_pe = int(st.randint(1, npes)[0])
        if op in (REQ_PUT, REQ_GET):
            nb = int(st.randint(1, max_bytes // w + 1)[0]) * w
        else:
            nb = 0
        wb = 4 if op == REQ_SIGNAL else (w if op in (REQ_P, REQ_G) else nb)
        skew_s = int(st.randint(1, 4)[0]) * 4 if mixed_alignment else 0
        skew_d = int(st.randint(1, 4)[0]) * 4 if mixed_alignment else 0
        if op in (REQ_P, REQ_G, REQ_SIGNAL):
            skew_d = 0 if w == 8 or op == REQ_SIGNAL else skew_d
            skew_s = 0 if w == 8 else skew_s
        src_off = (int(st.randint(1, max(1, (half - nb - 64) // align))[0]) * align // 16 * 16) + skew_s
        dst_off = cursor[dst_pe] + skew_d
        cursor[dst_pe] = (dst_off + wb + 15) // 16 * 16 + 16 * int(st.randint(1, 4)[0])
        if cursor[dst_pe] > heap:
            break
        row = dict(src_off=src_off, dst_off=dst_off, bytes=nb, src_pe=src_pe, dst_pe=dst_pe,
                   op=op, dtype=dt, value=int(st.randint(1, 1 << 30)[0]))
        if op == REQ_P:
            row["src_off"] = int(st.u64(1)[0]) & ((1 << (8 * w)) - 1)
        rows.append(row)
    return requests(rows)


def heap_images(sh, npes, nbytes):
    return np.stack([sh.read(pe, 0, nbytes) for pe in range(npes)])


def first_diff(a, b):
    d = np.nonzero(a.reshape(-1) != b.reshape(-1))[0]
    return None if len(d) == 0 else int(d[0])
