"""The picker at run time, through the C ABI (include/nvshmemx_picker.h):
nvshmemx_picker_pick takes the network's choice inside the measured table's
range and the table's nearest class outside it, and
nvshmemx_batch_execute_picked -- which groups a request array and runs each
group with its picked variant -- leaves every heap bit-identical to the
oracle whichever of the 12 variants runs."""
import ctypes
from ctypes import byref, c_float, c_int, c_void_p

import numpy as np
import pytest

from nvshmem_b200 import ERR_BOUNDS, PICKED_GROUP_DTYPE, REQ_PUT, _lib as L
from nvshmem_b200 import picker as P
from oracle.model import Model
from _util import first_diff, heap_images, random_requests, requests

pytestmark = pytest.mark.gpu

NV = 12


def _picker(net, tx, tt):
    h = c_void_p(0)
    tx = np.ascontiguousarray(tx, np.float32)
    tt = np.ascontiguousarray(tt, np.float32)
    assert L.lib.nvshmemx_picker_create(net.h, tx.ctypes.data, tt.ctypes.data, len(tx), byref(h)) == 0
    return h, (tx, tt)


def _pick(h, X):
    X = np.ascontiguousarray(X, np.float32)
    v = np.zeros(len(X), np.int32)
    s = np.zeros(len(X), np.int32)
    assert L.lib.nvshmemx_picker_pick(h, X.ctypes.data, len(X), v.ctypes.data, s.ctypes.data) == 0
    return v, s


def test_network_inside_the_range_table_outside():
    rng = np.random.default_rng(3)
    tx = rng.uniform(0, 10, size=(50, 6)).astype(np.float32)
    tt = rng.uniform(0.01, 1.0, size=(50, NV)).astype(np.float32)
    tt[:, 5] = np.nan  # a variant that never ran is never the table's choice
    net = P.MLP(seed=5)
    h, keep = _picker(net, tx, tt)
    try:
        inside = rng.uniform(1, 9, size=(40, 6)).astype(np.float32)
        v, s = _pick(h, inside)
        want, _ = net.pick(inside)
        assert np.all(s == 0) and np.array_equal(v, want)
        outside = inside.copy()
        outside[:, 2] = 20.0
        v, s = _pick(h, outside)
        assert np.all(s == 1)
        # the table's choice: the best measured variant of the nearest class
        mean, sd = tx.mean(0), np.maximum(tx.std(0), 1e-3)
        d = ((((outside[:, None, :] - tx[None]) / sd) ** 2).sum(-1))
        nn = d.argmin(1)
        assert np.array_equal(v, np.nanargmin(tt[nn], axis=1))
        tv = np.zeros(len(outside), np.int32)
        assert L.lib.nvshmemx_picker_table_pick(h, outside.ctypes.data, len(outside), tv.ctypes.data) == 0
        assert np.array_equal(tv, v)
    finally:
        L.lib.nvshmemx_picker_destroy(h)


def _execute(b, h, reqs, pattern=3):
    groups = np.zeros(64, PICKED_GROUP_DTYPE)
    ng, st, ms, run = c_int(), c_int(), c_float(), c_float()
    r = np.ascontiguousarray(reqs)
    rc = L.lib.nvshmemx_batch_execute_picked(b.h, h, r.ctypes.data, len(r), pattern, groups.ctypes.data, len(groups),
                                             byref(ng), byref(st), byref(ms), byref(run))
    if rc == 0:
        assert 0 < run.value <= ms.value
    return rc, groups[:ng.value], st.value, ms.value


@pytest.mark.parametrize("variant", range(NV))
def test_execute_picked_every_variant_bit_exact(shmem_factory, variant):
    """A one-class table where only `variant` was measured, so every group
    (all outside the table's single point) runs that variant."""
    npes, heap = 8, 2 << 20
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 9)
        om.fill_random(pe, 0, heap, 9)
    reqs = random_requests(300 + variant, 600, npes, heap, max_bytes=40000)
    net = P.MLP(seed=1)
    tt = np.full((1, NV), np.nan, np.float32)
    tt[0, variant] = 1.0
    h, keep = _picker(net, np.full((1, 6), 100.0, np.float32), tt)
    try:
        with sh.batch(len(reqs), int(reqs["bytes"].sum()) + 8 * len(reqs), 256) as b:
            rc, groups, st, ms = _execute(b, h, reqs)
            assert rc == 0 and st == 0 and ms > 0
            copy = groups[groups["source"] != 2]
            assert len(copy) > 1 and np.all(copy["variant"] == variant) and np.all(copy["source"] == 1)
            assert groups["count"].sum() == len(reqs)
            # the groups tile the grouped order
            order = np.argsort(groups["first"])
            assert np.array_equal(np.cumsum(groups["count"][order])[:-1], groups["first"][order][1:])
            rc, _, st, _ = _execute(b, h, reqs)  # idempotent: sources never overlap destinations
            assert rc == 0 and st == 0
        assert sh.status() == 0
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
    finally:
        L.lib.nvshmemx_picker_destroy(h)


def test_execute_picked_with_the_trained_picker_on_c4_traffic(shmem_factory):
    """The measured table and a trained network on C4-shaped traffic
    (random PE pairs): groups carry the features the call computed."""
    import os
    if not os.path.exists(P.DATA):
        pytest.skip("variant timings not measured yet")
    from nvshmem_b200.traffic import c4_batch
    npes, heap = 16, 4 << 20
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 11)
        om.fill_random(pe, 0, heap, 11)
    reqs = c4_batch(seed=12, n=3000, npes=npes, heap=heap, hi=256 << 10)
    d = np.load(P.DATA)
    pk = P.Picker(d["train_x"], d["train_t"], seed=0)
    pk.fit(epochs=200)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
        rc, groups, st, ms = _execute(b, pk.h, reqs, pattern=3)
        assert rc == 0 and st == 0
    assert sh.status() == 0
    f = groups["features"]
    assert np.all(f[:, 3] == np.log2(npes)) and np.all(f[:, 4] == 3)
    assert np.allclose(2 ** f[:, 5], groups["count"], rtol=1e-5)
    om.apply_requests(reqs)
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None
    pk.close()


def test_execute_picked_from_the_batch_pinned_buffer(shmem_factory):
    """The requests may already sit in the batch's pinned host buffer, which
    the call also uses to stage the grouped order."""
    npes, heap = 8, 2 << 20
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 13)
        om.fill_random(pe, 0, heap, 13)
    reqs = random_requests(77, 500, npes, heap, max_bytes=30000)
    net = P.MLP(seed=2)
    h, keep = _picker(net, np.full((1, 6), 100.0, np.float32), np.ones((1, NV), np.float32))
    try:
        with sh.batch(len(reqs), int(reqs["bytes"].sum()) + 8 * len(reqs), 256) as b:
            buf = b.host_buffer()
            buf[:len(reqs)] = reqs
            rc, groups, st, _ = _execute(b, h, buf[:len(reqs)])
            assert rc == 0 and st == 0 and groups["count"].sum() == len(reqs)
        assert sh.status() == 0
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
    finally:
        L.lib.nvshmemx_picker_destroy(h)


def test_execute_picked_rejects_before_running(shmem_factory):
    npes, heap = 4, 1 << 20
    sh = shmem_factory(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 2)
    before = heap_images(sh, npes, heap)
    good = random_requests(5, 50, npes, heap, max_bytes=4000)
    bad = requests([dict(src_off=(1 << 64) - 4, dst_off=heap // 2, bytes=8, src_pe=0, dst_pe=1, op=REQ_PUT,
                         dtype=0)])
    reqs = np.concatenate([good, bad])
    net = P.MLP(seed=1)
    h, keep = _picker(net, np.zeros((1, 6), np.float32), np.ones((1, NV), np.float32))
    try:
        with sh.batch(len(reqs), 1 << 20, 256) as b:
            rc, _, _, _ = _execute(b, h, reqs)
            assert rc == ERR_BOUNDS
    finally:
        L.lib.nvshmemx_picker_destroy(h)
    assert sh.status() == ERR_BOUNDS  # the host-side refusal, reported once
    assert np.array_equal(heap_images(sh, npes, heap), before)
