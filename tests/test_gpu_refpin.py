"""This library against the reference's own build on the same scenarios:
the heaps our CUDA path leaves must hash to what the reference's sources
(compiled for sm_100a, ranks on one GPU) left, as committed in
tests/golden/ref_heaps.json.  When the reference build is present on the
machine (oracle/_ref/ref_driver) it is also re-run live."""
import json
import os
import sys

import numpy as np
import pytest

from nvshmem_b200 import DT_FLOAT, MODE_BLOCK, MODE_THREAD, MODE_WARP, REQ_PUT
from oracle.model import fnv1a

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from ref_scenarios import (ALLOC_SIZES, REPO, SCENARIOS, halo_blocks,  # noqa: E402
                           request_list, scenario_id)

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(HERE, "golden", "ref_heaps.json")


def _golden(s):
    if not os.path.exists(GOLDEN):
        pytest.skip("tests/golden/ref_heaps.json not generated yet")
    with open(GOLDEN) as f:
        return json.load(f)["scenarios"][scenario_id(s)]["reference"]


def _hashes(sh, npes, heap):
    return {str(pe): f"{fnv1a(sh.read(pe, 0, heap)):016x}" for pe in range(npes)}


def _ours(s, shmem_factory, mode=MODE_THREAD):
    name, npes = s["name"], s["npes"]
    if name == "alloc":
        sh = shmem_factory(npes, 1 << 20)
        base = sh.alloc(0)
        offs = [sh.alloc(x) - base for x in ALLOC_SIZES]
        sh.cleanup()
        return {"offsets": offs, "after_cleanup": sh.alloc(16) - base}
    if name == "requests":
        sh = shmem_factory(npes, s["heap"])
        for pe in range(npes):
            sh.fill_random(pe, 0, s["heap"], s["seed"])
        sh.exec_requests(request_list(npes, s["heap"], s["nreq"], s["req_seed"]), mode)
        assert sh.status() == 0
        return _hashes(sh, npes, s["heap"])
    if name == "alltoall":
        heap = 2 * npes * s["bytes"]
        sh = shmem_factory(npes, heap)
        for pe in range(npes):
            sh.fill_random(pe, 0, heap, s["seed"])
        sh.alltoall(REQ_PUT, DT_FLOAT, 0, npes * s["bytes"], s["bytes"], rounds=s["rounds"],
                    mode=mode, ctas_per_pe=2)
        assert sh.status() == 0
        return _hashes(sh, npes, heap)
    if name == "halo":
        n = s["n"]
        block, ghosts = n ** 3 * 8, 6 * n * n * 8
        heap = (block + ghosts + 64 + 4095) // 4096 * 4096
        sh = shmem_factory(npes, heap)
        for pe, b in enumerate(halo_blocks(n, npes)):
            sh.memset(pe, 0, 0, heap)
            sh.write(pe, 0, b)
        sh.halo(2, 2, 2, n, 0, block, block + ghosts, s["iters"], 2)
        assert sh.status() == 0
        return _hashes(sh, npes, heap)
    if name == "pingpong":
        heap = (4096 + s["len"] * 4 + 4095) // 4096 * 4096
        sh = shmem_factory(2, heap)
        for pe in range(2):
            sh.fill_random(pe, 0, heap, s["seed"])
            sh.memset(pe, 0, 0, 4)
        sh.pingpong(0, 64, s["len"], s["iters"], skip=0)
        assert sh.status() == 0
        return _hashes(sh, 2, heap)
    raise ValueError(name)


@pytest.mark.parametrize("s", SCENARIOS, ids=scenario_id)
def test_library_matches_reference_build(s, shmem_factory):
    assert _ours(s, shmem_factory) == _golden(s)


@pytest.mark.parametrize("s", [x for x in SCENARIOS if x["name"] in ("requests", "alltoall")], ids=scenario_id)
@pytest.mark.parametrize("mode", [MODE_WARP, MODE_BLOCK])
def test_cooperative_modes_match_reference_build(s, mode, shmem_factory):
    assert _ours(s, shmem_factory, mode) == _golden(s)


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref", "ref_driver")),
                    reason="reference build not present")
@pytest.mark.parametrize("s", SCENARIOS[:4], ids=scenario_id)
def test_reference_build_live_rerun(s):
    from make_ref_golden import run_driver
    assert run_driver(s) == _golden(s)
