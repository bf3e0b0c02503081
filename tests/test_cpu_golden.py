"""The CPU oracle against the reference's own build: the heap hashes that
the reference's sources (compiled for sm_100a, all MPI ranks on one GPU)
produced for each scenario of tests/golden/ref_scenarios.py must equal what
the oracle predicts, bit for bit.  This is what pins the oracle."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from ref_scenarios import SCENARIOS, oracle_hashes, scenario_id  # noqa: E402

GOLDEN = os.path.join(HERE, "golden", "ref_heaps.json")


def _golden():
    if not os.path.exists(GOLDEN):
        pytest.skip("tests/golden/ref_heaps.json not generated yet")
    with open(GOLDEN) as f:
        return json.load(f)["scenarios"]


@pytest.mark.parametrize("s", SCENARIOS, ids=scenario_id)
def test_oracle_matches_reference_build(s):
    g = _golden()
    assert scenario_id(s) in g, "golden file lacks this scenario; regenerate it"
    assert oracle_hashes(s) == g[scenario_id(s)]["reference"]
