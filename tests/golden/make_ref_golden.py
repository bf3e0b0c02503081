"""Generates tests/golden/ref_heaps.json by running every scenario of
ref_scenarios.py through the REFERENCE's own build (oracle/_ref/ref_driver,
built by oracle/ref_build/Makefile from the reference sources), all MPI ranks
on one GPU.  Needs a GPU; run from the repository root:

  python tests/golden/make_ref_golden.py [--out tests/golden/ref_heaps.json]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from ref_scenarios import (REPO, SCENARIOS, halo_blocks, request_list,  # noqa: E402
                           scenario_id)

DRIVER = os.path.join(REPO, "oracle", "_ref", "ref_driver")


def run_driver(s: dict, timeout: int = 300) -> dict:
    env = dict(os.environ, MPI_SHIM_NP=str(s["npes"]), MPI_SHIM_TIMEOUT_S="60")
    with tempfile.TemporaryDirectory() as td:
        name = s["name"]
        if name == "alloc":
            args = ["alloc"]
        elif name == "requests":
            path = os.path.join(td, "reqs.bin")
            request_list(s["npes"], s["heap"], s["nreq"], s["req_seed"]).tofile(path)
            args = ["requests", path, str(s["heap"]), str(s["seed"])]
        elif name == "alltoall":
            args = ["alltoall", str(s["bytes"]), str(s["rounds"]), str(s["seed"])]
        elif name == "halo":
            prefix = os.path.join(td, "block")
            for pe, b in enumerate(halo_blocks(s["n"], s["npes"])):
                b.tofile(prefix + str(pe))
            args = ["halo", str(s["n"]), str(s["iters"]), prefix]
        elif name == "pingpong":
            args = ["pingpong", str(s["len"]), str(s["iters"]), str(s["seed"])]
        else:
            raise ValueError(name)
        p = subprocess.run([DRIVER] + args, env=env, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"{scenario_id(s)}: ref_driver exited {p.returncode}: {p.stderr[-2000:]}")
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    if name == "alloc":
        first = lines[0]
        return {"offsets": first["offsets"], "after_cleanup": first["after_cleanup"]}
    return {str(x["rank"]): x["fnv"] for x in sorted(lines, key=lambda x: x["rank"])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_heaps.json"))
    a = ap.parse_args()
    out = {"generator": "tests/golden/make_ref_golden.py", "driver": "oracle/_ref/ref_driver", "scenarios": {}}
    for s in SCENARIOS:
        out["scenarios"][scenario_id(s)] = {"spec": s, "reference": run_driver(s)}
        print(scenario_id(s), "ok", flush=True)
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
