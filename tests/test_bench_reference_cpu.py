"""The bench's reference arm on CPU: the reference's own engine (compiled from
its sources into oracle/_ref) timed on the host cores prints one JSON line in
the same contract as the GPU arm (metric, unit, direction), marked
impl = "reference", with its CPU-baseline description and an e2e block that
moves no bytes to or from a GPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libremcref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference harness not built here")
def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, lines
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "REMC replica-steps/s (batched persistent sweep + CUDA graph)"
    assert d["unit"] == "replica-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "batch64"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "MCSearch" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # the arm runs the reference alone: this repository's engine library is
    # never mapped into its process
    assert d["engine_library_mapped"] is False
    assert d["pair_energies_per_s"] > d["value"]
    # every system of the batch takes part (the batch's own mix of sizes)
    assert d["config"]["sample_systems"] == 64


def test_balanced_slices():
    sys.path.insert(0, ROOT)
    import bench
    costs = [100, 1, 50, 50, 3, 90, 10, 10, 20, 60, 5, 5]
    order = bench.balanced_order(costs, 4)
    assert sorted(order) == list(range(len(costs)))
    per = 3
    loads = [sum(costs[i] for i in order[k * per:(k + 1) * per]) for k in range(4)]
    assert max(loads) - min(loads) <= 40, loads
