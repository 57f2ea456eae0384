"""bench.py's reference arm on the host cores (no GPU needed).

The arm times the reference's own CPU MPM solver (built into oracle/_ref from
the reference's sources) on the bench workload and prints one JSON line with
the keys the bench contract names.  Under a multi-rank launch only rank 0
runs it and prints; the other ranks exit 0 without work.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_mpm.so")

pytestmark = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built")


def _json_lines(out):
    return [json.loads(s) for s in out.splitlines() if s.startswith("{")]


def _check_reference_line(d):
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"] == "two_material_drop" and d["config"]["n_particles"] == 2097152
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["warmup"] >= 3


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_reference_line(lines[0])


def test_reference_arm_under_two_ranks_prints_once():
    env = dict(os.environ, WORLD_SIZE="2", MASTER_ADDR="127.0.0.1")
    outs = []
    for rank in (1, 0):
        e = dict(env, RANK=str(rank), LOCAL_RANK=str(rank))
        r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                            "--warmup", "1"], cwd=ROOT, env=e, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(_json_lines(r.stdout))
    assert outs[0] == []  # rank 1: no work, no line
    assert len(outs[1]) == 1
    _check_reference_line(outs[1][0])
