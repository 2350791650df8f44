"""The bench's reference arm (`bench.py --impl reference`) on the host: the
reference's own CPU extract (its sources compiled under oracle/_ref) times whole
CoreSG::mst calls on a small case of the bench workload and prints the contract's
JSON line; under torchrun, ranks other than 0 exit 0 without output."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from checkers import Reference  # noqa: E402


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)


@pytest.mark.skipif(not Reference.available(), reason="reference not built (oracle/_ref)")
def test_reference_arm_prints_the_contract_line():
    p = _run({"RANK": "0"}, "--n", "3000", "--steps", "3", "--warmup", "1")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [x for x in p.stdout.splitlines() if x.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "MSTs/s" and d["higher_is_better"] is True
    # the bench raises the warm-up to at least 3 steps
    assert d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    assert d["config"]["workload"] == "blobs1m_d16" and d["config"]["n"] == 3000
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"RANK": "1"}, "--n", "3000", "--steps", "1", "--warmup", "1")
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
