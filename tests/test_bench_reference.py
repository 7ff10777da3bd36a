"""The benchmark's reference arm on the host: `bench.py --impl reference` times the reference's own complex64
executor (or its restatement) on the headline workload and prints one JSON line with the contract's keys; under a
multi-rank launch only rank 0 does any work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_the_contract_line():
    p = _run({"RANK": "0"})
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "amps/s" and line["value"] > 0
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 0
    assert line["config"]["workload"] == "matching_n70_d70_s2_w30" and line["config"]["width"] == 30
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "amps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_nothing():
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0 and p.stdout.strip() == "", (p.stdout, p.stderr[-2000:])
