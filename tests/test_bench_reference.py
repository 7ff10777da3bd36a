"""The benchmark's reference arm on the host: `bench.py --impl reference` times the reference's own complex64
executor (or its restatement) on the headline workload and prints one JSON line with the contract's keys; under a
multi-rank launch only rank 0 does any work.  The arm reads the committed headline plan, so its process maps no
shared object of this repository's package (the timed executor is the reference's, and nothing of the product is
loaded beside it)."""
import json
import os
import subprocess
import sys

from conftest import GOLDEN

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra, *extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0"] + list(extra), cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=900)


def test_reference_arm_prints_the_contract_line():
    p = _run({"RANK": "0"}, "--ref-samples", "0")
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "amps/s" and line["value"] > 0
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 0
    assert line["config"]["workload"] == "matching_n70_d70_s2_w30" and line["config"]["width"] == 30
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "amps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert not [p for p in line["repo_libraries_loaded"] if "libgsb" in p], line["repo_libraries_loaded"]
    assert not [p for p in line["repo_libraries_loaded"] if p.startswith("exact-graphstate-sampling_b200")]


def test_reference_arm_times_exact_samples(tmp_path):
    """s/sample of the reference executor's `sample` mode (gsamp2.cpp:149-152), here on a small plan."""
    case = json.load(open(os.path.join(GOLDEN, "planner_cases.json")))["cases"][0]
    path = tmp_path / "small_plan.txt"
    path.write_text(case["inplace_plan"])
    p = _run({"RANK": "0"}, "--ref-plan", str(path), "--ref-samples", "3")
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["samples_timed"] == 3 and line["s_per_sample"] > 0
    assert abs(line["samples_per_s"] * line["s_per_sample"] - 1) < 1e-9
    assert line["config"]["workload"] == "small_plan.txt"
    assert not [p for p in line["repo_libraries_loaded"] if p.startswith("exact-graphstate-sampling_b200")]


def test_reference_arm_other_ranks_do_nothing():
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0 and p.stdout.strip() == "", (p.stdout, p.stderr[-2000:])


def test_headline_plan_fixture_is_the_packages_plan():
    """The committed plan the reference arm reads equals the plan the package builds for the headline workload."""
    import workloads
    w = workloads.matching_n70_w30()
    assert open(os.path.join(GOLDEN, "headline", "matching_n70_w30_plan.txt")).read() == w["plan"]
