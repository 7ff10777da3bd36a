"""Test set-up: import paths, the `gpu` marker, in-tree builds and shared fixtures.

`-m "not gpu"` runs everything that needs no CUDA device: the planner against the reference's own outputs, the
oracle against the reference executor and its published vectors, host logic, the C ABI's exports.  `-m gpu` runs
the parity tests of the CUDA executor against the oracle and the golden vectors.
"""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "exact-graphstate-sampling_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

import build as _pkg_build  # noqa: E402  (the package's build script)
import oracle as _oracle  # noqa: E402

_pkg_build.build()
_oracle.build()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def planner_cases():
    return json.load(open(os.path.join(GOLDEN, "planner_cases.json")))


@pytest.fixture(scope="session")
def executor_cases():
    return json.load(open(os.path.join(GOLDEN, "executor_cases.json")))


@pytest.fixture(scope="session")
def w30_dir():
    return os.path.join(GOLDEN, "w30")


def case_plan_text(case):
    """In-place plan text of a planner case, built by this repository's planner."""
    from amp import Amplitudes
    from circuits import tableau_of
    from inplace import inplace_plan_text, plan_inplace
    n = case["n"]
    T = tableau_of(n, case["body"])
    am = Amplitudes(n, T, [tuple(x) for x in case["tail"]], case["order"])
    R = max(1, max(max(s["r"], s["rn"]) for s in am.steps))
    st = plan_inplace(am.A, case["order"], R)
    return inplace_plan_text(st, R, am.M, n), am, st, R


def parse_ref_lines(lines):
    return [ln.split() for ln in lines]
