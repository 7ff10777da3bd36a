"""The complex64 form on the headline workload (n = 70, depth 70, width 30: a 2^30-entry arena) against the
complex128 form, at the tolerance the form is held to: |d log2 Pr| <= 1e-5, unconditionally.

* 256 exact samples drawn with the same uniforms in both forms: identical bits, |d log2 Pr| <= 1e-5.
* 1,024 uniform random strings: the guarded complex64 form (complex128 re-evaluation below the error model's
  threshold) within 1e-5 of complex128 on every string; the unguarded complex64 results within the stated error
  (6 standard deviations of the error model) on every string; the strings re-evaluated are exactly those below
  the threshold.
* 2 of those strings against the reference's own complex128 executor (gsamp2 -DGS_DOUBLE, compiled from its
  sources into oracle/_ref) on the host: <= 1e-9 for complex128, <= 1e-5 for the guarded complex64 form.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
TOL = 1e-5
PLAN = os.path.join(GOLDEN, "headline", "matching_n70_w30_plan.txt")


@pytest.fixture(scope="module")
def engines():
    import gsb
    text = open(PLAN).read()
    e64 = gsb.Engine.from_text(text, precision=64)
    e128 = gsb.Engine.from_text(text, precision=128)
    yield e64, e128
    e64.close()
    e128.close()


def test_headline_samples_c64_vs_c128(engines):
    e64, e128 = engines
    ns = e64.ns
    u = np.random.default_rng(404).random((256, ns))
    e64.set_guard(None, 0.0)
    b64, lp64 = e64.sample_uniform(u)
    b128, lp128 = e128.sample_uniform(u)
    assert (b64 == b128).all()
    assert np.isfinite(lp128).all()
    assert np.abs(lp64 - lp128).max() <= TOL, np.abs(lp64 - lp128).max()


def test_headline_amplitudes_guarded_c64_vs_c128(engines):
    import gsb
    import workloads
    e64, e128 = engines
    ns = e64.ns
    strings = workloads.random_strings(ns, 1024, seed=4040)
    lp128, c128 = e128.chain(strings)
    e64.set_guard(None, 0.0)
    raw, _ = e64.chain(strings)
    # unguarded: within the stated error of each result
    sigma = gsb.c64_sigma(raw, ns)
    assert (np.abs(raw - lp128) <= 6 * sigma).all()
    lx = gsb.c64_guard_log2_xmin(ns, TOL)
    e64.set_guard(e128, lx)
    lp, cond = e64.chain(strings)
    flagged = ~(raw + ns >= lx)
    assert e64.guard_evaluations() == int(flagged.sum()) > 0
    assert (lp[flagged] == lp128[flagged]).all() and (cond[flagged] == c128[flagged]).all()
    assert (lp[~flagged] == raw[~flagged]).all()
    assert np.abs(lp - lp128).max() <= TOL, np.abs(lp - lp128).max()
    # the reference's complex128 executor on two of the strings (one re-evaluated, one not, when both exist)
    from oracle import ref_binary, run_ref
    if ref_binary(128) is None:
        pytest.skip("reference executor not built")
    pick = [int(np.flatnonzero(flagged)[0]), int(np.flatnonzero(~flagged)[0])]
    with tempfile.TemporaryDirectory() as td:
        sp = os.path.join(td, "s.txt")
        open(sp, "w").write("".join("".join(str(int(b)) for b in strings[i]) + "\n" for i in pick))
        out = run_ref(128, [PLAN, "chain", sp], threads=os.cpu_count())
    ref = np.array([float(ln.split()[0]) for ln in out.split("\n") if ln.strip()])
    assert np.abs(lp128[pick] - ref).max() <= 1e-9
    assert np.abs(lp[pick] - ref).max() <= TOL


def test_guard_rejects_mismatched_engines(engines):
    import gsb
    e64, e128 = engines
    with pytest.raises(gsb.GsbError):
        e128.set_guard(e64, 0.0)              # the guarded engine must be complex64
    with pytest.raises(gsb.GsbError):
        e64.set_guard(e64, 0.0)               # the guard must be complex128
    other = gsb.Engine.from_text(open(PLAN).read().replace(" 0.", " 0.5", 1), precision=128)
    with pytest.raises(gsb.GsbError):
        e64.set_guard(other, 0.0)             # another plan (different matrices)
    other.close()
