"""Batched persistent launch (gsb_batch_*): many instances of uneven width, strings sharing prefixes.

Every (prefix, suffix) string's log2 Pr equals the single-plan executor's 'chain' on the concatenated string
(complex128: <= 1e-9), the complex64 form stays within the stated tolerance of complex128, and the result does not
depend on the launch shape (block size, warp/CTA split, CTAs per SM) or on the autotuner's choice.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["search", "qubit"])
def small_batch(request):
    import workloads
    return workloads.batch_workload(count=14, seed=3, nmin=16, nmax=30, npre=3, nsuf=2, iters=2000,
                                    order=request.param)


def _strings(bw, i):
    p, s = bw["prefixes"][i], bw["suffixes"][i]
    return np.array([np.concatenate([p[a], s[a, b]]) for a in range(p.shape[0]) for b in range(s.shape[1])], np.int8)


def test_batch_c128_equals_executor(small_batch):
    import gsb
    bw = small_batch
    b = gsb.Batch([w["plan"] for w in bw["instances"]], precision=gsb.GSB_C128)
    b.set_strings(bw["K"], bw["prefixes"], bw["suffixes"])
    lp, ms = b.run()
    worst = 0.0
    for i, w in enumerate(bw["instances"]):
        with gsb.Engine.from_text(w["plan"], precision=gsb.GSB_C128) as eng:
            want = eng.chain(_strings(bw, i))[0]
        got = lp[i].reshape(-1)
        fin = np.isfinite(want)
        assert (np.isfinite(got) == fin).all()
        worst = max(worst, float(np.max(np.abs(got[fin] - want[fin]), initial=0.0)))
    assert worst <= 1e-9, worst
    assert ms > 0


def test_batch_shapes_and_c64(small_batch):
    import gsb
    bw = small_batch
    plans = [w["plan"] for w in bw["instances"]]
    ref = gsb.Batch(plans, precision=gsb.GSB_C128)
    ref.set_strings(bw["K"], bw["prefixes"], bw["suffixes"])
    want, _ = ref.run()
    b = gsb.Batch(plans, precision=gsb.GSB_C64)
    b.set_strings(bw["K"], bw["prefixes"], bw["suffixes"])
    outs = []
    for shape in [(256, 12, 2), (128, 0, 1), (512, 16, 1), (256, 8, 4)]:
        b.set_shape(*shape)
        outs.append(b.run()[0])
        assert b.shape() == shape
    for o in outs[1:]:
        assert np.max(np.abs(o - outs[0])) <= 1e-5     # complex64 sums in a shape-dependent order
    tuned = b.tune(reps=1)
    assert len(tuned) == 4 and tuned[3] > 0
    got, _ = b.run()
    d = np.abs(got - want)
    # complex64 (FP32 sums, FP64 norms and scales) against complex128; log2 amplifies the rounding of unlikely
    # strings, so the bound scales with -log2 Pr
    assert np.all(d <= 2e-5 * np.maximum(1.0, -want / 10)), float(d.max())


def test_batch_single_prefix_single_suffix_and_longest_prefix():
    """npre = nsuf = 1 and K = ns - 1 (a one-step suffix) against the single-plan executor (complex128)."""
    import gsb
    import workloads
    bw = workloads.batch_workload(count=5, seed=11, nmin=16, nmax=24, npre=1, nsuf=1, iters=2000)
    K = [len(w["steps"]) - 1 for w in bw["instances"]]
    rng = np.random.default_rng(2)
    pre = [rng.integers(0, 2, size=(1, k), dtype=np.int8) for k in K]
    suf = [rng.integers(0, 2, size=(1, 1, 1), dtype=np.int8) for _ in K]
    b = gsb.Batch([w["plan"] for w in bw["instances"]], precision=gsb.GSB_C128)
    b.set_strings(K, pre, suf)
    lp, _ = b.run()
    for i, w in enumerate(bw["instances"]):
        with gsb.Engine.from_text(w["plan"], precision=gsb.GSB_C128) as eng:
            want = eng.chain(np.concatenate([pre[i][0], suf[i][0, 0]])[None, :])[0][0]
        assert abs(lp[i, 0, 0] - want) <= 1e-9 or (not np.isfinite(want) and not np.isfinite(lp[i, 0, 0]))


def test_batch_rejects_shapes_it_cannot_launch():
    """A block larger than the batch kernel's register budget allows is refused up front (a usage error), and the
    autotuner only tries shapes that launch, in both precisions."""
    import gsb
    import workloads
    bw = workloads.batch_workload(count=4, seed=3, nmin=16, nmax=20, npre=2, nsuf=2, iters=2000)
    for prec in (gsb.GSB_C64, gsb.GSB_C128):
        b = gsb.Batch([w["plan"] for w in bw["instances"]], precision=prec)
        b.set_strings(bw["K"], bw["prefixes"], bw["suffixes"])
        with pytest.raises(gsb.GsbError) as e:
            b.set_shape(1024, 12, 1)
        assert e.value.code == 1
        block, small_R, per_sm, ms = b.tune(reps=1)
        assert block <= 512 and ms > 0
        b.run()


def test_l2_probe_measures_a_copy_bandwidth():
    """The L2 roofline's denominator: copying an L2-resident 24 MiB buffer runs well above HBM speed."""
    import gsb
    gbs = gsb.probe_l2_copy(mib=24, reps=100)
    assert 2000.0 < gbs < 1e6, gbs


def test_batch_vs_oracle(small_batch, tmp_path):
    """Both precisions of the batched launch against the oracle's chain (the reference executor's restatement) on
    every string of every instance: complex128 <= 1e-9; complex64 within 6 standard deviations of the complex64
    error model (gsb.c64_sigma) and <= 1e-5 where that model allows it."""
    import gsb
    from oracle import Oracle
    bw = small_batch
    plans = [w["plan"] for w in bw["instances"]]
    out = {}
    for prec in (gsb.GSB_C128, gsb.GSB_C64):
        b = gsb.Batch(plans, precision=prec)
        b.set_strings(bw["K"], bw["prefixes"], bw["suffixes"])
        out[prec] = b.run()[0]
        b.close()
    for i, w in enumerate(bw["instances"]):
        path = tmp_path / f"p{i}.txt"
        path.write_text(w["plan"])
        o = Oracle(str(path), 128)
        want = np.array([o.chain1(s)[0] for s in _strings(bw, i)])
        o.close()
        ns = len(w["steps"])
        fin = np.isfinite(want)
        got128 = out[gsb.GSB_C128][i].reshape(-1)
        got64 = out[gsb.GSB_C64][i].reshape(-1)
        assert (np.isfinite(got128) == fin).all()
        assert np.max(np.abs(got128[fin] - want[fin]), initial=0.0) <= 1e-9
        sig = gsb.c64_sigma(want[fin], ns)
        d64 = np.abs(got64[fin] - want[fin])
        assert (d64 <= 6 * sig).all(), (i, float(d64.max()))
        ok = 6 * sig <= 1e-5
        assert np.max(d64[ok], initial=0.0) <= 1e-5
