"""Parity of the wide-step kernels (steps of >= 2^10 / 2^11 cosets: the complex128 kernel and the complex64 paired
kernel) and of the fused passes with the oracle, in every executor mode, on instances wide enough to use them (one of
them with a wide single-output step, the fused passes' generic dataflow shape); and complex128 amplitudes against a
brute-force statevector at n = 24.

Modes: "c128" (complex128 arena), "c64x" (complex64 arena, exact pair sums + FP64 rotation: the oracle's own
complex64 arithmetic) and "c64" (complex64 arena, FP32 arithmetic, the default).  Tolerances: c128 |d log2 Pr| <=
1e-9; c64x <= 1e-5; c64 within 6 standard deviations of the complex64 error model (gsb.c64_sigma: complex64
rounding is absolute in units of the table norm, so the error grows as 1 / sqrt(Pr 2^n)), and the c64 form with its
complex128 guard attached <= 1e-5 on every string.  Sampled bits are identical to the oracle's (same mt19937_64
streams).
"""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = ["c128", "c64x", "c64"]


def engine(path, mode):
    import gsb
    e = gsb.Engine(path, precision=128 if mode == "c128" else 64)
    if mode == "c64x":
        e.set_arith(64)
    return e


def lp_tol(mode, lp, n):
    if mode == "c128":
        return 1e-9
    if mode == "c64x":
        return 1e-5
    import gsb
    return float(6 * gsb.c64_sigma(lp, n))


def cond_tol(mode):
    return {"c128": 1e-10, "c64x": 1e-6, "c64": 1e-5}[mode]


@pytest.fixture(scope="module")
def wide_case():
    import workloads
    w = workloads.matching_instance(38, 38, 7, 8, 20000)
    assert w["width"] >= 14
    td = tempfile.mkdtemp()
    path = os.path.join(td, "plan.txt")
    open(path, "w").write(w["plan"])
    w["path"] = path
    return w


@pytest.mark.parametrize("mode", MODES)
def test_wide_chain_prob_vs_oracle(wide_case, mode):
    import workloads
    from oracle import Oracle
    ns = n = len(wide_case["steps"])
    strings = workloads.random_strings(ns, 24, seed=31)
    o = Oracle(wide_case["path"], 128 if mode == "c128" else 64)
    with engine(wide_case["path"], mode) as eng:
        lp, cond = eng.chain(strings)
        lpp = eng.prob(strings[:6])
    for i in range(len(strings)):
        olp, ocond = o.chain1(strings[i])
        assert abs(lp[i] - olp) <= lp_tol(mode, olp, n), (i, lp[i], olp)
        if olp > -n - 3:
            assert np.abs(cond[i] - ocond).max() <= cond_tol(mode)
    for i in range(6):
        olp = o.prob(strings[i])
        assert abs(lpp[i] - olp) <= lp_tol(mode, olp, n)
    o.close()
    if mode == "c64":
        # the complex64 form with its complex128 guard: 1e-5 of the complex128 oracle on every string
        import gsb
        o = Oracle(wide_case["path"], 128)
        with engine(wide_case["path"], mode) as eng, gsb.Engine(wide_case["path"], precision=128) as e128:
            eng.set_guard(e128, gsb.c64_guard_log2_xmin(ns))
            lpg, _ = eng.chain(strings)
            lpgp = eng.prob(strings[:6])
        for i in range(len(strings)):
            assert abs(lpg[i] - o.chain1(strings[i])[0]) <= 1e-5, i
        for i in range(6):
            assert abs(lpgp[i] - o.prob(strings[i])) <= 1e-5, i
        o.close()


@pytest.mark.parametrize("mode", MODES)
def test_wide_samples_and_hybrid_vs_oracle(wide_case, mode):
    import gsb
    import workloads
    from oracle import Oracle
    ns = n = len(wide_case["steps"])
    o = Oracle(wide_case["path"], 128 if mode == "c128" else 64)
    with engine(wide_case["path"], mode) as eng:
        for seeding, seed in ((gsb.SEED_INT, 77), (gsb.SEED_SEQ, 78)):
            bits, lp = eng.sample(6, seed, seeding=seeding)
            for i in range(6):
                ob, olp = o.sample(seeding, seed, i)
                assert list(bits[i]) == list(ob) and abs(lp[i] - olp) <= lp_tol(mode, olp, n)
        lines = []
        base = workloads.random_strings(ns, 4, seed=5)
        for i in range(4):
            s = "".join(str(int(b)) for b in base[i])
            lines.append(s[:ns - 6] + "?" * 6)
        hb, hlp, hc = eng.hybrid(lines, 11)
        for i, ln in enumerate(lines):
            ob, olp, oc = o.hybrid(ln, 11, i)
            assert list(hb[i]) == list(ob) and abs(hlp[i] - olp) <= lp_tol(mode, olp, n)
            if olp > -n - 3:
                assert np.abs(hc[i] - oc).max() <= cond_tol(mode)
        # the same lines with their forced prefix declared: fused passes for steps < ns - 6, the same results
        eng.set_hybrid_prefix(ns - 6)
        assert any(p[3] == 1 for p in eng.passes(0))   # the plan has fused chain passes
        fb, flp, fc = eng.hybrid(lines, 11)
        for i, ln in enumerate(lines):
            ob, olp, oc = o.hybrid(ln, 11, i)
            assert list(fb[i]) == list(ob) and abs(flp[i] - olp) <= lp_tol(mode, olp, n)
            if olp > -n - 3:
                assert np.abs(fc[i] - oc).max() <= cond_tol(mode)
        with pytest.raises(gsb.GsbError) as e:
            eng.hybrid([lines[0][:ns - 7] + "?" * 7], 11)
        assert e.value.code == 8
        eng.set_hybrid_prefix(0)
    o.close()


@pytest.mark.parametrize("mode", MODES)
def test_wide_prefix_resume_two_slices(wide_case, mode):
    """prefix dump at a wide step, then resume over two half tables (the slice sum of gsamp2.cpp:196-205)."""
    import workloads
    from oracle import Oracle
    prec = 128 if mode == "c128" else 64
    ns = n = len(wide_case["steps"])
    K = max(range(ns), key=lambda k: wide_case["steps"][k]["r"])
    s = "".join(str(int(b)) for b in workloads.random_strings(ns, 1, seed=6)[0])
    line = s[:K] + "?" * (ns - K)
    o = Oracle(wide_case["path"], prec)
    with engine(wide_case["path"], mode) as eng:
        d, ls, lp = eng.prefix(line, K)
        od, ols, olp = o.prefix(line, K)
        assert abs(lp - olp) <= lp_tol(mode, olp, K) and abs(ls - ols) <= 1e-6
        scale = max(1e-300, np.abs(od).max())
        assert np.abs(d.astype(np.complex128) - od).max() <= (1e-12 if prec == 128 else 1e-5) * scale
        half = (d / 2).astype(d.dtype)
        bits, lpf, lpp, cond = eng.resume(line, K, 21, 0, [half, half], [ls, ls])
        ob, olpf, olpp, oc = o.resume(line, K, 21, 0, [half.astype(np.complex128)] * 2, [ls, ls])
    assert list(bits) == list(ob)
    assert abs(lpf - olpf) <= lp_tol(mode, olpf, n) and abs(lpp - olpp) <= 1e-9
    assert np.abs(cond[K:] - oc[K:]).max() <= cond_tol(mode)
    o.close()


def test_statevector_n24():
    """complex128 amplitudes of 64 strings of an n = 24 random-matching circuit against a brute-force 2^24
    statevector (simulated with torch on the GPU): |d Pr| <= 1e-12 absolute, |d log2 Pr| <= 1e-9."""
    import gsb
    import workloads
    from oracle import statevector
    w = workloads.matching_instance(24, 24, 5, 6, 20000)
    psi = statevector.dense_state_torch(24, list(w["body"]) + list(w["tail"]), device="cuda")
    p = (psi.abs() ** 2).cpu().numpy()
    rng = np.random.default_rng(3)
    idx = list(rng.integers(0, 1 << 24, 56)) + list(np.argsort(p)[-8:])
    strings = []
    for ix in idx:
        bits = [(int(ix) >> (23 - q)) & 1 for q in range(24)]
        strings.append([bits[s["v"]] for s in w["steps"]])
    with gsb.Engine.from_text(w["plan"], precision=128) as eng:
        lp = eng.chain(np.array(strings, np.int8))[0]
    ref = p[idx]
    assert np.abs(np.exp2(lp) - ref).max() <= 1e-12
    big = ref > 1e-10                   # log2 amplifies the absolute rounding of very unlikely strings
    assert big.sum() >= 48 and np.abs(lp[big] - np.log2(ref[big])).max() <= 1e-9


@pytest.mark.parametrize("mode", MODES)
def test_fused_chain_depths_vs_oracle(wide_case, mode):
    """'chain' mode with 1, 2 and 3 DP steps fused per pass gives the oracle's log2 Pr and conditionals; 'prob' and
    'sample' (fused passes that carry the next step's branch norms) give the oracle's probabilities and
    bit-identical samples; so do the pass lists the autotuner picks."""
    import workloads
    from oracle import Oracle
    ns = n = len(wide_case["steps"])
    strings = workloads.random_strings(ns, 12, seed=41)
    o = Oracle(wide_case["path"], 128 if mode == "c128" else 64)
    ref = [o.chain1(s) for s in strings]
    samples_ref = [o.sample(0, 123, i) for i in range(4)]
    o.close()
    with engine(wide_case["path"], mode) as eng:
        for depth in (1, 2, 3):
            eng.set_fusion(depth)
            glen, _ = eng.fusion_groups()
            assert sum(glen) == ns and (depth == 1 or max(glen) >= 2)
            lp, cond = eng.chain(strings)
            for i, (olp, ocond) in enumerate(ref):
                assert abs(lp[i] - olp) <= lp_tol(mode, olp, n), (depth, i, lp[i], olp)
                if olp > -n - 3:
                    assert np.abs(cond[i] - ocond).max() <= cond_tol(mode), depth
            # 'prob' and 'sample' run fused passes with trailing branch norms when fusion is on
            lpp = eng.prob(strings[:4])
            for i in range(4):
                assert abs(lpp[i] - ref[i][0]) <= lp_tol(mode, ref[i][0], n), (depth, i)
            bits, slp = eng.sample(4, 123)
            for i in range(4):
                ob, olp = samples_ref[i]
                assert list(bits[i]) == list(ob) and abs(slp[i] - olp) <= lp_tol(mode, olp, n), (depth, i)
        # the autotuner's pass lists (measured on this device) must give the same results
        before, after = eng.autotune(mode=2, reps=1)
        assert before > 0 and after > 0
        glen, _ = eng.fusion_groups()
        assert sum(glen) == ns
        lp, cond = eng.chain(strings)
        for i, (olp, ocond) in enumerate(ref):
            assert abs(lp[i] - olp) <= lp_tol(mode, olp, n), ("tuned", i, lp[i], olp)
            if olp > -n - 3:
                assert np.abs(cond[i] - ocond).max() <= cond_tol(mode)
        lpp = eng.prob(strings[:4])
        for i in range(4):
            assert abs(lpp[i] - ref[i][0]) <= lp_tol(mode, ref[i][0], n), ("tuned", i)
        bits, slp = eng.sample(4, 123)
        for i in range(4):
            ob, olp = samples_ref[i]
            assert list(bits[i]) == list(ob) and abs(slp[i] - olp) <= lp_tol(mode, olp, n), ("tuned", i)
        # new matrices keep the tuned pass lists (rebuilt with the new M): the same plan's M gives the same results
        tuned = eng.fusion_groups()[0]
        eng.set_matrices_from_text(open(wide_case["path"]).read())
        assert eng.fusion_groups()[0] == tuned
        assert np.array_equal(eng.chain(strings)[0], lp)


@pytest.fixture(scope="module")
def twin_case():
    import workloads
    w = workloads.twin_graph_instance()
    w["m1"] = [k for k, s in enumerate(w["steps"]) if s["m"] == 1 and s["r"] >= 12]
    assert w["m1"], "the twin instance must keep a wide one-output step"
    td = tempfile.mkdtemp()
    path = os.path.join(td, "plan.txt")
    open(path, "w").write(w["plan"])
    w["path"] = path
    return w


@pytest.mark.parametrize("mode", MODES)
def test_fused_one_output_step_vs_oracle(twin_case, mode):
    """A wide step with a single output class (m = 1: a twin vertex measured after its original) runs the fused
    passes' generic dataflow shape (GK_ANY): in 'chain' passes at depths 2 and 3, and in the sampling passes both as a
    written step and as the trailing branch-norm step (the packed FP32 form in mode "c64").  The pass lists must
    cover it that way, and chain, prob and sample must give the oracle's results."""
    import workloads
    from oracle import Oracle
    ns = n = len(twin_case["steps"])
    m1 = twin_case["m1"]
    strings = workloads.random_strings(ns, 8, seed=3)
    o = Oracle(twin_case["path"], 128 if mode == "c128" else 64)
    ref = [o.chain1(s) for s in strings]
    sref = [o.sample(0, 9, i) for i in range(4)]
    o.close()
    in_chain = in_written = in_trailing = False
    with engine(twin_case["path"], mode) as eng:
        for depth in (2, 3):
            eng.set_fusion(depth)
            for k0, d, tr, fused in eng.passes(0):
                in_chain |= bool(fused) and d >= 2 and any(k0 <= k < k0 + d for k in m1)
            for k0, d, tr, fused in eng.passes(1):
                in_written |= bool(fused) and any(k0 <= k < k0 + d for k in m1)
                in_trailing |= bool(fused and tr) and (k0 + d) in m1
            lp, cond = eng.chain(strings)
            lpp = eng.prob(strings)
            bits, slp = eng.sample(4, 9)
            for i, (olp, ocond) in enumerate(ref):
                assert abs(lp[i] - olp) <= lp_tol(mode, olp, n), (depth, i, lp[i], olp)
                assert abs(lpp[i] - olp) <= lp_tol(mode, olp, n), (depth, i, lpp[i], olp)
                if olp > -n - 3:
                    assert np.abs(cond[i] - ocond).max() <= cond_tol(mode), depth
            for i in range(4):
                ob, olp = sref[i]
                assert list(bits[i]) == list(ob) and abs(slp[i] - olp) <= lp_tol(mode, olp, n), (depth, i)
    assert in_chain and in_written and in_trailing, (in_chain, in_written, in_trailing)


def test_pass_lists_cover_every_step_once(wide_case):
    """gsb_pass_list: both modes' passes cover the steps in order, each once, agree with the group lengths that
    gsb_fusion_groups / gsb_sample_groups report, and only fused passes carry a trailing branch-norm step."""
    ns = len(wide_case["steps"])
    with engine(wide_case["path"], "c64") as eng:
        for depth in (1, 2, 3):
            eng.set_fusion(depth)
            for mode, groups in ((0, eng.fusion_groups), (1, eng.sample_groups)):
                passes = eng.passes(mode)
                glen, _ = groups()
                k = 0
                for k0, d, tr, fused in passes:
                    assert k0 == k and d >= 1 and (fused or (d == 1 and tr == 0)), (mode, depth, k0, d, tr, fused)
                    assert glen[k0] == d and (tr == 0 or k0 + d < ns), (mode, depth, k0)
                    k += d
                assert k == ns, (mode, depth)
                assert mode == 1 or all(tr == 0 for _, _, tr, _ in passes)
