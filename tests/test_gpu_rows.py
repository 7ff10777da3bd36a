"""GPU parity of the rows around the executor: the out-of-place amplitude engine (dp.cpp, engine.run_dp), the
sampler_ref call signatures, and sliced prefix / resume with a twist file; all against the reference's own outputs
(tests/golden/extras_cases.json)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def extras():
    return json.load(open(os.path.join(GOLDEN, "extras_cases.json")))


def _am(planner_cases, name):
    from amp import Amplitudes
    from circuits import tableau_of
    c = {c["name"]: c for c in planner_cases["cases"]}[name]
    return Amplitudes(c["n"], tableau_of(c["n"], c["body"]), [tuple(t) for t in c["tail"]], c["order"]), c


def test_run_dp_matches_reference_dp(extras, tmp_path):
    """engine.run_dp on the GPU equals the reference's dp.cpp and ref.run (complex amplitudes, slicing included),
    complex128 to 1e-12 relative, complex64 storage to 1e-6."""
    import engine
    for d in extras["dp"]:
        (tmp_path / "p.txt").write_text(d["plan"])
        (tmp_path / "j.txt").write_text(d["jobs"])
        ref = [complex(*map(float, ln.split())) for ln in d["ref_dp"]]
        for prec, tol in ((128, 1e-12), (64, 1e-6)):
            got = engine.run_dp(str(tmp_path), "p.txt", "j.txt", precision=prec)
            for a, b, r in zip(got, ref, d["ref_run"]):
                scale = max(1.0, abs(b))
                assert abs(a - b) <= tol * scale and abs(a - complex(*r)) <= tol * scale


def test_sampler_ref_signatures(extras, planner_cases):
    """sampler.extend / conditionals / sample / chain_distribution against sampler_ref's outputs."""
    import sampler
    for d in extras["sampler"]:
        am, c = _am(planner_cases, d["name"])
        st = am.steps[d["extend_step"]]
        old = np.array([complex(*z) for z in d["extend_in"]])
        out = sampler.extend(old, st, (am.M[st["v"]][0, 0], am.M[st["v"]][0, 1]))
        assert np.abs(out - np.array([complex(*z) for z in d["extend_out"]])).max() <= 1e-12
        for p, (cond, nrm) in zip(d["prefixes"], d["conditionals"]):
            gc, gn = sampler.conditionals(am, p)
            assert np.abs(gc - np.array(cond)).max() <= 1e-10 and np.abs(gn - np.array(nrm)).max() <= 1e-12
        for seed, b in zip((1, 2, 3, 4), d["samples"]):
            assert sampler.sample(am, np.random.default_rng(seed)) == b
        if d["chain_distribution"] is not None:
            dist = sampler.chain_distribution(am)
            ref = {k: v for k, v in d["chain_distribution"]}
            for k, v in ref.items():
                assert abs(dist.get(tuple(int(ch) for ch in k), 0.0) - v) <= 1e-12
            assert sum(dist.values()) == pytest.approx(1.0, abs=1e-10)


def test_sliced_prefix_resume_with_twist(extras, planner_cases, tmp_path):
    """Slice plans of make_sliced_plans: prefix on every slice, resume with the twist file = the unsliced
    probability of the full string (the identity the reference's test_twist.py checks)."""
    import gsb
    from inplace import inplace_plan_text, plan_inplace, plan_width
    from sliced_plans import make_sliced_plans
    for d in extras["sliced"]:
        am, c = _am(planner_cases, d["name"])
        n = c["n"]
        out = str(tmp_path / "sp")
        info = make_sliced_plans(am.A, [m.copy() for m in am.M], c["order"], d["S"], out, K=d["K"], ND=n)
        K = info["K"]
        twist = [tuple(int(x) for x in ln.split()) for ln in open(f"{out}_twist.txt") if ln.strip()]
        R = max(1, plan_width(am.steps))
        full = gsb.Engine.from_text(inplace_plan_text(plan_inplace(am.A, c["order"], R), R, am.M, n), precision=128)
        rng = np.random.default_rng(5)
        for prec in (128, 64):
            engs = [gsb.Engine(f"{out}_s{tag}.txt", precision=prec) for tag in sorted(d["plans"])]
            for _ in range(6):
                line = [int(x) for x in rng.integers(0, 2, n)]
                dumps, lss = [], []
                for e in engs:
                    dd, ls, _ = e.prefix(line, K)
                    dumps.append(dd)
                    lss.append(ls)
                bits, lpf, lpp, cond = engs[0].resume(line, K, 3, 0, dumps, lss, twist=twist)
                ref = full.chain([line])[0][0]
                assert abs(lpf - ref) <= (1e-9 if prec == 128 else 1e-5) or abs(2 ** lpf - 2 ** ref) <= 1e-12
            for e in engs:
                e.close()
        full.close()


def _fields(line):
    t = line.split()
    if not t or t[0] == "#":
        return None
    return t


def test_hybrid_driver_matches_reference_driver(extras, tmp_path):
    """hybrid_sampler (in process) against the reference's doped_sampler.py run with its own gsamp2 as --bin: the same
    accept/reject decisions, bits, log2 Pr and z, unsliced and sliced with a twist; score mode too."""
    import hybrid_sampler
    for d in extras["driver"]:
        n = len(d["strings"][0])
        (tmp_path / "str.txt").write_text("\n".join(d["strings"]) + "\n")
        for name, run in d["runs"].items():
            args = list(run["args"])
            # the plan / slice files of the fixture live in the planner fixtures: rebuild them here
            _write_inputs(extras, d, tmp_path)
            outf = args[args.index("sv.json") + (4 if args[0] == "sample" else 2)]
            out = tmp_path / outf
            if out.exists():
                out.unlink()
            cwd = os.getcwd()
            os.chdir(tmp_path)
            try:
                hybrid_sampler.main(["hybrid_sampler.py"] + args + ["--na", "0", "--nd", str(n), "--precision", "64"])
            finally:
                os.chdir(cwd)
            got = [f for f in map(_fields, out.read_text().split("\n")) if f]
            ref = [f for f in map(_fields, run["lines"]) if f]
            assert len(got) == len(ref), name
            for g, r in zip(got, ref):
                if args[0] == "sample":
                    assert g[0] == r[0] and g[1] == r[1], (name, g, r)
                    assert abs(float(g[2]) - float(r[2])) <= 1e-5
                    assert abs(float(g[3][2:]) - float(r[3][2:])) <= 1e-5 * max(1.0, float(r[3][2:]))
                else:
                    assert g[0] == r[0] and abs(float(g[1]) - float(r[1])) <= 1e-5


def _write_inputs(extras, d, tmp_path):
    import json as _json
    from conftest import GOLDEN
    from amp import Amplitudes
    from circuits import tableau_of
    from inplace import plan_inplace, write_inplace_plan, plan_width
    cases = {c["name"]: c for c in _json.load(open(os.path.join(GOLDEN, "planner_cases.json")))["cases"]}
    c = cases[d["name"]]
    n = c["n"]
    am = Amplitudes(n, tableau_of(n, c["body"]), [tuple(t) for t in c["tail"]], c["order"])
    R = max(1, plan_width(am.steps))
    write_inplace_plan(str(tmp_path / "full.txt"), plan_inplace(am.A, c["order"], R), R, am.M, n)
    (tmp_path / "sv.json").write_text(_json.dumps(c["order"]))
    sl = [s for s in extras["sliced"] if s["name"] == d["name"]][0]
    for tag, text in sl["plans"].items():
        (tmp_path / f"sl_s{tag}.txt").write_text(text)
    (tmp_path / "sl_twist.txt").write_text(sl["twist"])


def test_slices_summed_after_the_last_step(planner_cases, tmp_path):
    """Slicing with every slice vertex's neighbours in the sweep (K = ns, no twist): 'prefix' through the last step
    on every slice plan and 'resume' with no steps left give the unsliced log2 Pr (the width-34 cross-check's use)."""
    import gsb
    from inplace import inplace_plan_text, plan_inplace, plan_width
    from sliced_plans import make_sliced_plans
    case = [c for c in planner_cases["cases"] if c["n"] >= 10][0]
    am, c = _am(planner_cases, case["name"])
    n = c["n"]
    S = [c["order"][1], c["order"][n // 2]]
    out = str(tmp_path / "sp")
    info = make_sliced_plans(am.A, [m.copy() for m in am.M], c["order"], S, out, ND=n)
    assert info["K"] == n and not info["twist"]
    R = max(1, plan_width(am.steps))
    rng = np.random.default_rng(9)
    with gsb.Engine.from_text(inplace_plan_text(plan_inplace(am.A, c["order"], R), R, am.M, n), precision=128) as full, \
            gsb.Engine(f"{out}_s00.txt", precision=128) as e:
        texts = [open(f"{out}_s{a}{b}.txt").read() for a in (0, 1) for b in (0, 1)]
        for _ in range(5):
            line = [int(x) for x in rng.integers(0, 2, n)]
            dumps, lss = [], []
            for t in texts:
                e.set_matrices_from_text(t)
                d, ls, _ = e.prefix(line, n)
                dumps.append(d)
                lss.append(ls)
            _, lpf, _, _ = e.resume(line, n, 0, 0, dumps, lss)
            ref = full.chain([line])[0][0]
            assert abs(lpf - ref) <= 1e-9 or abs(2 ** lpf - 2 ** ref) <= 1e-12
