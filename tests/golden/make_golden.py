"""Generate the golden fixtures of this directory from the reference implementation.

    python tests/golden/make_golden.py            (needs the reference checkout at $GSB_REFERENCE_DIR, by default
                                                    the sibling directory "reference" of this checkout, and
                                                    `make -C oracle ref`)
    python tests/golden/make_golden.py --w30      (slow: the reference executor on the width-30 gate strings)

Three phases, each in its own process so the reference's flat module names (tableau, plan, amp, ...) never mix
with this repository's modules of the same names:

  inputs    (this repository on sys.path)  seeded circuits and orders: random small circuits with the reference's
            test gate set and either the #151 tail (tdg; h; rz(theta); h) or a U3 layer; the n=20 G(n,1/2)
            instance and the n=70 random-matching instance of the benchmark configurations, with orders from the
            native order search.
  expected  (reference on sys.path)  the reference's graph form A, out-of-place plan steps and in-place plan text
            for every case (U3 tails fold into M_j = W_j U_j^dag exactly as amp.py:26 does); the reference's
            width-30 plan regenerated from its #151 circuit and order (w30/nq70_inplace_plan_regen.txt).
  executor  (compiled reference executor, oracle/_ref)  gsamp2 outputs on small plans: prob / chain on every
            string (complex128 and complex64 builds), sample / sample2 / hybrid lines, a prefix + resume run.
  extras    (reference on sys.path + oracle/_ref/dp)  engine.py plan/jobs with vertex slicing and dp.cpp's
            amplitudes, ref.run amplitudes, sampler_ref conditionals / samples / extend / chain_distribution, and
            make_sliced_plans slice plans with their twist files.

Reference data files copied verbatim (the pinned width-30 instance and its published outputs):
  w30/nq70.qasm, w30/order_w30.json, w30/nq70_inplace_plan.txt (as shipped), w30/gate_strings.txt,
  w30/ibm_strings_64.txt + w30/ibm_log2p_64.txt + w30/ibm_chain_64.txt (first 64 of 1,726 IBM shots),
  w30/laptop_samples_w30.txt, w30/samples2_16.txt (first 16 'sample2' samples), w30/rngbits_2000000.txt.
"""
import itertools
import json
import os
import random
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "exact-graphstate-sampling_b200")
REF = os.environ.get("GSB_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
GATES = ["h", "s", "sdg", "sx", "sxdg", "x", "z", "cz", "cz", "cz"]
TH = 0.9553166181245092


def tail_151(n):
    t = []
    for q in range(n):
        t += [["tdg", [q]], ["h", [q]], [f"rz({TH})", [q]], ["h", [q]]]
    return t


def phase_inputs(out):
    sys.path.insert(0, PKG)
    import circuits
    import gsb
    from graphform import graph_form
    cases = []
    rng = random.Random(20261203)
    for i in range(40):
        n = rng.randint(2, 10)
        body = []
        for _ in range(rng.randint(5, 90)):
            g = rng.choice(GATES)
            body.append([g, rng.sample(range(n), 2)] if g == "cz" else [g, [rng.randrange(n)]])
        if i % 4 == 3:
            tail = [[circuits.u3_op(q, rng.uniform(0, 6.283), rng.uniform(0, 6.283), rng.uniform(0, 6.283))[0], [q]]
                    for q in range(n)]
        else:
            tail = tail_151(n)
        order = list(range(n))
        rng.shuffle(order)
        cases.append(dict(name=f"small{i}", n=n, body=body, tail=tail, order=order))
    for name, (n, body, tail), seed in (("config1_n20", circuits.graph_state_circuit(20, 0.5, seed=1), 11),
                                         ("config2_n70", circuits.matching_circuit(70, 70, seed=2), 12)):
        A, _ = graph_form(circuits.tableau_of(n, body))
        order, w = gsb.order_search(A, seed=seed, ngreedy=4, iters=20000 if n < 40 else 60000)
        cases.append(dict(name=name, n=n, body=[list(x) for x in body], tail=[list(x) for x in tail], order=order,
                          search_width=w))
    json.dump(cases, open(out, "w"))


def phase_expected(inp, out):
    sys.path.insert(0, REF)
    import math
    import numpy as np
    from tableau import Tableau, clifford_body
    from graphform import graph_form
    from amp import tail_matrix, Amplitudes
    from plan import plan
    from inplace import plan_inplace, write_inplace_plan

    def W_of(ops):
        M = np.eye(2, dtype=complex)
        for name, _ in ops:
            if name.startswith("u3("):
                th, ph, la = (float(x) for x in name[3:-1].split(","))
                c, s = math.cos(th / 2), math.sin(th / 2)
                G = np.array([[c, -np.exp(1j * la) * s], [np.exp(1j * ph) * s, np.exp(1j * (ph + la)) * c]])
            else:
                G = tail_matrix([(name, None)])
            M = G @ M
        return M

    res = []
    with tempfile.TemporaryDirectory() as td:
        for c in json.load(open(inp)):
            n = c["n"]
            T = Tableau(n)
            for g, qs in c["body"]:
                T.apply(g, qs)
            A, U = graph_form(T)
            per = [[] for _ in range(n)]
            for g, qs in c["tail"]:
                per[qs[0]].append((g, qs))
            M = [W_of(per[q]) @ U[q].conj().T for q in range(n)]
            steps = plan(A, c["order"])
            R = max(1, max(max(s["r"], s["rn"]) for s in steps))
            st = plan_inplace(A, c["order"], R)
            pth = os.path.join(td, "p.txt")
            write_inplace_plan(pth, st, R, M, n)
            c["A"] = ["".join(str(int(x)) for x in row) for row in A]
            c["plan"] = [dict(v=s["v"], r=s["r"], rn=s["rn"], rho=s["rho"], piv=s["piv"], ker=s["ker"]) for s in steps]
            c["R"] = R
            c["inplace_plan"] = open(pth).read()
            c["U"] = [[[float(z.real).hex(), float(z.imag).hex()] for z in u.reshape(-1)] for u in U]
            res.append(c)
        # the pinned width-30 instance: regenerate the shipped plan from its circuit and order
        n, T, tail = clifford_body(os.path.join(REF, "cloud_nq76", "nq70.qasm"))
        order = json.load(open(os.path.join(REF, "orders", "order_w30.json")))
        am = Amplitudes(n, T, tail, order)
        st = plan_inplace(am.A, order, 30)
        pth = os.path.join(td, "w30.txt")
        write_inplace_plan(pth, st, 30, am.M, n)
        # The shipped plan predates the reference's current planner (kept coordinates are now ordered by physical
        # address, inplace.py:50): the current code writes an equivalent plan with a different layout, and its M
        # entries also differ from the shipped ones in the last ulps (another platform's numpy).  Planner parity is
        # therefore pinned to the plan the current reference code writes here; the shipped plan stays the input of
        # the executor golden vectors it was used to produce.
        w30_text_here = open(pth).read()
        same = w30_text_here == open(os.path.join(REF, "cloud_ibmxeb", "nq70_inplace_plan.txt")).read()
    open(os.path.join(HERE, "w30", "nq70_inplace_plan_regen.txt"), "w").write(w30_text_here)
    json.dump(dict(cases=res, w30_shipped_plan_equal_regenerated=same), open(out, "w"))


def _ref(prec, args, cwd):
    exe = os.path.join(ROOT, "oracle", "_ref", "gsamp2_c128" if prec == 128 else "gsamp2")
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, cwd=cwd,
                       env={**os.environ, "OMP_NUM_THREADS": os.environ.get("OMP_NUM_THREADS", "4")})
    assert r.returncode == 0, r.stderr
    return r.stdout.strip().split("\n") if r.stdout.strip() else []


def phase_executor(exp, out):
    import itertools
    data = json.load(open(exp))
    outs = []
    with tempfile.TemporaryDirectory() as td:
        chosen = [c for c in data["cases"] if c["name"].startswith("small") and c["n"] <= 7][:10]
        for c in chosen:
            n = c["n"]
            open(os.path.join(td, "p.txt"), "w").write(c["inplace_plan"])
            ns = n
            strings = ["".join(s) for s in itertools.product("01", repeat=ns)]
            open(os.path.join(td, "s.txt"), "w").write("\n".join(strings) + "\n")
            rr = random.Random(sum(map(ord, c["name"])))
            hyb = []
            for _ in range(8):
                s = [rr.choice("01") for _ in range(ns)]
                for k in range(max(0, ns - 2), ns):
                    s[k] = "?"
                hyb.append("".join(s))
            open(os.path.join(td, "h.txt"), "w").write("\n".join(hyb) + "\n")
            K = ns // 2
            pre = ["".join(rr.choice("01") for _ in range(K)) + "?" * (ns - K) for _ in range(3)]
            open(os.path.join(td, "pre.txt"), "w").write("\n".join(pre) + "\n")
            rec = dict(name=c["name"], strings=strings, hybrid_lines=hyb, prefix_lines=pre, K=K)
            for prec in (128, 64):
                rec[f"prob{prec}"] = _ref(prec, ["p.txt", "prob", "s.txt"], td)
                rec[f"chain{prec}"] = _ref(prec, ["p.txt", "chain", "s.txt"], td)
                rec[f"sample{prec}"] = _ref(prec, ["p.txt", "sample", 40, 1000], td)
                rec[f"sample2_{prec}"] = _ref(prec, ["p.txt", "sample2", 12, 5], td)
                rec[f"hybrid{prec}"] = _ref(prec, ["p.txt", "hybrid", "h.txt", 9], td)
                rec[f"prefix{prec}"] = _ref(prec, ["p.txt", "prefix", "pre.txt", K, "d"], td)
                rec[f"resume{prec}"] = _ref(prec, ["p.txt", "resume", "pre.txt", K, 3, "d"], td)
            outs.append(rec)
    json.dump(outs, open(out, "w"))


def copy_w30():
    d = os.path.join(HERE, "w30")
    os.makedirs(d, exist_ok=True)
    shutil.copy(os.path.join(REF, "cloud_nq76", "nq70.qasm"), d)
    shutil.copy(os.path.join(REF, "orders", "order_w30.json"), d)
    shutil.copy(os.path.join(REF, "cloud_ibmxeb", "nq70_inplace_plan.txt"), d)
    shutil.copy(os.path.join(REF, "cloud_ibmxeb", "gate_strings.txt"), d)
    shutil.copy(os.path.join(REF, "results", "laptop_samples_w30.txt"), d)
    shutil.copy(os.path.join(REF, "results", "rngbits_seeds_2000000.txt"), os.path.join(d, "rngbits_2000000.txt"))

    def head(src, dst, k):
        with open(os.path.join(REF, src)) as f:
            lines = [next(f) for _ in range(k)]
        open(os.path.join(d, dst), "w").write("".join(lines))
    head("cloud_ibmxeb/ibm_qiskit.txt", "ibm_strings_64.txt", 64)
    head("results/ibmxeb/ibm_out.txt", "ibm_log2p_64.txt", 64)
    head("results/chain/ibm_fwd_chain.txt", "ibm_chain_64.txt", 64)
    head("results/samples_nq70_reseeded.txt", "samples2_16.txt", 16)
    # the gate constants of cloud_ibmxeb/run.sh:19-21
    json.dump(dict(log2p=[-69.508530214929, -68.876165103181], tol=1e-5),
              open(os.path.join(d, "gate_log2p.json"), "w"))


def phase_extras(exp, out):
    """Reference outputs of the rows around the executor: dp.cpp jobs with slicing (engine.py), sampler_ref, and
    make_sliced_plans with a twist file."""
    sys.path.insert(0, REF)
    import numpy as np
    from tableau import Tableau
    from amp import Amplitudes
    from engine import Sliced, write_plan, write_jobs
    from ref import run
    import sampler_ref
    from sliced_plans import make_sliced_plans
    data = json.load(open(exp))
    cases = [c for c in data["cases"] if c["name"].startswith("small") and c["n"] >= 5 and all(
        t[0] in ("tdg", "h") or t[0].startswith("rz(") for t in c["tail"])][:6]
    res = dict(dp=[], sampler=[], sliced=[])
    with tempfile.TemporaryDirectory() as td:
        for c in cases:
            n = c["n"]
            T = Tableau(n)
            for g, qs in c["body"]:
                T.apply(g, qs)
            am = Amplitudes(n, T, [tuple(t) for t in c["tail"]], c["order"])
            rr = random.Random(n * 101)
            S = sorted(rr.sample(range(n), 2))
            sl = Sliced(am.A, c["order"], S)
            bs = [[rr.randrange(2) for _ in range(n)] for _ in range(3)]
            ws = [am.weights(b) for b in bs]
            write_plan(os.path.join(td, "dp_plan.txt"), sl.steps, sl.m)
            write_jobs(os.path.join(td, "dp_jobs.txt"), sl, ws)
            lines = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "dp"), "dp_plan.txt", "dp_jobs.txt"],
                                   capture_output=True, text=True, cwd=td, check=True).stdout.split("\n")
            res["dp"].append(dict(name=c["name"], S=S, bits=bs, plan=open(os.path.join(td, "dp_plan.txt")).read(),
                                  jobs=open(os.path.join(td, "dp_jobs.txt")).read(),
                                  ref_dp=[ln for ln in lines if ln.strip()],
                                  ref_run=[[run(am.steps, w).real, run(am.steps, w).imag] for w in ws]))
            prefs = [[rr.randrange(2) for _ in range(t)] for t in (0, 1, n // 2, n - 1)]
            conds = [[list(map(float, x)) for x in sampler_ref.conditionals(am, p)] for p in prefs]
            samples = [sampler_ref.sample(am, np.random.default_rng(seed)) for seed in (1, 2, 3, 4)]
            st0 = am.steps[min(2, n - 1)]
            old = np.array([complex(rr.gauss(0, 1), rr.gauss(0, 1)) for _ in range(1 << st0["r"])])
            wv = (am.M[st0["v"]][0, 0], am.M[st0["v"]][0, 1])
            ext = sampler_ref.extend(old, st0, wv)
            dist = sampler_ref.chain_distribution(am) if n <= 7 else None
            res["sampler"].append(dict(name=c["name"], prefixes=prefs, conditionals=conds, samples=samples,
                                       extend_step=min(2, n - 1),
                                       extend_in=[[z.real, z.imag] for z in old],
                                       extend_out=[[z.real, z.imag] for z in ext],
                                       chain_distribution=None if dist is None else
                                       [["".join(map(str, k)), v] for k, v in sorted(dist.items())]))
        # sliced plans with a suffix neighbour: the first case whose slice vertices have suffix neighbours
        for c in data["cases"]:
            if not c["name"].startswith("small") or c["n"] < 7 or any(t[0].startswith("u3(") for t in c["tail"]):
                continue
            n = c["n"]
            T = Tableau(n)
            for g, qs in c["body"]:
                T.apply(g, qs)
            am = Amplitudes(n, T, [tuple(t) for t in c["tail"]], c["order"])
            order = c["order"]
            K = n - 2
            S = [order[1]]
            try:
                info = make_sliced_plans(am.A, [m.copy() for m in am.M], order, S, os.path.join(td, "sp"), K=K, ND=n)
            except AssertionError:
                continue
            if not info["twist"]:
                continue
            files = {}
            for bits in itertools.product([0, 1], repeat=len(S)):
                tag = "".join(map(str, bits))
                files[tag] = open(os.path.join(td, f"sp_s{tag}.txt")).read()
            res["sliced"].append(dict(name=c["name"], S=S, K=K, info=info, plans=files,
                                      twist=open(os.path.join(td, "sp_twist.txt")).read(),
                                      slices_json=open(os.path.join(td, "sp_slices.json")).read()))
            if len(res["sliced"]) >= 3:
                break
        # the reference's hybrid rejection driver (doped_sampler.py) run on an undoped instance (--na 0 --nd n)
        # with the compiled reference executor as --bin: unsliced sample + score, and the sliced variant
        res["driver"] = []
        gs2 = os.path.join(ROOT, "oracle", "_ref", "gsamp2")
        for d in res["sliced"][:1]:
            c = {x["name"]: x for x in data["cases"]}[d["name"]]
            n = c["n"]
            T = Tableau(n)
            for g, qs in c["body"]:
                T.apply(g, qs)
            am = Amplitudes(n, T, [tuple(t) for t in c["tail"]], c["order"])
            from inplace import plan_inplace as _pi, write_inplace_plan as _wi
            R = max(1, max(max(st["r"], st["rn"]) for st in am.steps))
            _wi(os.path.join(td, "full.txt"), _pi(am.A, c["order"], R), R, am.M, n)
            json.dump(c["order"], open(os.path.join(td, "sv.json"), "w"))
            for tag, text in d["plans"].items():
                open(os.path.join(td, f"sl_s{tag}.txt"), "w").write(text)
            open(os.path.join(td, "sl_twist.txt"), "w").write(d["twist"])
            rr = random.Random(7)
            strings = ["".join(str(rr.randrange(2)) for _ in range(n)) for _ in range(6)]
            open(os.path.join(td, "str.txt"), "w").write("\n".join(strings) + "\n")
            drv = os.path.join(REF, "doped_sampler.py")
            common = ["--na", "0", "--nd", str(n), "--bin", gs2, "--threads", "2"]
            runs = {}
            for name, args in (("sample", ["sample", "full.txt", "sv.json", "24", "5", "2.0", "o_sample.txt", "--m", "2"]),
                               ("score", ["score", "full.txt", "sv.json", "str.txt", "o_score.txt"]),
                               ("sample_sliced", ["sample", "sl_s0.txt", "sv.json", "12", "6", "2.0", "o_ss.txt",
                                                  "--slices", "sl_s0.txt,sl_s1.txt", "--K", str(d["K"]), "--twist",
                                                  "sl_twist.txt", "--m", "2"]),
                               ("score_sliced", ["score", "sl_s0.txt", "sv.json", "str.txt", "o_sc.txt", "--slices",
                                                 "sl_s0.txt,sl_s1.txt", "--K", str(d["K"]), "--twist", "sl_twist.txt"])):
                outf = args[args.index("sv.json") + (4 if args[0] == "sample" else 2)]
                if os.path.exists(os.path.join(td, outf)):
                    os.unlink(os.path.join(td, outf))
                subprocess.run([sys.executable, drv] + args + common, cwd=td, check=True, capture_output=True)
                runs[name] = dict(args=args, lines=open(os.path.join(td, outf)).read().split("\n"))
            res["driver"].append(dict(name=d["name"], strings=strings, K=d["K"], runs=runs))
    json.dump(res, open(out, "w"))


def w30_reference_outputs():
    """The compiled reference executor (complex64 and complex128 builds) on the width-30 gate strings: 'prob' and
    'chain' lines for the shipped plan and 'prob' for the regenerated one (about a minute per run on 8 cores)."""
    d = os.path.join(HERE, "w30")
    out = {}
    for prec in (64, 128):
        out[f"prob{prec}"] = _ref(prec, ["nq70_inplace_plan.txt", "prob", "gate_strings.txt"], d)
        out[f"chain{prec}"] = _ref(prec, ["nq70_inplace_plan.txt", "chain", "gate_strings.txt"], d)
        out[f"regen_prob{prec}"] = _ref(prec, ["nq70_inplace_plan_regen.txt", "prob", "gate_strings.txt"], d)
    json.dump(out, open(os.path.join(d, "gate_ref_outputs.json"), "w"), indent=1)


if __name__ == "__main__":
    if sys.argv[1:] == ["--w30"]:
        w30_reference_outputs()
        sys.exit(0)
    if len(sys.argv) > 1 and sys.argv[1] == "--phase":
        ph = sys.argv[2]
        if ph == "inputs":
            phase_inputs(sys.argv[3])
        elif ph == "expected":
            phase_expected(sys.argv[3], sys.argv[4])
        elif ph == "executor":
            phase_executor(sys.argv[3], sys.argv[4])
        elif ph == "extras":
            phase_extras(sys.argv[3], sys.argv[4])
        sys.exit(0)
    me = os.path.abspath(__file__)
    os.makedirs(os.path.join(HERE, "w30"), exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "inputs.json")
        subprocess.run([sys.executable, me, "--phase", "inputs", inp], check=True)
        subprocess.run([sys.executable, me, "--phase", "expected", inp, os.path.join(HERE, "planner_cases.json")],
                       check=True, cwd=td)
        subprocess.run([sys.executable, me, "--phase", "executor", os.path.join(HERE, "planner_cases.json"),
                        os.path.join(HERE, "executor_cases.json")], check=True, cwd=td)
        subprocess.run([sys.executable, me, "--phase", "extras", os.path.join(HERE, "planner_cases.json"),
                        os.path.join(HERE, "extras_cases.json")], check=True, cwd=td)
    copy_w30()
    print("golden fixtures written to", HERE)
