"""Record the executor calls of the reference's hybrid driver, for replay against gsb2 on the GPU.

    python tests/golden/record_driver_calls.py      (needs the reference checkout at $GSB_REFERENCE_DIR, by default
                                                     the sibling directory "reference" of this checkout, and the
                                                     compiled reference executor, `make -C oracle ref`)

The reference's doped_sampler.py runs its executor as a subprocess chosen by --bin (doped_sampler.py:28).  This script
runs the unmodified driver on the driver runs of extras_cases.json (sample and score, unsliced and sliced with a twist
file) with --bin pointing at a small recording wrapper.  The wrapper runs the compiled reference executor
(oracle/_ref/gsamp2) with the same arguments and logs, per call, its argv, the text files it reads (strings and twist
files) and its stdout and exit status.  The driver cannot travel to the GPU machine, so its calls are kept as
driver_calls.json, and tests/test_gpu_cli.py replays them in order against gsb2.
"""
import json
import os
import re
import stat
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("GSB_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
GSAMP2 = os.path.join(ROOT, "oracle", "_ref", "gsamp2")

WRAPPER = r'''#!{python}
import json, subprocess, sys
argv = sys.argv[1:]
mode = argv[1]
files = {{}}
if mode in ("prob", "chain", "hybrid", "prefix", "resume"):
    files[argv[2]] = open(argv[2]).read()
if mode == "resume" and "--twist" in argv:
    t = argv[argv.index("--twist") + 1]
    files[t] = open(t).read()
p = subprocess.run([{exe!r}] + argv, capture_output=True, text=True)
with open({log!r}, "a") as f:
    f.write(json.dumps({{"argv": ["gsamp2"] + argv, "inputs": files, "stdout": p.stdout, "rc": p.returncode}}) + "\n")
sys.stdout.write(p.stdout)
sys.stderr.write(p.stderr)
sys.exit(p.returncode)
'''


def _untimed(lines):
    """Driver output lines without their wall-time fields ("0.0" / "0.0s")."""
    return [" ".join(t for t in ln.split() if not re.fullmatch(r"[0-9.]+s?", t) or t == ln.split()[0])
            if ln and not ln.startswith("#") else ln for ln in lines]


def main():
    extras = json.load(open(os.path.join(HERE, "extras_cases.json")))
    cases = {c["name"]: c for c in json.load(open(os.path.join(HERE, "planner_cases.json")))["cases"]}
    sys.path.insert(0, os.path.join(ROOT, "exact-graphstate-sampling_b200"))
    from amp import Amplitudes
    from circuits import tableau_of
    from inplace import inplace_plan_text, plan_inplace, plan_width
    out = {"driver": "doped_sampler.py", "executor": "oracle/_ref/gsamp2 (complex64)", "runs": []}
    for d in extras["driver"]:
        c = cases[d["name"]]
        n = c["n"]
        am = Amplitudes(n, tableau_of(n, c["body"]), [tuple(t) for t in c["tail"]], c["order"])
        R = max(1, plan_width(am.steps))
        full = inplace_plan_text(plan_inplace(am.A, c["order"], R), R, am.M, n)
        assert full == c["inplace_plan"]
        sl = [s for s in extras["sliced"] if s["name"] == d["name"]][0]
        files = {"full.txt": "@plan:" + d["name"], "sv.json": json.dumps(c["order"]),
                 "sl_twist.txt": sl["twist"], "str.txt": "\n".join(d["strings"]) + "\n"}
        files.update({f"sl_s{tag}.txt": text for tag, text in sl["plans"].items()})
        for name, run in d["runs"].items():
            with tempfile.TemporaryDirectory() as td:
                for f, text in files.items():
                    open(os.path.join(td, f), "w").write(c["inplace_plan"] if text.startswith("@plan:") else text)
                log = os.path.join(td, "calls.jsonl")
                wrap = os.path.join(td, "rec_exec")
                open(wrap, "w").write(WRAPPER.format(python=sys.executable, exe=GSAMP2, log=log))
                os.chmod(wrap, os.stat(wrap).st_mode | stat.S_IEXEC)
                args = list(run["args"])
                subprocess.run([sys.executable, os.path.join(REF, "doped_sampler.py")] + args +
                               ["--na", "0", "--nd", str(n), "--bin", wrap, "--threads", "2"], cwd=td, check=True,
                               capture_output=True)
                calls = [json.loads(ln) for ln in open(log)]
                outf = args[args.index("sv.json") + (4 if args[0] == "sample" else 2)]
                lines = open(os.path.join(td, outf)).read().split("\n")
                # the driver's own output must be the one recorded in extras_cases.json (same seeds, same executor)
                strip, ref = _untimed(lines), _untimed(run["lines"])
                assert strip == ref, (name, [(a, b) for a, b in zip(strip, ref) if a != b][:3])
            out["runs"].append({"name": f"{d['name']}_{name}", "driver_args": args, "files": files, "calls": calls})
    json.dump(out, open(os.path.join(HERE, "driver_calls.json"), "w"), indent=0)
    print(f"recorded {sum(len(r['calls']) for r in out['runs'])} executor calls of {len(out['runs'])} driver runs")


if __name__ == "__main__":
    main()
