#!/usr/bin/env python
"""Benchmark of the B200 cut-rank DP executor on the n=70, width-30 workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gsb|reference]

Workload: n = 70 random graph-state circuit of depth 70 (CZ on seeded random perfect matchings + seeded random
single-qubit Cliffords, seed 2), Haar-random U3 layer, order of width 30 from the native order search (seed 12):
an arena of 2^30 entries (8.6 GB complex64, 17.2 GB complex128).  The arena is far larger than L2 (126 MB), so
every pass streams from HBM and no flush is needed between steps.

One step = the exact amplitudes (log2 Pr and all 70 conditionals, 'chain' mode: one pass per DP step) of
--amps-per-step uniform random bitstrings in the complex64 form.  `value` is amplitudes/s with the strings already
in HBM (device-resident entry point), timed with CUDA events on the engine's stream, max over ranks; `e2e` is the
same metric through the host-buffer C-ABI call (strings copied in from pinned host memory, log2 Pr and
conditionals copied back, every step).  Extra keys report exact samples (s/sample), the complex128 form (with the
same fused passes, and its samples also with one norm and one write pass per step), the complex64-vs-complex128
agreement, the roofline of the dominant kernel and the reference's CPU executor timed on this host.

Multi-GPU: replicas only (the arena sweep does not shard without an all-to-all per step): each rank evaluates its
own strings on its own GPU; value = all ranks' amplitudes / the slowest rank's time.

--impl reference times the reference's own CPU executor (gsamp2 compiled from its sources into oracle/_ref, complex64,
'chain' mode, every host core) on one string of the same workload per step, on rank 0 only.

--form batch|grad|wide34 measures the other workloads instead, one JSON line each (1 GPU):
  batch : 512 matching instances, n uniform in [16, 40], 16 prefixes x 4 suffixes each, one persistent launch
          (complex64, autotuned shape, complex128 agreement);
  grad  : n = 48 rotation layer, loss -mean log2 Pr over 2048 targets drawn exactly from a second instance,
          gradient by the adjoint sweep;
  wide34: n = 80, width 34 (2^34-entry complex64 arena, 137 GB): 256 amplitudes and 16 exact samples.
"""
import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "exact-graphstate-sampling_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)
import replicas  # noqa: E402  (package module: torchrun rank bookkeeping)

METRIC = "s/sample & amps/s at n=70 w=30, c64 form vs c128 plain, |Δlog2P|≤1e-5; HBM GB/s"
WORKLOAD = "matching_n70_d70_s2_w30"
K_GROUP_TRAFFIC_RATIO = 0.9726
# the headline workload's plan text (tests/golden/make_headline_plan.py writes it; a host test pins it to the package)
HEADLINE_PLAN = os.path.join(ROOT, "tests", "golden", "headline", "matching_n70_w30_plan.txt")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gsb", choices=["gsb", "reference"])
    ap.add_argument("--amps-per-step", type=int, default=16)
    ap.add_argument("--samples", type=int, default=16)
    ap.add_argument("--c128-amps", type=int, default=16,
                    help="strings timed for the complex128 amplitudes/s (every timed string is checked against it)")
    ap.add_argument("--no-c128", dest="c128", action="store_false")
    ap.add_argument("--tol", type=float, default=1e-5, help="|d log2 Pr| the complex64 form is held to")
    ap.add_argument("--no-guard", dest="guard", action="store_false",
                    help="complex64 without the complex128 re-evaluation of unlikely strings")
    ap.add_argument("--no-ref-gpu-port", dest="ref_gpu_port", action="store_false",
                    help="skip timing the reference's own GPU port (oracle/_ref/gsamp_cuda)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-plan", default=HEADLINE_PLAN,
                    help="--impl reference: plan file to time (default: the committed headline plan)")
    ap.add_argument("--ref-samples", type=int, default=2,
                    help="--impl reference: exact samples drawn by the reference executor for s/sample (0 = none)")
    ap.add_argument("--arith", type=int, default=32, choices=[32, 64],
                    help="arithmetic of the complex64 wide-step kernels (32: FP32; 64: exact sums + FP64 rotation)")
    ap.add_argument("--fusion", type=int, default=2, choices=[1, 2, 3],
                    help="'chain' mode: DP steps fused into one pass over the arena (1 = none)")
    ap.add_argument("--profile-chain", type=int, default=0, metavar="N",
                    help="only evaluate N strings in chain mode on --profile-workload (for ncu captures)")
    ap.add_argument("--profile-workload", default="n70", choices=["n70", "n64", "n62"])
    ap.add_argument("--profile-mode", default="chain", choices=["chain", "sample"],
                    help="with --profile-chain: evaluate strings (chain) or draw exact samples (sample)")
    ap.add_argument("--profile-precision", type=int, default=64, choices=[64, 128])
    ap.add_argument("--proposals", type=int, default=64, help="--form hybrid: proposals per timed run")
    ap.add_argument("--no-forms", dest="forms", action="store_false",
                    help="headline line without the hybrid-driver and batched-launch sub-measurements")
    ap.add_argument("--form", default="headline", choices=["headline", "batch", "grad", "wide34", "hybrid"],
                    help="workload to measure (the default line is the headline n = 70, width-30 workload)")
    ap.add_argument("--batch-instances", type=int, default=512)
    ap.add_argument("--wide34-amps", type=int, default=256, help="--form wide34: amplitudes timed")
    ap.add_argument("--wide34-samples", type=int, default=16, help="--form wide34: exact samples timed")
    ap.add_argument("--no-wide34-check", dest="wide34_check", action="store_false",
                    help="--form wide34: skip the complex128 cross-check through the width-30 sliced order")
    ap.add_argument("--batch-order", default="qubit", choices=["qubit", "search"],
                    help="--form batch: qubit index order (widths 7-20, the configuration's) or the native search")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the byte-model pass lists (skip the guarded autotuner)")
    return ap.parse_args()


def profile_chain(args):
    """A bare run for profilers: build the workload, evaluate N strings in chain mode, print nothing else."""
    import gsb
    import workloads
    w = {"n70": workloads.matching_n70_w30,
         "n64": lambda: workloads.matching_instance(64, 64, 2, 12),     # width 27: a 1.07 GB complex64 arena
         "n62": lambda: workloads.matching_instance(62, 62, 3, 13)}[args.profile_workload]()
    with gsb.Engine.from_text(w["plan"], precision=args.profile_precision) as eng:
        eng.set_arith(args.arith)
        eng.set_fusion(args.fusion)
        if args.profile_mode == "sample":
            _, lp = eng.sample(args.profile_chain, seed=5)
        else:
            lp, _ = eng.chain(workloads.random_strings(len(w["steps"]), args.profile_chain, seed=9))
    print(json.dumps({"workload": w["name"], "width": w["width"], "log2p": [float(x) for x in lp]}))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples every 200 ms while running (SM clock, max clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        for ln in open(self.f.name):
            t = [x.strip() for x in ln.split(",")]
            if len(t) >= 9:
                try:
                    rows.append((float(t[1]), float(t[2]), t[5:9]))
                except ValueError:
                    pass
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def ref_time(plan_path, mode_args, threads, precision=64):
    """Wall time and stdout of the reference executor (oracle/_ref/gsamp2, compiled from the reference's sources)
    on `gsamp2 <plan> <mode_args...>`; without that build, the C restatement of the same executor ('port')."""
    from oracle import ref_binary, run_ref
    t0 = time.perf_counter()
    if ref_binary(precision):
        out = run_ref(precision, [plan_path] + list(mode_args), threads=threads)
        return time.perf_counter() - t0, out, "reference"
    from oracle import Oracle
    o = Oracle(plan_path, precision)
    lines = []
    if mode_args[0] == "chain":
        for ln in open(mode_args[1]):
            if ln.strip():
                lp, _ = o.chain1(ln.strip())
                lines.append(f"{lp:.12f}")
    else:                                                    # sample N seed
        for i in range(int(mode_args[1])):
            bits, lp = o.sample(0, int(mode_args[2]), i)
            lines.append("".join(map(str, bits)) + f" {lp:.12f}")
    o.close()
    return time.perf_counter() - t0, "\n".join(lines) + "\n", "port"


def repo_libraries():
    """Shared objects of this repository mapped into this process (from /proc/self/maps), relative paths."""
    root = os.path.realpath(ROOT) + os.sep
    seen = set()
    try:
        for ln in open("/proc/self/maps"):
            f = ln.split()
            if len(f) >= 6 and (f[-1].endswith(".so") or ".so." in f[-1]):
                p = os.path.realpath(f[-1])
                if p.startswith(root):
                    seen.add(os.path.relpath(p, root))
    except OSError:
        pass
    return sorted(seen)


def run_reference(args):
    """The reference's own CPU executor on the headline workload, every host thread, rank 0 only.  The plan comes
    from a committed file, so this process loads nothing of this repository's package or library."""
    if int(os.environ.get("RANK", "0")) != 0:   # rank 0 alone times the host reference; no process group needed
        return
    import numpy as np
    from oracle import ref_isa
    plan_text = open(args.ref_plan).read()
    head = plan_text.split(None, 3)
    n, ns, width = int(head[0]), int(head[1]), int(head[2])
    cores = os.cpu_count() or 1
    strings = np.random.default_rng(4242).integers(0, 2, size=(args.warmup + args.steps, ns), dtype=np.int8)
    with tempfile.TemporaryDirectory() as td:
        plan = os.path.join(td, "plan.txt")
        open(plan, "w").write(plan_text)
        times = []
        kind = "reference"
        for i in range(args.warmup + args.steps):
            sp = os.path.join(td, f"s{i}.txt")
            open(sp, "w").write("".join(str(int(b)) for b in strings[i]) + "\n")
            t, _, kind = ref_time(plan, ["chain", sp], cores)
            if i >= args.warmup:
                times.append(t)
        samples = {}
        if args.ref_samples > 0:
            t, out, _ = ref_time(plan, ["sample", str(args.ref_samples), "2000000"], cores)
            samples = {"s_per_sample": t / args.ref_samples, "samples_per_s": args.ref_samples / t,
                       "samples_timed": args.ref_samples,
                       "sample_mode": f"gsamp2 sample {args.ref_samples} 2000000 (one process, wall clock)"}
    tot = sum(times)
    v = args.steps / tot
    isa = ref_isa(64) if kind == "reference" else None
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "amps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 arena, f64 arithmetic", "data": "synthetic",
        "config": {"workload": WORKLOAD if args.ref_plan == HEADLINE_PLAN else os.path.basename(args.ref_plan),
                   "n": n, "width": width, "strings_per_step": 1, "mode": "chain", "l2": "arena 8.6 GB >> L2"},
        "cpu_baseline": {"value": v, "unit": "amps/s", "cores": cores, "kind": kind,
                         "sample": f"{args.steps} uniform random strings of the workload, one per step, gsamp2 chain "
                                   f"mode, OMP_NUM_THREADS={cores}" + (f", built -march=x86-64-{isa}" if isa else "")},
        "e2e": {"value": v, "unit": "amps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "repo_libraries_loaded": repo_libraries(),
    }
    line.update(samples)
    print(json.dumps(line), flush=True)


def ref_gpu_port_time(plan_path, strings, ns):
    """The reference's own GPU port (gsamp_cuda.cu built for sm_100a into oracle/_ref) in 'chain' mode on the first
    strings of the workload: seconds per string from two runs (1 string and len(strings) strings, so its start-up and
    arena allocation cancel), and its log2 Pr.  None when that build is absent."""
    from oracle import ref_gpu_binary
    exe = ref_gpu_binary()
    if not exe:
        return None
    with tempfile.TemporaryDirectory() as td:
        def run(k):
            sp = os.path.join(td, f"s{k}.txt")
            open(sp, "w").write("".join("".join(str(int(b)) for b in strings[i]) + "\n" for i in range(k)))
            t0 = time.perf_counter()
            out = subprocess.run([exe, plan_path, "chain", sp], capture_output=True, text=True, timeout=600)
            t = time.perf_counter() - t0
            if out.returncode:
                raise RuntimeError(f"gsamp_cuda exit {out.returncode}: {out.stderr[-300:]}")
            return t, [float(ln.split()[0]) for ln in out.stdout.split("\n") if ln.strip()]
        k = len(strings)
        t1, _ = run(1)
        tk, lp = run(k)
    per = (tk - t1) / (k - 1)
    return {"s_per_string": per, "amps_per_s": 1.0 / per, "strings_timed": k,
            "timing": f"wall clock of gsamp_cuda chain on {k} strings minus 1 string (start-up and arena set-up "
                      f"cancel)", "log2p": lp}


def run_gsb(args):
    import numpy as np
    import torch
    rank, world, local = replicas.init()
    torch.cuda.set_device(local)
    import gsb
    import workloads
    w = workloads.matching_n70_w30()
    steps = w["steps"]
    ns = len(steps)
    A, K, W = args.amps_per_step, args.steps, args.warmup
    hbm_peak, peak_kind = peaks()

    eng = gsb.Engine.from_text(w["plan"], precision=64, device=local)
    eng.set_arith(args.arith)
    eng.set_fusion(args.fusion)
    e128 = gsb.Engine.from_text(w["plan"], precision=128, device=local)
    e128.set_fusion(args.fusion)
    stream = torch.cuda.Stream()                  # a real stream: the engines' kernels and the events share it
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    e128.set_stream(stream.cuda_stream)
    # the byte-model pass lists (fused passes of up to two steps), step-timed before the autotuner replaces them:
    # their executed bytes over their own time, the bandwidth figure of the two-step fused kernel in sequence
    R0 = 32
    d_b0 = torch.from_numpy(workloads.random_strings(ns, R0, seed=999)).to("cuda")
    d_l0 = torch.empty(R0, dtype=torch.float64, device="cuda")
    eng.chain_device(d_b0[:2], d_l0[:2])
    torch.cuda.synchronize()
    t0e, t1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0e.record(stream)
    eng.chain_device(d_b0, d_l0)
    t1e.record(stream)
    torch.cuda.synchronize()
    ms_bytemodel = t0e.elapsed_time(t1e) / R0
    bytes_bytemodel = float(np.sum(eng.fusion_groups()[1])) * 8
    # guarded autotuner of the pass lists (kept only where a whole item gets faster), outside every timed region
    tune64 = eng.autotune(mode=2, reps=3) if args.autotune else None
    tune128 = e128.autotune(mode=2, reps=3) if args.autotune else None
    # the complex64 form: complex64 arena, FP32 arithmetic, complex128 re-evaluation of the strings whose complex64
    # probability lies below the error model's threshold for |d log2 Pr| <= TOL
    lx = gsb.c64_guard_log2_xmin(ns, args.tol) if args.guard else float("-inf")
    if args.guard:
        eng.set_guard(e128, lx)
    strings = workloads.random_strings(ns, (W + K) * A, seed=1000 + rank)
    d_bits = torch.from_numpy(strings).to("cuda")
    d_lp = torch.empty((W + K) * A, dtype=torch.float64, device="cuda")
    d_cond = torch.empty(((W + K) * A, ns), dtype=torch.float64, device="cuda")

    def amp_step(i):
        sl = slice(i * A, (i + 1) * A)
        eng.chain_device(d_bits[sl], d_lp[sl], d_cond[sl])

    for i in range(W):
        amp_step(i)
    torch.cuda.synchronize()
    replicas.barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0 = eng.guard_evaluations()
    with Clocks(local) as clk:
        ev0.record(stream)
        for i in range(W, W + K):
            amp_step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
    replicas.barrier(world)
    torch.cuda.synchronize()
    guarded_timed = eng.guard_evaluations() - g0
    ms = ev0.elapsed_time(ev1)
    ms_max = replicas.max_over_ranks(ms, world)
    value = world * K * A / (ms_max / 1000.0)
    lp64 = d_lp.cpu().numpy()

    # e2e: host strings (pinned) -> C ABI -> host results, every step
    pinned = torch.from_numpy(strings[W * A:(W + K) * A].copy()).pin_memory()
    host = pinned.numpy()
    eng.chain(host[:A])
    torch.cuda.synchronize()
    replicas.barrier(world)
    t0 = time.perf_counter()
    for i in range(K):
        eng.chain(host[i * A:(i + 1) * A])
    e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, world)
    e2e = {"value": world * K * A / e2e_s, "unit": "amps/s", "h2d_bytes_per_step": A * ns,
           "d2h_bytes_per_step": A * 8 + A * ns * 8}

    # exact samples (fused sampling passes), device-resident uniforms, guarded like the amplitudes
    S = args.samples
    rng = np.random.default_rng(77 + rank)
    d_u = torch.from_numpy(rng.random((S, ns))).to("cuda")
    d_sb = torch.empty((S, ns), dtype=torch.int8, device="cuda")
    d_slp = torch.empty(S, dtype=torch.float64, device="cuda")
    eng.sample_device(d_u[:1], d_sb[:1], d_slp[:1])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    eng.sample_device(d_u, d_sb, d_slp)
    e1.record(stream)
    torch.cuda.synchronize()
    s_per_sample64 = replicas.max_over_ranks(e0.elapsed_time(e1) / 1000.0 / S, world)
    sbits64 = d_sb.cpu().numpy()
    slp64 = d_slp.cpu().numpy()

    # unguarded complex64 on the same strings (its raw error), and a step-timed unguarded batch for the roofline
    eng.set_guard(None, 0.0)
    nt = (W + K) * A
    d_lpr = torch.empty(nt, dtype=torch.float64, device="cuda")
    eng.chain_device(d_bits, d_lpr)
    torch.cuda.synchronize()
    lp64_raw = d_lpr.cpu().numpy()
    R = min(nt, 32)
    e0.record(stream)
    eng.chain_device(d_bits[:R], d_lpr[:R])
    e1.record(stream)
    torch.cuda.synchronize()
    ms_per_string = e0.elapsed_time(e1) / R

    # roofline of the dominant kernels (the chain-mode passes: fused groups k_group and single steps).  achieved =
    # the bytes the executed passes must read and write (fused groups keep intermediate tables in shared memory)
    # over the step-timed time per string; the per-pass event sum and the unfused per-step byte model are reported
    # beside it
    tot_bytes, per = workloads.pass_bytes(steps, 8, "chain")
    glen, gent = eng.fusion_groups()
    wsum = np.zeros(ns)
    nprof = 3
    for j in range(nprof):
        wm, _ = eng.profile_steps(strings[j])
        wsum += wm
    wmean = wsum / nprof
    pass_bytes = float(np.sum(gent)) * 8
    kernel_ms = float(wmean.sum())
    achieved = pass_bytes / (ms_per_string / 1000.0) / 1e9
    fused = [k for k in range(ns) if glen[k] >= 2]
    fused_bytes = float(sum(gent[k] for k in fused)) * 8
    fused_ms = float(sum(wmean[k] for k in fused))
    # DRAM bytes per algorithmic byte of the dominant pass, from one ncu capture of k_group<float2, float, 2, 0> on the
    # width-27 instance (no re-reads; writes still dirty in L2 at kernel end make it < 1), scaled to one string
    traffic = pass_bytes * K_GROUP_TRAFFIC_RATIO
    sw, sn = eng.profile_steps(strings[0], mode=1)
    sample_kernel_ms = float(sw.sum() + sn.sum())
    _, sent = eng.sample_groups()
    sample_pass_bytes = float(np.sum(sent)) * 8
    sample_bytes = float(sum((2 * (1 << st["r"]) + (1 << st["rn"])) for st in steps)) * 8
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": traffic, "traffic_source": "ncu dram bytes of one k_group launch (width-27 capture) per "
                                                      "algorithmic byte, times the pass bytes of one string",
                "peak_kind": peak_kind,
                "kernel": "chain passes: k_group<float2,float,*> (fused) + k_pair64/k_step (single steps)",
                "pass_bytes_per_string": pass_bytes,
                "step_timed_ms_per_string": ms_per_string,
                "step_timed": f"{R} strings in one unguarded chain_device call, CUDA events",
                "kernel_ms_per_string_event_sum": kernel_ms,
                "fused_passes_frac": (fused_bytes / (fused_ms / 1000.0) / 1e9) / hbm_peak if fused_ms > 0 else None,
                "model_unfused_bytes_per_string": float(sum(p[0] for p in per)),
                "model_unfused_GBps": float(sum(p[0] for p in per)) / (ms_per_string / 1000.0) / 1e9,
                "model_note": "the unfused per-step byte model E*sum(2^r_k + 2^r_k+1); the fused passes move fewer "
                              "bytes, so this model's GB/s exceeds the copy peak",
                "passes_per_string": int(sum(1 for x in glen if x > 0)), "fusion": args.fusion,
                "passes_note": "the timed lists are the autotuner's: fused passes of up to three steps, which move "
                               "fewer bytes for more arithmetic per byte, so they run below the copy peak while "
                               "the item as a whole gets faster",
                "byte_model_lists": {"ms_per_string": ms_bytemodel, "pass_bytes_per_string": bytes_bytemodel,
                                     "achieved": bytes_bytemodel / (ms_bytemodel / 1e3) / 1e9,
                                     "frac": bytes_bytemodel / (ms_bytemodel / 1e3) / 1e9 / hbm_peak,
                                     "what": "the same chain with the byte-model lists (fused passes of up to two "
                                             "steps, the dominant kernel k_group<float2,float,2,0,2,1>), step-timed "
                                             "on 32 strings before the autotuner ran"},
                "sample_kernel_ms": sample_kernel_ms, "sample_norm_ms": float(sn.sum()),
                "sample_write_ms": float(sw.sum()), "model_unfused_sample_bytes": sample_bytes,
                "sample_pass_bytes": sample_pass_bytes,
                "sample_achieved": sample_pass_bytes / (sample_kernel_ms / 1000.0) / 1e9,
                "sample_frac": sample_pass_bytes / (sample_kernel_ms / 1000.0) / 1e9 / hbm_peak}

    # kernel launches of one chain item (begin, passes with each run of small steps as one launch, finish)
    lpi64, lpi128 = eng.launches_per_item(0), e128.launches_per_item(0)

    # complex128 plain form: amplitudes/s, every timed string and every sample again, s/sample
    c128 = {}
    if args.c128:
        B = min(args.c128_amps, K * A)
        d_lp128 = torch.empty(nt, dtype=torch.float64, device="cuda")
        d_cond128 = torch.empty((nt, ns), dtype=torch.float64, device="cuda")
        sl = slice(W * A, W * A + B)
        e128.chain_device(d_bits[:1], d_lp128[:1], d_cond128[:1])
        torch.cuda.synchronize()
        e0.record(stream)
        e128.chain_device(d_bits[sl], d_lp128[sl], d_cond128[sl])
        e1.record(stream)
        torch.cuda.synchronize()
        amps128 = B / (e0.elapsed_time(e1) / 1000.0)
        e128.chain_device(d_bits, d_lp128, d_cond128)
        torch.cuda.synchronize()
        lp128 = d_lp128.cpu().numpy()
        dlp = np.abs(lp128 - lp64)
        dlp_raw = np.abs(lp128 - lp64_raw)
        d_sb128 = torch.empty((S, ns), dtype=torch.int8, device="cuda")
        d_slp128 = torch.empty(S, dtype=torch.float64, device="cuda")

        def time_samples128():
            e128.sample_device(d_u[:1], d_sb128[:1], d_slp128[:1])   # graph built outside the timed region
            torch.cuda.synchronize()
            e0.record(stream)
            e128.sample_device(d_u, d_sb128, d_slp128)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / 1000.0 / S

        s_per_sample128 = time_samples128()
        same_bits = bool((d_sb128.cpu().numpy() == sbits64).all())
        dslp = np.abs(d_slp128.cpu().numpy() - slp64)
        # the same complex128 form without fusion: one norm pass and one write pass per DP step, the structure of
        # the reference executor's two-pass sampler (gsamp2.cpp:39-55)
        e128.set_fusion(1)
        s_per_sample128_unfused = time_samples128()
        x = lp128 + ns
        c128 = {"amps_per_s": amps128, "autotune_ms_item_before_after": tune128,
                "s_per_sample": s_per_sample128, "s_per_sample_unfused_two_pass": s_per_sample128_unfused,
                "samples_per_s_ratio_c64_over_c128": s_per_sample128 / s_per_sample64,
                "check": {"strings": int(nt), "samples": int(S), "tol": args.tol,
                          "max_abs_dlog2p_c64_vs_c128": float(dlp.max()),
                          "strings_above_tol": int((dlp > args.tol).sum()),
                          "max_abs_dlog2p_c64_unguarded": float(dlp_raw.max()),
                          "unguarded_above_tol": int((dlp_raw > args.tol).sum()),
                          "median_abs_dlog2p_times_sqrt_x_unguarded": float(np.median(dlp_raw * np.sqrt(2.0 ** x))),
                          "samples_max_abs_dlog2p": float(dslp.max()), "samples_same_bits_c64_c128": same_bits}}
    eng.close()
    e128.close()

    guard = {"enabled": bool(args.guard), "log2_xmin": lx, "tol": args.tol,
             "strings_reevaluated_in_timed_region": int(guarded_timed),
             "fraction_of_timed_strings": guarded_timed / float(K * A),
             "model": "|d log2 Pr| ~ N(0, (s1 sqrt(ns) / sqrt(x))^2), x = Pr 2^ns; re-evaluated where "
                      "z s1 sqrt(ns) / sqrt(x) > tol"}
    # per string: one chain item (begin, passes, finish); one item reset per batch; the guard's complex128 items
    launches = lpi64 * K * A + K + guarded_timed * lpi128
    out = {
        "metric": METRIC, "value": value, "unit": "amps/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": f"c64 arena, f{args.arith} arithmetic" + (", c128 guard" if args.guard else ""), "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": 70, "width": w["width"], "strings_per_step": A, "mode": "chain",
                   "arith": args.arith, "fusion": args.fusion, "guard": bool(args.guard),
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2: arena 8.6 GB >> 126 MB"},
        "s_per_sample": s_per_sample64, "samples_per_s": world / s_per_sample64,
        "c128": c128, "guard": guard, "e2e": e2e, "roofline": roofline, "gpu_launches": launches,
        "autotune_ms_item_before_after": tune64,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and args.ref_gpu_port:
        try:
            with tempfile.TemporaryDirectory() as td:
                plan = os.path.join(td, "plan.txt")
                open(plan, "w").write(w["plan"])
                rg = ref_gpu_port_time(plan, strings[W * A:W * A + 4], ns)
            if rg:
                rg["max_abs_dlog2p_vs_c128"] = float(np.abs(np.array(rg.pop("log2p")) - lp128[W * A:W * A + 4]).max()) \
                    if c128 else None
                rg["value_over_port"] = value / rg["amps_per_s"]
                out["reference_gpu_port"] = rg
        except Exception as ex:   # the port is a reported comparison only
            out["reference_gpu_port"] = {"unavailable": str(ex)[:200]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as td:
            plan = os.path.join(td, "plan.txt")
            open(plan, "w").write(w["plan"])
            sp = os.path.join(td, "s.txt")
            open(sp, "w").write("".join(str(int(b)) for b in strings[W * A]) + "\n")
            cores = os.cpu_count() or 1
            t, txt, kind = ref_time(plan, ["chain", sp], cores)
            ref_lp = float(txt.split()[0])
            from oracle import ref_isa
            out["cpu_baseline"] = {"value": 1.0 / t, "unit": "amps/s", "cores": cores, "kind": kind,
                                   "sample": "1 uniform random string of the workload, gsamp2 chain mode (complex64"
                                             + (f", -march=x86-64-{ref_isa(64)}" if kind == "reference" else "") + ")",
                                   "abs_dlog2p_vs_gpu_c128": abs(ref_lp - float(lp128[W * A])) if c128 else None}
    if rank == 0 and world == 1 and args.forms:
        # the hybrid driver, the batched launch, the adjoint sweep and the width-34 arena on the same GPU, reported
        # inside this line (the width-34 form with 16 amplitudes and 4 samples, without its sliced complex128
        # cross-check, which `--form wide34` runs); the width-30 engines are closed, so the 137 GB arena fits
        torch.cuda.empty_cache()
        out["forms"] = {}
        for name, fn in (("hybrid", run_form_hybrid), ("batch", run_form_batch), ("grad", run_form_grad),
                         ("wide34", run_form_wide34)):
            try:
                sub = argparse.Namespace(**vars(args))
                sub.steps, sub.warmup = 5, 3
                sub.wide34_amps, sub.wide34_samples, sub.wide34_check = 16, 4, False
                out["forms"][name] = fn(sub, emit=False)
            except Exception as ex:   # a reported extra only
                out["forms"][name] = {"unavailable": str(ex)[:200]}
            gc.collect()
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(out), flush=True)
    replicas.finish(world)


def _form_line(form, metric, value, unit, hib, extra, emit=True):
    d = {"form": form, "metric": metric, "value": value, "unit": unit, "n_gpus": 1, "higher_is_better": hib,
         "data": "synthetic"}
    d.update(extra)
    if emit:
        print(json.dumps(d), flush=True)
    return d


def run_form_batch(args, emit=True):
    """Batched uneven workload: one persistent launch over all (instance, prefix) items."""
    import numpy as np
    import gsb
    import workloads
    t0 = time.perf_counter()
    bw = workloads.batch_workload(count=args.batch_instances, seed=0, npre=16, nsuf=4, order=args.batch_order)
    t_plan = time.perf_counter() - t0
    plans = [w["plan"] for w in bw["instances"]]
    widths = [w["width"] for w in bw["instances"]]
    b = gsb.Batch(plans, precision=gsb.GSB_C64)
    b.set_strings(bw["K"], bw["prefixes"], bw["suffixes"])
    if args.autotune:
        block, small_R, per_sm, tune_ms = b.tune(reps=2)
    else:
        block, small_R, per_sm = b.shape()
    for _ in range(max(3, args.warmup)):
        b.run()
    times = []
    for _ in range(args.steps):
        lp, ms = b.run()
        times.append(ms)
    ms = statistics.median(times)
    ref = gsb.Batch(plans, precision=gsb.GSB_C128)
    ref.set_strings(bw["K"], bw["prefixes"], bw["suffixes"])
    lp128, ms128 = ref.run()
    fin = np.isfinite(lp128)
    d = np.abs(lp - lp128)[fin]
    nstr = lp.size
    # algorithmic bytes: per item one prefix sweep plus nsuf suffix sweeps (one write pass per step), the
    # snapshot and its restores
    E = 8
    byt = 0
    for w, K in zip(bw["instances"], bw["K"]):
        st = w["steps"]
        pre = sum((1 << s["r"]) + (1 << s["rn"]) for s in st[:K])
        suf = sum((1 << s["r"]) + (1 << s["rn"]) for s in st[K:])
        snap = 1 << st[K]["r"]
        byt += 16 * E * (pre + 4 * suf + 2 * snap + 3 * 2 * snap)
    peak, kind = peaks()
    l2 = max(gsb.probe_l2_copy(mib=mib) for mib in (16, 24, 32))
    # working set of the items in flight: each CTA team holds one wide item's arena and snapshot (2 x 2^R x E)
    wide = [1 << r for r in widths if r > small_R] or [0]
    working_set = min(len(wide), per_sm * 148) * 2 * E * float(np.mean(wide))
    l2_bytes = 126e6
    roof_l2 = {"bound": "l2", "achieved": byt / (ms / 1e3) / 1e9, "peak": l2, "unit": "GB/s",
               "frac": byt / (ms / 1e3) / 1e9 / l2,
               "peak_kind": "measured here: L2 copy bandwidth (gsb_probe_l2_copy, best of 16/24/32 MiB buffers, one "
                            "launch of 400 passes)"}
    roof_hbm = {"bound": "hbm", "achieved": byt / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                "frac": byt / (ms / 1e3) / 1e9 / peak, "peak_kind": kind}
    return _form_line("batch", "amps/s, 512 instances n in [16,40] x 64 strings, one persistent launch", nstr / (ms / 1e3),
               "amps/s", True, {
                   "ms_per_launch": ms, "strings": int(nstr), "instances": len(plans),
                   "widths": {"min": int(min(widths)), "max": int(max(widths)), "mean": float(np.mean(widths))},
                   "dtype": "c64 arena, f32 sums, f64 norms/scales", "shape": {"block": block, "small_R": small_R,
                                                                                 "ctas_per_sm": per_sm},
                   "c128": {"ms_per_launch": ms128, "max_abs_dlog2p_c64_vs_c128": float(d.max()),
                            "median_abs_dlog2p": float(np.median(d))},
                   "roofline": roof_l2 if working_set <= l2_bytes else roof_hbm,
                   "roofline_other": roof_hbm if working_set <= l2_bytes else roof_l2,
                   "working_set_bytes": working_set,
                   "roofline_choice": "the L2 line when the wide items in flight (one per CTA team: arena and "
                                      "snapshot) fit the 126 MB L2, else the HBM line",
                   "orders": args.batch_order,
                   "host_planning_s": t_plan, "steps": args.steps, "warmup": args.warmup,
               }, emit=emit)


def run_form_grad(args, emit=True):
    """Gradient of -mean log2 Pr over 2048 exact targets w.r.t. the 48 x 3 rotation angles (adjoint sweep)."""
    import math
    import numpy as np
    import torch
    import adjoint
    import gsb
    import workloads
    w = workloads.rotation_instance(48, 48, seed=7, order_seed=12, iters=20000)
    w2 = workloads.matching_instance(48, 48, 8, 12, 20000)
    with gsb.Engine.from_text(w2["plan"], precision=gsb.GSB_C128) as eng2:
        tb, _ = eng2.sample(2048, seed=99)
    v2 = [s["v"] for s in w2["steps"]]
    q = np.zeros((len(tb), 48), np.int8)
    q[:, v2] = tb                                       # targets by qubit
    bits = np.ascontiguousarray(q[:, w["step_vertices"]])   # in this instance's step order
    theta = torch.tensor(np.random.default_rng(5).uniform(0, 2 * math.pi, (48, 3)), requires_grad=True)
    sweep = gsb.GradSweep(w["plan"], every=4)
    times = []
    for i in range(max(3, args.warmup) + args.steps):
        theta.grad = None
        t0 = time.perf_counter()
        loss = -adjoint.log2_prob(theta, w["M0"], w["step_vertices"], bits, sweep).mean()
        loss.backward()
        if i >= max(3, args.warmup):
            times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    # algorithmic bytes of the sweep (complex128): per string, every step's forward pass twice (the sweep and the
    # recompute of its checkpoint segment: read 2^r, write 2^r') and its reverse pass (read the step's input table and
    # lambda_{k+1}, write lambda_k: 2^r + 2^r' + 2^r); the time is the whole loss + gradient, host work included
    fwd = sum((1 << s["r"]) + (1 << s["rn"]) for s in w["steps"])
    bwd = sum(2 * (1 << s["r"]) + (1 << s["rn"]) for s in w["steps"])
    byt = 16.0 * len(bits) * (2 * fwd + bwd)
    peak, kind = peaks()
    sweep.close()
    return _form_line("grad", "s per loss+gradient, n=48 rotation layer, 2048 exact targets", t, "s", False, {
        "roofline": {"bound": "hbm", "achieved": byt / t / 1e9, "peak": peak, "unit": "GB/s", "frac": byt / t / 1e9 / peak,
                     "peak_kind": kind, "bytes_per_string": byt / len(bits)},
        "strings_per_s": len(bits) / t, "loss": loss.item(), "grad_norm": float(theta.grad.norm()),
        "step_times_s": [round(x, 4) for x in times],
        "width": w["width"], "checkpoint_every": 4, "dtype": "c128 arena, f64",
        "targets": "2048 exact samples of a second seeded n=48 instance (complex128 executor)",
        "steps": args.steps, "warmup": max(3, args.warmup)}, emit=emit)


def run_form_wide34(args, emit=True):
    """n = 80, width 34 in complex64: 256 amplitudes and 16 exact samples on one GPU (fewer with --wide34-amps /
    --wide34-samples), and 4 amplitudes against complex128 through a width-30 sliced order (--no-wide34-check: none)."""
    import numpy as np
    import torch
    import gsb
    import workloads
    t0 = time.perf_counter()
    w = workloads.wide34_instance()
    t_plan = time.perf_counter() - t0
    ns = len(w["steps"])
    NA, NS = args.wide34_amps, args.wide34_samples
    strings = workloads.random_strings(ns, 256, seed=2024)[:NA]
    with gsb.Engine.from_text(w["plan"], precision=gsb.GSB_C64) as eng:
        stream = torch.cuda.Stream()
        eng.set_stream(stream.cuda_stream)
        eng.chain(strings[:1])
        t1 = time.perf_counter()
        lp, _ = eng.chain(strings)
        t_amp = time.perf_counter() - t1
        t2 = time.perf_counter()
        sbits, slp = eng.sample(NS, seed=7)
        t_smp = time.perf_counter() - t2
        chain_bytes = 8.0 * float(eng.fusion_groups()[1].sum())     # bytes the executed passes move per string
        sample_bytes = 8.0 * float(eng.sample_groups()[1].sum())
    check_line = {"skipped": "--no-wide34-check"}
    if args.wide34_check:
        check_line = wide34_sliced_check(w, strings[:4], lp[:4])
    return _form_line("wide34", "amps/s and s/sample at n=80, width 34, complex64 (137 GB arena)", NA / t_amp, "amps/s",
                      True, {
        "s_per_sample": t_smp / NS, "amplitudes": NA, "samples": NS, "width": w["width"],
        "arena_gb": (1 << w["width"]) * 8 / 1e9,
        "log2p_first": [float(x) for x in lp[:4]], "sample_log2p": [float(x) for x in slp[:4]],
        "dtype": "c64 arena, f32 sums, f64 norms/scales", "host_planning_s": t_plan,
        "timing": "wall clock around the host-buffer C-ABI calls (whole batches, one synchronisation each)",
        "roofline": {"bound": "hbm", "achieved": NA * chain_bytes / t_amp / 1e9, "peak": peaks()[0], "unit": "GB/s",
                     "frac": NA * chain_bytes / t_amp / 1e9 / peaks()[0], "peak_kind": peaks()[1],
                     "pass_bytes_per_string": chain_bytes, "sample_pass_bytes": sample_bytes,
                     "sample_achieved": NS * sample_bytes / t_smp / 1e9,
                     "note": "wall clock (host calls included), so a lower bound on the kernels' rate"},
        "c128_sliced_check": check_line}, emit=emit)


def wide34_sliced_check(w, strings, lp):
    """complex128 cross-check of 4 amplitudes of the width-34 instance: a second order with 10 slice vertices cut out
    (width 30), every slice's final table from 'prefix' through the last step, summed by 'resume' (the reference's
    slicing identity, gsamp2.cpp:176-208); one complex128 arena serves all 1,024 slice plans (they differ only in M)"""
    import numpy as np
    import gsb
    import workloads
    t3 = time.perf_counter()
    sl = workloads.wide34_slices(w)
    v1 = [s["v"] for s in w["steps"]]
    lines = []
    for i in range(4):
        q = np.zeros(w["n"], np.int8)
        q[v1] = strings[i]
        lines.append(q[sl["step_vertices"]])
    dumps = [[] for _ in lines]
    lss = [[] for _ in lines]
    check = []
    with gsb.Engine.from_text(sl["plans"][0], precision=gsb.GSB_C128) as e128:
        ns2 = e128.ns
        for text in sl["plans"]:
            e128.set_matrices_from_text(text)
            for i, line in enumerate(lines):
                d, ls, _ = e128.prefix(line, ns2)
                dumps[i].append(d)
                lss[i].append(ls)
        e128.set_matrices_from_text(sl["plans"][0])
        for i, line in enumerate(lines):
            _, lpf, _, _ = e128.resume(line, ns2, 0, 0, dumps[i], lss[i])
            check.append((float(lp[i]), float(lpf)))
    t_check = time.perf_counter() - t3
    return {"slices": len(sl["plans"]), "slice_vertices": sl["S"], "width": sl["width"],
            "arena_gb": (1 << sl["width"]) * 16 / 1e9, "log2p_c64_vs_c128": check,
            "max_abs_dlog2p": max(abs(a - b) for a, b in check), "seconds": t_check}


def run_form_hybrid(args, emit=True):
    """Hybrid rejection sampling of the headline instance in process (hybrid_sampler, the reference's doped_sampler
    driver with the executor kept loaded): proposals draw the first 70 - m step bits uniformly and sample the last
    m = 16 exactly.  Seconds per proposal as the driver runs them (forced prefix in fused passes, 64 proposals per
    gsb_hybrid call), with one call per proposal, and with every step a single-step pass (no declared prefix: the
    structure of the reference's executor, without its process start-up)."""
    import gsb
    import hybrid_sampler
    import workloads
    w = workloads.matching_n70_w30()
    with tempfile.TemporaryDirectory() as td:
        plan = os.path.join(td, "plan.txt")
        open(plan, "w").write(w["plan"])
        sv = os.path.join(td, "sv.json")
        json.dump([s["v"] for s in w["steps"]], open(sv, "w"))
        hs = hybrid_sampler.HybridSampler(plan, sv, na=0, nd=70, m=16, precision=64)
        res = {}
        K = hs.ns - hs.m_suffix
        for name, batch, prefix in (("batched", 64, K), ("one_call_per_proposal", 1, K), ("unfused_steps", 64, 0)):
            hs.BATCH = batch
            hs.eng.set_hybrid_prefix(prefix)
            hs.sample(2, 3, 2.0, os.path.join(td, f"warm_{name}.txt"))
            gsb.Engine.synchronize(hs.eng)
            t0 = time.perf_counter()
            acc, zmax = hs.sample(args.proposals, 7, 2.0, os.path.join(td, f"{name}.txt"))
            gsb.Engine.synchronize(hs.eng)
            res[name] = (time.perf_counter() - t0) / args.proposals
        same = open(os.path.join(td, "batched.txt")).read().split("\n")
        one = open(os.path.join(td, "one_call_per_proposal.txt")).read().split("\n")
        unf = open(os.path.join(td, "unfused_steps.txt")).read().split("\n")
        import re

        def strip(ls):   # the lines without their wall-time fields
            return [" ".join(t for t in ln.split() if not re.fullmatch(r"[0-9.]+s", t)) for ln in ls]
        hs.close()
    return _form_line("hybrid", "s/proposal (hybrid rejection sampling, n=70 w=30, m=16, complex64)", res["batched"],
               "s/proposal", False,
               {"config": {"workload": WORKLOAD, "proposals": args.proposals, "m_suffix": 16, "cap": 2.0},
                "one_call_per_proposal_s": res["one_call_per_proposal"],
                "unfused_steps_s": res["unfused_steps"],
                "speedup_over_unfused": res["unfused_steps"] / res["batched"],
                "same_lines_all_three": strip(same) == strip(one),
                "same_decisions_unfused": [ln.split()[:2] for ln in strip(same) if ln and not ln.startswith("#")] ==
                                          [ln.split()[:2] for ln in strip(unf) if ln and not ln.startswith("#")],
                "accepted": acc, "max_z": zmax}, emit=emit)


if __name__ == "__main__":
    a = parse()
    if a.form == "hybrid":
        run_form_hybrid(a)
        raise SystemExit(0)
    if a.form == "batch":
        run_form_batch(a)
    elif a.form == "grad":
        run_form_grad(a)
    elif a.form == "wide34":
        run_form_wide34(a)
    elif a.profile_chain:
        profile_chain(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_gsb(a)
