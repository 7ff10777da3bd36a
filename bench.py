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
    ap.add_argument("--c128-amps", type=int, default=8)
    ap.add_argument("--c128-samples", type=int, default=4)
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
    ap.add_argument("--form", default="headline", choices=["headline", "batch", "grad", "wide34"],
                    help="workload to measure (the default line is the headline n = 70, width-30 workload)")
    ap.add_argument("--batch-instances", type=int, default=512)
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
    # guarded autotuner of the pass lists (kept only where a whole item gets faster), outside every timed region
    tune64 = eng.autotune(mode=2, reps=3) if args.autotune else None
    stream = torch.cuda.Stream()                  # a real stream: the engine's kernels and the events share it
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
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
    with Clocks(local) as clk:
        ev0.record(stream)
        for i in range(W, W + K):
            amp_step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
    replicas.barrier(world)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms_max = replicas.max_over_ranks(ms, world)
    value = world * K * A / (ms_max / 1000.0)
    lp64 = d_lp.cpu().numpy()
    cond64 = d_cond.cpu().numpy()

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

    # exact samples (two passes per DP step), device-resident uniforms
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

    # roofline of the dominant kernels (the chain-mode passes: fused groups k_group and single steps), timed per
    # pass with CUDA events; bytes = the table entries each executed pass must read and write (fused groups keep
    # their intermediate tables in shared memory, so they move fewer bytes than the unfused step model)
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
    achieved = pass_bytes / (kernel_ms / 1000.0) / 1e9
    fused = [k for k in range(ns) if glen[k] >= 2]
    fused_bytes = float(sum(gent[k] for k in fused)) * 8
    fused_ms = float(sum(wmean[k] for k in fused))
    # DRAM bytes per algorithmic byte of the dominant pass, from one ncu capture of k_group<float2, float, 2, 0> on the
    # width-27 instance (2.0880 GB read + written for 2.1475 GB algorithmic: no re-reads; writes still dirty in L2
    # at kernel end make it < 1), scaled to the chain passes of one string
    traffic = pass_bytes * K_GROUP_TRAFFIC_RATIO
    # exact-sample passes (a norm pass where a pass has no other source for its first bit, then the pass)
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
                "pass_bytes_per_string": pass_bytes, "kernel_ms_per_string": kernel_ms,
                "fused_passes_frac": (fused_bytes / (fused_ms / 1000.0) / 1e9) / hbm_peak if fused_ms > 0 else None,
                "unfused_model_bytes_per_string": float(sum(p[0] for p in per)),
                "unfused_model_GBps": float(sum(p[0] for p in per)) / (kernel_ms / 1000.0) / 1e9,
                "passes_per_string": int(sum(1 for x in glen if x > 0)), "fusion": args.fusion,
                "sample_kernel_ms": sample_kernel_ms, "sample_norm_ms": float(sn.sum()),
                "sample_write_ms": float(sw.sum()), "sample_unfused_model_bytes": sample_bytes,
                "sample_pass_bytes": sample_pass_bytes,
                "sample_achieved": sample_pass_bytes / (sample_kernel_ms / 1000.0) / 1e9,
                "sample_frac": sample_pass_bytes / (sample_kernel_ms / 1000.0) / 1e9 / hbm_peak}
    eng.close()

    # complex128 plain form on the first strings of the timed batch, and the c64-vs-c128 agreement
    c128 = {}
    if args.c128_amps > 0:
        e128 = gsb.Engine.from_text(w["plan"], precision=128, device=local)
        e128.set_fusion(args.fusion)
        tune128 = e128.autotune(mode=2, reps=3) if args.autotune else None
        e128.set_stream(stream.cuda_stream)
        B = args.c128_amps
        d_lp128 = torch.empty(B, dtype=torch.float64, device="cuda")
        d_cond128 = torch.empty((B, ns), dtype=torch.float64, device="cuda")
        sl = slice(W * A, W * A + B)
        e128.chain_device(d_bits[:1], d_lp128[:1], d_cond128[:1])
        torch.cuda.synchronize()
        e0.record(stream)
        e128.chain_device(d_bits[sl], d_lp128, d_cond128)
        e1.record(stream)
        torch.cuda.synchronize()
        amps128 = B / (e0.elapsed_time(e1) / 1000.0)
        lp128 = d_lp128.cpu().numpy()
        dlp = float(np.abs(lp128 - lp64[sl]).max())
        dcond = float(np.abs(d_cond128.cpu().numpy() - cond64[sl]).max())
        S2 = args.c128_samples

        def time_samples128():
            e128.sample_device(d_u[:1], d_sb[:1], d_slp[:1])      # graph built outside the timed region
            torch.cuda.synchronize()
            e0.record(stream)
            e128.sample_device(d_u[:S2], d_sb[:S2], d_slp[:S2])
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / 1000.0 / S2

        s_per_sample128 = time_samples128()
        same_bits = bool((d_sb[:S2].cpu().numpy() == sbits64[:S2]).all())
        # the same complex128 form without fusion: one norm pass and one write pass per DP step, the structure of
        # the reference executor's two-pass sampler (gsamp2.cpp:39-55)
        e128.set_fusion(1)
        s_per_sample128_unfused = time_samples128()
        e128.close()
        c128 = {"amps_per_s": amps128, "autotune_ms_item_before_after": tune128,
                "s_per_sample": s_per_sample128, "s_per_sample_unfused_two_pass": s_per_sample128_unfused,
                "max_abs_dlog2p_c64_vs_c128": dlp,
                "max_abs_dcond_c64_vs_c128": dcond, "samples_same_bits_c64_c128": same_bits}

    # per string: begin + one launch per chain pass + finish; one item reset per batch
    launches = (roofline["passes_per_string"] + 2) * K * A + K
    out = {
        "metric": METRIC, "value": value, "unit": "amps/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": f"c64 arena, f{args.arith} arithmetic", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": 70, "width": w["width"], "strings_per_step": A, "mode": "chain",
                   "arith": args.arith, "fusion": args.fusion, "parallelism": f"replicas{world}", "l2": "inputs larger than L2: arena 8.6 GB >> 126 MB"},
        "s_per_sample": s_per_sample64, "samples_per_s": world / s_per_sample64,
        "c128": c128, "e2e": e2e, "roofline": roofline, "gpu_launches": launches,
        "autotune_ms_item_before_after": tune64,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as td:
            plan = os.path.join(td, "plan.txt")
            open(plan, "w").write(w["plan"])
            sp = os.path.join(td, "s.txt")
            open(sp, "w").write("".join(str(int(b)) for b in strings[W * A]) + "\n")
            cores = os.cpu_count() or 1
            t, txt, kind = ref_time(plan, ["chain", sp], cores)
            ref_lp = float(txt.split()[0])
            out["cpu_baseline"] = {"value": 1.0 / t, "unit": "amps/s", "cores": cores, "kind": kind,
                                   "sample": "1 uniform random string of the workload, gsamp2 chain mode (complex64)",
                                   "abs_dlog2p_vs_gpu_c64": abs(ref_lp - float(lp64[W * A]))}
    if rank == 0:
        print(json.dumps(out), flush=True)
    replicas.finish(world)


def _form_line(form, metric, value, unit, hib, extra):
    d = {"form": form, "metric": metric, "value": value, "unit": unit, "n_gpus": 1, "higher_is_better": hib,
         "data": "synthetic"}
    d.update(extra)
    print(json.dumps(d), flush=True)


def run_form_batch(args):
    """Batched uneven workload: one persistent launch over all (instance, prefix) items."""
    import numpy as np
    import gsb
    import workloads
    t0 = time.perf_counter()
    bw = workloads.batch_workload(count=args.batch_instances, seed=0, npre=16, nsuf=4)
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
    _form_line("batch", "amps/s, 512 instances n in [16,40] x 64 strings, one persistent launch", nstr / (ms / 1e3),
               "amps/s", True, {
                   "ms_per_launch": ms, "strings": int(nstr), "instances": len(plans),
                   "widths": {"min": int(min(widths)), "max": int(max(widths)), "mean": float(np.mean(widths))},
                   "dtype": "c64 arena, f32 sums, f64 norms/scales", "shape": {"block": block, "small_R": small_R,
                                                                                 "ctas_per_sm": per_sm},
                   "c128": {"ms_per_launch": ms128, "max_abs_dlog2p_c64_vs_c128": float(d.max()),
                            "median_abs_dlog2p": float(np.median(d))},
                   "roofline": {"bound": "hbm", "achieved": byt / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                "frac": byt / (ms / 1e3) / 1e9 / peak, "peak_kind": kind,
                                "note": "team tables <= 2^20 entries: many items are L2-resident"},
                   "roofline_l2": {"bound": "l2", "achieved": byt / (ms / 1e3) / 1e9, "peak": l2, "unit": "GB/s",
                                   "frac": byt / (ms / 1e3) / 1e9 / l2,
                                   "peak_kind": "measured here: L2 copy bandwidth (gsb_probe_l2_copy, best of "
                                                "16/24/32 MiB buffers, one launch of 400 passes)"},
                   "host_planning_s": t_plan, "steps": args.steps, "warmup": args.warmup,
               })


def run_form_grad(args):
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
    _form_line("grad", "s per loss+gradient, n=48 rotation layer, 2048 exact targets", t, "s", False, {
        "roofline": {"bound": "hbm", "achieved": byt / t / 1e9, "peak": peak, "unit": "GB/s", "frac": byt / t / 1e9 / peak,
                     "peak_kind": kind, "bytes_per_string": byt / len(bits)},
        "strings_per_s": len(bits) / t, "loss": loss.item(), "grad_norm": float(theta.grad.norm()),
        "step_times_s": [round(x, 4) for x in times],
        "width": w["width"], "checkpoint_every": 4, "dtype": "c128 arena, f64",
        "targets": "2048 exact samples of a second seeded n=48 instance (complex128 executor)",
        "steps": args.steps, "warmup": max(3, args.warmup)})


def run_form_wide34(args):
    """n = 80, width 34 in complex64: 256 amplitudes and 16 exact samples on one GPU."""
    import numpy as np
    import torch
    import gsb
    import workloads
    t0 = time.perf_counter()
    w = workloads.wide34_instance()
    t_plan = time.perf_counter() - t0
    ns = len(w["steps"])
    strings = workloads.random_strings(ns, 256, seed=2024)
    with gsb.Engine.from_text(w["plan"], precision=gsb.GSB_C64) as eng:
        stream = torch.cuda.Stream()
        eng.set_stream(stream.cuda_stream)
        eng.chain(strings[:1])
        t1 = time.perf_counter()
        lp, _ = eng.chain(strings)
        t_amp = time.perf_counter() - t1
        t2 = time.perf_counter()
        sbits, slp = eng.sample(16, seed=7)
        t_smp = time.perf_counter() - t2
        chain_bytes = 8.0 * float(eng.fusion_groups()[1].sum())     # bytes the executed passes move per string
        sample_bytes = 8.0 * float(eng.sample_groups()[1].sum())
    # complex128 cross-check of 4 amplitudes: a second order with 3 slice vertices cut out (width 33), every slice's
    # final table from 'prefix', summed by 'resume' (the reference's slicing identity)
    t3 = time.perf_counter()
    sl = workloads.wide34_slices(w)
    v1 = [s["v"] for s in w["steps"]]
    check = []
    with gsb.Engine.from_text(sl["plans"][0], precision=gsb.GSB_C128) as e128:
        ns2 = e128.ns
        for i in range(4):
            q = np.zeros(w["n"], np.int8)
            q[v1] = strings[i]
            line = q[sl["step_vertices"]]
            dumps, lss = [], []
            for text in sl["plans"]:
                e128.set_matrices_from_text(text)
                d, ls, _ = e128.prefix(line, ns2)
                dumps.append(d)
                lss.append(ls)
            _, lpf, _, _ = e128.resume(line, ns2, 0, 0, dumps, lss)
            check.append((float(lp[i]), float(lpf)))
    t_check = time.perf_counter() - t3
    _form_line("wide34", "amps/s and s/sample at n=80, width 34, complex64 (137 GB arena)", 256 / t_amp, "amps/s", True, {
        "s_per_sample": t_smp / 16, "width": w["width"], "arena_gb": (1 << w["width"]) * 8 / 1e9,
        "log2p_first": [float(x) for x in lp[:4]], "sample_log2p": [float(x) for x in slp[:4]],
        "dtype": "c64 arena, f32 sums, f64 norms/scales", "host_planning_s": t_plan,
        "timing": "wall clock around the host-buffer C-ABI calls (whole batches, one synchronisation each)",
        "roofline": {"bound": "hbm", "achieved": 256 * chain_bytes / t_amp / 1e9, "peak": peaks()[0], "unit": "GB/s",
                     "frac": 256 * chain_bytes / t_amp / 1e9 / peaks()[0], "peak_kind": peaks()[1],
                     "pass_bytes_per_string": chain_bytes, "sample_pass_bytes": sample_bytes,
                     "sample_achieved": 16 * sample_bytes / t_smp / 1e9,
                     "note": "wall clock (host calls included), so a lower bound on the kernels' rate"},
        "c128_sliced_check": {"slices": len(sl["plans"]), "slice_vertices": sl["S"], "width": sl["width"],
                              "arena_gb": (1 << sl["width"]) * 16 / 1e9,
                              "log2p_c64_vs_c128": check,
                              "max_abs_dlog2p": max(abs(a - b) for a, b in check), "seconds": t_check}})


if __name__ == "__main__":
    a = parse()
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
