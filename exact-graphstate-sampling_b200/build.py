"""Build the executor in-tree: libgsb.so (CUDA, sm_100a) and the gsb2 / gsb2_c128 command lines.

    python build.py [--force]

nvcc cross-compiles for sm_100a without a GPU, so this runs on any machine with the CUDA toolkit.  Outputs sit next
to this file, where gsb.py loads them.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libgsb.so")
CLI = os.path.join(HERE, "gsb2")
CLI128 = os.path.join(HERE, "gsb2_c128")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
# the complex64 FP32 fused passes sit in translation units of their own (gsb_group_*.cu): the largest objects, compiled
# in parallel with the rest
LIB_SOURCES = ["gsb_engine.cu", "gsb_group_ws.cu", "gsb_group_wst.cu", "gsb_group_f32.cu", "gsb_group3.cu",
               "gsb_dp.cu", "gsb_grad.cu", "gsb_batch.cu", "gsb_probe.cu", "gsb_plan.cpp", "gsb_order.cpp", "gsb_fuse.cpp"]
LIB_DEPS = LIB_SOURCES + ["gsb_kernels.cuh", "gsb_group.cuh", "gsb_step.h", "gsb_plan.h", "gsb_common.h", "gsb_fuse.h",
                          "gsb_pick.h"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose_ptxas=False):
    deps = [os.path.join(CSRC, f) for f in LIB_DEPS] + [os.path.join(INCLUDE, "gsb.h")]
    if force or _stale(LIB, deps):
        # one object per source, compiled in parallel (the sources share no device code), then one link
        objdir = os.path.join(ROOT, "_build", "gsb")
        os.makedirs(objdir, exist_ok=True)
        cmds, objs = [], []
        for f in LIB_SOURCES:
            obj = os.path.join(objdir, f + ".o")
            objs.append(obj)
            cmds.append([_nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) +
                        ["-c", "-I" + INCLUDE, "-I" + CSRC, "-o", obj, os.path.join(CSRC, f)])
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
            list(ex.map(_run, cmds))
        _run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + objs)
    cli_src = os.path.join(CSRC, "gsb_cli.cpp")
    if force or _stale(CLI, [cli_src, LIB, os.path.join(INCLUDE, "gsb.h")]):
        _run(["g++", "-O2", "-std=c++17", "-Wall", "-I" + INCLUDE, cli_src, "-L" + HERE, "-lgsb",
              "-Wl,-rpath,$ORIGIN", "-o", CLI])
    if not os.path.lexists(CLI128):
        os.symlink("gsb2", CLI128)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
