"""Python access to the CPU oracle of the in-place cut-rank DP executor.

TEST INFRASTRUCTURE ONLY.  Only tests, the smoke check and the benchmark's CPU-baseline leg use this module, and only
as the checker / the reported CPU baseline; the product never imports it.

* ``Oracle``: ctypes binding of liboracle.so, the plain-C restatement of the reference executor (gsamp_oracle.c).
* ``ref_binary`` / ``run_ref``: the reference's own gsamp2 compiled from its sources into oracle/_ref (see the
  Makefile), when that build exists.
* ``build()``: runs the Makefile (the oracle always; the reference binaries when the reference checkout is present).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


# the reference checkout: $GSB_REFERENCE_DIR, else the sibling directory "reference" of this repository's checkout
REF_SRC = os.environ.get("GSB_REFERENCE_DIR",
                         os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
_AVX512 = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def build(with_ref=None):
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if with_ref is None:
        with_ref = os.path.exists(os.path.join(REF_SRC, "gsamp2.cpp"))
    if with_ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={os.path.abspath(REF_SRC)}"], check=True)


def host_has_avx512():
    """True when this host's CPU has the x86-64-v4 extensions (AVX-512 F, BW, CD, DQ, VL)."""
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("flags"):
                fl = set(ln.split(":", 1)[1].split())
                return all(f in fl for f in _AVX512)
    except OSError:
        pass
    return False


def ref_binary(precision=64, isa=None):
    """Path of the compiled reference executor (None when not built).  isa: "v4" (AVX-512), "v3" (AVX2), or None
    for the best level this host runs."""
    base = "gsamp2_c128" if precision == 128 else "gsamp2"
    if isa is None:
        isa = "v4" if host_has_avx512() and os.path.exists(os.path.join(REF_DIR, base + "_v4")) else "v3"
    p = os.path.join(REF_DIR, base + ("_v4" if isa == "v4" else ""))
    return p if os.path.exists(p) else None


def ref_isa(precision=64):
    """The instruction-set level ref_binary(precision) picks on this host ("v4" or "v3")."""
    p = ref_binary(precision)
    return "v4" if p and p.endswith("_v4") else "v3"


def ref_gpu_binary():
    """Path of the reference's own GPU port (gsamp_cuda.cu built for sm_100a), or None."""
    p = os.path.join(REF_DIR, "gsamp_cuda")
    return p if os.path.exists(p) else None


def run_ref(precision, args, threads=None, cwd=None, timeout=None):
    """stdout of the compiled reference executor: gsamp2 <args...>."""
    exe = ref_binary(precision)
    if exe is None:
        raise FileNotFoundError("reference executor not built (oracle/_ref)")
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    out = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, env=env, cwd=cwd,
                         timeout=timeout)
    if out.returncode:
        raise RuntimeError(f"gsamp2 exit {out.returncode}: {out.stderr[-500:]}")
    return out.stdout


_lib = None


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build(with_ref=False)
    lib = ctypes.CDLL(LIB_PATH)
    c = ctypes
    P = c.c_void_p
    ip, dp, u64p = c.POINTER(c.c_int), c.POINTER(c.c_double), c.POINTER(c.c_uint64)
    sig = {
        "orc_load": (P, [c.c_char_p, c.c_int]),
        "orc_free": (None, [P]),
        "orc_last_error": (c.c_char_p, []),
        "orc_n": (c.c_int, [P]), "orc_ns": (c.c_int, [P]), "orc_R": (c.c_int, [P]),
        "orc_prob": (c.c_double, [P, ip]),
        "orc_sample": (c.c_double, [P, c.c_int, c.c_uint64, c.c_uint64, ip]),
        "orc_chain1": (c.c_double, [P, ip, dp]),
        "orc_hybrid": (c.c_double, [P, ip, c.c_uint64, c.c_uint64, ip, dp]),
        "orc_coset_offsets": (c.c_int, [P, c.c_int, u64p]),
        "orc_dump_nk": (c.c_int, [P, c.c_int]),
        "orc_prefix": (c.c_double, [P, ip, c.c_int, dp, dp]),
        "orc_resume": (c.c_int, [P, ip, c.c_int, c.c_uint64, c.c_uint64, c.c_int, c.POINTER(dp), dp, u64p, u64p,
                                 ip, dp, dp, dp]),
        "orc_uniforms": (None, [c.c_int, c.c_uint64, c.c_uint64, c.c_int, dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def uniforms(mode, seed, i, count):
    """First `count` uniforms of the stream 'sample' (mode 0: mt19937_64(seed+i)) or 'sample2' (mode 1)."""
    lib = _load()
    out = np.zeros(count, np.float64)
    lib.orc_uniforms(int(mode), int(seed), int(i), int(count), _dp(out))
    return out


class Oracle:
    """The C restatement of the reference executor on one plan file; precision 64 or 128 (arena element type)."""

    def __init__(self, plan_path, precision=128):
        lib = _load()
        self._lib = lib
        self._h = lib.orc_load(os.fsencode(plan_path), int(precision))
        if not self._h:
            raise ValueError(lib.orc_last_error().decode())
        self.n, self.ns, self.R = lib.orc_n(self._h), lib.orc_ns(self._h), lib.orc_R(self._h)

    def close(self):
        if self._h:
            self._lib.orc_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _bits(self, b):
        a = np.ascontiguousarray([(-1 if ch == "?" else int(ch)) for ch in b] if isinstance(b, str) else b, np.int32)
        assert a.shape == (self.ns,)
        return a

    def prob(self, bits):
        return self._lib.orc_prob(self._h, _ip(self._bits(bits)))

    def chain1(self, bits):
        cond = np.zeros(max(self.ns, 1), np.float64)
        lp = self._lib.orc_chain1(self._h, _ip(self._bits(bits)), _dp(cond))
        return lp, cond[:self.ns]

    def sample(self, mode, seed, i):
        bits = np.zeros(max(self.ns, 1), np.int32)
        lp = self._lib.orc_sample(self._h, int(mode), int(seed), int(i), _ip(bits))
        return bits[:self.ns], lp

    def hybrid(self, forced, seed, line):
        bits = np.zeros(max(self.ns, 1), np.int32)
        cond = np.zeros(max(self.ns, 1), np.float64)
        lp = self._lib.orc_hybrid(self._h, _ip(self._bits(forced)), int(seed), int(line), _ip(bits), _dp(cond))
        return bits[:self.ns], lp, cond[:self.ns]

    def dump_shape(self, K):
        tq = np.zeros(16, np.uint64)
        ntq = self._lib.orc_coset_offsets(self._h, int(K), tq.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
        return self._lib.orc_dump_nk(self._h, int(K)), ntq

    def prefix(self, forced, K):
        nk, ntq = self.dump_shape(K)
        d = np.zeros(2 * (1 << nk) * ntq, np.float64)
        ls = ctypes.c_double()
        lp = self._lib.orc_prefix(self._h, _ip(self._bits(forced)), int(K), _dp(d), ctypes.byref(ls))
        return d[0::2] + 1j * d[1::2], ls.value, lp

    def resume(self, forced, K, seed, line, dumps, logscales, twist=None):
        tabs = []
        for t in dumps:
            t = np.asarray(t, np.complex128)
            x = np.empty(2 * len(t), np.float64)
            x[0::2], x[1::2] = t.real, t.imag
            tabs.append(x)
        arr = (ctypes.POINTER(ctypes.c_double) * len(tabs))(*[_dp(t) for t in tabs])
        ls = np.ascontiguousarray(logscales, np.float64)
        u64 = ctypes.POINTER(ctypes.c_uint64)
        cs = tq = None
        if twist is not None:
            cs = np.ascontiguousarray([t[0] for t in twist], np.uint64)
            tq = np.ascontiguousarray([t[1] for t in twist], np.uint64)
        bits = np.zeros(max(self.ns, 1), np.int32)
        cond = np.zeros(max(self.ns, 1), np.float64)
        lpf, lpp = ctypes.c_double(), ctypes.c_double()
        rc = self._lib.orc_resume(self._h, _ip(self._bits(forced)), int(K), int(seed), int(line), len(tabs), arr,
                                  _dp(ls), None if cs is None else cs.ctypes.data_as(u64),
                                  None if tq is None else tq.ctypes.data_as(u64), _ip(bits), _dp(cond),
                                  ctypes.byref(lpf), ctypes.byref(lpp))
        if rc:
            raise ValueError(f"resume failed with reference exit code {rc}")
        return bits[:self.ns], lpf.value, lpp.value, cond[:self.ns]
