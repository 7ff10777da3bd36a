"""Python binding (ctypes) of libgsb, the B200 executor of the in-place cut-rank DP (C ABI: include/gsb.h).

Each method is one mode of the reference's executor command line (gsamp2.cpp:149-225): ``prob``, ``chain``,
``sample`` (``sample`` / ``sample2`` seeding), ``hybrid``, ``prefix`` and ``resume``.  Strings are in STEP order
(element k is the bit of the vertex processed at step k), given as str ('0', '1', '?') or int arrays (0, 1, -1).

The library must be built (``python build.py``); there is no fallback: importing this module without
libgsb.so, or opening an engine without a CUDA device, raises.
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgsb.so")

GSB_C64, GSB_C128 = 64, 128
SEED_INT, SEED_SEQ = 0, 1

ERROR_NAMES = {1: "usage", 2: "plan header", 3: "plan step", 4: "plan Tkeep", 5: "plan term", 6: "plan M",
               7: "plan range", 8: "'?' before K", 9: "dump missing", 10: "bad dump", 11: "allocation",
               12: "twist missing", 13: "twist line", 14: "twist range", 15: "plan layout", 20: "CUDA", 21: "state"}


class GsbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gsb error {code} ({ERROR_NAMES.get(code, '?')}): {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run build.py (the executor has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    c = ctypes
    P = c.c_void_p
    i8p, dp, u64p = c.POINTER(c.c_int8), c.POINTER(c.c_double), c.POINTER(c.c_uint64)
    sig = {
        "gsb_version": (c.c_char_p, []),
        "gsb_last_error": (c.c_char_p, []),
        "gsb_open_file": (c.c_int, [c.c_char_p, c.c_int, c.c_int, c.POINTER(P)]),
        "gsb_open_text": (c.c_int, [c.c_char_p, c.c_size_t, c.c_int, c.c_int, c.POINTER(P)]),
        "gsb_close": (c.c_int, [P]),
        "gsb_info": (c.c_int, [P, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_int)]),
        "gsb_step_vertices": (c.c_int, [P, c.POINTER(c.c_int)]),
        "gsb_prob": (c.c_int, [P, i8p, c.c_int64, dp]),
        "gsb_chain": (c.c_int, [P, i8p, c.c_int64, dp, dp]),
        "gsb_sample": (c.c_int, [P, c.c_int, c.c_uint64, c.c_int64, c.c_int64, i8p, dp]),
        "gsb_sample_uniform": (c.c_int, [P, dp, c.c_int64, i8p, dp]),
        "gsb_hybrid": (c.c_int, [P, i8p, c.c_int64, c.c_uint64, c.c_int64, i8p, dp, dp]),
        "gsb_dump_shape": (c.c_int, [P, c.c_int, c.POINTER(c.c_int), c.POINTER(c.c_int)]),
        "gsb_prefix": (c.c_int, [P, i8p, c.c_int, P, dp, dp]),
        "gsb_resume": (c.c_int, [P, i8p, c.c_int, c.c_uint64, c.c_int64, c.c_int, c.POINTER(P), dp, u64p, u64p,
                                 i8p, dp, dp, dp]),
        "gsb_chain_device": (c.c_int, [P, P, c.c_int64, P, P]),
        "gsb_sample_device": (c.c_int, [P, P, c.c_int64, P, P]),
        "gsb_synchronize": (c.c_int, [P]),
        "gsb_set_stream": (c.c_int, [P, P]),
        "gsb_set_arith": (c.c_int, [P, c.c_int]),
        "gsb_set_matrices": (c.c_int, [P, dp]),
        "gsb_set_fusion": (c.c_int, [P, c.c_int]),
        "gsb_fusion_groups": (c.c_int, [P, c.POINTER(c.c_int), dp]),
        "gsb_profile_steps": (c.c_int, [P, i8p, c.c_int, c.POINTER(c.c_float), c.POINTER(c.c_float)]),
        "gsb_launches_per_item": (c.c_int, [P, c.c_int, c.POINTER(c.c_int64)]),
        "gsb_dp_open_text": (c.c_int, [c.c_char_p, c.c_size_t, c.c_int, c.c_int, c.POINTER(P)]),
        "gsb_dp_close": (c.c_int, [P]),
        "gsb_dp_info": (c.c_int, [P, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_int)]),
        "gsb_dp_run": (c.c_int, [P, c.c_int64, dp, dp, dp]),
        "gsb_dp_extend": (c.c_int, [c.c_int, c.c_int, c.c_uint64, c.c_uint64, c.c_int, u64p, dp, dp, dp, c.c_int]),
        "gsb_dp_extend_static": (c.c_int, [c.c_int, c.c_int, c.c_uint64, c.c_uint64, c.c_int, u64p, dp, dp, dp,
                                           c.c_int]),
        "gsb_grad_open_text": (c.c_int, [c.c_char_p, c.c_size_t, c.c_int, c.c_int, c.POINTER(P)]),
        "gsb_grad_close": (c.c_int, [P]),
        "gsb_grad_info": (c.c_int, [P, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_int)]),
        "gsb_grad_run": (c.c_int, [P, dp, c.POINTER(c.c_int8), c.c_int64, dp, dp]),
        "gsb_sample_groups": (c.c_int, [P, c.POINTER(c.c_int), dp]),
        "gsb_probe_l2_copy": (c.c_int, [c.c_int, c.c_uint64, c.c_int, c.POINTER(c.c_float)]),
        "gsb_pass_list": (c.c_int, [P, c.c_int, c.c_int, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_int),
                                    c.POINTER(c.c_int), c.POINTER(c.c_int)]),
        "gsb_test_withhold_tile_loads": (c.c_int, [P, c.c_int]),
        "gsb_set_guard": (c.c_int, [P, P, c.c_double]),
        "gsb_set_hybrid_prefix": (c.c_int, [P, c.c_int]),
        "gsb_guard_evaluations": (c.c_int, [P, c.POINTER(c.c_int64)]),
        "gsb_autotune": (c.c_int, [P, c.c_int, c.c_int, c.POINTER(c.c_float), c.POINTER(c.c_float)]),
        "gsb_batch_open": (c.c_int, [c.POINTER(c.c_char_p), c.POINTER(c.c_size_t), c.c_int, c.c_int, c.c_int,
                                     c.POINTER(P)]),
        "gsb_batch_close": (c.c_int, [P]),
        "gsb_batch_set_strings": (c.c_int, [P, c.POINTER(c.c_int), c.c_int, c.c_int, i8p, i8p]),
        "gsb_batch_run": (c.c_int, [P, dp, c.POINTER(c.c_float)]),
        "gsb_batch_set_shape": (c.c_int, [P, c.c_int, c.c_int, c.c_int]),
        "gsb_batch_get_shape": (c.c_int, [P, c.POINTER(c.c_int), c.POINTER(c.c_int), c.POINTER(c.c_int)]),
        "gsb_batch_tune": (c.c_int, [P, c.c_int, c.c_size_t, c.POINTER(c.c_int), c.POINTER(c.c_int),
                                     c.POINTER(c.c_int), c.POINTER(c.c_float)]),
        "gsb_validate_text": (c.c_int, [c.c_char_p, c.c_size_t, c.POINTER(c.c_int), c.POINTER(c.c_int),
                                        c.POINTER(c.c_int)]),
        "gsb_cut_profile": (c.c_int, [c.c_int, c.POINTER(c.c_uint8), c.POINTER(c.c_int), c.POINTER(c.c_int)]),
        "gsb_order_search": (c.c_int, [c.c_int, c.POINTER(c.c_uint8), c.c_uint64, c.c_int, c.c_int64,
                                       c.POINTER(c.c_int), c.POINTER(c.c_int)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = _load()
EXPORTS = ("gsb_version", "gsb_last_error", "gsb_open_file", "gsb_open_text", "gsb_close", "gsb_info",
           "gsb_step_vertices", "gsb_prob", "gsb_chain", "gsb_sample", "gsb_sample_uniform", "gsb_hybrid",
           "gsb_dump_shape", "gsb_prefix", "gsb_resume", "gsb_chain_device", "gsb_sample_device",
           "gsb_synchronize", "gsb_set_stream", "gsb_set_arith", "gsb_set_matrices", "gsb_set_fusion", "gsb_fusion_groups", "gsb_sample_groups", "gsb_pass_list", "gsb_probe_l2_copy", "gsb_test_withhold_tile_loads", "gsb_set_guard", "gsb_guard_evaluations", "gsb_set_hybrid_prefix", "gsb_profile_steps", "gsb_launches_per_item", "gsb_validate_text",
           "gsb_cut_profile", "gsb_order_search", "gsb_dp_open_text", "gsb_dp_close", "gsb_dp_info", "gsb_dp_run",
           "gsb_dp_extend", "gsb_dp_extend_static", "gsb_grad_open_text", "gsb_grad_close", "gsb_grad_info",
           "gsb_grad_run", "gsb_autotune", "gsb_batch_open", "gsb_batch_close", "gsb_batch_set_strings", "gsb_batch_run",
           "gsb_batch_set_shape", "gsb_batch_get_shape", "gsb_batch_tune")


def lib():
    return _lib


def _check(rc):
    if rc:
        raise GsbError(rc, _lib.gsb_last_error().decode(errors="replace"))


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def as_bits(strings, ns, allow_free=False):
    """list of str / 2-D array -> contiguous int8 array [nstr][ns] with 0, 1 (and -1 for '?')."""
    if isinstance(strings, np.ndarray):
        a = np.ascontiguousarray(strings, dtype=np.int8)
        if a.ndim == 1:
            a = a[None, :]
    else:
        rows = []
        for s in strings:
            if isinstance(s, str):
                s = s.strip()
                rows.append([-1 if ch == "?" else int(ch) for ch in s])
            else:
                rows.append([int(x) for x in s])
        a = np.array(rows, dtype=np.int8).reshape(len(rows), -1) if rows else np.zeros((0, ns), np.int8)
    if a.shape[1] != ns:
        raise ValueError(f"strings must have {ns} step bits, got {a.shape[1]}")
    if not allow_free and (a < 0).any():
        raise ValueError("'?' is only allowed in hybrid / resume strings")
    return a


# Error model of the complex64 form (complex64 arena, FP32 arithmetic), measured against complex128 on 2,048
# uniform strings of the n = 70, width-30 workload: the log2 Pr error of a string is close to normal with mean 0
# and standard deviation
#     sigma(x) = C64_SIGMA_STEP * sqrt(nsteps) / sqrt(x),   x = Pr * 2^nsteps,
# since the rounding of the stored table is absolute in units of its norm and each step adds its own
# (measured: sigma * sqrt(x) = 5.5e-7 at nsteps = 70).
C64_SIGMA_STEP = 6.6e-8
C64_GUARD_Z = 5.5


def c64_sigma(log2p, nsteps):
    """Estimated standard deviation of a complex64 log2 Pr (the stated error of each result)."""
    x = np.exp2(np.asarray(log2p, np.float64) + nsteps)
    with np.errstate(divide="ignore"):
        return C64_SIGMA_STEP * math.sqrt(nsteps) / np.sqrt(x)


def c64_guard_log2_xmin(nsteps, tol=1e-5, z=C64_GUARD_Z):
    """log2 of the probability ratio x = Pr 2^nsteps below which z standard deviations of the complex64 error
    exceed tol: the threshold of Engine.set_guard for |d log2 Pr| <= tol."""
    return 2.0 * math.log2(z * C64_SIGMA_STEP * math.sqrt(nsteps) / tol)


class Engine:
    """One plan on one GPU at one precision (64 = complex64 arena, 128 = complex128 arena)."""

    def __init__(self, plan_path=None, precision=GSB_C64, device=0, text=None):
        h = ctypes.c_void_p()
        if text is None:
            with open(plan_path) as f:
                text = f.read()
        self.plan_text = text if isinstance(text, str) else bytes(text).decode()
        b = self.plan_text.encode()
        _check(_lib.gsb_open_text(b, len(b), int(precision), int(device), ctypes.byref(h)))
        self._h = h
        n, ns, R, p = (ctypes.c_int() for _ in range(4))
        _check(_lib.gsb_info(h, ctypes.byref(n), ctypes.byref(ns), ctypes.byref(R), ctypes.byref(p)))
        self.n, self.ns, self.R, self.precision = n.value, ns.value, R.value, p.value
        sv = np.zeros(max(self.ns, 1), np.int32)
        _check(_lib.gsb_step_vertices(h, _ptr(sv, ctypes.c_int)))
        self.step_vertices = [int(v) for v in sv[:self.ns]]
        self.entry_dtype = np.complex128 if self.precision == 128 else np.complex64

    @classmethod
    def from_text(cls, text, precision=GSB_C64, device=0):
        return cls(precision=precision, device=device, text=text)

    @property
    def handle(self):
        if self._h is None:
            raise GsbError(21, "engine is closed")
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.gsb_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- modes ---
    def prob(self, strings):
        """'prob': log2 Pr of each string (two passes per step)."""
        b = as_bits(strings, self.ns)
        out = np.zeros(len(b), np.float64)
        if len(b):
            _check(_lib.gsb_prob(self.handle, _ptr(b, ctypes.c_int8), len(b), _ptr(out, ctypes.c_double)))
        return out

    def chain(self, strings):
        """'chain': (log2 Pr [nstr], conditionals [nstr][ns]) with one pass per step."""
        b = as_bits(strings, self.ns)
        lp = np.zeros(len(b), np.float64)
        cond = np.zeros((len(b), max(self.ns, 1)), np.float64)
        if len(b):
            _check(_lib.gsb_chain(self.handle, _ptr(b, ctypes.c_int8), len(b), _ptr(lp, ctypes.c_double),
                                  _ptr(cond, ctypes.c_double)))
        return lp, cond[:, :self.ns]

    def sample(self, count, seed, first=0, seeding=SEED_INT):
        """'sample' (seeding=SEED_INT) / 'sample2' (SEED_SEQ): (bits [count][ns], log2 Pr [count])."""
        bits = np.zeros((count, max(self.ns, 1)), np.int8)
        lp = np.zeros(count, np.float64)
        if count:
            _check(_lib.gsb_sample(self.handle, int(seeding), int(seed), int(first), int(count),
                                   _ptr(bits, ctypes.c_int8), _ptr(lp, ctypes.c_double)))
        return bits[:, :self.ns], lp

    def sample_uniform(self, u):
        """Chain-rule samples from caller uniforms u [count][ns]: bit k = u[k] < Pr(b_k = 1 | prefix)."""
        u = np.ascontiguousarray(u, np.float64).reshape(-1, self.ns)
        bits = np.zeros((len(u), max(self.ns, 1)), np.int8)
        lp = np.zeros(len(u), np.float64)
        if len(u):
            _check(_lib.gsb_sample_uniform(self.handle, _ptr(u, ctypes.c_double), len(u), _ptr(bits, ctypes.c_int8),
                                           _ptr(lp, ctypes.c_double)))
        return bits[:, :self.ns], lp

    def hybrid(self, strings, seed, first_line=0):
        """'hybrid': '?' bits drawn from mt19937_64(seed + line); (bits, log2 Pr, conditionals)."""
        f = as_bits(strings, self.ns, allow_free=True)
        bits = np.zeros((len(f), max(self.ns, 1)), np.int8)
        lp = np.zeros(len(f), np.float64)
        cond = np.zeros((len(f), max(self.ns, 1)), np.float64)
        if len(f):
            _check(_lib.gsb_hybrid(self.handle, _ptr(f, ctypes.c_int8), len(f), int(seed), int(first_line),
                                   _ptr(bits, ctypes.c_int8), _ptr(lp, ctypes.c_double), _ptr(cond, ctypes.c_double)))
        return bits[:, :self.ns], lp, cond[:, :self.ns]

    def dump_shape(self, K):
        nk, ntq = ctypes.c_int(), ctypes.c_int()
        _check(_lib.gsb_dump_shape(self.handle, int(K), ctypes.byref(nk), ctypes.byref(ntq)))
        return nk.value, ntq.value

    def prefix(self, string, K, want_dump=True):
        """'prefix': (dump [2^nk * ntq] of the arena dtype in (c, tq) order, logscale, log2 Pr(prefix)).
        With want_dump=False only (None, logscale, log2 Pr of the first K steps) -- a marginal probability."""
        f = as_bits([string], self.ns, allow_free=True)[0].copy()
        dump = None
        if want_dump:
            nk, ntq = self.dump_shape(K)
            dump = np.zeros((1 << nk) * ntq, self.entry_dtype)
        ls, lp = ctypes.c_double(), ctypes.c_double()
        _check(_lib.gsb_prefix(self.handle, _ptr(f, ctypes.c_int8), int(K),
                               None if dump is None else dump.ctypes.data_as(ctypes.c_void_p),
                               ctypes.byref(ls), ctypes.byref(lp)))
        return dump, ls.value, lp.value

    def resume(self, string, K, seed, line, dumps, logscales, twist=None):
        """'resume': sum slice dumps, run steps K.. with '?' drawn; (bits, log2 Pr full, log2 Pr prefix, cond)."""
        f = as_bits([string], self.ns, allow_free=True)[0].copy()
        tabs = [np.ascontiguousarray(d, self.entry_dtype) for d in dumps]
        ptrs = (ctypes.c_void_p * len(tabs))(*[t.ctypes.data for t in tabs])
        ls = np.ascontiguousarray(logscales, np.float64)
        cs = tq = None
        if twist is not None:
            cs = np.ascontiguousarray([t[0] for t in twist], np.uint64)
            tq = np.ascontiguousarray([t[1] for t in twist], np.uint64)
        bits = np.zeros(max(self.ns, 1), np.int8)
        cond = np.zeros(max(self.ns, 1), np.float64)
        lpf, lpp = ctypes.c_double(), ctypes.c_double()
        _check(_lib.gsb_resume(self.handle, _ptr(f, ctypes.c_int8), int(K), int(seed), int(line), len(tabs), ptrs,
                               _ptr(ls, ctypes.c_double), None if cs is None else _ptr(cs, ctypes.c_uint64),
                               None if tq is None else _ptr(tq, ctypes.c_uint64), _ptr(bits, ctypes.c_int8),
                               ctypes.byref(lpf), ctypes.byref(lpp), _ptr(cond, ctypes.c_double)))
        return bits[:self.ns], lpf.value, lpp.value, cond[:self.ns]

    # --- device-resident batches (torch tensors on this engine's GPU) ---
    def chain_device(self, d_bits, d_log2p, d_cond=None):
        _check(_lib.gsb_chain_device(self.handle, d_bits.data_ptr(), d_bits.shape[0], d_log2p.data_ptr(),
                                     None if d_cond is None else d_cond.data_ptr()))

    def sample_device(self, d_u, d_bits, d_log2p):
        _check(_lib.gsb_sample_device(self.handle, d_u.data_ptr(), d_u.shape[0], d_bits.data_ptr(), d_log2p.data_ptr()))

    def set_stream(self, cuda_stream):
        """Queue work on a cudaStream_t (int handle, e.g. torch.cuda.current_stream().cuda_stream); 0 = own."""
        _check(_lib.gsb_set_stream(self.handle, ctypes.c_void_p(int(cuda_stream) or None)))

    def set_matrices_from_text(self, plan_text):
        """Load the M matrices of another plan with this plan's layout (a slice plan) into this engine."""
        rows = [ln.split() for ln in plan_text.strip().split("\n")]
        mine = [ln.split() for ln in self.plan_text.strip().split("\n")]
        if len(rows) != len(mine) or rows[0] != mine[0] or any(a[:-8] != b[:-8] for a, b in zip(rows[1:], mine[1:])):
            raise ValueError("the plan's layout differs from this engine's (only M may differ)")
        rows = rows[1:]
        M = np.array([[float(x) for x in r[-8:]] for r in rows], np.float64).reshape(-1)
        _check(_lib.gsb_set_matrices(self.handle, _ptr(np.ascontiguousarray(M), ctypes.c_double)))

    def set_matrices(self, M):
        """Replace every step's matrix: M [ns][2][2] complex, step order (same plan layout)."""
        Mc = np.ascontiguousarray(M, np.complex128).reshape(self.ns, 2, 2)
        _check(_lib.gsb_set_matrices(self.handle, _ptr(Mc.view(np.float64), ctypes.c_double)))

    def set_fusion(self, depth):
        """'chain' mode: fuse up to `depth` consecutive wide steps per pass (1 = no fusion)."""
        _check(_lib.gsb_set_fusion(self.handle, int(depth)))

    def autotune(self, mode=2, reps=3):
        """Time every candidate pass on this device and keep the fastest covers of the steps (mode 0: 'chain',
        1: 'prob' / 'sample', 2: both); returns (ms of one item before, after)."""
        a, b = ctypes.c_float(), ctypes.c_float()
        _check(_lib.gsb_autotune(self.handle, int(mode), int(reps), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def fusion_groups(self):
        """(group length per step: the pass starting at step k spans that many steps, 0 inside a pass;
        table entries read + written by each pass, at its first step)."""
        g = np.zeros(max(self.ns, 1), np.int32)
        e = np.zeros(max(self.ns, 1), np.float64)
        _check(_lib.gsb_fusion_groups(self.handle, _ptr(g, ctypes.c_int), _ptr(e, ctypes.c_double)))
        return [int(x) for x in g[:self.ns]], e[:self.ns]

    def test_withhold_tile_loads(self, on, partial=False):
        """Test hook: the fused passes issue no tile loads (partial=True: only in their odd CTAs), so those CTAs'
        bounded waits run out and calls raise GsbError (GSB_E_CUDA); off again, the engine runs normally."""
        _check(_lib.gsb_test_withhold_tile_loads(self.handle, (2 if partial else 1) if on else 0))

    def sample_groups(self):
        """The sampling passes: (steps written per pass at its first step, 0 inside a pass; table entries read +
        written by each pass, its norm pass included)."""
        g = np.zeros(max(self.ns, 1), np.int32)
        e = np.zeros(max(self.ns, 1), np.float64)
        _check(_lib.gsb_sample_groups(self.handle, _ptr(g, ctypes.c_int), _ptr(e, ctypes.c_double)))
        return [int(x) for x in g[:self.ns]], e[:self.ns]

    def passes(self, mode=0):
        """The passes of 'chain' (mode 0) or 'prob' / 'sample' (mode 1) in launch order: a list of
        (first step, steps written, trailing branch-norm step 0/1, fused 0/1)."""
        n = ctypes.c_int()
        _check(_lib.gsb_pass_list(self.handle, int(mode), 0, None, None, None, None, ctypes.byref(n)))
        cols = [np.zeros(max(n.value, 1), np.int32) for _ in range(4)]
        _check(_lib.gsb_pass_list(self.handle, int(mode), n.value, *[_ptr(a, ctypes.c_int) for a in cols],
                                  ctypes.byref(n)))
        return [tuple(int(a[i]) for a in cols) for i in range(n.value)]

    def set_guard(self, guard, log2_xmin):
        """Re-evaluate this complex64 engine's unlikely strings (log2 Pr + nsteps < log2_xmin) on `guard`, a
        complex128 Engine of the same plan (None detaches).  The guard must stay open while attached."""
        _check(_lib.gsb_set_guard(self.handle, None if guard is None else guard.handle, float(log2_xmin)))
        self._guard = guard          # keeps the guard alive as long as it is attached

    def set_hybrid_prefix(self, K):
        """hybrid() strings force their first K steps: those run as fused 'chain' passes (0 undoes it)."""
        _check(_lib.gsb_set_hybrid_prefix(self.handle, int(K)))

    def guard_evaluations(self):
        n = ctypes.c_int64()
        _check(_lib.gsb_guard_evaluations(self.handle, ctypes.byref(n)))
        return n.value

    def set_arith(self, bits):
        """complex64 wide-step arithmetic: 32 (FP32 sums and rotation, default) or 64 (exact sums + FP64 rotation,
        the reference's complex64 arithmetic)."""
        _check(_lib.gsb_set_arith(self.handle, int(bits)))

    def synchronize(self):
        _check(_lib.gsb_synchronize(self.handle))

    def profile_steps(self, string, mode=0):
        """Per-step kernel times (ms) of one forced string: (write [ns], norm [ns]); mode 0 chain, 1 prob."""
        f = as_bits([string], self.ns)[0].copy()
        w = np.zeros(max(self.ns, 1), np.float32)
        nrm = np.zeros(max(self.ns, 1), np.float32)
        _check(_lib.gsb_profile_steps(self.handle, _ptr(f, ctypes.c_int8), int(mode), _ptr(w, ctypes.c_float),
                                      _ptr(nrm, ctypes.c_float)))
        return w[:self.ns], nrm[:self.ns]

    def launches_per_item(self, mode):
        n = ctypes.c_int64()
        _check(_lib.gsb_launches_per_item(self.handle, int(mode), ctypes.byref(n)))
        return n.value


class DpEngine:
    """The out-of-place amplitude engine (the reference's dp.cpp) on one plan: complex amplitudes Z(w)."""

    def __init__(self, plan_text, precision=GSB_C128, device=0):
        h = ctypes.c_void_p()
        b = plan_text.encode() if isinstance(plan_text, str) else bytes(plan_text)
        _check(_lib.gsb_dp_open_text(b, len(b), int(precision), int(device), ctypes.byref(h)))
        self._h = h
        m, ns, mr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(_lib.gsb_dp_info(h, ctypes.byref(m), ctypes.byref(ns), ctypes.byref(mr)))
        self.m, self.ns, self.maxr = m.value, ns.value, mr.value

    def run(self, slices):
        """sum over slices (pre, weights [(w0, w1) per vertex]) of pre * Z(weights) (one reference job)."""
        pre = np.zeros(2 * max(len(slices), 1))
        w = np.zeros(max(len(slices), 1) * max(self.m, 1) * 4)
        for i, (p, ww) in enumerate(slices):
            pre[2 * i], pre[2 * i + 1] = complex(p).real, complex(p).imag
            for q, (a, b) in enumerate(ww):
                j = (i * self.m + q) * 4
                w[j:j + 4] = complex(a).real, complex(a).imag, complex(b).real, complex(b).imag
        out = np.zeros(2)
        _check(_lib.gsb_dp_run(self._h, len(slices), _ptr(pre, ctypes.c_double), _ptr(w, ctypes.c_double),
                               _ptr(out, ctypes.c_double)))
        return complex(out[0], out[1])

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.gsb_dp_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GradSweep:
    """The adjoint sweep (complex128) on one in-place plan: Z(b) and dZ/dM_k[b_k][x] for a batch of strings."""

    def __init__(self, plan_text, device=0, every=4):
        h = ctypes.c_void_p()
        b = plan_text.encode() if isinstance(plan_text, str) else bytes(plan_text)
        _check(_lib.gsb_grad_open_text(b, len(b), int(device), int(every), ctypes.byref(h)))
        self._h = h
        n, ns, R = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(_lib.gsb_grad_info(h, ctypes.byref(n), ctypes.byref(ns), ctypes.byref(R)))
        self.n, self.ns, self.R = n.value, ns.value, R.value

    def run(self, M, bits):
        """M: [ns][2][2] complex (step order); bits: [nstr][ns] (step order).  Returns (Z [nstr] complex128,
        dZ [nstr][ns][2] complex128 with dZ[s, k, x] = dZ(b_s)/dM_k[b_sk][x])."""
        Mc = np.ascontiguousarray(M, np.complex128).reshape(self.ns, 2, 2)
        b = as_bits(bits, self.ns)
        z = np.zeros(max(len(b), 1), np.complex128)
        dz = np.zeros((max(len(b), 1), self.ns, 2), np.complex128)
        if len(b):
            _check(_lib.gsb_grad_run(self._h, _ptr(Mc.view(np.float64), ctypes.c_double), _ptr(b, ctypes.c_int8),
                                     len(b), _ptr(z.view(np.float64), ctypes.c_double),
                                     _ptr(dz.view(np.float64), ctypes.c_double)))
        return z[:len(b)], dz[:len(b)]

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.gsb_grad_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many instances (in-place plans of uneven width) in one persistent launch; strings share prefixes."""

    def __init__(self, plan_texts, precision=GSB_C64, device=0):
        bs = [t.encode() if isinstance(t, str) else bytes(t) for t in plan_texts]
        arr = (ctypes.c_char_p * len(bs))(*bs)
        lens = (ctypes.c_size_t * len(bs))(*[len(b) for b in bs])
        h = ctypes.c_void_p()
        _check(_lib.gsb_batch_open(arr, lens, len(bs), int(precision), int(device), ctypes.byref(h)))
        self._h = h
        self.ninst = len(bs)
        self._shape = None

    def set_strings(self, K, prefixes, suffixes):
        """K[i]: prefix length; prefixes[i]: [npre][K[i]]; suffixes[i]: [npre][nsuf][ns_i - K[i]] (0/1, step order)."""
        pre = [np.ascontiguousarray(p, np.int8) for p in prefixes]
        suf = [np.ascontiguousarray(s, np.int8) for s in suffixes]
        self.npre, self.nsuf = pre[0].shape[0], suf[0].shape[1]
        Kc = np.ascontiguousarray(K, np.int32)
        pb = np.concatenate([p.reshape(-1) for p in pre])
        sb = np.concatenate([s.reshape(-1) for s in suf])
        _check(_lib.gsb_batch_set_strings(self._h, _ptr(Kc, ctypes.c_int), self.npre, self.nsuf,
                                          _ptr(pb, ctypes.c_int8), _ptr(sb, ctypes.c_int8)))

    def run(self):
        """(log2 Pr [ninst][npre][nsuf], device milliseconds of the launch)."""
        out = np.zeros(self.ninst * self.npre * self.nsuf)
        ms = ctypes.c_float()
        _check(_lib.gsb_batch_run(self._h, _ptr(out, ctypes.c_double), ctypes.byref(ms)))
        return out.reshape(self.ninst, self.npre, self.nsuf), ms.value

    def set_shape(self, block, small_R, per_sm):
        _check(_lib.gsb_batch_set_shape(self._h, int(block), int(small_R), int(per_sm)))

    def shape(self):
        v = [ctypes.c_int() for _ in range(3)]
        _check(_lib.gsb_batch_get_shape(self._h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def tune(self, reps=2, max_bytes=8 << 30):
        """Autotune the launch shape on the current strings; returns (block, small_R, per_sm, mean ms)."""
        v = [ctypes.c_int() for _ in range(3)]
        ms = ctypes.c_float()
        _check(_lib.gsb_batch_tune(self._h, int(reps), int(max_bytes), *[ctypes.byref(x) for x in v], ctypes.byref(ms)))
        return tuple(x.value for x in v) + (ms.value,)

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.gsb_batch_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _extend(fn, old, r, rn, rho, piv, ker, wv, device):
    old = np.ascontiguousarray(old, np.complex128)
    assert old.shape == (1 << r,)
    out = np.zeros(1 << rn, np.complex128)
    k = np.ascontiguousarray(list(ker) or [0], np.uint64)
    w = np.array([complex(wv[0]).real, complex(wv[0]).imag, complex(wv[1]).real, complex(wv[1]).imag])
    pm = sum(1 << p for p in piv)
    _check(fn(int(r), int(rn), int(rho), int(pm), len(ker), _ptr(k, ctypes.c_uint64), _ptr(w, ctypes.c_double),
              _ptr(old.view(np.float64), ctypes.c_double), _ptr(out.view(np.float64), ctypes.c_double), int(device)))
    return out


def dp_extend(old, r, rn, rho, piv, ker, wv, device=0):
    """One out-of-place DP step on the GPU (complex128): new table of 2^rn entries."""
    return _extend(_lib.gsb_dp_extend, old, r, rn, rho, piv, ker, wv, device)


def dp_extend_static(old, r, rn, rho, piv, ker, wv, device=0):
    """dp_extend without device allocation (static scratch in the library; r, rn <= 16; calls must not overlap)."""
    return _extend(_lib.gsb_dp_extend_static, old, r, rn, rho, piv, ker, wv, device)


def probe_l2_copy(device=0, mib=24, reps=400):
    """L2 copy bandwidth of a device (GB/s, bytes read + written): one launch copies an L2-resident buffer of `mib`
    MiB onto another `reps` times.  The denominator of the L2 roofline of L2-resident work."""
    g = ctypes.c_float()
    _check(_lib.gsb_probe_l2_copy(int(device), int(mib) << 20, int(reps), ctypes.byref(g)))
    return float(g.value)


def validate_text(text):
    """Parse + validate plan text on the host (no GPU): (n, nsteps, R); raises GsbError."""
    b = text.encode() if isinstance(text, str) else bytes(text)
    n, ns, R = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(_lib.gsb_validate_text(b, len(b), ctypes.byref(n), ctypes.byref(ns), ctypes.byref(R)))
    return n.value, ns.value, R.value


def cut_profile(A, order):
    A = np.ascontiguousarray(np.asarray(A) & 1, np.uint8)
    n = len(A)
    o = np.ascontiguousarray(order, np.int32)
    prof = np.zeros(max(n - 1, 1), np.int32)
    _check(_lib.gsb_cut_profile(n, _ptr(A, ctypes.c_uint8), _ptr(o, ctypes.c_int), _ptr(prof, ctypes.c_int)))
    return [int(x) for x in prof[:max(n - 1, 0)]]


def order_search(A, seed=0, ngreedy=4, iters=20000):
    A = np.ascontiguousarray(np.asarray(A) & 1, np.uint8)
    n = len(A)
    out = np.zeros(n, np.int32)
    w = ctypes.c_int()
    _check(_lib.gsb_order_search(n, _ptr(A, ctypes.c_uint8), int(seed), int(ngreedy), int(iters),
                                 _ptr(out, ctypes.c_int), ctypes.byref(w)))
    return [int(x) for x in out], w.value


def version():
    return _lib.gsb_version().decode()
