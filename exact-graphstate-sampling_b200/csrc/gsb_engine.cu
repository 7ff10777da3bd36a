// libgsb: the C ABI of include/gsb.h on top of the kernels in gsb_kernels.cuh.
//
// An engine = one validated plan + one arena (2^R entries) + one stream + device-resident state.  Every mode of the
// reference executor (gsamp2.cpp:149-225) becomes a sequence of kernel launches per string or sample:
//   begin (unit table) -> per step [norm pass] write pass -> finish (log2 Pr, next item)
// with all scalar decisions made on the device.  The per-item sequences of the batch modes are captured once as
// CUDA graphs and replayed per item; the item index advances on the device, so a batch of strings is one H2D copy,
// N graph launches and one D2H copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <random>
#include <string>
#include <tuple>
#include <vector>

#include "gsb.h"
#include "gsb_common.h"
#include "gsb_fuse.h"
#include "gsb_group.cuh"
#include "gsb_kernels.cuh"
#include "gsb_pick.h"
#include "gsb_plan.h"

namespace gsb {

static thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define GSB_CK(x)                                                                                         \
    do {                                                                                                  \
        cudaError_t e_ = (x);                                                                             \
        if (e_ != cudaSuccess) {                                                                          \
            return fail(GSB_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #x);    \
        }                                                                                                 \
    } while (0)

struct Launch {
    int grid = 1, block = 1, U = 1, tl = 0, cl = 0;
    unsigned int nchunks = 1;
    void *fn = nullptr;
};

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int d) {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~DevGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

template <typename E, int NTQ, int M, int U>
static void *pick_w(bool write) {
    return write ? (void *)k_step<E, NTQ, M, U, true> : (void *)k_step<E, NTQ, M, U, false>;
}
template <typename E, int NTQ, int M>
static void *pick_u(int U, bool write) {
    return U == 4 ? pick_w<E, NTQ, M, 4>(write) : pick_w<E, NTQ, M, 1>(write);
}
template <typename E, int NTQ>
static void *pick_m(int m, int U, bool write) {
    return m == 2 ? pick_u<E, NTQ, 2>(U, write) : pick_u<E, NTQ, 1>(U, write);
}
template <typename E>
static void *pick_step_kernel(int ntq, int m, int U, bool write) {
    if (ntq == 4) return pick_m<E, 4>(m, U, write);
    if (ntq == 2) return pick_m<E, 2>(m, U, write);
    return pick_m<E, 1>(m, U, write);
}

// wide-step kernels: U = 4 coset groups per thread for 1-2 offsets, 2 for 4 offsets (register budget)
template <int NTQ, int M>
static void *pick_pair64(bool write, bool fp32) {
    constexpr int U = NTQ == 4 ? 2 : 4;
    if (fp32) return write ? (void *)k_pair64<float, NTQ, M, U, true> : (void *)k_pair64<float, NTQ, M, U, false>;
    return write ? (void *)k_pair64<double, NTQ, M, U, true> : (void *)k_pair64<double, NTQ, M, U, false>;
}
template <int NTQ, int M>
static void *pick_wide128(bool write) {
    constexpr int U = NTQ == 4 ? 2 : 4;
    return write ? (void *)k_wide128<NTQ, M, U, true> : (void *)k_wide128<NTQ, M, U, false>;
}
static void *pick_wide(int prec, int ntq, int m, bool write, bool fp32) {
    if (prec == 64) {
        if (ntq == 4) return m == 2 ? pick_pair64<4, 2>(write, fp32) : pick_pair64<4, 1>(write, fp32);
        if (ntq == 2) return m == 2 ? pick_pair64<2, 2>(write, fp32) : pick_pair64<2, 1>(write, fp32);
        return m == 2 ? pick_pair64<1, 2>(write, fp32) : pick_pair64<1, 1>(write, fp32);
    }
    if (ntq == 4) return m == 2 ? pick_wide128<4, 2>(write) : pick_wide128<4, 1>(write);
    if (ntq == 2) return m == 2 ? pick_wide128<2, 2>(write) : pick_wide128<2, 1>(write);
    return m == 2 ? pick_wide128<1, 2>(write) : pick_wide128<1, 1>(write);
}

template <typename E, typename T>
static void *pick_group(int d, int tr) {
    if (tr) return d == 2 ? (void *)k_group<E, T, 2, 1> : (void *)k_group<E, T, 1, 1>;
    return d == 3 ? (void *)k_group<E, T, 3, 0> : (void *)k_group<E, T, 2, 0>;
}

// One pass of an item: a single step (group == false: norm pass + write pass when sampling) or a fused group that
// writes d steps and, with tr = 1, evaluates the next step's branch norms (sampling only).
// A fused pass's kernel parameters (GroupArgs, the arena pointer, Ctx) stay within the 4 KB of a classic launch.
static_assert(sizeof(GroupArgs) + sizeof(void *) + sizeof(Ctx) <= 4096, "fused-pass parameters exceed 4 KB");

struct Op {
    int k0 = 0, d = 1, tr = 0, lcap = 0;   // lcap: the tile-size cap the pass was built with (fused passes)
    int minb = 2;                          // CTAs per SM the fused kernel is built for (2, or 3: pick_group3)
    int threads = GROUP_NCT;               // block size: GROUP_NCT, or GROUP_NCT + 32 (warp-specialised build)
    int ws = 0;                            // the warp-specialised build (1) or not (0)
    bool group = false;
    bool norm_first = false;  // sampling: a norm pass of step k0 runs first (its bit has no other source)
    GroupArgs ga;
    void *fn = nullptr;
    int grid = 1;
    size_t smem = 0;
    unsigned int ntiles = 0;
    double entries = 0;       // entries read + written by the pass (the norm pass not included)
};

#ifndef GSB_GROUP_SMEM_PREF
#define GSB_GROUP_SMEM_PREF (100 * 1024)
#endif
#ifndef GSB_GROUP_MAX_L
#define GSB_GROUP_MAX_L 10
#endif
constexpr uint32_t GROUP_SMEM_BUDGET = 200 * 1024;  // shared memory of one fused-pass CTA at most
constexpr uint32_t GROUP_SMEM_PREF = GSB_GROUP_SMEM_PREF;   // tiles are shrunk to this first (two CTAs per SM)
constexpr int GROUP_MAX_L = GSB_GROUP_MAX_L;                // at most 2^GROUP_MAX_L classes per tile
constexpr int GROUP_MIN_R = 12;                     // steps below 2^12 entries run unfused

// What a pass is, without its arguments: rebuilt with the current matrices whenever they change.
struct OpShape {
    int k0 = 0, d = 1, tr = 0, lcap = 0, src = 0, minb = 2;
    int ws = -1;   // warp-specialised build: 1 yes, 0 no, -1 the default rule (fill_group)
    bool group = false, norm_first = false;
};
constexpr uint32_t GROUP_SMEM_3 = 72 * 1024;        // shared memory of a fused-pass CTA when three share an SM

template <typename E, typename T>
static uint32_t group_smem_bytes(int D, int TR, const int (&ssz)[4], int L, bool fold = false) {
    if (TR) return D == 2 ? group_smem<E, T, 2, 1>(ssz, L, fold).total : group_smem<E, T, 1, 1>(ssz, L).total;
    return D == 3 ? group_smem<E, T, 3, 0>(ssz, L).total : group_smem<E, T, 2, 0>(ssz, L).total;
}

struct Engine {
    HPlan plan;
    int prec = 64, dev = 0, sms = 0;
    int arith = 32;                      // arithmetic of the complex64 wide-step kernels: 32 (FP32) or 64 (FP64)
    int fuse_depth = 2;                  // chain mode: largest number of DP steps fused into one pass (1 = none)
    std::vector<Op> chain_ops;           // 'chain' passes
    int hyb_K = 0;                       // gsb_set_hybrid_prefix: hybrid strings force their first hyb_K steps
    std::vector<Op> hyb_ops;             // fused 'chain' passes over those steps
    std::vector<Op> sample_ops;          // 'prob' / 'sample' passes (build_sample_ops)
    int withhold_loads = 0;              // test hook: fused passes issue no tile loads (their bounded waits run out)
    std::vector<OpShape> chain_shapes;   // pass lists chosen by gsb_autotune (empty: the byte-model defaults)
    std::vector<OpShape> sample_shapes;
    size_t esize = 8;
    void *mem = nullptr;
    cudaStream_t stream = nullptr;       // where work is queued (own_stream unless the caller set one)
    cudaStream_t own_stream = nullptr;
    DevState *st = nullptr;
    double *partials = nullptr;
    int cap = 1024;                      // items per device batch
    int8_t *d_forced = nullptr, *d_bits = nullptr;
    double *d_unif = nullptr, *d_cond = nullptr, *d_logp = nullptr, *d_aux = nullptr;
    void *d_dump = nullptr;
    size_t dump_bytes = 0;
    std::vector<StepArgs> args;
    StepArgs *d_args = nullptr;          // device copy of args (read by the small-step runs, k_small_run)
    bool args_dirty = true;              // args changed since d_args was last written
    std::vector<Launch> lw, ln;
    std::map<int, cudaGraphExec_t> graphs;   // key: graph kind
    std::map<void *, int> occ;
    // complex128 re-evaluation of unlikely strings (gsb_set_guard): the engine that re-evaluates this one's strings
    // whose log2 Pr + ns < guard_lx, and the engine this one re-evaluates for
    Engine *guard = nullptr, *guarded = nullptr;
    double guard_lx = 0;
    int64_t guard_evals = 0;
    // FP32 coefficients of a complex64 engine with FP32 arithmetic (apply_coeffs): per step, the M entries and the
    // factored steps' pivot and ratio, rounded to float values
    struct Coef32 {
        double Mr[2][2], Mi[2][2];
        int piv[2];
        double br[2], bi[2], cp[2];
    };
    std::vector<Coef32> c32;

    ~Engine() {
        if (guard) guard->guarded = nullptr;
        if (guarded) guarded->guard = nullptr;
        DevGuard g(dev);
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        cudaFree(mem);
        cudaFree(d_args);
        cudaFree(st);
        cudaFree(partials);
        cudaFree(d_forced);
        cudaFree(d_bits);
        cudaFree(d_unif);
        cudaFree(d_cond);
        cudaFree(d_logp);
        cudaFree(d_aux);
        cudaFree(d_dump);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    int occupancy(void *fn, int block) {
        auto it = occ.find(fn);
        if (it != occ.end()) return it->second;
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, 0) != cudaSuccess || nb < 1) nb = 1;
        occ[fn] = nb;
        return nb;
    }

    void *step_fn(int ntq, int m, int U, bool write) const {
        return prec == 128 ? pick_step_kernel<double2>(ntq, m, U, write) : pick_step_kernel<float2>(ntq, m, U, write);
    }

    Launch shape(const StepArgs &a, bool write) {
        Launch L;
        const uint64_t N = 1ULL << a.nk;
        // wide steps: the pair kernel (complex64, needs coset bit 0 = arena bit 0) or the complex128 kernel
        const int uw = a.ntq == 4 ? 2 : 4;
        const bool wide64 = prec == 64 && a.nk >= 11 && a.tk[0] == 1;
        const bool wide128 = prec == 128 && a.nk >= 10;
        if (wide64 || wide128) {
            L.block = 256;
            L.U = uw;
            L.tl = 8;
            L.cl = (wide64 ? 9 : 8) + (uw == 4 ? 2 : 1);
            L.nchunks = (unsigned int)(N >> L.cl);
            L.fn = pick_wide(prec, a.ntq, a.m, write, arith == 32);
            const int cap_blocks = occupancy(L.fn, L.block) * sms;
            L.grid = (int)std::min<uint64_t>(L.nchunks, (uint64_t)cap_blocks);
            return L;
        }
        // blocks of at least one full warp (the reductions shuffle over 32 lanes); below 32 cosets the threads
        // tid >= 2^nk idle
        if (N >= 1024) { L.block = 256; L.U = 4; L.tl = 8; }
        else if (N >= 256) { L.block = 256; L.U = 1; L.tl = 8; }
        else { L.block = (int)std::max<uint64_t>(32, N); L.U = 1; L.tl = a.nk; }
        L.cl = L.tl + (L.U == 4 ? 2 : 0);
        L.nchunks = (unsigned int)(N >> L.cl);
        L.fn = step_fn(a.ntq, a.m, L.U, write);
        const int cap_blocks = occupancy(L.fn, L.block) * sms;
        L.grid = (int)std::min<uint64_t>(L.nchunks, (uint64_t)cap_blocks);
        return L;
    }

    Ctx ctx(int driver, int k1, const Launch &L, bool use_forced, bool use_unif) const {
        Ctx c;
        c.st = st;
        c.partials = partials;
        c.forced = use_forced ? d_forced : nullptr;
        c.unif = use_unif ? d_unif : nullptr;
        c.bits_out = d_bits;
        c.cond_out = d_cond;
        c.ns = plan.ns;
        c.driver = driver;
        c.k1 = k1;
        c.tpb_log2 = L.tl;
        c.chunk_log2 = L.cl;
        c.nchunks = L.nchunks;
        return c;
    }

    cudaError_t launch_step(int k, bool write, int driver, int k1, bool use_forced, bool use_unif) {
        const Launch &L = write ? lw[(size_t)k] : ln[(size_t)k];
        StepArgs a = args[(size_t)k];
        Ctx c = ctx(driver, k1, L, use_forced, use_unif);
        void *memp = mem;
        void *kargs[] = {&a, &memp, &c};
        return cudaLaunchKernel(L.fn, dim3((unsigned)L.grid), dim3((unsigned)L.block), kargs, 0, stream);
    }

    // Whether step k runs in a small-step run (k_small_run) when it is a single-step pass.
    bool small_step(int k) const { return args[(size_t)k].nk <= SMALL_NK; }

    // Steps k0 .. k1-1 as one k_small_run launch; norm: each step's norm pass runs before its write pass.
    cudaError_t launch_small_run(int k0, int k1, int driver, bool norm, bool use_forced, bool use_unif) {
        Launch L;
        Ctx c = ctx(driver, plan.ns, L, use_forced, use_unif);
        const StepArgs *sa = d_args;
        int a0 = k0, a1 = k1, nm = norm ? 1 : 0;
        void *memp = mem;
        void *kargs[] = {&sa, &a0, &a1, &nm, &memp, &c};
        void *fn = prec == 128 ? (void *)k_small_run<double2> : (void *)k_small_run<float2>;
        return cudaLaunchKernel(fn, dim3(1), dim3(SMALL_THREADS), kargs, 0, stream);
    }

    // Length of the run of consecutive single small-step passes that starts at ops[i] (0 or 1: no run).
    size_t small_run_len(const std::vector<Op> &ops, size_t i) const {
        size_t j = i;
        while (j < ops.size() && !ops[j].group && small_step(ops[j].k0)) j++;
        return j - i >= 2 ? j - i : 0;
    }

    // Launches of one item over a pass list (small-step runs count once), begin and finish included.
    int64_t item_launches(const std::vector<Op> &ops, bool norm) const {
        int64_t n = 2;
        for (size_t i = 0; i < ops.size();) {
            const size_t r = small_run_len(ops, i);
            if (r) { n++; i += r; continue; }
            n += 1 + ((norm && !ops[i].group) || ops[i].norm_first ? 1 : 0);
            i++;
        }
        return n;
    }

    cudaError_t launch_begin() {
        if (prec == 128) k_begin<double2><<<1, 1, 0, stream>>>((double2 *)mem, st);
        else k_begin<float2><<<1, 1, 0, stream>>>((float2 *)mem, st);
        return cudaGetLastError();
    }

    // One item: begin, steps k0..k1-1, finish.  driver decides the passes:
    //   CHAIN: norm + write per step; CHAIN1: write; HYBRID: norm (skipped on device when forced) + write.
    cudaError_t launch_op(const Op &op, int driver, bool use_forced = true, bool use_unif = false) {
        if (!op.group) return launch_step(op.k0, true, driver, plan.ns, use_forced, use_unif);
        Launch L;
        L.tl = 8;
        L.cl = op.ga.L;
        L.nchunks = op.ntiles;
        Ctx c = ctx(driver, plan.ns, L, use_forced, use_unif);
        GroupArgs ga = op.ga;
        ga.withhold_loads = withhold_loads;
        void *memp = mem;
        void *kargs[] = {&ga, &memp, &c};
        return cudaLaunchKernel(op.fn, dim3((unsigned)op.grid), dim3((unsigned)op.threads), kargs, op.smem, stream);
    }

    cudaError_t enqueue_item(int driver, bool use_forced, bool use_unif) {
        cudaError_t e = launch_begin();
        if (e != cudaSuccess) return e;
        if (driver == DRV_CHAIN1 && !chain_ops.empty()) {
            for (size_t i = 0; i < chain_ops.size();) {
                if (const size_t r = small_run_len(chain_ops, i)) {
                    e = launch_small_run(chain_ops[i].k0, chain_ops[i + r - 1].k0 + 1, driver, false, use_forced,
                                         use_unif);
                    if (e != cudaSuccess) return e;
                    i += r;
                    continue;
                }
                e = launch_op(chain_ops[i++], driver);
                if (e != cudaSuccess) return e;
            }
            k_finish<<<1, 1, 0, stream>>>(st, d_logp, d_aux, driver, plan.ns);
            return cudaGetLastError();
        }
        if (driver == DRV_CHAIN && !sample_ops.empty()) {
            for (size_t i = 0; i < sample_ops.size();) {
                if (const size_t r = small_run_len(sample_ops, i)) {
                    e = launch_small_run(sample_ops[i].k0, sample_ops[i + r - 1].k0 + 1, driver, true, use_forced,
                                         use_unif);
                    if (e != cudaSuccess) return e;
                    i += r;
                    continue;
                }
                const Op &op = sample_ops[i++];
                if (!op.group || op.norm_first) {
                    e = launch_step(op.k0, false, driver, plan.ns, use_forced, use_unif);
                    if (e != cudaSuccess) return e;
                }
                e = op.group ? launch_op(op, driver, use_forced, use_unif)
                             : launch_step(op.k0, true, driver, plan.ns, use_forced, use_unif);
                if (e != cudaSuccess) return e;
            }
            k_finish<<<1, 1, 0, stream>>>(st, d_logp, d_aux, driver, plan.ns);
            return cudaGetLastError();
        }
        int k0 = 0;
        if (driver == DRV_HYBRID && hyb_K > 0) {
            // forced prefix: 'chain' passes (fused where possible), then the run_steps state for the sampled steps
            for (size_t i = 0; i < hyb_ops.size();) {
                if (const size_t r = small_run_len(hyb_ops, i)) {
                    e = launch_small_run(hyb_ops[i].k0, hyb_ops[i + r - 1].k0 + 1, DRV_CHAIN1, false, true, false);
                    if (e != cudaSuccess) return e;
                    i += r;
                    continue;
                }
                e = launch_op(hyb_ops[i++], DRV_CHAIN1);
                if (e != cudaSuccess) return e;
            }
            k_hybrid_switch<<<1, 1, 0, stream>>>(st, d_forced, d_bits, plan.ns, hyb_K);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            k0 = hyb_K;
        }
        for (int k = k0; k < plan.ns; k++) {
            int k1 = k;
            while (k1 < plan.ns && small_step(k1)) k1++;
            if (k1 - k >= 2) {
                e = launch_small_run(k, k1, driver, driver != DRV_CHAIN1, use_forced, use_unif);
                if (e != cudaSuccess) return e;
                k = k1 - 1;
                continue;
            }
            if (driver != DRV_CHAIN1) {
                e = launch_step(k, false, driver, plan.ns, use_forced, use_unif);
                if (e != cudaSuccess) return e;
            }
            e = launch_step(k, true, driver, plan.ns, use_forced, use_unif);
            if (e != cudaSuccess) return e;
        }
        k_finish<<<1, 1, 0, stream>>>(st, d_logp, d_aux, driver, plan.ns);
        return cudaGetLastError();
    }

    int graph(int kind, cudaGraphExec_t *out) {
        auto it = graphs.find(kind);
        if (it != graphs.end()) { *out = it->second; return 0; }
        int driver = kind == 0 ? DRV_CHAIN1 : kind == 3 ? DRV_HYBRID : DRV_CHAIN;
        bool use_forced = kind != 2, use_unif = kind >= 2;
        if (args_dirty) {   // the small-step runs read the step descriptors from the device
            GSB_CK(cudaMemcpyAsync(d_args, args.data(), args.size() * sizeof(StepArgs), cudaMemcpyHostToDevice, stream));
            GSB_CK(cudaStreamSynchronize(stream));
            args_dirty = false;
        }
        cudaGraph_t g = nullptr;
        GSB_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = enqueue_item(driver, use_forced, use_unif);
        cudaError_t e2 = cudaStreamEndCapture(stream, &g);
        if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); GSB_CK(e); }
        GSB_CK(e2);
        cudaGraphExec_t ex = nullptr;
        e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        GSB_CK(e);
        graphs[kind] = ex;
        *out = ex;
        return 0;
    }

    // Run `n` items of graph `kind` with inputs already in d_forced / d_unif rows 0..n-1.
    int run_graph_items(int kind, int64_t n) {
        cudaGraphExec_t ex;
        int rc = graph(kind, &ex);
        if (rc) return rc;
        k_set_item<<<1, 1, 0, stream>>>(st, 0);
        GSB_CK(cudaGetLastError());
        for (int64_t i = 0; i < n; i++) GSB_CK(cudaGraphLaunch(ex, stream));
        return 0;
    }
};

// Float rounding of the FP32 kernels' coefficients by error diffusion.  A rounded coefficient c' = c (1 + d)
// scales every amplitude path through it; the real part of d biases log2 Pr, the same way for every string, and
// with round-to-nearest a plan whose steps repeat one matrix (a circuit with one rotation on every qubit) adds
// those biases up step after step.  Each occurrence of a value is therefore rounded up or down (either is within
// one ulp) so that the running sum of Re d over that value's occurrences stays within about one ulp of zero; the
// first occurrence rounds to nearest, so a plan of distinct matrices keeps round-to-nearest throughout.
static std::complex<double> round_diffused(std::complex<double> v, double &cum) {
    if (v == 0.0) return v;
    auto pair = [](double x, float &lo, float &hi) {
        const float f = (float)x;
        if ((double)f == x) { lo = hi = f; return; }
        if ((double)f > x) { hi = f; lo = std::nextafter(f, -INFINITY); }
        else { lo = f; hi = std::nextafter(f, INFINITY); }
    };
    float rl, rh, il, ih;
    pair(v.real(), rl, rh);
    pair(v.imag(), il, ih);
    std::complex<double> best = v;
    double bd = 0, bs = INFINITY;
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) {
            const std::complex<double> c((double)(a ? rh : rl), (double)(b ? ih : il));
            const double d = ((c - v) / v).real();
            const double sc = std::fabs(cum + d) + 1e-3 * std::abs((c - v) / v);   // ties: the nearer value
            if (sc < bs) { bs = sc; best = c; bd = d; }
        }
    cum += bd;
    return best;
}

// The coefficients a complex64 engine with FP32 arithmetic uses: M entries (single-step kernels, the fused passes'
// general shape) and, per bit, the factored step's pivot (the larger of the row's two entries), its ratio
// beta = M[b][1-piv] / M[b][piv] and cp = |M[b][piv]|^2 (exact), all rounded by round_diffused in step order.
// Other engines use the plan's M as it is (FP64 arithmetic, or complex128).
static void apply_coeffs(Engine &E) {
    const HPlan &p = E.plan;
    const bool f32 = E.prec == 64 && E.arith == 32;
    E.c32.assign((size_t)p.ns, Engine::Coef32());
    // running sums of Re d per (role, exact value): roles 0-3 the M entries [b][x], 4-5 the ratios of bit b
    std::map<std::tuple<int, double, double>, double> cum;
    auto rnd = [&](int role, std::complex<double> v) {
        auto key = std::make_tuple(role, v.real(), v.imag());
        auto it = cum.find(key);
        if (it == cum.end()) {   // first occurrence: round to nearest
            const std::complex<double> c((double)(float)v.real(), (double)(float)v.imag());
            cum[key] = v == 0.0 ? 0.0 : ((c - v) / v).real();
            return c;
        }
        return round_diffused(v, it->second);
    };
    for (int k = 0; k < p.ns; k++) {
        const HStep &hs = p.st[(size_t)k];
        Engine::Coef32 &c = E.c32[(size_t)k];
        for (int b = 0; b < 2; b++) {
            for (int x = 0; x < 2; x++) {
                std::complex<double> m(hs.Mr[b][x], hs.Mi[b][x]);
                if (f32) m = rnd(2 * b + x, m);
                c.Mr[b][x] = m.real();
                c.Mi[b][x] = m.imag();
            }
            const double n0 = std::norm(std::complex<double>(hs.Mr[b][0], hs.Mi[b][0]));
            const double n1 = std::norm(std::complex<double>(hs.Mr[b][1], hs.Mi[b][1]));
            c.piv[b] = -1;
            c.br[b] = c.bi[b] = 0;
            c.cp[b] = 1;
            if (f32 && std::max(n0, n1) > 0) {
                const int pv = n0 >= n1 ? 0 : 1;
                const std::complex<double> w(hs.Mr[b][pv], hs.Mi[b][pv]), o(hs.Mr[b][1 - pv], hs.Mi[b][1 - pv]);
                const std::complex<double> beta = rnd(4 + b, o / w);
                c.piv[b] = pv;
                c.br[b] = beta.real();
                c.bi[b] = beta.imag();
                c.cp[b] = std::norm(w);
            }
        }
        if ((size_t)k < E.args.size())
            for (int b = 0; b < 2; b++)
                for (int x = 0; x < 2; x++) {
                    E.args[(size_t)k].Mr32[b][x] = c.Mr[b][x];
                    E.args[(size_t)k].Mi32[b][x] = c.Mi[b][x];
                }
    }
    E.args_dirty = true;   // every change of the descriptors (matrices, arithmetic) ends here
}

static int make_args(Engine &E) {
    const HPlan &p = E.plan;
    E.args.resize((size_t)p.ns);
    for (int k = 0; k < p.ns; k++) {
        const HStep &s = p.st[(size_t)k];
        StepArgs a;
        memset(&a, 0, sizeof a);
        for (int j = 0; j < s.nk; j++) a.tk[j] = s.tk[(size_t)j];
        a.ntq = (int)s.tqs.size();
        for (int i = 0; i < a.ntq; i++) {
            a.tq[i] = s.tqs[(size_t)i];
            a.tau0[i] = s.tau0[i];
            a.tau1[i] = s.tau1[i];
            a.par[i] = s.par[i];
        }
        a.g = s.m == 2 ? s.g : 0;
        a.rhoc = s.rhoc;
        for (int b = 0; b < 2; b++)
            for (int x = 0; x < 2; x++) { a.Mr[b][x] = s.Mr[b][x]; a.Mi[b][x] = s.Mi[b][x]; }
        a.nk = s.nk;
        a.k = k;
        a.m = s.m;
        E.args[(size_t)k] = a;
    }
    apply_coeffs(E);
    size_t maxgrid = 1;
    E.lw.resize((size_t)p.ns);
    E.ln.resize((size_t)p.ns);
    for (int k = 0; k < p.ns; k++) {
        E.lw[(size_t)k] = E.shape(E.args[(size_t)k], true);
        E.ln[(size_t)k] = E.shape(E.args[(size_t)k], false);
        maxgrid = std::max(maxgrid, (size_t)std::max(E.lw[(size_t)k].grid, E.ln[(size_t)k].grid));
    }
    maxgrid = std::max(maxgrid, (size_t)E.sms * 8);
    GSB_CK(cudaMalloc(&E.partials, maxgrid * 8 * sizeof(double)));   // up to 6 sums per block (fused groups)
    GSB_CK(cudaMalloc(&E.d_args, (size_t)std::max(1, p.ns) * sizeof(StepArgs)));
    E.args_dirty = true;
    return 0;
}

// Whether a step's branch norms are exact functions of M (one coset offset, x = 0 and x = 1 terms in different
// outputs): n(b) = (|M[b][0]|^2 + |M[b][1]|^2) |T|^2.
static bool analytic_step(const HStep &hs) {
    return hs.tqs.size() == 1 && hs.m == 2 && hs.tau1[0] == 1 - hs.tau0[0];
}

// Group arguments of a fused pass from the host derivation and the steps' descriptors.  The pass writes stage gp.ws;
// with gp.ws = gp.d - 1 the last step is the trailing norm step.
static bool fill_group(Engine &E, const GroupPlan &gp, Op &op, int lcap = GROUP_MAX_L, int minb = 2, int ws_req = -1) {
    const HPlan &p = E.plan;
    const int D = gp.ws, TR = gp.d - gp.ws;
    if (gp.stage_size[0] > 32 || gp.stage_size[D] > 32) return false;
    if (minb != 2 && (minb != 3 || E.prec != 64 || E.arith != 32)) return false;
    // Canonical offset order per step (the kernel's compile-time dataflow shapes, GK_*): for m = 2 with every x = 1
    // term in the other output than its offset's x = 0 term, offsets whose x = 0 term goes to output 0 come first,
    // and the outputs are relabelled when more than half go to output 1.  Other steps keep their order (GK_ANY).
    GroupPlan::Step cs[FUSE_MAX_STEPS];
    int kinds[FUSE_MAX_STEPS], perm[FUSE_MAX_STEPS][4], swp[FUSE_MAX_STEPS];
    for (int s = 0; s < gp.d; s++) {
        const HStep &hs = p.st[(size_t)(gp.k0 + s)];
        const GroupPlan::Step &g = gp.step[s];
        bool shaped = g.m == 2;
        int h = 0;
        for (int t = 0; t < g.ntq; t++) {
            shaped = shaped && hs.tau1[t] == 1 - hs.tau0[t];
            h += hs.tau0[t];
        }
        swp[s] = shaped && 2 * h > g.ntq;
        if (swp[s]) h = g.ntq - h;
        int n = 0;
        for (int pass = 0; pass < 2; pass++)
            for (int t = 0; t < g.ntq; t++)
                if (!shaped ? pass == 0 : ((hs.tau0[t] ^ swp[s]) == pass)) perm[s][n++] = t;
        kinds[s] = GK_ANY;
        if (shaped) {
            if (g.ntq == 1 && h == 0) kinds[s] = GK_1_0;
            else if (g.ntq == 2) kinds[s] = h == 0 ? GK_2_0 : GK_2_1;
            else if (g.ntq == 4) kinds[s] = h == 0 ? GK_4_0 : h == 1 ? GK_4_1 : GK_4_2;
        }
        cs[s] = g;
        for (int j = 0; j < g.nmem; j++) {
            for (int t = 0; t < g.ntq; t++) cs[s].in_idx[j][t] = g.in_idx[j][perm[s][t]];
            if (swp[s]) std::swap(cs[s].out_idx[j][0], cs[s].out_idx[j][1]);
        }
    }
    // Folded sampling pass (GroupArgs::fold): two written steps whose second is a one-offset growth step of the
    // factored complex64 form for both bits, then a shaped trailing step.  The trailing step then reads stage 1
    // through the growth step's map, and the written stage needs no shared memory.
    bool fold = false;
    if (E.prec == 64 && E.arith == 32 && minb == 2 && D == 2 && TR == 1 && kinds[1] == GK_1_0 && kinds[2] != GK_ANY) {
        const Engine::Coef32 &cg = E.c32[(size_t)(gp.k0 + 1)];
        fold = cg.piv[0] >= 0 && cg.piv[1] >= 0;
    }
    // trailing member j, offset t reads written-stage index i = in_idx[j][t]: the growth step's member m with
    // out_idx[m][tau] = i, whose input is stage-1 index in_idx[m][0]
    unsigned char fsrc[16][4] = {}, ftau[16][4] = {}, fmem[16][4] = {};
    if (fold) {
        const GroupPlan::Step &g1 = cs[1], &g2 = cs[2];
        for (int j2 = 0; j2 < g2.nmem && fold; j2++)
            for (int t = 0; t < g2.ntq && fold; t++) {
                const int i2 = g2.in_idx[j2][t];
                int found = -1, tau_f = 0;
                for (int m = 0; m < g1.nmem && found < 0; m++)
                    for (int tau = 0; tau < 2; tau++)
                        if (g1.out_idx[m][tau] == i2) { found = m; tau_f = tau; break; }
                if (found < 0) { fold = false; break; }   // not a value the growth step writes: leave it unfolded
                fsrc[j2][t] = (unsigned char)g1.in_idx[found][0];
                ftau[j2][t] = (unsigned char)tau_f;
                fmem[j2][t] = (unsigned char)found;
            }
    }
    // tile size: the largest 2^L classes whose pipeline buffers fit the budget (6 <= L: a warp needs 32 class pairs)
    auto smem_at = [&](int L) -> uint32_t {
        const int ssz[4] = {gp.stage_size[0], gp.stage_size[1], gp.stage_size[2], gp.stage_size[3]};
        if (E.prec == 128) return group_smem_bytes<double2, double>(D, TR, ssz, L);
        if (E.arith == 64) return group_smem_bytes<float2, double>(D, TR, ssz, L);
        return group_smem_bytes<float2, float>(D, TR, ssz, L, fold);
    };
    int L = std::min(gp.L, std::min(lcap, GROUP_MAX_L));
    const uint32_t pref = minb == 3 ? GROUP_SMEM_3 : GROUP_SMEM_PREF, budget = minb == 3 ? GROUP_SMEM_3 : GROUP_SMEM_BUDGET;
    while (L > 6 && smem_at(L) > pref) L--;
    if (smem_at(L) > budget || L < 6) return false;
    GroupArgs &ga = op.ga;
    memset(&ga, 0, sizeof ga);
    ga.d = gp.d;
    ga.L = L;
    std::vector<uint64_t> bhi;
    for (int j = L; j < gp.L; j++) bhi.push_back(1ULL << j);    // low unit vectors beyond the tile
    bhi.insert(bhi.end(), gp.bhi.begin(), gp.bhi.end());
    if (bhi.size() > 30) return false;                           // tile index fits 32 bits with room
    ga.nbhi = (int)bhi.size();
    for (size_t j = 0; j < bhi.size(); j++) ga.bhi[j] = bhi[j];
    for (int s = 0; s <= gp.d; s++) ga.ssz[s] = gp.stage_size[s];
    {
        const GroupPlan::Step &g0 = cs[0], &gd = cs[gp.ws - 1];
        const uint64_t mask = (1ULL << L) - 1;
        for (size_t i = 0; i < gp.z_in.size(); i++) ga.blk_in[i] = gp.z_in[i] & ~mask;
        for (size_t i = 0; i < gp.z_out.size(); i++) ga.blk_out[i] = gp.z_out[i] & ~mask;
        for (int j = 0; j < g0.nmem; j++)
            for (int t = 0; t < g0.ntq; t++) ga.z0lo[j][t] = (uint32_t)(gp.z_in[(size_t)g0.in_idx[j][t]] & mask);
        for (int j = 0; j < gd.nmem; j++)
            for (int tau = 0; tau < gd.m; tau++) ga.zdlo[j][tau] = (uint32_t)(gp.z_out[(size_t)gd.out_idx[j][tau]] & mask);
    }
    for (int s = 0; s < gp.d; s++) {
        const HStep &hs = p.st[(size_t)(gp.k0 + s)];
        const GroupPlan::Step &g = cs[s];
        GroupStepArgs &a = ga.st[s];
        a.nmem = g.nmem;
        a.ntq = g.ntq;
        a.m = g.m;
        a.k = gp.k0 + s;
        a.kind = kinds[s];
        a.lambda = g.lambda;
        for (int t = 0; t < g.ntq; t++) {
            a.tau0[t] = hs.tau0[perm[s][t]] ^ swp[s];
            a.tau1[t] = hs.tau1[perm[s][t]] ^ swp[s];
            a.par[t] = hs.par[perm[s][t]];
        }
        const Engine::Coef32 &cf = E.c32[(size_t)(gp.k0 + s)];
        for (int b = 0; b < 2; b++) {
            for (int x = 0; x < 2; x++) { a.Mr[b][x] = cf.Mr[b][x]; a.Mi[b][x] = cf.Mi[b][x]; }
            a.c[b] = hs.Mr[b][0] * hs.Mr[b][0] + hs.Mi[b][0] * hs.Mi[b][0] + hs.Mr[b][1] * hs.Mr[b][1] +
                     hs.Mi[b][1] * hs.Mi[b][1];
            // factored form of a written complex64 step (FP32 arithmetic, compile-time shapes only)
            const bool fact = kinds[s] != GK_ANY && cf.piv[b] >= 0;
            a.piv[b] = fact ? cf.piv[b] : -1;
            a.br[b] = fact ? cf.br[b] : 0;
            a.bi[b] = fact ? cf.bi[b] : 0;
            a.cp[b] = fact ? cf.cp[b] : 1;
        }
        for (int j = 0; j < g.nmem; j++) {
            for (int t = 0; t < g.ntq; t++) {
                a.in_idx[j][t] = (unsigned char)g.in_idx[j][t];
                a.ioff[j][t] = ((uint32_t)g.in_idx[j][t] << L) | (s == 0 ? ga.z0lo[j][t] : 0u);
            }
            for (int tau = 0; tau < g.m; tau++) {
                a.out_idx[j][tau] = (unsigned char)g.out_idx[j][tau];
                a.soff[j][tau] = (uint32_t)g.out_idx[j][tau] << L;
            }
            a.mpar[j] = (unsigned char)g.mpar[j];
        }
    }
    {
        const GroupPlan::Step &gd = cs[gp.ws - 1];
        for (int j = 0; j < gd.nmem; j++)
            for (int tau = 0; tau < gd.m; tau++) ga.ooff[j][tau] = gp.z_out[(size_t)gd.out_idx[j][tau]];
    }
    if (fold) {
        // mode 2 when every trailing member reads one growth output in all its offsets
        bool uni = true;
        for (int j2 = 0; j2 < cs[2].nmem; j2++)
            for (int t = 1; t < cs[2].ntq; t++) uni = uni && ftau[j2][t] == ftau[j2][0];
        ga.fold = uni ? 2 : 1;
        memcpy(ga.fsrc, fsrc, sizeof fsrc);
        memcpy(ga.ftau, ftau, sizeof ftau);
        memcpy(ga.fmem, fmem, sizeof fmem);
    }
    op.group = true;
    op.k0 = gp.k0;
    op.d = gp.ws;
    op.tr = gp.d - gp.ws;
    op.lcap = lcap;
    op.minb = minb;
    op.smem = smem_at(L);
    op.ntiles = 1u << ga.nbhi;
    // The warp-specialised build needs complex64 FP32 and tiles of 2^9 classes or more (a step thread's class pairs
    // then are the same in every step).  By default the chain passes take it (complex64 chain 9.77 -> 9.29 ms per
    // string of pass time on the headline plan); the sampling passes measured even with it (18.88 vs 18.89 ms, some
    // passes faster, the folded ones 3 % slower), so there the autotuner times both.
    const bool ws_ok = E.prec == 64 && E.arith == 32 && minb == 2 && L >= 9;
    if (ws_req == 1 && !ws_ok) return false;
    const bool ws = ws_ok && (ws_req < 0 ? TR == 0 : ws_req == 1);
    op.ws = ws ? 1 : 0;
    op.threads = ws ? GROUP_NCT + 32 : GROUP_NCT;
    if (E.prec == 128) op.fn = pick_group<double2, double>(op.d, op.tr);
    else if (E.arith == 64) op.fn = pick_group<float2, double>(op.d, op.tr);
    else if (minb == 3) op.fn = pick_group3(op.d, op.tr);
    else if (ws) op.fn = pick_group_ws(op.d, op.tr);
    else op.fn = pick_group_f32(op.d, op.tr);
    if (cudaFuncSetAttribute(op.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GROUP_SMEM_BUDGET) != cudaSuccess)
        return false;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, op.fn, op.threads, op.smem) != cudaSuccess || nb < 1) nb = 1;
    op.grid = (int)std::min<uint64_t>(op.ntiles, (uint64_t)nb * E.sms);
    op.entries = gp.entries_moved;
    return true;
}

static double single_entries(const HPlan &p, int k) {
    const HStep &hs = p.st[(size_t)k];
    const int r = hs.nk + (hs.tqs.size() == 4 ? 2 : hs.tqs.size() == 2 ? 1 : 0);
    return std::ldexp(1.0, r) + std::ldexp(1.0, hs.nk + (hs.m == 2 ? 1 : 0));
}

// The pass of a shape with the engine's current matrices; false when the group cannot be built.
static bool make_op(Engine &E, const OpShape &sh, Op &op) {
    op = Op();
    if (!sh.group) {
        op.k0 = sh.k0;
        op.d = 1;
        op.entries = single_entries(E.plan, sh.k0);
        return true;
    }
    GroupPlan gp;
    if (!plan_group(E.plan, sh.k0, sh.d + sh.tr, 6, sh.lcap, gp, sh.d) || !fill_group(E, gp, op, sh.lcap, sh.minb, sh.ws))
        return false;
    op.norm_first = sh.norm_first;
    op.ga.src = sh.src;
    return true;
}

static bool ops_from_shapes(Engine &E, const std::vector<OpShape> &shapes, std::vector<Op> &ops) {
    std::vector<Op> out;
    for (const OpShape &sh : shapes) {
        Op op;
        if (!make_op(E, sh, op)) return false;
        out.push_back(op);
    }
    ops.swap(out);
    return true;
}

// Sampling pass list ('prob' / 'sample'): the cheapest cover of the steps, by table entries moved, with
//   * single steps: norm pass + write pass (read, read, write);
//   * fused passes of steps k .. k+d-1 (k+1 .. k+d-1 analytic, so their bits need no data), optionally with the
//     branch norms of step k+d (trailing, tr = 1; at most 3 steps evaluated in one pass).  Step k's bit comes from
//     the previous pass's trailing norms, from M when step k is analytic, or else from a norm pass launched first.
static void build_sample_ops(Engine &E) {
    E.sample_ops.clear();
    if (!E.sample_shapes.empty() && ops_from_shapes(E, E.sample_shapes, E.sample_ops)) return;
    if (E.fuse_depth < 2) return;
    const HPlan &p = E.plan;
    const int ns = p.ns;
    auto rof = [&](int k) { const HStep &h = p.st[(size_t)k]; return h.nk + (h.tqs.size() == 4 ? 2 : h.tqs.size() == 2 ? 1 : 0); };
    auto size_in = [&](int k) { return k < ns ? std::ldexp(1.0, rof(k)) : 0.0; };
    auto size_out = [&](int k) { const HStep &h = p.st[(size_t)k]; return std::ldexp(1.0, h.nk + (h.m == 2 ? 1 : 0)); };
    const double INF = 1e300;
    // cost[k][t]: entries moved from step k on, t = step k's trailing norms are available
    std::vector<std::array<double, 2>> cost((size_t)ns + 1, {INF, INF});
    std::vector<std::array<Op, 2>> best((size_t)ns + 1);
    cost[(size_t)ns] = {0, 0};
    for (int k = ns - 1; k >= 0; k--) {
        const bool an = analytic_step(p.st[(size_t)k]);
        for (int t = 0; t < 2; t++) {
            // single step: norm pass + write pass
            Op single;
            single.k0 = k;
            double c = 2 * size_in(k) + size_out(k) + cost[(size_t)k + 1][0];
            Op pick = single;
            if (rof(k) >= GROUP_MIN_R) {
                for (int d = 1; d <= FUSE_MAX_STEPS; d++) {
                    if (k + d > ns) break;
                    if (d > 1 && !analytic_step(p.st[(size_t)(k + d - 1)])) break;
                    for (int tr = 0; tr < 2; tr++) {
                        if (d + tr < 2 || d + tr > FUSE_MAX_STEPS) continue;
                        if (tr && (k + d >= ns || analytic_step(p.st[(size_t)(k + d)]))) continue;
                        const bool nf = !an && !t;
                        const double cc = (nf ? size_in(k) : 0) + size_in(k) + size_out(k + d - 1) + cost[(size_t)(k + d)][tr];
                        if (cc >= c) continue;
                        GroupPlan gp;
                        Op op;
                        if (!plan_group(p, k, d + tr, 6, GROUP_MAX_L, gp, d) || !fill_group(E, gp, op)) continue;
                        op.norm_first = nf;
                        op.ga.src = an ? GSRC_ANALYTIC : t ? GSRC_TRAILING : GSRC_NORM;
                        c = cc;
                        pick = op;
                    }
                }
            }
            cost[(size_t)k][(size_t)t] = c;
            best[(size_t)k][(size_t)t] = pick;
        }
    }
    for (int k = 0, t = 0; k < ns;) {
        const Op &op = best[(size_t)k][(size_t)t];
        E.sample_ops.push_back(op);
        t = op.group ? op.tr : 0;
        k += op.group ? op.d : 1;
    }
}

// Chain-mode pass list: wide steps fused greedily into groups of up to fuse_depth steps.
// The fused 'chain' passes of steps 0 .. hyb_K - 1 (groups do not cross hyb_K), for hybrid strings whose first
// hyb_K steps are forced.
static void build_hyb_ops(Engine &E) {
    E.hyb_ops.clear();
    const HPlan &p = E.plan;
    for (int k = 0; k < E.hyb_K;) {
        const HStep &hs = p.st[(size_t)k];
        const int r = hs.nk + (hs.tqs.size() == 4 ? 2 : hs.tqs.size() == 2 ? 1 : 0);
        bool done = false;
        if (E.fuse_depth >= 2 && r >= GROUP_MIN_R) {
            for (int d = std::min(std::min(E.fuse_depth, FUSE_MAX_STEPS), E.hyb_K - k); d >= 2 && !done; d--) {
                GroupPlan gp;
                if (!plan_group(p, k, d, 6, GROUP_MAX_L, gp)) continue;
                Op op;
                if (!fill_group(E, gp, op)) continue;
                E.hyb_ops.push_back(op);
                k += d;
                done = true;
            }
        }
        if (!done) {
            Op op;
            op.k0 = k;
            op.d = 1;
            E.hyb_ops.push_back(op);
            k++;
        }
    }
}

static void build_chain_ops(Engine &E) {
    build_hyb_ops(E);
    build_sample_ops(E);
    E.chain_ops.clear();
    if (!E.chain_shapes.empty() && ops_from_shapes(E, E.chain_shapes, E.chain_ops)) return;
    const HPlan &p = E.plan;
    for (int k = 0; k < p.ns;) {
        const HStep &hs = p.st[(size_t)k];
        const int r = hs.nk + (hs.tqs.size() == 4 ? 2 : hs.tqs.size() == 2 ? 1 : 0);
        bool done = false;
        if (E.fuse_depth >= 2 && r >= GROUP_MIN_R) {
            for (int d = std::min(E.fuse_depth, FUSE_MAX_STEPS); d >= 2 && !done; d--) {
                GroupPlan gp;
                if (!plan_group(p, k, d, 6, GROUP_MAX_L, gp)) continue;
                Op op;
                if (!fill_group(E, gp, op)) continue;
                E.chain_ops.push_back(op);
                k += d;
                done = true;
            }
        }
        if (!done) {
            Op op;
            op.k0 = k;
            op.d = 1;
            const double r1 = (double)(1ULL << r), r2 = (double)(1ULL << (hs.nk + (hs.m == 2 ? 1 : 0)));
            op.entries = r1 + r2;
            E.chain_ops.push_back(op);
            k++;
        }
    }
}

static int open_plan(const char *text, size_t len, int precision, int device, gsb_engine **out) {
    if (!out) return fail(GSB_E_USAGE, "null output handle");
    *out = nullptr;
    if (precision != 64 && precision != 128) return fail(GSB_E_USAGE, "precision must be 64 or 128");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(GSB_E_CUDA, "no CUDA device is visible");
    if (device < 0 || device >= ndev) return fail(GSB_E_USAGE, "device index out of range");
    Engine *E = new Engine();
    E->prec = precision;
    E->esize = precision == 128 ? 16 : 8;
    E->dev = device;
    std::string err;
    int rc = parse_plan_text(text, len, E->plan, err);
    if (!rc) rc = validate_plan(E->plan, err);
    if (rc) { delete E; return fail(rc, err); }
    DevGuard g(device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { delete E; return fail(GSB_E_CUDA, "cudaGetDeviceProperties failed"); }
    E->sms = prop.multiProcessorCount;
    auto cuda_fail = [&](cudaError_t e, const char *what) {
        delete E;
        return fail(GSB_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e = cudaStreamCreateWithFlags(&E->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "stream");
    E->stream = E->own_stream;
    const size_t arena = ((size_t)1 << E->plan.R) * E->esize;
    e = cudaMalloc(&E->mem, arena);
    if (e != cudaSuccess) {
        cudaGetLastError();
        char b[160];
        snprintf(b, sizeof b, "allocation of %zu bytes for the 2^%d arena failed", arena, E->plan.R);
        delete E;
        return fail(GSB_E_ALLOC, b);
    }
    e = cudaMemsetAsync(E->mem, 0, arena, E->stream);
    if (e != cudaSuccess) return cuda_fail(e, "arena clear");
    const size_t ns = (size_t)std::max(1, E->plan.ns), cap = (size_t)E->cap;
    if ((e = cudaMalloc(&E->st, sizeof(DevState))) != cudaSuccess) return cuda_fail(e, "state");
    if ((e = cudaMemsetAsync(E->st, 0, sizeof(DevState), E->stream)) != cudaSuccess) return cuda_fail(e, "state");
    if ((e = cudaMalloc(&E->d_forced, cap * ns)) != cudaSuccess) return cuda_fail(e, "buffers");
    if ((e = cudaMalloc(&E->d_bits, cap * ns)) != cudaSuccess) return cuda_fail(e, "buffers");
    if ((e = cudaMalloc(&E->d_unif, cap * ns * 8)) != cudaSuccess) return cuda_fail(e, "buffers");
    if ((e = cudaMalloc(&E->d_cond, cap * ns * 8)) != cudaSuccess) return cuda_fail(e, "buffers");
    if ((e = cudaMalloc(&E->d_logp, cap * 8)) != cudaSuccess) return cuda_fail(e, "buffers");
    if ((e = cudaMalloc(&E->d_aux, cap * 8)) != cudaSuccess) return cuda_fail(e, "buffers");
    if ((e = cudaMemsetAsync(E->d_forced, 0, cap * ns, E->stream)) != cudaSuccess) return cuda_fail(e, "buffers");
    rc = make_args(*E);
    if (rc) { std::string m = g_err; delete E; return fail(rc, m); }
    build_chain_ops(*E);
    if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return cuda_fail(e, "set-up");
    *out = reinterpret_cast<gsb_engine *>(E);
    return 0;
}

static Engine *eng(gsb_engine *e) { return reinterpret_cast<Engine *>(e); }
static const Engine *eng(const gsb_engine *e) { return reinterpret_cast<const Engine *>(e); }

// uniforms of one 'sample'/'sample2' stream item: one draw per step, in step order (gsamp2.cpp:46-47,151,159-160)
static void sample_uniforms(int seeding, uint64_t seed, uint64_t i, int ns, double *u) {
    std::uniform_real_distribution<double> U(0, 1);
    if (seeding == GSB_SEED_SEQ) {
        std::seed_seq sq{(unsigned)(seed & 0xffffffffu), (unsigned)(seed >> 32), (unsigned)(i & 0xffffffffu),
                         (unsigned)(i >> 32), 0x9E3779B9u};
        std::mt19937_64 rng(sq);
        for (int k = 0; k < ns; k++) u[k] = U(rng);
    } else {
        std::mt19937_64 rng(seed + i);
        for (int k = 0; k < ns; k++) u[k] = U(rng);
    }
}

// uniforms of a hybrid / resume line: one draw per '?' step from k0 on, in step order (gsamp2.cpp:86, 206, 215)
static void free_uniforms(uint64_t seed, const int8_t *forced, int k0, int ns, double *u) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(0, 1);
    for (int k = 0; k < ns; k++) u[k] = 0;
    for (int k = k0; k < ns; k++)
        if (forced[k] < 0) u[k] = U(rng);
}

}  // namespace gsb

using namespace gsb;

extern "C" {

const char *gsb_version(void) { return "gsb 0.1 (sm_100a)"; }
const char *gsb_last_error(void) { return g_err.c_str(); }

int gsb_open_text(const char *plan_text, size_t len, int precision, int device, gsb_engine **out) {
    if (!plan_text) return fail(GSB_E_USAGE, "null plan text");
    return open_plan(plan_text, len, precision, device, out);
}

int gsb_validate_text(const char *plan_text, size_t len, int *n, int *nsteps, int *R) {
    if (!plan_text) return fail(GSB_E_USAGE, "null plan text");
    HPlan p;
    std::string err;
    int rc = parse_plan_text(plan_text, len, p, err);
    if (!rc) rc = validate_plan(p, err);
    if (rc) return fail(rc, err);
    if (n) *n = p.n;
    if (nsteps) *nsteps = p.ns;
    if (R) *R = p.R;
    return 0;
}

int gsb_open_file(const char *plan_path, int precision, int device, gsb_engine **out) {
    if (!plan_path) return fail(GSB_E_USAGE, "null plan path");
    FILE *f = fopen(plan_path, "rb");
    if (!f) return fail(GSB_E_PLAN_HEADER, std::string("cannot open plan ") + plan_path);
    std::string text;
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    fclose(f);
    return open_plan(text.data(), text.size(), precision, device, out);
}

int gsb_close(gsb_engine *e) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    delete eng(e);
    return 0;
}

int gsb_info(const gsb_engine *e, int *n, int *nsteps, int *R, int *precision) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    const Engine *E = eng(e);
    if (n) *n = E->plan.n;
    if (nsteps) *nsteps = E->plan.ns;
    if (R) *R = E->plan.R;
    if (precision) *precision = E->prec;
    return 0;
}

int gsb_step_vertices(const gsb_engine *e, int *out) {
    if (!e || !out) return fail(GSB_E_USAGE, "null argument");
    const Engine *E = eng(e);
    for (int k = 0; k < E->plan.ns; k++) out[k] = E->plan.st[(size_t)k].v;
    return 0;
}

static int check_bits(const int8_t *b, int64_t n, int ns, bool allow_free) {
    for (int64_t i = 0; i < n * ns; i++)
        if (!(b[i] == 0 || b[i] == 1 || (allow_free && b[i] == -1)))
            return fail(GSB_E_USAGE, allow_free ? "bits must be 0, 1 or -1" : "bits must be 0 or 1");
    return 0;
}

// A fused pass whose tile loads did not complete within its bounded wait sets DevState::err and stops the item;
// report it (and clear it) after the work has been synchronised.
static int check_device(Engine *E) {
    int v = 0;
    GSB_CK(cudaMemcpy(&v, &E->st->err, sizeof v, cudaMemcpyDeviceToHost));
    if (!v) return 0;
    v = 0;
    GSB_CK(cudaMemcpy(&E->st->err, &v, sizeof v, cudaMemcpyHostToDevice));
    return fail(GSB_E_CUDA, "a fused pass gave up waiting for its tile loads; results of this call are invalid");
}

// forced-string batch through graph `kind` (0 chain, 1 prob)
static int forced_batch(Engine *E, int kind, const int8_t *bits, int64_t nstr, double *log2p, double *cond) {
    const int ns = E->plan.ns;
    for (int64_t off = 0; off < nstr; off += E->cap) {
        const int64_t nb = std::min<int64_t>(E->cap, nstr - off);
        if (ns) GSB_CK(cudaMemcpyAsync(E->d_forced, bits + off * ns, (size_t)(nb * ns), cudaMemcpyHostToDevice, E->stream));
        int rc = E->run_graph_items(kind, nb);
        if (rc) return rc;
        if (log2p) GSB_CK(cudaMemcpyAsync(log2p + off, E->d_logp, (size_t)nb * 8, cudaMemcpyDeviceToHost, E->stream));
        if (cond && ns) GSB_CK(cudaMemcpyAsync(cond + off * ns, E->d_cond, (size_t)(nb * ns) * 8, cudaMemcpyDeviceToHost, E->stream));
        GSB_CK(cudaStreamSynchronize(E->stream));
        if ((rc = check_device(E))) return rc;
    }
    return 0;
}

// ---- complex128 guard (gsb_set_guard) ----
// A complex64 log2 Pr carries a rounding error that grows as 1 / sqrt(Pr 2^ns) (the table's rounding is absolute
// in units of its norm, and an unlikely string's amplitude is a small remainder of it); strings below the guard's
// threshold are evaluated again by the complex128 engine, whose results replace the complex64 ones.
static void guard_pick(const Engine *E, const double *lp, int64_t n, std::vector<int64_t> &idx) {
    const double ns = E->plan.ns;
    for (int64_t i = 0; i < n; i++)
        if (!(lp[i] + ns >= E->guard_lx)) idx.push_back(i);   // -inf and NaN too
}

// host arrays: kind 0 (chain: log2 Pr and conditionals) or 1 (prob: log2 Pr)
static int guard_host(Engine *E, int kind, const int8_t *bits, int64_t nstr, double *log2p, double *cond) {
    if (!E->guard || nstr <= 0) return 0;
    std::vector<int64_t> idx;
    guard_pick(E, log2p, nstr, idx);
    if (idx.empty()) return 0;
    const int ns = E->plan.ns;
    const size_t m = idx.size(), nsz = (size_t)std::max(ns, 1);
    std::vector<int8_t> b(m * nsz);
    std::vector<double> lp(m), cd(cond ? m * nsz : 0);
    for (size_t j = 0; j < m; j++) memcpy(b.data() + j * nsz, bits + idx[j] * ns, (size_t)ns);
    Engine *G = E->guard;
    {
        DevGuard g(G->dev);
        int rc = forced_batch(G, kind, b.data(), (int64_t)m, lp.data(), cond ? cd.data() : nullptr);
        if (rc) return rc;
    }
    for (size_t j = 0; j < m; j++) {
        log2p[idx[j]] = lp[j];
        if (cond) memcpy(cond + idx[j] * ns, cd.data() + j * nsz, (size_t)ns * 8);
    }
    E->guard_evals += (int64_t)m;
    return 0;
}

// device arrays (the engines share a device): the strings' rows are copied to the guard, its results copied back
static int guard_device(Engine *E, int kind, const int8_t *d_bits, int64_t nstr, double *d_log2p, double *d_cond) {
    if (!E->guard || nstr <= 0) return 0;
    GSB_CK(cudaStreamSynchronize(E->stream));
    std::vector<double> lp((size_t)nstr);
    GSB_CK(cudaMemcpy(lp.data(), d_log2p, (size_t)nstr * 8, cudaMemcpyDeviceToHost));
    std::vector<int64_t> idx;
    guard_pick(E, lp.data(), nstr, idx);
    if (idx.empty()) return 0;
    Engine *G = E->guard;
    DevGuard g(G->dev);
    const int ns = E->plan.ns;
    for (size_t off = 0; off < idx.size(); off += (size_t)G->cap) {
        const size_t m = std::min(idx.size() - off, (size_t)G->cap);
        for (size_t j = 0; j < m && ns; j++)
            GSB_CK(cudaMemcpyAsync(G->d_forced + j * ns, d_bits + idx[off + j] * ns, (size_t)ns, cudaMemcpyDeviceToDevice,
                                   G->stream));
        int rc = G->run_graph_items(kind, (int64_t)m);
        if (rc) return rc;
        for (size_t j = 0; j < m; j++) {
            GSB_CK(cudaMemcpyAsync(d_log2p + idx[off + j], G->d_logp + j, 8, cudaMemcpyDeviceToDevice, G->stream));
            if (d_cond && ns)
                GSB_CK(cudaMemcpyAsync(d_cond + idx[off + j] * ns, G->d_cond + j * ns, (size_t)ns * 8,
                                       cudaMemcpyDeviceToDevice, G->stream));
        }
    }
    GSB_CK(cudaStreamSynchronize(G->stream));
    int rc = check_device(G);
    if (rc) return rc;
    E->guard_evals += (int64_t)idx.size();
    return 0;
}

static bool same_plan(const HPlan &a, const HPlan &b) {
    if (a.n != b.n || a.ns != b.ns || a.R != b.R || a.st.size() != b.st.size()) return false;
    for (size_t k = 0; k < a.st.size(); k++) {
        const HStep &x = a.st[k], &y = b.st[k];
        if (x.v != y.v || x.nk != y.nk || x.m != y.m || x.g != y.g || x.rhoc != y.rhoc || x.tk != y.tk ||
            x.t.size() != y.t.size())
            return false;
        for (size_t i = 0; i < x.t.size(); i++)
            if (x.t[i].tq != y.t[i].tq || x.t[i].x != y.t[i].x || x.t[i].tau != y.t[i].tau || x.t[i].par != y.t[i].par)
                return false;
        for (int r = 0; r < 2; r++)
            for (int c = 0; c < 2; c++)
                if (x.Mr[r][c] != y.Mr[r][c] || x.Mi[r][c] != y.Mi[r][c]) return false;
    }
    return true;
}

int gsb_prob(gsb_engine *e, const int8_t *bits, int64_t nstr, double *log2p) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (nstr < 0 || (nstr && (!bits || !log2p))) return fail(GSB_E_USAGE, "null argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    int rc = check_bits(bits, nstr, E->plan.ns, false);
    if (rc) return rc;
    if ((rc = forced_batch(E, 1, bits, nstr, log2p, nullptr))) return rc;
    return guard_host(E, 1, bits, nstr, log2p, nullptr);
}

int gsb_chain(gsb_engine *e, const int8_t *bits, int64_t nstr, double *log2p, double *cond) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (nstr < 0 || (nstr && (!bits || !log2p))) return fail(GSB_E_USAGE, "null argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    int rc = check_bits(bits, nstr, E->plan.ns, false);
    if (rc) return rc;
    if ((rc = forced_batch(E, 0, bits, nstr, log2p, cond))) return rc;
    return guard_host(E, 0, bits, nstr, log2p, cond);
}

static int uniform_batch(Engine *E, const double *u, int64_t count, int8_t *bits, double *log2p) {
    const int ns = E->plan.ns;
    for (int64_t off = 0; off < count; off += E->cap) {
        const int64_t nb = std::min<int64_t>(E->cap, count - off);
        if (ns) GSB_CK(cudaMemcpyAsync(E->d_unif, u + off * ns, (size_t)(nb * ns) * 8, cudaMemcpyHostToDevice, E->stream));
        int rc = E->run_graph_items(2, nb);
        if (rc) return rc;
        if (log2p) GSB_CK(cudaMemcpyAsync(log2p + off, E->d_logp, (size_t)nb * 8, cudaMemcpyDeviceToHost, E->stream));
        if (bits && ns) GSB_CK(cudaMemcpyAsync(bits + off * ns, E->d_bits, (size_t)(nb * ns), cudaMemcpyDeviceToHost, E->stream));
        GSB_CK(cudaStreamSynchronize(E->stream));
        if ((rc = check_device(E))) return rc;
        // guarded: the log2 Pr of an unlikely sample again in complex128 (its bits are the complex64 draw's)
        if (bits && log2p && (rc = guard_host(E, 0, bits + off * ns, nb, log2p + off, nullptr))) return rc;
    }
    return 0;
}

int gsb_sample_uniform(gsb_engine *e, const double *u, int64_t count, int8_t *bits, double *log2p) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (count < 0 || (count && (!u || !bits || !log2p))) return fail(GSB_E_USAGE, "null argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    return uniform_batch(E, u, count, bits, log2p);
}

int gsb_sample(gsb_engine *e, int seeding, uint64_t seed, int64_t first, int64_t count, int8_t *bits, double *log2p) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (seeding != GSB_SEED_INT && seeding != GSB_SEED_SEQ) return fail(GSB_E_USAGE, "unknown seeding");
    if (count < 0 || first < 0 || (count && (!bits || !log2p))) return fail(GSB_E_USAGE, "bad argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    const int ns = E->plan.ns;
    std::vector<double> u((size_t)std::max<int64_t>(1, std::min<int64_t>(count, E->cap)) * (size_t)std::max(ns, 1));
    for (int64_t off = 0; off < count; off += E->cap) {
        const int64_t nb = std::min<int64_t>(E->cap, count - off);
        for (int64_t i = 0; i < nb; i++) sample_uniforms(seeding, seed, (uint64_t)(first + off + i), ns, u.data() + i * ns);
        int rc = uniform_batch(E, u.data(), nb, bits + off * ns, log2p + off);
        if (rc) return rc;
    }
    return 0;
}

int gsb_hybrid(gsb_engine *e, const int8_t *forced, int64_t nstr, uint64_t seed, int64_t first_line, int8_t *bits,
               double *log2p, double *cond) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (nstr < 0 || (nstr && (!forced || !bits || !log2p))) return fail(GSB_E_USAGE, "null argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    const int ns = E->plan.ns;
    int rc = check_bits(forced, nstr, ns, true);
    if (rc) return rc;
    for (int64_t i = 0; i < nstr; i++)
        for (int k = 0; k < E->hyb_K; k++)
            if (forced[i * ns + k] < 0) return fail(GSB_E_PREFIX_FREE, "'?' before the forced prefix set by gsb_set_hybrid_prefix");
    std::vector<double> u((size_t)std::max<int64_t>(1, std::min<int64_t>(nstr, E->cap)) * (size_t)std::max(ns, 1));
    for (int64_t off = 0; off < nstr; off += E->cap) {
        const int64_t nb = std::min<int64_t>(E->cap, nstr - off);
        for (int64_t i = 0; i < nb; i++)
            free_uniforms(seed + (uint64_t)(first_line + off + i), forced + (off + i) * ns, 0, ns, u.data() + i * ns);
        if (ns) {
            GSB_CK(cudaMemcpyAsync(E->d_forced, forced + off * ns, (size_t)(nb * ns), cudaMemcpyHostToDevice, E->stream));
            GSB_CK(cudaMemcpyAsync(E->d_unif, u.data(), (size_t)(nb * ns) * 8, cudaMemcpyHostToDevice, E->stream));
        }
        rc = E->run_graph_items(3, nb);
        if (rc) return rc;
        GSB_CK(cudaMemcpyAsync(log2p + off, E->d_logp, (size_t)nb * 8, cudaMemcpyDeviceToHost, E->stream));
        if (ns) GSB_CK(cudaMemcpyAsync(bits + off * ns, E->d_bits, (size_t)(nb * ns), cudaMemcpyDeviceToHost, E->stream));
        if (cond && ns) GSB_CK(cudaMemcpyAsync(cond + off * ns, E->d_cond, (size_t)(nb * ns) * 8, cudaMemcpyDeviceToHost, E->stream));
        GSB_CK(cudaStreamSynchronize(E->stream));
        if ((rc = check_device(E))) return rc;
    }
    return 0;
}

int gsb_dump_shape(const gsb_engine *e, int K, int *nk, int *ntq) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    const Engine *E = eng(e);
    if (K < 0) return fail(GSB_E_USAGE, "K must be >= 0");
    if (K >= E->plan.ns) {
        if (nk) *nk = 0;
        if (ntq) *ntq = 1;
    } else {
        if (nk) *nk = E->plan.st[(size_t)K].nk;
        if (ntq) *ntq = (int)E->plan.st[(size_t)K].tqs.size();
    }
    return 0;
}

static StepArgs dump_args(const Engine *E, int K) {
    if (K < E->plan.ns) return E->args[(size_t)K];
    StepArgs a;
    memset(&a, 0, sizeof a);
    a.ntq = 1;
    return a;
}

static int ensure_dump(Engine *E, size_t bytes) {
    if (E->dump_bytes >= bytes) return 0;
    cudaFree(E->d_dump);
    E->d_dump = nullptr;
    E->dump_bytes = 0;
    cudaError_t e = cudaMalloc(&E->d_dump, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(GSB_E_ALLOC, "allocation of the dump buffer failed"); }
    E->dump_bytes = bytes;
    return 0;
}

int gsb_prefix(gsb_engine *e, const int8_t *forced, int K, void *dump, double *logscale, double *log2p_prefix) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    Engine *E = eng(e);
    const int ns = E->plan.ns;
    if (!forced || K < 0) return fail(GSB_E_USAGE, "bad argument");
    for (int k = 0; k < std::min(K, ns); k++)
        if (forced[k] < 0) return fail(GSB_E_PREFIX_FREE, "'?' before K in prefix mode");
        else if (forced[k] > 1) return fail(GSB_E_USAGE, "bits must be 0 or 1");
    DevGuard g(E->dev);
    const int Kr = std::min(K, ns);
    std::vector<int8_t> row((size_t)std::max(ns, 1), 0);
    for (int k = 0; k < Kr; k++) row[(size_t)k] = forced[k];
    if (ns) GSB_CK(cudaMemcpyAsync(E->d_forced, row.data(), (size_t)ns, cudaMemcpyHostToDevice, E->stream));
    k_set_item<<<1, 1, 0, E->stream>>>(E->st, 0);
    GSB_CK(E->launch_begin());
    for (int k = 0; k < Kr; k++) GSB_CK(E->launch_step(k, true, DRV_HYBRID, Kr, true, false));
    if (dump) {   // dump == NULL: only the prefix probability (a marginal) is wanted
        int nk, ntq;
        gsb_dump_shape(e, K, &nk, &ntq);
        const size_t nent = ((size_t)1 << nk) * (size_t)ntq, bytes = nent * E->esize;
        int rc = ensure_dump(E, bytes);
        if (rc) return rc;
        StepArgs a = dump_args(E, K);
        const int grid = (int)std::min<size_t>((nent + 255) / 256, (size_t)E->sms * 8);
        if (E->prec == 128) k_gather<double2><<<grid, 256, 0, E->stream>>>(a, (const double2 *)E->mem, ntq, (double2 *)E->d_dump);
        else k_gather<float2><<<grid, 256, 0, E->stream>>>(a, (const float2 *)E->mem, ntq, (float2 *)E->d_dump);
        GSB_CK(cudaGetLastError());
        GSB_CK(cudaMemcpyAsync(dump, E->d_dump, bytes, cudaMemcpyDeviceToHost, E->stream));
    }
    DevState hs;
    GSB_CK(cudaMemcpyAsync(&hs, E->st, sizeof hs, cudaMemcpyDeviceToHost, E->stream));
    GSB_CK(cudaStreamSynchronize(E->stream));
    if (logscale) *logscale = hs.logscale;
    if (log2p_prefix) *log2p_prefix = hs.logp;
    return 0;
}

int gsb_resume(gsb_engine *e, const int8_t *forced, int K, uint64_t seed, int64_t line, int nslices,
               const void *const *dumps, const double *logscales, const uint64_t *cshift, const uint64_t *tqshift,
               int8_t *bits, double *log2p_full, double *log2p_prefix, double *cond) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    Engine *E = eng(e);
    const int ns = E->plan.ns;
    if (!forced || !dumps || !logscales || !bits || !log2p_full || nslices < 1 || K < 0) return fail(GSB_E_USAGE, "bad argument");
    for (int s = 0; s < nslices; s++)
        if (!dumps[s]) return fail(GSB_E_DUMP_MISSING, "missing dump table");
    int rc = check_bits(forced, 1, ns, true);
    if (rc) return rc;
    DevGuard g(E->dev);
    int nk, ntq;
    gsb_dump_shape(e, K, &nk, &ntq);
    const StepArgs a = dump_args(E, K);
    // twist translation (gsamp2.cpp:184-195)
    std::vector<uint64_t> cs((size_t)nslices, 0);
    std::vector<int> tperm((size_t)nslices * 4, 0);
    for (int s = 0; s < nslices; s++) {
        if (cshift) {
            if (cshift[s] >> nk) return fail(GSB_E_TWIST_RANGE, "twist cshift exceeds the kept coordinates");
            cs[(size_t)s] = cshift[s];
        }
        for (int t = 0; t < ntq; t++) {
            int pos = t;
            if (tqshift) {
                pos = -1;
                for (int u = 0; u < ntq; u++)
                    if (a.tq[u] == (a.tq[t] ^ tqshift[s])) pos = u;
                if (pos < 0) return fail(GSB_E_TWIST_RANGE, "twist tqshift does not map the coset offsets of step K onto themselves");
            }
            tperm[(size_t)s * 4 + (size_t)t] = pos;
        }
    }
    double L = -1e300;
    for (int s = 0; s < nslices; s++) L = std::max(L, logscales[s]);
    std::vector<double> f((size_t)nslices);
    for (int s = 0; s < nslices; s++) f[(size_t)s] = std::exp2(logscales[s] - L);
    const size_t nent = ((size_t)1 << nk) * (size_t)ntq, tbytes = nent * E->esize;
    // device copies: slice tables back to back, then the small arrays
    rc = ensure_dump(E, tbytes * (size_t)nslices);
    if (rc) return rc;
    std::vector<const void *> dptr((size_t)nslices);
    for (int s = 0; s < nslices; s++) {
        dptr[(size_t)s] = (const char *)E->d_dump + tbytes * (size_t)s;
        GSB_CK(cudaMemcpyAsync((void *)dptr[(size_t)s], dumps[s], tbytes, cudaMemcpyHostToDevice, E->stream));
    }
    void *small = nullptr;
    const size_t sbytes = (size_t)nslices * (8 + 8 + 8 + 16);
    GSB_CK(cudaMallocAsync(&small, sbytes, E->stream));
    char *sp = (char *)small;
    GSB_CK(cudaMemcpyAsync(sp, dptr.data(), (size_t)nslices * 8, cudaMemcpyHostToDevice, E->stream));
    GSB_CK(cudaMemcpyAsync(sp + (size_t)nslices * 8, f.data(), (size_t)nslices * 8, cudaMemcpyHostToDevice, E->stream));
    GSB_CK(cudaMemcpyAsync(sp + (size_t)nslices * 16, cs.data(), (size_t)nslices * 8, cudaMemcpyHostToDevice, E->stream));
    GSB_CK(cudaMemcpyAsync(sp + (size_t)nslices * 24, tperm.data(), (size_t)nslices * 16, cudaMemcpyHostToDevice, E->stream));
    ResumeArgs ra;
    ra.dumps = (const void *const *)sp;
    ra.f = (const double *)(sp + (size_t)nslices * 8);
    ra.cshift = (const uint64_t *)(sp + (size_t)nslices * 16);
    ra.tperm = (const int *)(sp + (size_t)nslices * 24);
    ra.nsl = nslices;
    ra.ntq = ntq;
    ra.K = K;
    ra.L = L;
    // forced row and the uniforms of the '?' steps (mt19937_64(seed + line), gsamp2.cpp:206)
    std::vector<int8_t> row((size_t)std::max(ns, 1), 0);
    for (int k = 0; k < ns; k++) row[(size_t)k] = forced[k];
    std::vector<double> u((size_t)std::max(ns, 1), 0.0);
    if (ns) free_uniforms(seed + (uint64_t)line, row.data(), std::min(K, ns), ns, u.data());
    if (ns) {
        GSB_CK(cudaMemcpyAsync(E->d_forced, row.data(), (size_t)ns, cudaMemcpyHostToDevice, E->stream));
        GSB_CK(cudaMemcpyAsync(E->d_unif, u.data(), (size_t)ns * 8, cudaMemcpyHostToDevice, E->stream));
    }
    k_set_item<<<1, 1, 0, E->stream>>>(E->st, 0);
    const uint64_t Nc = 1ULL << nk;
    Launch L1;
    L1.block = (int)std::max<uint64_t>(32, std::min<uint64_t>(256, Nc));
    Ctx c = E->ctx(DRV_HYBRID, ns, L1, true, true);
    const int grid = (int)std::min<uint64_t>((Nc + 255) / 256, (uint64_t)E->sms * 8);
    if (E->prec == 128) k_resume_sum<double2><<<grid, L1.block, 0, E->stream>>>(a, (double2 *)E->mem, ra, c);
    else k_resume_sum<float2><<<grid, L1.block, 0, E->stream>>>(a, (float2 *)E->mem, ra, c);
    GSB_CK(cudaGetLastError());
    for (int k = K; k < ns; k++) {
        GSB_CK(E->launch_step(k, false, DRV_HYBRID, ns, true, true));
        GSB_CK(E->launch_step(k, true, DRV_HYBRID, ns, true, true));
    }
    DevState hs;
    GSB_CK(cudaMemcpyAsync(&hs, E->st, sizeof hs, cudaMemcpyDeviceToHost, E->stream));
    std::vector<int8_t> hb((size_t)std::max(ns, 1), 0);
    std::vector<double> hc((size_t)std::max(ns, 1), 0.0);
    if (ns) {
        GSB_CK(cudaMemcpyAsync(hb.data(), E->d_bits, (size_t)ns, cudaMemcpyDeviceToHost, E->stream));
        GSB_CK(cudaMemcpyAsync(hc.data(), E->d_cond, (size_t)ns * 8, cudaMemcpyDeviceToHost, E->stream));
    }
    GSB_CK(cudaFreeAsync(small, E->stream));
    GSB_CK(cudaStreamSynchronize(E->stream));
    for (int k = 0; k < ns; k++) bits[k] = k < K ? forced[k] : hb[(size_t)k];
    if (cond)
        for (int k = K; k < ns; k++) cond[k] = hc[(size_t)k];
    *log2p_full = hs.aux + hs.logp;
    if (log2p_prefix) *log2p_prefix = hs.aux;
    return 0;
}

int gsb_chain_device(gsb_engine *e, const int8_t *d_bits, int64_t nstr, double *d_log2p, double *d_cond) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (nstr < 0 || (nstr && (!d_bits || !d_log2p))) return fail(GSB_E_USAGE, "null argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    const int ns = E->plan.ns;
    for (int64_t off = 0; off < nstr; off += E->cap) {
        const int64_t nb = std::min<int64_t>(E->cap, nstr - off);
        if (ns) GSB_CK(cudaMemcpyAsync(E->d_forced, d_bits + off * ns, (size_t)(nb * ns), cudaMemcpyDeviceToDevice, E->stream));
        int rc = E->run_graph_items(0, nb);
        if (rc) return rc;
        GSB_CK(cudaMemcpyAsync(d_log2p + off, E->d_logp, (size_t)nb * 8, cudaMemcpyDeviceToDevice, E->stream));
        if (d_cond && ns) GSB_CK(cudaMemcpyAsync(d_cond + off * ns, E->d_cond, (size_t)(nb * ns) * 8, cudaMemcpyDeviceToDevice, E->stream));
    }
    return guard_device(E, 0, d_bits, nstr, d_log2p, d_cond);
}

int gsb_sample_device(gsb_engine *e, const double *d_u, int64_t count, int8_t *d_bits, double *d_log2p) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (count < 0 || (count && (!d_u || !d_bits || !d_log2p))) return fail(GSB_E_USAGE, "null argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    const int ns = E->plan.ns;
    for (int64_t off = 0; off < count; off += E->cap) {
        const int64_t nb = std::min<int64_t>(E->cap, count - off);
        if (ns) GSB_CK(cudaMemcpyAsync(E->d_unif, d_u + off * ns, (size_t)(nb * ns) * 8, cudaMemcpyDeviceToDevice, E->stream));
        int rc = E->run_graph_items(2, nb);
        if (rc) return rc;
        GSB_CK(cudaMemcpyAsync(d_log2p + off, E->d_logp, (size_t)nb * 8, cudaMemcpyDeviceToDevice, E->stream));
        if (ns) GSB_CK(cudaMemcpyAsync(d_bits + off * ns, E->d_bits, (size_t)(nb * ns), cudaMemcpyDeviceToDevice, E->stream));
    }
    return guard_device(E, 0, d_bits, count, d_log2p, nullptr);
}

int gsb_synchronize(gsb_engine *e) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    GSB_CK(cudaStreamSynchronize(E->stream));
    return check_device(E);
}

int gsb_set_hybrid_prefix(gsb_engine *e, int K) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    Engine *E = eng(e);
    if (K < 0 || K > E->plan.ns) return fail(GSB_E_USAGE, "prefix length out of range");
    DevGuard g(E->dev);
    GSB_CK(cudaStreamSynchronize(E->stream));
    E->hyb_K = K;
    auto it = E->graphs.find(3);
    if (it != E->graphs.end()) {
        cudaGraphExecDestroy(it->second);
        E->graphs.erase(it);
    }
    build_hyb_ops(*E);
    return 0;
}

int gsb_set_guard(gsb_engine *e, gsb_engine *g, double log2_xmin) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    Engine *E = eng(e);
    if (E->prec != 64) return fail(GSB_E_USAGE, "the guarded engine must be complex64");
    if (E->guard) {
        E->guard->guarded = nullptr;
        E->guard = nullptr;
    }
    E->guard_evals = 0;
    if (!g) return 0;
    Engine *G = eng(g);
    if (G->prec != 128) return fail(GSB_E_USAGE, "the guard engine must be complex128");
    if (G->dev != E->dev) return fail(GSB_E_USAGE, "the guard engine must be on the same device");
    if (G->guarded && G->guarded != E) return fail(GSB_E_USAGE, "the guard engine already guards another engine");
    if (!same_plan(E->plan, G->plan)) return fail(GSB_E_USAGE, "the guard engine's plan differs");
    if (!(log2_xmin == log2_xmin)) return fail(GSB_E_USAGE, "threshold is NaN");
    E->guard = G;
    G->guarded = E;
    E->guard_lx = log2_xmin;
    return 0;
}

int gsb_guard_evaluations(const gsb_engine *e, int64_t *count) {
    if (!e || !count) return fail(GSB_E_USAGE, "null argument");
    *count = eng(e)->guard_evals;
    return 0;
}

int gsb_set_arith(gsb_engine *e, int bits) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (bits != 32 && bits != 64) return fail(GSB_E_USAGE, "arithmetic must be 32 or 64");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    GSB_CK(cudaStreamSynchronize(E->stream));
    if (bits == E->arith) return 0;
    E->arith = bits;
    for (auto &kv : E->graphs) cudaGraphExecDestroy(kv.second);
    E->graphs.clear();
    apply_coeffs(*E);
    for (int k = 0; k < E->plan.ns; k++) {
        E->lw[(size_t)k] = E->shape(E->args[(size_t)k], true);
        E->ln[(size_t)k] = E->shape(E->args[(size_t)k], false);
    }
    build_chain_ops(*E);
    return 0;
}

int gsb_set_fusion(gsb_engine *e, int depth) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (depth < 1 || depth > FUSE_MAX_STEPS) return fail(GSB_E_USAGE, "fusion depth must be 1..3");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    GSB_CK(cudaStreamSynchronize(E->stream));
    E->fuse_depth = depth;
    E->chain_shapes.clear();     // an explicit depth replaces the autotuner's choice
    E->sample_shapes.clear();
    for (auto &kv : E->graphs) cudaGraphExecDestroy(kv.second);
    E->graphs.clear();
    build_chain_ops(*E);
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------
// Autotuner of the pass lists: every candidate pass (one step; 2 or 3 fused steps; with or without the next step's
// branch norms for sampling; tile caps 2^8, 2^9, 2^10) is timed on the device, alone, with CUDA events on the
// engine's stream, and the cover of the steps with the least measured time replaces the byte-model choice.  A pass's
// time does not depend on the table's values (no data-dependent control flow besides the dead flag, which the device
// state reset before each launch clears), so the candidates run on whatever the arena holds, with bits chosen so that
// no analytic step takes a zero-probability branch.

struct Timer {
    Engine &E;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int reps;
    explicit Timer(Engine &e, int r) : E(e), reps(r) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
    }
    ~Timer() {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    // mean milliseconds of `launch` after a device-state reset, or a negative value on a CUDA error
    template <typename F>
    double operator()(F launch) {
        double tot = 0;
        for (int r = -1; r < reps; r++) {   // r = -1: untimed warm-up
            k_set_item<<<1, 1, 0, E.stream>>>(E.st, 0);
            if (E.launch_begin() != cudaSuccess) return -1;
            if (cudaEventRecord(e0, E.stream) != cudaSuccess) return -1;
            if (launch() != cudaSuccess) return -1;
            if (cudaEventRecord(e1, E.stream) != cudaSuccess) return -1;
            if (cudaEventSynchronize(e1) != cudaSuccess) return -1;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (r >= 0) tot += ms;
        }
        return tot / reps;
    }
};

static int autotune(Engine &E, int mode, int reps) {
    const HPlan &p = E.plan;
    const int ns = p.ns;
    if (ns < 1) return 0;
    // forced bits for timing: the likelier branch of every analytic step, 0 elsewhere
    std::vector<int8_t> row((size_t)ns, 0);
    for (int k = 0; k < ns; k++) {
        const HStep &h = p.st[(size_t)k];
        const double c0 = h.Mr[0][0] * h.Mr[0][0] + h.Mi[0][0] * h.Mi[0][0] + h.Mr[0][1] * h.Mr[0][1] + h.Mi[0][1] * h.Mi[0][1];
        const double c1 = h.Mr[1][0] * h.Mr[1][0] + h.Mi[1][0] * h.Mi[1][0] + h.Mr[1][1] * h.Mr[1][1] + h.Mi[1][1] * h.Mi[1][1];
        row[(size_t)k] = (int8_t)(c1 > c0 ? 1 : 0);
    }
    GSB_CK(cudaMemcpyAsync(E.d_forced, row.data(), (size_t)ns, cudaMemcpyHostToDevice, E.stream));
    Timer timer(E, reps);
    auto rof = [&](int k) { const HStep &h = p.st[(size_t)k]; return h.nk + (h.tqs.size() == 4 ? 2 : h.tqs.size() == 2 ? 1 : 0); };
    const double INF = 1e300;
    std::vector<double> t_write((size_t)ns), t_norm((size_t)ns);
    const int drv = mode == 0 ? DRV_CHAIN1 : DRV_CHAIN;
    for (int k = 0; k < ns; k++) {
        t_write[(size_t)k] = timer([&] { return E.launch_step(k, true, drv, ns, true, false); });
        t_norm[(size_t)k] = mode == 0 ? 0 : timer([&] { return E.launch_step(k, false, drv, ns, true, false); });
        if (t_write[(size_t)k] < 0 || t_norm[(size_t)k] < 0) return fail(GSB_E_CUDA, "autotuner: a timing launch failed");
    }
    // fused candidates starting at k, with their times (distinct tile sizes only)
    auto fused = [&](int k, int d, int tr, std::vector<std::pair<OpShape, double>> &out) -> int {
        const bool c64f = E.prec == 64 && E.arith == 32;
        for (int minb : {2, 3}) {
          if (minb == 3 && !c64f) continue;
          for (int ws : {0, 1}) {   // the warp-specialised build: complex64 FP32, two CTAs per SM
            if (ws && (minb != 2 || !c64f)) continue;
            int lastL = -1;
            for (int lcap : {GROUP_MAX_L, GROUP_MAX_L - 1, GROUP_MAX_L - 2}) {
              OpShape sh;
              sh.group = true;
              sh.k0 = k;
              sh.d = d;
              sh.tr = tr;
              sh.lcap = lcap;
              sh.minb = minb;
              sh.ws = ws;
              sh.src = GSRC_NORM;   // timing: the bit of step k as a norm pass would leave it
              Op op;
              if (!make_op(E, sh, op) || op.ga.L == lastL) continue;
              lastL = op.ga.L;
              const double t = timer([&] { return E.launch_op(op, drv, true, false); });
              if (t < 0) return fail(GSB_E_CUDA, "autotuner: a timing launch failed");
              out.push_back({sh, t});
            }
          }
        }
        return 0;
    };
    if (mode == 0) {
        std::vector<double> cost((size_t)ns + 1, INF);
        std::vector<OpShape> pick((size_t)ns + 1);
        cost[(size_t)ns] = 0;
        for (int k = ns - 1; k >= 0; k--) {
            OpShape single;
            single.k0 = k;
            cost[(size_t)k] = t_write[(size_t)k] + cost[(size_t)k + 1];
            pick[(size_t)k] = single;
            if (rof(k) < GROUP_MIN_R) continue;
            for (int d = 2; d <= FUSE_MAX_STEPS && k + d <= ns; d++) {
                std::vector<std::pair<OpShape, double>> c;
                if (int rc = fused(k, d, 0, c)) return rc;
                for (auto &x : c)
                    if (x.second + cost[(size_t)(k + d)] < cost[(size_t)k]) {
                        cost[(size_t)k] = x.second + cost[(size_t)(k + d)];
                        pick[(size_t)k] = x.first;
                    }
            }
        }
        E.chain_shapes.clear();
        for (int k = 0; k < ns;) {
            E.chain_shapes.push_back(pick[(size_t)k]);
            k += pick[(size_t)k].group ? pick[(size_t)k].d : 1;
        }
        return 0;
    }
    // sampling: state t = step k's branch norms come from the previous pass
    std::vector<std::array<double, 2>> cost((size_t)ns + 1, {INF, INF});
    std::vector<std::array<OpShape, 2>> pick((size_t)ns + 1);
    cost[(size_t)ns] = {0, 0};
    std::vector<std::vector<std::pair<OpShape, double>>> cands((size_t)ns);
    for (int k = 0; k < ns; k++) {
        if (rof(k) < GROUP_MIN_R) continue;
        for (int d = 1; d <= FUSE_MAX_STEPS && k + d <= ns; d++) {
            if (d > 1 && !analytic_step(p.st[(size_t)(k + d - 1)])) break;
            for (int tr = 0; tr < 2; tr++) {
                if (d + tr < 2 || d + tr > FUSE_MAX_STEPS) continue;
                if (tr && (k + d >= ns || analytic_step(p.st[(size_t)(k + d)]))) continue;
                if (int rc = fused(k, d, tr, cands[(size_t)k])) return rc;
            }
        }
    }
    for (int k = ns - 1; k >= 0; k--) {
        const bool an = analytic_step(p.st[(size_t)k]);
        for (int t = 0; t < 2; t++) {
            OpShape single;
            single.k0 = k;
            double best = t_norm[(size_t)k] + t_write[(size_t)k] + cost[(size_t)k + 1][0];
            OpShape bp = single;
            for (auto &x : cands[(size_t)k]) {
                const OpShape &sh = x.first;
                const bool nf = !an && !t;
                const double c = (nf ? t_norm[(size_t)k] : 0) + x.second + cost[(size_t)(k + sh.d)][(size_t)sh.tr];
                if (c < best) {
                    best = c;
                    bp = sh;
                    bp.norm_first = nf;
                    bp.src = an ? GSRC_ANALYTIC : t ? GSRC_TRAILING : GSRC_NORM;
                }
            }
            cost[(size_t)k][(size_t)t] = best;
            pick[(size_t)k][(size_t)t] = bp;
        }
    }
    E.sample_shapes.clear();
    for (int k = 0, t = 0; k < ns;) {
        const OpShape &sh = pick[(size_t)k][(size_t)t];
        E.sample_shapes.push_back(sh);
        t = sh.group ? sh.tr : 0;
        k += sh.group ? sh.d : 1;
    }
    return 0;
}

extern "C" {

int gsb_autotune(gsb_engine *e, int mode, int reps, float *ms_before, float *ms_after) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (mode < 0 || mode > 2 || reps < 1) return fail(GSB_E_USAGE, "mode must be 0 (chain), 1 (sampling) or 2 (both)");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    GSB_CK(cudaStreamSynchronize(E->stream));
    const HPlan &p = E->plan;
    {   // the timed items' bits: the likelier branch of every analytic step, 0 elsewhere (as the autotuner uses)
        std::vector<int8_t> row((size_t)std::max(p.ns, 1), 0);
        for (int k = 0; k < p.ns; k++) {
            const HStep &h = p.st[(size_t)k];
            const double c0 = h.Mr[0][0] * h.Mr[0][0] + h.Mi[0][0] * h.Mi[0][0] + h.Mr[0][1] * h.Mr[0][1] + h.Mi[0][1] * h.Mi[0][1];
            const double c1 = h.Mr[1][0] * h.Mr[1][0] + h.Mi[1][0] * h.Mi[1][0] + h.Mr[1][1] * h.Mr[1][1] + h.Mi[1][1] * h.Mi[1][1];
            row[(size_t)k] = (int8_t)(c1 > c0 ? 1 : 0);
        }
        if (p.ns) GSB_CK(cudaMemcpyAsync(E->d_forced, row.data(), (size_t)p.ns, cudaMemcpyHostToDevice, E->stream));
    }
    // device time of one item of graph `kind` (replayed: one warm-up, then the mean of `reps`)
    auto item_ms = [&](int kind, float *out) -> int {
        cudaGraphExec_t ex;
        if (int rc = E->graph(kind, &ex)) return rc;
        cudaEvent_t a, b;
        GSB_CK(cudaEventCreate(&a));
        GSB_CK(cudaEventCreate(&b));
        k_set_item<<<1, 1, 0, E->stream>>>(E->st, 0);
        GSB_CK(cudaGraphLaunch(ex, E->stream));
        float tot = 0;
        for (int r = 0; r < reps; r++) {
            k_set_item<<<1, 1, 0, E->stream>>>(E->st, 0);
            GSB_CK(cudaEventRecord(a, E->stream));
            GSB_CK(cudaGraphLaunch(ex, E->stream));
            GSB_CK(cudaEventRecord(b, E->stream));
            GSB_CK(cudaEventSynchronize(b));
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            tot += ms;
        }
        *out = tot / reps;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return 0;
    };
    auto rebuild = [&]() {
        for (auto &kv : E->graphs) cudaGraphExecDestroy(kv.second);
        E->graphs.clear();
        build_chain_ops(*E);
    };
    float tb = 0, ta = 0;
    // per pass list: tune, then keep the tuned list only if a whole item got faster (passes timed alone do not
    // always add up to their time in sequence)
    for (int m = 0; m < 2; m++) {
        if (mode != 2 && mode != m) continue;
        const int kind = m == 0 ? 0 : 1;   // the 'chain' graph, or 'prob' (the sampling passes with forced bits)
        float before = 0, after = 0;
        if (int rc = item_ms(kind, &before)) return rc;
        std::vector<OpShape> keep = m == 0 ? E->chain_shapes : E->sample_shapes;
        rebuild();
        if (int rc = autotune(*E, m, reps)) return rc;
        rebuild();
        if (int rc = item_ms(kind, &after)) return rc;
        if (after > before) {
            (m == 0 ? E->chain_shapes : E->sample_shapes) = keep;
            rebuild();
            after = before;
        }
        tb += before;
        ta += after;
    }
    GSB_CK(cudaStreamSynchronize(E->stream));
    if (ms_before) *ms_before = tb;
    if (ms_after) *ms_after = ta;
    return check_device(E);
}

int gsb_test_withhold_tile_loads(gsb_engine *e, int on) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    GSB_CK(cudaStreamSynchronize(E->stream));
    if (on < 0 || on > 2) return fail(GSB_E_USAGE, "withhold mode must be 0, 1 or 2");
    E->withhold_loads = on;
    for (auto &kv : E->graphs) cudaGraphExecDestroy(kv.second);   // the graphs hold the pass arguments by value
    E->graphs.clear();
    return 0;
}

int gsb_sample_groups(const gsb_engine *e, int *group_len, double *entries) {
    if (!e || !group_len) return fail(GSB_E_USAGE, "null argument");
    const Engine *E = eng(e);
    const HPlan &p = E->plan;
    for (int k = 0; k < p.ns; k++) {
        group_len[k] = 0;
        if (entries) entries[k] = 0;
    }
    auto table = [&](int k) { const HStep &h = p.st[(size_t)k]; return std::ldexp(1.0, h.nk) * (double)h.tqs.size(); };
    if (E->sample_ops.empty()) {   // no fusion: a norm pass and a write pass per step
        for (int k = 0; k < p.ns; k++) {
            group_len[k] = 1;
            if (entries) entries[k] = table(k) + single_entries(p, k);
        }
        return 0;
    }
    for (const Op &op : E->sample_ops) {
        group_len[op.k0] = op.group ? op.d : 1;
        if (entries) entries[op.k0] = (op.group ? op.entries : single_entries(p, op.k0)) +
                                      ((!op.group || op.norm_first) ? table(op.k0) : 0.0);
    }
    return 0;
}

int gsb_pass_list(const gsb_engine *e, int mode, int cap, int *k0, int *d, int *tr, int *fused, int *count) {
    if (!e || !count || cap < 0 || (mode != 0 && mode != 1)) return fail(GSB_E_USAGE, "bad argument");
    if (cap > 0 && (!k0 || !d || !tr || !fused)) return fail(GSB_E_USAGE, "null argument");
    const Engine *E = eng(e);
    const std::vector<Op> &ops = mode == 0 ? E->chain_ops : E->sample_ops;
    int n = 0;
    auto put = [&](int a, int b, int c, int f) {
        if (n < cap) {
            k0[n] = a;
            d[n] = b;
            tr[n] = c;
            fused[n] = f;
        }
        n++;
    };
    if (ops.empty()) {   // no fusion: one pass per step
        for (int k = 0; k < E->plan.ns; k++) put(k, 1, 0, 0);
    } else {
        for (const Op &op : ops) put(op.k0, op.group ? op.d : 1, op.group ? op.tr : 0, op.group ? 1 : 0);
    }
    *count = n;
    return 0;
}

int gsb_fusion_groups(const gsb_engine *e, int *group_len, double *entries) {
    if (!e || !group_len) return fail(GSB_E_USAGE, "null argument");
    const Engine *E = eng(e);
    for (int k = 0; k < E->plan.ns; k++) {
        group_len[k] = 0;
        if (entries) entries[k] = 0;
    }
    for (const Op &op : E->chain_ops) {
        group_len[op.k0] = op.d;
        if (entries) entries[op.k0] = op.entries;
    }
    return 0;
}

int gsb_set_matrices(gsb_engine *e, const double *M) {
    if (!e || !M) return fail(GSB_E_USAGE, "null argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    GSB_CK(cudaStreamSynchronize(E->stream));
    for (int k = 0; k < E->plan.ns; k++) {
        HStep &s = E->plan.st[(size_t)k];
        StepArgs &a = E->args[(size_t)k];
        for (int b = 0; b < 2; b++)
            for (int x = 0; x < 2; x++) {
                const double re = M[(size_t)k * 8 + (size_t)(4 * b + 2 * x)], im = M[(size_t)k * 8 + (size_t)(4 * b + 2 * x + 1)];
                s.Mr[b][x] = a.Mr[b][x] = re;
                s.Mi[b][x] = a.Mi[b][x] = im;
            }
    }
    apply_coeffs(*E);
    for (auto &kv : E->graphs) cudaGraphExecDestroy(kv.second);   // the captured graphs hold M by value
    E->graphs.clear();
    build_chain_ops(*E);
    return 0;
}

int gsb_set_stream(gsb_engine *e, void *cuda_stream) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    GSB_CK(cudaStreamSynchronize(E->stream));
    E->stream = cuda_stream ? (cudaStream_t)cuda_stream : E->own_stream;
    return 0;
}

int gsb_profile_steps(gsb_engine *e, const int8_t *bits, int mode, float *ms_write, float *ms_norm) {
    if (!e) return fail(GSB_E_STATE, "null engine");
    if (!bits || !ms_write || (mode != 0 && mode != 1)) return fail(GSB_E_USAGE, "bad argument");
    Engine *E = eng(e);
    DevGuard g(E->dev);
    const int ns = E->plan.ns;
    int rc = check_bits(bits, 1, ns, false);
    if (rc) return rc;
    const int driver = mode == 0 ? DRV_CHAIN1 : DRV_CHAIN;
    std::vector<cudaEvent_t> ev((size_t)(2 * ns + 1));
    for (auto &x : ev) GSB_CK(cudaEventCreate(&x));
    if (ns) GSB_CK(cudaMemcpyAsync(E->d_forced, bits, (size_t)ns, cudaMemcpyHostToDevice, E->stream));
    k_set_item<<<1, 1, 0, E->stream>>>(E->st, 0);
    GSB_CK(E->launch_begin());
    GSB_CK(cudaEventRecord(ev[0], E->stream));
    if (driver == DRV_CHAIN1 && !E->chain_ops.empty()) {   // one timing per pass, reported at its first step
        std::vector<float> t((size_t)ns, 0.f);
        for (size_t i = 0; i < E->chain_ops.size(); i++) {
            GSB_CK(E->launch_op(E->chain_ops[i], driver));
            GSB_CK(cudaEventRecord(ev[i + 1], E->stream));
        }
        k_finish<<<1, 1, 0, E->stream>>>(E->st, E->d_logp, E->d_aux, driver, ns);
        GSB_CK(cudaStreamSynchronize(E->stream));
        for (size_t i = 0; i < E->chain_ops.size(); i++) {
            float a = 0;
            GSB_CK(cudaEventElapsedTime(&a, ev[i], ev[i + 1]));
            t[(size_t)E->chain_ops[i].k0] = a;
        }
        for (int k = 0; k < ns; k++) {
            ms_write[k] = t[(size_t)k];
            if (ms_norm) ms_norm[k] = 0.f;
        }
        for (auto &x : ev) cudaEventDestroy(x);
        return 0;
    }
    if (driver == DRV_CHAIN && !E->sample_ops.empty()) {   // per pass: its norm pass (if any), then the pass
        std::vector<float> tw((size_t)ns, 0.f), tn((size_t)ns, 0.f);
        std::vector<cudaEvent_t> ev2(2 * E->sample_ops.size() + 1);
        for (auto &x : ev2) GSB_CK(cudaEventCreate(&x));
        GSB_CK(cudaEventRecord(ev2[0], E->stream));
        for (size_t i = 0; i < E->sample_ops.size(); i++) {
            const Op &op = E->sample_ops[i];
            if (!op.group || op.norm_first) GSB_CK(E->launch_step(op.k0, false, driver, ns, true, false));
            GSB_CK(cudaEventRecord(ev2[2 * i + 1], E->stream));
            if (op.group) GSB_CK(E->launch_op(op, driver, true, false));
            else GSB_CK(E->launch_step(op.k0, true, driver, ns, true, false));
            GSB_CK(cudaEventRecord(ev2[2 * i + 2], E->stream));
        }
        k_finish<<<1, 1, 0, E->stream>>>(E->st, E->d_logp, E->d_aux, driver, ns);
        GSB_CK(cudaStreamSynchronize(E->stream));
        for (size_t i = 0; i < E->sample_ops.size(); i++) {
            float a = 0, b = 0;
            GSB_CK(cudaEventElapsedTime(&a, ev2[2 * i], ev2[2 * i + 1]));
            GSB_CK(cudaEventElapsedTime(&b, ev2[2 * i + 1], ev2[2 * i + 2]));
            tn[(size_t)E->sample_ops[i].k0] = a;
            tw[(size_t)E->sample_ops[i].k0] = b;
        }
        for (int k = 0; k < ns; k++) {
            ms_write[k] = tw[(size_t)k];
            if (ms_norm) ms_norm[k] = tn[(size_t)k];
        }
        for (auto &x : ev2) cudaEventDestroy(x);
        for (auto &x : ev) cudaEventDestroy(x);
        return 0;
    }
    for (int k = 0; k < ns; k++) {
        if (driver == DRV_CHAIN) GSB_CK(E->launch_step(k, false, driver, ns, true, false));
        GSB_CK(cudaEventRecord(ev[(size_t)(2 * k + 1)], E->stream));
        GSB_CK(E->launch_step(k, true, driver, ns, true, false));
        GSB_CK(cudaEventRecord(ev[(size_t)(2 * k + 2)], E->stream));
    }
    k_finish<<<1, 1, 0, E->stream>>>(E->st, E->d_logp, E->d_aux, driver, ns);
    GSB_CK(cudaStreamSynchronize(E->stream));
    for (int k = 0; k < ns; k++) {
        float a = 0, b = 0;
        GSB_CK(cudaEventElapsedTime(&a, ev[(size_t)(2 * k)], ev[(size_t)(2 * k + 1)]));
        GSB_CK(cudaEventElapsedTime(&b, ev[(size_t)(2 * k + 1)], ev[(size_t)(2 * k + 2)]));
        if (ms_norm) ms_norm[k] = driver == DRV_CHAIN ? a : 0.f;
        ms_write[k] = b;
    }
    for (auto &x : ev) cudaEventDestroy(x);
    return 0;
}

int gsb_launches_per_item(const gsb_engine *e, int mode, int64_t *launches) {
    if (!e || !launches) return fail(GSB_E_USAGE, "null argument");
    const Engine *E = eng(e);
    const int64_t ns = E->plan.ns;
    if (mode == 0 && !E->chain_ops.empty()) *launches = E->item_launches(E->chain_ops, false);
    else if (mode == 1 && !E->sample_ops.empty()) *launches = E->item_launches(E->sample_ops, true);
    else {   // one norm and one write pass per step ('chain' mode: write only), small-step runs counted once
        int64_t n = 2;
        for (int k = 0; k < ns;) {
            int k1 = k;
            while (k1 < ns && E->small_step(k1)) k1++;
            if (k1 - k >= 2) { n++; k = k1; continue; }
            n += mode == 0 ? 1 : 2;
            k++;
        }
        *launches = n;
    }
    return 0;
}

}  // extern "C"
