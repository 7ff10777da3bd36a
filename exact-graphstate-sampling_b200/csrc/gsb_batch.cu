// Batched evaluation of many instances of uneven width in one persistent launch (the batching form).
//
// Work: for every instance i (its own in-place plan, ns_i steps, width R_i) and each of its npre prefixes, the
// forced bits of steps [0, K_i) are applied once, the live table before step K_i is kept, and each of nsuf suffixes
// resumes from it through steps [K_i, ns_i): one log2 Pr per (prefix, suffix) string.  Strings that share a prefix
// share its DP work (the reference's prefix / resume, gsamp2.cpp:162-208, done in memory).
//
// A work item is (instance, prefix).  Items sit in two queues, each sorted by decreasing cost: wide instances are
// run by a whole CTA ("block team"), narrow ones (R <= small_R) by one warp ("warp team").  The kernel is
// persistent: every CTA first takes block-team items from the first queue, then each of its warps takes warp-team
// items from the second, with one atomic per item.  A team owns an arena of 2^R entries and a snapshot buffer in its
// slot, so a whole item runs without any grid-wide synchronisation: a step is a strided loop of the team over the
// step's cosets (each coset reads and writes only its own slots, gsamp2.cpp:32-38 and 59-66), then a team reduction
// of the written norm; the one-pass chain logic (power-of-two rescaling, gsamp2.cpp:59-70) runs redundantly in every
// thread of the team.  Block size, the narrow-width threshold and CTAs per SM are chosen by an autotuner that times
// the actual batch; each shape's launch is captured once as a CUDA graph (queue reset + kernel).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "gsb.h"
#include "gsb_common.h"
#include "gsb_plan.h"
#include "gsb_step.h"

namespace gsb {

struct BStep {
    uint64_t g, rhoc, tq[4];
    double M[8];             // M[b][x] (re, im)
    int nk, ntq, m, tk_off;
    int tau0[4], tau1[4], par[4];
};

struct BInst {
    int ns, R, K, n;
    int step_off;            // first BStep
    int64_t pre_off;         // prefix bits: [npre][K]
    int64_t suf_off;         // suffix bits: [npre][nsuf][ns - K]
    int64_t out_off;         // log2 Pr: [npre][nsuf]
};

struct BatchArgs {
    const BStep *steps;
    const uint64_t *tk;
    const BInst *inst;
    const int *items_big, *items_small;   // item = inst * npre + prefix
    int n_big, n_small, npre, nsuf;
    const int8_t *pre_bits, *suf_bits;
    double *log2p;
    unsigned int *queues;    // [0] block-team queue, [1] warp-team queue
    void *big_arena;         // per CTA: arena + snapshot of 2^big_R entries each
    void *small_arena;       // per warp: arena + snapshot of 2^small_R entries each
    int big_R, small_R;
};

struct BlockTeam {
    __device__ int rank() const { return threadIdx.x; }
    __device__ int size() const { return blockDim.x; }
    __device__ int log2size() const { return __ffs((int)blockDim.x) - 1; }   // blockDim.x: a power of two
    __device__ void sync() const { __syncthreads(); }
    __device__ double sum(double v) const {
        __shared__ double red[32];
        v = warp_sum(v);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        __syncthreads();
        if (lane == 0) red[w] = v;
        __syncthreads();
        double t = 0;
        for (int i = 0; i < nw; i++) t += red[i];
        return t;
    }
};

struct WarpTeam {
    __device__ int rank() const { return threadIdx.x & 31; }
    __device__ int size() const { return 32; }
    __device__ int log2size() const { return 5; }
    __device__ void sync() const { __syncwarp(); }
    __device__ double sum(double v) const {
        __syncwarp();
        return warp_sum(v);
    }
};

template <typename E> struct ArithOf;
template <> struct ArithOf<float2> { typedef float T; };
template <> struct ArithOf<double2> { typedef double T; };

__device__ __forceinline__ void ld_e(const float2 *m, uint64_t a, float &r, float &i) { const float2 v = m[a]; r = v.x; i = v.y; }
__device__ __forceinline__ void ld_e(const double2 *m, uint64_t a, double &r, double &i) { const double2 v = m[a]; r = v.x; i = v.y; }
__device__ __forceinline__ void st_e(float2 *m, uint64_t a, float r, float i) { m[a] = make_float2(r, i); }
__device__ __forceinline__ void st_e(double2 *m, uint64_t a, double r, double i) { m[a] = make_double2(r, i); }
__device__ __forceinline__ void ld_e(const float2 *m, uint64_t a, double &r, double &i) { const float2 v = m[a]; r = v.x; i = v.y; }
__device__ __forceinline__ void st_e(float2 *m, uint64_t a, double r, double i) { m[a] = make_float2((float)r, (float)i); }

__device__ __forceinline__ uint64_t bcoset_base(const uint64_t *tk, uint64_t c) {
    uint64_t b = 0;
    while (c) {
        b ^= tk[__ffsll((long long)c) - 1];
        c &= c - 1;
    }
    return b;
}

// The cosets of a step a team member visits: c = rank | (g << log2 team size) for the Gray codes g of the high bits,
// so consecutive cosets differ in one high bit and the base is the member's fixed low part XOR one running value
// (one XOR per coset instead of a loop over the bits of c).  f(c, base) is called for each.
template <typename TM, typename F>
__device__ __forceinline__ void team_cosets(const TM &tm, int nk, const uint64_t *tk, F f) {
    const int ls = tm.log2size();
    const uint64_t r = (uint64_t)tm.rank();
    if (nk < ls && r >= (1ULL << nk)) return;
    const uint64_t lo = bcoset_base(tk, r);
    const uint64_t nh = nk > ls ? 1ULL << (nk - ls) : 1;
    uint64_t hi = 0;
    for (uint64_t n = 0; n < nh; n++) {
        if (n) hi ^= tk[ls + __ffsll((long long)n) - 1];
        f(r | ((n ^ (n >> 1)) << ls), lo ^ hi);
    }
}

// One coset of step s: inputs already loaded (v), outputs stored, their squared norm returned.
template <typename E, typename T, int NTQ>
__device__ __forceinline__ T coset_out(const BStep &s, E *arena, uint64_t c, uint64_t base, const T (&vr)[NTQ],
                                       const T (&vi)[NTQ], T m0r, T m0i, T m1r, T m1i) {
    const int pc = __popcll(c & s.rhoc) & 1;
    // x = 0 and signed x = 1 sums of the two outputs, in scalars (no runtime-indexed arrays)
    T a0r = 0, a0i = 0, a1r = 0, a1i = 0, b0r = 0, b0i = 0, b1r = 0, b1i = 0;
#pragma unroll
    for (int t = 0; t < NTQ; t++) {
        T xr = vr[t], xi = vi[t];
        if (s.tau0[t]) { a1r += xr; a1i += xi; } else { a0r += xr; a0i += xi; }
        if ((pc ^ s.par[t]) & 1) { xr = -xr; xi = -xi; }
        if (s.tau1[t]) { b1r += xr; b1i += xi; } else { b0r += xr; b0i += xi; }
    }
    const T r0 = m0r * a0r - m0i * a0i + m1r * b0r - m1i * b0i;
    const T i0 = m0r * a0i + m0i * a0r + m1r * b0i + m1i * b0r;
    st_e(arena, base, r0, i0);
    T n = r0 * r0 + i0 * i0;
    if (s.m == 2) {
        const T r1 = m0r * a1r - m0i * a1i + m1r * b1r - m1i * b1i;
        const T i1 = m0r * a1i + m0i * a1r + m1r * b1i + m1i * b1r;
        st_e(arena, base ^ s.g, r1, i1);
        n += r1 * r1 + i1 * i1;
    }
    return n;
}

// The write pass over the member's cosets (team_cosets' order), CPI cosets per iteration: every coset's inputs are
// loaded before any output is stored (distinct cosets never share a slot, so this order is safe in place), which
// multiplies the loads in flight of a latency-bound team.  Four cosets for complex64 (the big items' tables spill
// from L2, and 4 cut the batch launch by 11 %); two for complex128, where four cost registers and ran 21 % slower.
template <typename E, typename TM, int NTQ>
__device__ double team_step_n(const TM &tm, const BStep &s, const uint64_t *tk, E *arena, int bit, double scale) {
    typedef typename ArithOf<E>::T T;
    constexpr int CPI = sizeof(E) == 8 ? 4 : 2;
    const T m0r = (T)(scale * s.M[4 * bit + 0]), m0i = (T)(scale * s.M[4 * bit + 1]);
    const T m1r = (T)(scale * s.M[4 * bit + 2]), m1i = (T)(scale * s.M[4 * bit + 3]);
    double nb = 0;
    const int ls = tm.log2size();
    const uint64_t r = (uint64_t)tm.rank();
    if (!(s.nk < ls && r >= (1ULL << s.nk))) {
        const uint64_t lo = bcoset_base(tk, r);
        const uint64_t nh = s.nk > ls ? 1ULL << (s.nk - ls) : 1;   // a power of two
        uint64_t hi = 0;
        for (uint64_t n = 0; n < nh; n += CPI) {
            // cosets n .. n + CPI - 1 (n a multiple of CPI): Gray step n + q flips high bit ctz(q); a bit is read
            // only when that coset exists, so tk stays within the step's kept columns
            if (n) hi ^= tk[ls + __ffsll((long long)n) - 1];
            uint64_t h[CPI];
            h[0] = hi;
#pragma unroll
            for (int q = 1; q < CPI; q++) h[q] = n + (uint64_t)q < nh ? h[q - 1] ^ tk[ls + __ffs(q) - 1] : h[q - 1];
            const int cnt = nh - n >= (uint64_t)CPI ? CPI : (int)(nh - n);
            T vr[CPI][NTQ], vi[CPI][NTQ];
#pragma unroll
            for (int q = 0; q < CPI; q++)
#pragma unroll
                for (int t = 0; t < NTQ; t++) {
                    if (q < cnt) ld_e(arena, (lo ^ h[q]) ^ s.tq[t], vr[q][t], vi[q][t]);
                    else { vr[q][t] = 0; vi[q][t] = 0; }
                }
            T nn = 0;
#pragma unroll
            for (int q = 0; q < CPI; q++)
                if (q < cnt) {
                    const uint64_t m = n + (uint64_t)q;
                    nn += coset_out<E, T, NTQ>(s, arena, r | ((m ^ (m >> 1)) << ls), lo ^ h[q], vr[q], vi[q], m0r, m0i,
                                               m1r, m1i);
                }
            nb += (double)nn;
            hi = h[CPI - 1];
        }
    }
    tm.sync();
    return tm.sum(nb);
}

// One write pass of step s with bit `bit`, outputs scaled by `scale`; returns the written norm (to every thread).
template <typename E, typename TM>
__device__ double team_step(const TM &tm, const BStep &s, const uint64_t *tk, E *arena, int bit, double scale) {
    switch (s.ntq) {
        case 1: return team_step_n<E, TM, 1>(tm, s, tk, arena, bit, scale);
        case 2: return team_step_n<E, TM, 2>(tm, s, tk, arena, bit, scale);
        default: return team_step_n<E, TM, 4>(tm, s, tk, arena, bit, scale);
    }
}

// Live table before step s, in (coset, offset) order, to / from a compact buffer.
template <typename E, typename TM>
__device__ void team_copy(const TM &tm, const BStep &s, const uint64_t *tk, E *arena, E *snap, bool save) {
    team_cosets(tm, s.nk, tk, [&](uint64_t c, uint64_t base) {
        for (int t = 0; t < s.ntq; t++) {
            if (save) snap[c * (uint64_t)s.ntq + (uint64_t)t] = arena[base ^ s.tq[t]];
            else arena[base ^ s.tq[t]] = snap[c * (uint64_t)s.ntq + (uint64_t)t];
        }
    });
    tm.sync();
}

struct ChainState {
    double prev, lsc, scale;
    int ek, dead;
};

// The one-pass chain scalars after a write of norm nb (gsamp2.cpp:59-70, executor write_epilogue).
__device__ __forceinline__ void chain_update(ChainState &cs, double nb) {
    cs.lsc += cs.ek;
    cs.prev = nb;
    if (!(nb > 0)) {
        cs.dead = 1;
        return;
    }
    int ex;
    frexp(nb, &ex);
    cs.ek = (ex - 1) >> 1;
    cs.scale = ldexp(1.0, -cs.ek);
}

template <typename E, typename TM>
__device__ void run_item(const TM &tm, const BatchArgs &a, int item, E *arena, E *snap) {
    const int ii = item / a.npre, pre = item % a.npre;
    const BInst in = a.inst[ii];
    const BStep *st = a.steps + in.step_off;
    const int8_t *pb = a.pre_bits + in.pre_off + (int64_t)pre * in.K;
    if (tm.rank() == 0) st_e(arena, 0, 1.0, 0.0);
    tm.sync();
    ChainState cs{1.0, 0.0, 1.0, 0, 0};
    for (int k = 0; k < in.K && !cs.dead; k++) chain_update(cs, team_step(tm, st[k], a.tk + st[k].tk_off, arena, pb[k], cs.scale));
    const ChainState at_k = cs;
    if (!cs.dead) team_copy(tm, st[in.K], a.tk + st[in.K].tk_off, arena, snap, true);
    const int nsuf_steps = in.ns - in.K;
    for (int sidx = 0; sidx < a.nsuf; sidx++) {
        cs = at_k;
        double lp = -INFINITY;
        if (!cs.dead) {
            if (sidx > 0) team_copy(tm, st[in.K], a.tk + st[in.K].tk_off, arena, snap, false);
            const int8_t *sb = a.suf_bits + in.suf_off + ((int64_t)pre * a.nsuf + sidx) * nsuf_steps;
            for (int k = in.K; k < in.ns && !cs.dead; k++)
                chain_update(cs, team_step(tm, st[k], a.tk + st[k].tk_off, arena, sb[k - in.K], cs.scale));
            if (!cs.dead) lp = log2(cs.prev) + 2.0 * cs.lsc - in.n;
        }
        if (tm.rank() == 0) a.log2p[in.out_off + (int64_t)pre * a.nsuf + sidx] = lp;
    }
    tm.sync();
}

template <typename E>
__global__ void k_batch(const BatchArgs a) {
    __shared__ int s_item;
    const size_t big = (size_t)1 << a.big_R, small = (size_t)1 << a.small_R;
    E *arena = reinterpret_cast<E *>(a.big_arena) + (size_t)blockIdx.x * 2 * big;
    BlockTeam bt;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(&a.queues[0], 1u);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= a.n_big) break;
        run_item<E>(bt, a, a.items_big[it], arena, arena + big);
    }
    const int warps = (int)(blockDim.x >> 5), w = (int)(threadIdx.x >> 5);
    E *wa = reinterpret_cast<E *>(a.small_arena) + ((size_t)blockIdx.x * warps + (size_t)w) * 2 * small;
    WarpTeam wt;
    for (;;) {
        int it = 0;
        if ((threadIdx.x & 31) == 0) it = (int)atomicAdd(&a.queues[1], 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= a.n_small) break;
        run_item<E>(wt, a, a.items_small[it], wa, wa + small);
    }
}

struct BatchShape {
    int block = 256, small_R = 12, per_sm = 2;
    bool operator<(const BatchShape &o) const {
        return std::tie(block, small_R, per_sm) < std::tie(o.block, o.small_R, o.per_sm);
    }
};

struct BatchEngine {
    int prec = 64, dev = 0, sms = 0;
    size_t esize = 8;
    std::vector<HPlan> plans;
    std::vector<BStep> h_steps;
    std::vector<uint64_t> h_tk;
    std::vector<double> cost;       // per instance: entries moved by one prefix + its suffixes (relative)
    BStep *d_steps = nullptr;
    uint64_t *d_tk = nullptr;
    BInst *d_inst = nullptr;
    int *d_items = nullptr;
    int8_t *d_pre = nullptr, *d_suf = nullptr;
    double *d_out = nullptr;
    unsigned int *d_q = nullptr;
    void *d_arena = nullptr;
    size_t arena_bytes = 0;
    int npre = 0, nsuf = 0;
    int64_t pre_total = 0, suf_total = 0, out_total = 0;
    std::vector<BInst> h_inst;
    cudaStream_t stream = nullptr;
    BatchShape shape;
    bool tuned = false;
    std::map<BatchShape, cudaGraphExec_t> graphs;

    ~BatchEngine() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        cudaFree(d_steps);
        cudaFree(d_tk);
        cudaFree(d_inst);
        cudaFree(d_items);
        cudaFree(d_pre);
        cudaFree(d_suf);
        cudaFree(d_out);
        cudaFree(d_q);
        cudaFree(d_arena);
        if (stream) cudaStreamDestroy(stream);
        cudaSetDevice(prev);
    }

    int max_R() const {
        int r = 0;
        for (const HPlan &p : plans) r = std::max(r, p.R);
        return r;
    }
};

}  // namespace gsb

using namespace gsb;

#define BT_CK(x)                                                                                                  \
    do {                                                                                                          \
        cudaError_t e_ = (x);                                                                                     \
        if (e_ != cudaSuccess) return fail(GSB_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #x); \
    } while (0)

struct gsb_batch {
    BatchEngine E;
};

// Lay out the items of a shape: wide instances to the block-team queue, narrow ones to the warp-team queue, each in
// decreasing cost; size the team arenas.  Returns the device bytes the shape needs.
static size_t shape_layout(const BatchEngine &E, const BatchShape &sh, std::vector<int> &big, std::vector<int> &small,
                           int &big_R, int &small_R, int &grid) {
    big.clear();
    small.clear();
    big_R = 0;
    small_R = 0;
    std::vector<int> order(E.plans.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int x, int y) { return E.cost[(size_t)x] > E.cost[(size_t)y]; });
    for (int i : order) {
        const int R = E.plans[(size_t)i].R;
        auto &q = R <= sh.small_R ? small : big;
        for (int p = 0; p < E.npre; p++) q.push_back(i * E.npre + p);
        if (R <= sh.small_R) small_R = std::max(small_R, R);
        else big_R = std::max(big_R, R);
    }
    grid = E.sms * sh.per_sm;
    const size_t warps = (size_t)grid * (size_t)(sh.block / 32);
    return E.esize * 2 * ((size_t)grid * ((size_t)1 << big_R) + warps * ((size_t)1 << small_R));
}

static int batch_graph(BatchEngine &E, const BatchShape &sh, cudaGraphExec_t *out) {
    auto it = E.graphs.find(sh);
    if (it != E.graphs.end()) {
        *out = it->second;
        return 0;
    }
    std::vector<int> big, small;
    int big_R, small_R, grid;
    const size_t need = shape_layout(E, sh, big, small, big_R, small_R, grid);
    if (need > E.arena_bytes) {
        cudaFree(E.d_arena);
        E.d_arena = nullptr;
        E.arena_bytes = 0;
        for (auto &kv : E.graphs) cudaGraphExecDestroy(kv.second);   // they point at the old arena
        E.graphs.clear();
        BT_CK(cudaMalloc(&E.d_arena, need));
        E.arena_bytes = need;
    }
    cudaFree(E.d_items);
    E.d_items = nullptr;
    std::vector<int> items(big);
    items.insert(items.end(), small.begin(), small.end());
    BT_CK(cudaMalloc(&E.d_items, std::max<size_t>(items.size(), 1) * sizeof(int)));
    if (!items.empty())
        BT_CK(cudaMemcpy(E.d_items, items.data(), items.size() * sizeof(int), cudaMemcpyHostToDevice));
    for (auto &kv : E.graphs) cudaGraphExecDestroy(kv.second);   // items buffer changed
    E.graphs.clear();
    BatchArgs a;
    a.steps = E.d_steps;
    a.tk = E.d_tk;
    a.inst = E.d_inst;
    a.items_big = E.d_items;
    a.items_small = E.d_items + big.size();
    a.n_big = (int)big.size();
    a.n_small = (int)small.size();
    a.npre = E.npre;
    a.nsuf = E.nsuf;
    a.pre_bits = E.d_pre;
    a.suf_bits = E.d_suf;
    a.log2p = E.d_out;
    a.queues = E.d_q;
    a.big_arena = E.d_arena;
    a.small_arena = static_cast<char *>(E.d_arena) + E.esize * 2 * (size_t)grid * ((size_t)1 << big_R);
    a.big_R = big_R;
    a.small_R = small_R;
    cudaGraph_t g = nullptr;
    BT_CK(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(E.d_q, 0, 2 * sizeof(unsigned int), E.stream);
    if (E.prec == 128) k_batch<double2><<<grid, sh.block, 0, E.stream>>>(a);
    else k_batch<float2><<<grid, sh.block, 0, E.stream>>>(a);
    cudaError_t e = cudaGetLastError();
    cudaError_t e2 = cudaStreamEndCapture(E.stream, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        BT_CK(e);
    }
    BT_CK(e2);
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    BT_CK(e);
    E.graphs[sh] = ex;
    *out = ex;
    return 0;
}

extern "C" {

int gsb_batch_open(const char *const *texts, const size_t *lens, int ninst, int precision, int device, gsb_batch **out) {
    if (!texts || !lens || !out || ninst < 1) return fail(GSB_E_USAGE, "bad argument");
    *out = nullptr;
    if (precision != 64 && precision != 128) return fail(GSB_E_USAGE, "precision must be 64 or 128");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(GSB_E_CUDA, "no CUDA device is visible");
    if (device < 0 || device >= ndev) return fail(GSB_E_USAGE, "device out of range");
    gsb_batch *h = new gsb_batch();
    BatchEngine &E = h->E;
    E.prec = precision;
    E.esize = precision == 128 ? 16 : 8;
    E.dev = device;
    E.plans.resize((size_t)ninst);
    for (int i = 0; i < ninst; i++) {
        std::string err;
        int rc = parse_plan_text(texts[i], lens[i], E.plans[(size_t)i], err);
        if (!rc) rc = validate_plan(E.plans[(size_t)i], err);
        if (!rc && E.plans[(size_t)i].ns < 2) {
            rc = GSB_E_USAGE;
            err = "a batched instance needs at least 2 steps";
        }
        if (!rc && E.plans[(size_t)i].R > 24) {
            rc = GSB_E_USAGE;
            err = "batched instances are limited to width 24 (one team arena each)";
        }
        if (rc) {
            delete h;
            return fail(rc, "instance " + std::to_string(i) + ": " + err);
        }
    }
    for (const HPlan &p : E.plans) {
        double c = 0;
        for (int k = 0; k < p.ns; k++) {
            const HStep &s = p.st[(size_t)k];
            BStep b;
            memset(&b, 0, sizeof b);
            b.nk = s.nk;
            b.ntq = (int)s.tqs.size();
            b.m = s.m;
            b.g = s.m == 2 ? s.g : 0;
            b.rhoc = s.rhoc;
            for (int t = 0; t < b.ntq; t++) {
                b.tq[t] = s.tqs[(size_t)t];
                b.tau0[t] = s.tau0[t];
                b.tau1[t] = s.tau1[t];
                b.par[t] = s.par[t];
            }
            for (int bb = 0; bb < 2; bb++)
                for (int x = 0; x < 2; x++) {
                    b.M[4 * bb + 2 * x] = s.Mr[bb][x];
                    b.M[4 * bb + 2 * x + 1] = s.Mi[bb][x];
                }
            b.tk_off = (int)E.h_tk.size();
            for (int j = 0; j < s.nk; j++) E.h_tk.push_back(s.tk[(size_t)j]);
            E.h_steps.push_back(b);
            c += std::ldexp(1.0, s.nk) * (double)(b.ntq + b.m);
        }
        E.cost.push_back(c);
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    struct Restore {
        int p;
        ~Restore() { cudaSetDevice(p); }
    } restore{prev};
    cudaDeviceGetAttribute(&E.sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&E.d_steps, E.h_steps.size() * sizeof(BStep));
    if (e == cudaSuccess) e = cudaMalloc(&E.d_tk, std::max<size_t>(E.h_tk.size(), 1) * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc(&E.d_q, 2 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemcpy(E.d_steps, E.h_steps.data(), E.h_steps.size() * sizeof(BStep), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !E.h_tk.empty())
        e = cudaMemcpy(E.d_tk, E.h_tk.data(), E.h_tk.size() * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        delete h;
        return fail(GSB_E_ALLOC, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    *out = h;
    return 0;
}

int gsb_batch_close(gsb_batch *h) {
    delete h;
    return 0;
}

int gsb_batch_set_strings(gsb_batch *h, const int *K, int npre, int nsuf, const int8_t *prefix_bits,
                          const int8_t *suffix_bits) {
    if (!h || !K || npre < 1 || nsuf < 1 || !prefix_bits || !suffix_bits) return fail(GSB_E_USAGE, "bad argument");
    BatchEngine &E = h->E;
    const int ninst = (int)E.plans.size();
    std::vector<BInst> inst((size_t)ninst);
    int64_t po = 0, so = 0, oo = 0;
    int step_off = 0;
    for (int i = 0; i < ninst; i++) {
        const HPlan &p = E.plans[(size_t)i];
        if (K[i] < 1 || K[i] >= p.ns) return fail(GSB_E_USAGE, "prefix length must be in [1, ns) for instance " + std::to_string(i));
        BInst b;
        b.ns = p.ns;
        b.R = p.R;
        b.K = K[i];
        b.n = p.n;
        b.step_off = step_off;
        b.pre_off = po;
        b.suf_off = so;
        b.out_off = oo;
        step_off += p.ns;
        po += (int64_t)npre * K[i];
        so += (int64_t)npre * nsuf * (p.ns - K[i]);
        oo += (int64_t)npre * nsuf;
        inst[(size_t)i] = b;
    }
    for (int64_t i = 0; i < po; i++)
        if (prefix_bits[i] != 0 && prefix_bits[i] != 1) return fail(GSB_E_USAGE, "bits must be 0 or 1");
    for (int64_t i = 0; i < so; i++)
        if (suffix_bits[i] != 0 && suffix_bits[i] != 1) return fail(GSB_E_USAGE, "bits must be 0 or 1");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(E.dev);
    struct Restore {
        int p;
        ~Restore() { cudaSetDevice(p); }
    } restore{prev};
    const bool resize = po != E.pre_total || so != E.suf_total || oo != E.out_total || npre != E.npre || nsuf != E.nsuf;
    if (resize) {
        for (auto &kv : E.graphs) cudaGraphExecDestroy(kv.second);
        E.graphs.clear();
        cudaFree(E.d_pre);
        cudaFree(E.d_suf);
        cudaFree(E.d_out);
        cudaFree(E.d_inst);
        E.d_pre = nullptr;
        E.d_suf = nullptr;
        E.d_out = nullptr;
        E.d_inst = nullptr;
        BT_CK(cudaMalloc(&E.d_pre, (size_t)std::max<int64_t>(po, 1)));
        BT_CK(cudaMalloc(&E.d_suf, (size_t)std::max<int64_t>(so, 1)));
        BT_CK(cudaMalloc(&E.d_out, (size_t)std::max<int64_t>(oo, 1) * sizeof(double)));
        BT_CK(cudaMalloc(&E.d_inst, (size_t)ninst * sizeof(BInst)));
        E.pre_total = po;
        E.suf_total = so;
        E.out_total = oo;
        E.npre = npre;
        E.nsuf = nsuf;
    }
    BT_CK(cudaMemcpy(E.d_inst, inst.data(), (size_t)ninst * sizeof(BInst), cudaMemcpyHostToDevice));
    BT_CK(cudaMemcpy(E.d_pre, prefix_bits, (size_t)po, cudaMemcpyHostToDevice));
    BT_CK(cudaMemcpy(E.d_suf, suffix_bits, (size_t)so, cudaMemcpyHostToDevice));
    E.h_inst = inst;
    return 0;
}

// Run the batch with the current shape (the tuned one after gsb_batch_tune); log2p: per instance [npre][nsuf].
int gsb_batch_run(gsb_batch *h, double *log2p, float *ms) {
    if (!h || !log2p) return fail(GSB_E_USAGE, "null argument");
    BatchEngine &E = h->E;
    if (!E.d_out) return fail(GSB_E_STATE, "no strings set (gsb_batch_set_strings)");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(E.dev);
    struct Restore {
        int p;
        ~Restore() { cudaSetDevice(p); }
    } restore{prev};
    cudaGraphExec_t ex;
    if (int rc = batch_graph(E, E.shape, &ex)) return rc;
    cudaEvent_t e0, e1;
    BT_CK(cudaEventCreate(&e0));
    BT_CK(cudaEventCreate(&e1));
    BT_CK(cudaEventRecord(e0, E.stream));
    BT_CK(cudaGraphLaunch(ex, E.stream));
    BT_CK(cudaEventRecord(e1, E.stream));
    BT_CK(cudaMemcpyAsync(log2p, E.d_out, (size_t)E.out_total * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    BT_CK(cudaStreamSynchronize(E.stream));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

// The largest block the batch kernel of this precision can launch with (its registers per thread bound it), or 0.
static int batch_max_block(const BatchEngine &E) {
    cudaFuncAttributes fa{};
    const cudaError_t e = E.prec == 128 ? cudaFuncGetAttributes(&fa, k_batch<double2>) : cudaFuncGetAttributes(&fa, k_batch<float2>);
    return e == cudaSuccess ? fa.maxThreadsPerBlock : 0;
}

int gsb_batch_set_shape(gsb_batch *h, int block, int small_R, int per_sm) {
    if (!h || (block != 64 && block != 128 && block != 256 && block != 512 && block != 1024) || small_R < 0 ||
        small_R > 24 || per_sm < 1 || per_sm > 16 || block * per_sm > 2048)
        return fail(GSB_E_USAGE, "bad shape");
    if (block > batch_max_block(h->E)) return fail(GSB_E_USAGE, "block larger than the batch kernel can launch");
    h->E.shape = BatchShape{block, small_R, per_sm};
    return 0;
}

int gsb_batch_get_shape(const gsb_batch *h, int *block, int *small_R, int *per_sm) {
    if (!h) return fail(GSB_E_STATE, "null handle");
    if (block) *block = h->E.shape.block;
    if (small_R) *small_R = h->E.shape.small_R;
    if (per_sm) *per_sm = h->E.shape.per_sm;
    return 0;
}

// Autotuner: times every candidate shape on the current strings (one warm-up and `reps` timed runs each, CUDA
// events on the batch stream) and keeps the fastest.  Candidates whose arenas exceed `max_bytes` are skipped.
int gsb_batch_tune(gsb_batch *h, int reps, size_t max_bytes, int *block, int *small_R, int *per_sm, float *best_ms) {
    if (!h || reps < 1) return fail(GSB_E_USAGE, "bad argument");
    BatchEngine &E = h->E;
    if (!E.d_out) return fail(GSB_E_STATE, "no strings set (gsb_batch_set_strings)");
    std::vector<double> out((size_t)std::max<int64_t>(E.out_total, 1));
    float best = 1e30f;
    BatchShape bs = E.shape;
    const int maxR = E.max_R();
    const int max_block = batch_max_block(E);   // shapes the kernel cannot launch are skipped
    for (int blk : {128, 256, 512})
        for (int sr : {0, 8, 10, 12, 14})
            for (int ps : {1, 2, 4}) {
                if (blk * ps > 2048 || sr > maxR + 1 || blk > max_block) continue;
                BatchShape sh{blk, sr, ps};
                std::vector<int> big, small;
                int bR, sR, grid;
                if (shape_layout(E, sh, big, small, bR, sR, grid) > max_bytes) continue;
                E.shape = sh;
                float ms = 0, tot = 0;
                if (int rc = gsb_batch_run(h, out.data(), &ms)) return rc;
                for (int r = 0; r < reps; r++) {
                    if (int rc = gsb_batch_run(h, out.data(), &ms)) return rc;
                    tot += ms;
                }
                if (tot / reps < best) {
                    best = tot / reps;
                    bs = sh;
                }
            }
    E.shape = bs;
    E.tuned = true;
    if (block) *block = bs.block;
    if (small_R) *small_R = bs.small_R;
    if (per_sm) *per_sm = bs.per_sm;
    if (best_ms) *best_ms = best;
    return 0;
}

}  // extern "C"
