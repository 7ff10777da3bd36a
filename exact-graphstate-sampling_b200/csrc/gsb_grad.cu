// Adjoint sweep of the in-place cut-rank DP (complex128): gradients of log Pr(b) with respect to the step matrices.
//
// The forward sweep of a string b is linear in every table and in every step's M row:
//   T_{k+1} = L_k(M_k[b_k]) T_k,   Z(b) = T_ns[0],   Pr(b) = 2^-n |Z(b)|^2,
// with the step map of the executor (gsamp2.cpp:32-38, 59-66): for every coset c of step k, base = XOR of Tkeep
// over the bits of c, the inputs v_t = T_k[base ^ tq_t] and
//   out[tau] = sum_{t: tau0_t = tau} m0 v_t + sum_{t: tau1_t = tau} m1 s_t v_t,   s_t = (-1)^(parity(c & rhoc) ^ par_t),
// m_x = M_k[b_k][x], stored at base (tau 0) and base ^ g (tau 1).  The reverse sweep carries lambda_k = dZ/dT_k
// backwards through the transposed step map (the same cosets and slots, read and written the other way round):
//   lambda_k[base ^ tq_t] = m0 lambda_{k+1}[tau0_t] + m1 s_t lambda_{k+1}[tau1_t],
//   dZ/dm0 = sum_t lambda_{k+1}[tau0_t] v_t,       dZ/dm1 = sum_t s_t lambda_{k+1}[tau1_t] v_t,
// with lambda_ns = 1 at the final entry.  Each coset reads and writes only its own slots, so the reverse pass is
// in place and race-free like the forward one.  The reverse pass needs T_k: the forward sweep keeps a compact copy
// of the live table ([coset][offset], 2^{r_k} entries) every `every` steps, and each segment between two
// checkpoints is recomputed forward once, keeping its tables, before the reverse pass walks it.  Up to 32 strings
// are swept together (grid dimension y: each string owns its arenas, checkpoints, segment tables and reduction
// slots), and the whole sequence of such a launch (forward, then per segment: restore, recompute, reverse) is one
// CUDA graph; the first string's index lives in device memory and advances at its end.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "gsb.h"
#include "gsb_common.h"
#include "gsb_plan.h"
#include "gsb_step.h"

namespace gsb {

// A launch sweeps `bs` strings at once: string y = blockIdx.y is item *item + y and owns slot y of every buffer.
struct GradCtx {
    const double *M;         // [ns][2][2] (re, im): the caller's matrices
    const int8_t *bits;      // [cap][ns]
    const int *item;         // first string of the launch
    int ns, maxgrid;
    size_t arena;            // entries per string: T and Lam arenas
};

__device__ __forceinline__ uint64_t coset_base(const StepArgs &s, uint64_t c) {
    uint64_t b = 0;
    while (c) {
        const int j = __ffsll((long long)c) - 1;
        b ^= s.tk[j];
        c &= c - 1;
    }
    return b;
}

// The cosets a thread visits (grid x times block: a power of two, 2^ls threads): c = t | (g << ls) for the Gray
// codes g of the high bits, so the base is the thread's fixed low part XOR one running value (one XOR per coset).
template <typename F>
__device__ __forceinline__ void grid_cosets(const StepArgs &s, F f) {
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const int ls = __ffsll((long long)nthreads) - 1;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s.nk < ls && t >= (1ULL << s.nk)) return;
    const uint64_t lo = coset_base(s, t);
    const uint64_t nh = s.nk > ls ? 1ULL << (s.nk - ls) : 1;
    uint64_t hi = 0;
    for (uint64_t n = 0; n < nh; n++) {
        if (n) hi ^= s.tk[ls + __ffsll((long long)n) - 1];
        f(t | ((n ^ (n >> 1)) << ls), lo ^ hi);
    }
}

// The same walk, two consecutive Gray-code cosets per call: f(c0, base0, c1, base1, two), the second only when two.
template <typename F>
__device__ __forceinline__ void grid_cosets2(const StepArgs &s, F f) {
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const int ls = __ffsll((long long)nthreads) - 1;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s.nk < ls && t >= (1ULL << s.nk)) return;
    const uint64_t lo = coset_base(s, t);
    const uint64_t nh = s.nk > ls ? 1ULL << (s.nk - ls) : 1;
    uint64_t hi = 0;
    for (uint64_t n = 0; n < nh; n += 2) {
        if (n) hi ^= s.tk[ls + __ffsll((long long)n) - 1];
        const bool two = n + 1 < nh;
        const uint64_t hi1 = two ? hi ^ s.tk[ls] : hi;   // Gray step n -> n + 1 flips high bit 0
        f(t | ((n ^ (n >> 1)) << ls), lo ^ hi, t | (((n + 1) ^ ((n + 1) >> 1)) << ls), lo ^ hi1, two);
        hi = hi1;
    }
}

__device__ __forceinline__ void step_row(const StepArgs &s, const GradCtx &g, double2 &m0, double2 &m1) {
    const int b = g.bits[(size_t)(*g.item + (int)blockIdx.y) * (size_t)g.ns + (size_t)s.k];
    const double *Mk = g.M + (size_t)s.k * 8 + 4 * b;
    m0 = make_double2(Mk[0], Mk[1]);
    m1 = make_double2(Mk[2], Mk[3]);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }

__global__ void k_gr_begin(double2 *T, const GradCtx g) { T[blockIdx.y * g.arena] = make_double2(1.0, 0.0); }

// Forward step on the T arena: gathers the input table to `gather` ([c][t], if given) and, if `write`, stores the
// step's outputs in place.  Two cosets per iteration, both cosets' loads first (distinct cosets never share a slot),
// so a thread has twice the loads in flight (7 % off the sweep); NTQ (the step's offsets) is a template parameter, so
// the loaded values stay in registers.
template <int NTQ>
__global__ void __launch_bounds__(256) k_gr_fwd(const StepArgs s, double2 *__restrict__ T, double2 *__restrict__ gather,
                                                size_t gather_stride, int write, const GradCtx g) {
    double2 m0, m1;
    step_row(s, g, m0, m1);
    T += blockIdx.y * g.arena;
    if (gather) gather += blockIdx.y * gather_stride;
    auto one = [&](uint64_t c, uint64_t base, const double2 (&v)[NTQ]) {
        const int pc = __popcll(c & s.rhoc) & 1;
        double2 o0 = make_double2(0, 0), o1 = make_double2(0, 0);   // scalars: no runtime-indexed arrays
#pragma unroll
        for (int t = 0; t < NTQ; t++) {
            if (gather) gather[c * (uint64_t)NTQ + (uint64_t)t] = v[t];
            const double2 a = cmul(m0, v[t]), b = cscale((pc ^ s.par[t]) ? -1.0 : 1.0, cmul(m1, v[t]));
            if (s.tau0[t]) o1 = cadd(o1, a); else o0 = cadd(o0, a);
            if (s.tau1[t]) o1 = cadd(o1, b); else o0 = cadd(o0, b);
        }
        if (!write) return;
        T[base] = o0;
        if (s.m == 2) T[base ^ s.g] = o1;
    };
    grid_cosets2(s, [&](uint64_t c0, uint64_t b0, uint64_t c1, uint64_t b1, bool two) {
        double2 v0[NTQ], v1[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) {
            v0[t] = T[b0 ^ s.tq[t]];
            v1[t] = two ? T[b1 ^ s.tq[t]] : make_double2(0, 0);
        }
        one(c0, b0, v0);
        if (two) one(c1, b1, v1);
    });
}

// Restore a checkpoint: the compact table [c][t] back to its arena slots.
__global__ void __launch_bounds__(256) k_gr_scatter(const StepArgs s, const double2 *__restrict__ src, size_t src_stride,
                                                    double2 *__restrict__ T, const GradCtx g) {
    src += blockIdx.y * src_stride;
    T += blockIdx.y * g.arena;
    grid_cosets(s, [&](uint64_t c, uint64_t base) {
        for (int t = 0; t < s.ntq; t++) T[base ^ s.tq[t]] = src[c * (uint64_t)s.ntq + (uint64_t)t];
    });
}

// End of the forward sweep: Z = T[0]; lambda_ns = 1.
__global__ void k_gr_final(const double2 *T, double2 *Lam, double2 *z_out, const GradCtx g) {
    z_out[*g.item + (int)blockIdx.y] = T[blockIdx.y * g.arena];
    Lam[blockIdx.y * g.arena] = make_double2(1.0, 0.0);
}

__global__ void k_gr_next(int *item, int bs) { *item += bs; }
__global__ void k_gr_set_item(int *item, int v) { *item = v; }

// Reverse step: lambda_{k+1} (output slots of the Lam arena) -> lambda_k (input slots, in place), and
// dZ/dM_k[b_k][x] from the step's input table Tk ([c][t]).  Deterministic reduction: per-block partials, the last
// block sums them in block order and writes grad[item][k] = (dZ/dm0, dZ/dm1).
template <int NTQ>
__global__ void __launch_bounds__(256) k_gr_bwd(const StepArgs s, const double2 *__restrict__ Tk, size_t tk_stride,
                                                double2 *__restrict__ Lam, const GradCtx g, double *partials,
                                                unsigned int *counter, double *grad) {
    double2 m0, m1;
    step_row(s, g, m0, m1);
    Tk += blockIdx.y * tk_stride;
    Lam += blockIdx.y * g.arena;
    partials += (size_t)blockIdx.y * 4 * (size_t)g.maxgrid;
    counter += blockIdx.y;
    double a[4] = {0, 0, 0, 0};   // dZ/dm0 (re, im), dZ/dm1 (re, im)
    // two cosets per iteration: both cosets' lambda and input values are read before either writes (a coset writes
    // only its own slots)
    auto one = [&](uint64_t c, uint64_t base, double2 lam0, double2 lam1, const double2 (&v)[NTQ]) {
        const int pc = __popcll(c & s.rhoc) & 1;
#pragma unroll
        for (int t = 0; t < NTQ; t++) {
            const double sg = (pc ^ s.par[t]) ? -1.0 : 1.0;
            const double2 la = s.tau0[t] ? lam1 : lam0, lb = cscale(sg, s.tau1[t] ? lam1 : lam0);
            const double2 p0 = cmul(la, v[t]), p1 = cmul(lb, v[t]);
            a[0] += p0.x;
            a[1] += p0.y;
            a[2] += p1.x;
            a[3] += p1.y;
            Lam[base ^ s.tq[t]] = cadd(cmul(m0, la), cmul(m1, lb));
        }
    };
    grid_cosets2(s, [&](uint64_t c0, uint64_t b0, uint64_t c1, uint64_t b1, bool two) {
        const double2 z = make_double2(0, 0);
        const double2 l00 = Lam[b0], l01 = s.m == 2 ? Lam[b0 ^ s.g] : z;
        const double2 l10 = two ? Lam[b1] : z, l11 = two && s.m == 2 ? Lam[b1 ^ s.g] : z;
        double2 v0[NTQ], v1[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) {
            v0[t] = Tk[c0 * (uint64_t)NTQ + (uint64_t)t];
            v1[t] = two ? Tk[c1 * (uint64_t)NTQ + (uint64_t)t] : z;
        }
        one(c0, b0, l00, l01, v0);
        if (two) one(c1, b1, l10, l11, v1);
    });
    __shared__ double red[4][8];
    __shared__ int last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < 4; i++) a[i] = warp_sum(a[i]);
    if (lane == 0)
        for (int i = 0; i < 4; i++) red[i][warp] = a[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < 4; i++) {
            double t = 0;
            for (int w = 0; w < nw; w++) t += red[i][w];
            partials[4 * blockIdx.x + i] = t;
        }
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double t[4] = {0, 0, 0, 0};
    for (unsigned int b = 0; b < gridDim.x; b++)
        for (int i = 0; i < 4; i++) t[i] += __ldcg(partials + 4 * b + i);
    double *out = grad + ((size_t)(*g.item + (int)blockIdx.y) * (size_t)g.ns + (size_t)s.k) * 4;
    for (int i = 0; i < 4; i++) out[i] = t[i];
    *counter = 0;
}

// Blocks per launch: at most GSB_GRAD_GRID_MUL x maxgrid (8 per SM) over the launch's bs strings together.  Every
// block ends in a block reduction and an atomic (the reverse step) or is short-lived (forward), so a thread should
// walk several cosets: with the x extent sized per string alone, a launch of 32 strings made 32768 blocks of one or two
// cosets per thread, and the sweep ran 28 % slower than with 4 (timed 1, 2, 4, 8: 0.400, 0.370, 0.364, 0.383 s for
// 2048 strings at width 20, against 0.507 s uncapped).
#ifndef GSB_GRAD_GRID_MUL
#define GSB_GRAD_GRID_MUL 4
#endif

struct GradEngine {
    HPlan plan;
    int dev = 0, sms = 0, every = 4, cap = 1024, bs = 1;   // cap: strings per host batch, a multiple of bs
    std::vector<StepArgs> args;
    std::vector<size_t> ckpt_off;      // offset (entries) of step k's checkpoint in a string's checkpoint slot
    size_t arena = 0, ckpt_n = 0;      // entries per string: arena, checkpoints
    double2 *T = nullptr, *Lam = nullptr, *d_ckpt = nullptr, *d_seg = nullptr;
    size_t seg_stride = 0;             // entries per segment table
    double *d_M = nullptr, *partials = nullptr, *d_grad = nullptr;
    double2 *d_z = nullptr;
    int8_t *d_bits = nullptr;
    int *d_item = nullptr;
    unsigned int *d_counter = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int maxgrid = 1;

    ~GradEngine() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
        if (graph) cudaGraphExecDestroy(graph);
        cudaFree(T);
        cudaFree(Lam);
        cudaFree(d_ckpt);
        cudaFree(d_seg);
        cudaFree(d_M);
        cudaFree(partials);
        cudaFree(d_grad);
        cudaFree(d_z);
        cudaFree(d_bits);
        cudaFree(d_item);
        cudaFree(d_counter);
        if (stream) cudaStreamDestroy(stream);
        cudaSetDevice(prev);
    }

    // a power of two of blocks per string (grid_cosets splits a coset index into thread and Gray-walk bits), with
    // the launch's bs strings together at most GSB_GRAD_GRID_MUL * maxgrid blocks
    dim3 grid_of(const StepArgs &s) const {
        const uint64_t N = 1ULL << s.nk;
        const uint64_t cap = std::max<uint64_t>(1, (uint64_t)GSB_GRAD_GRID_MUL * (uint64_t)maxgrid / (uint64_t)bs);
        uint64_t want = std::max<uint64_t>(1, std::min<uint64_t>((N + 255) / 256, std::min<uint64_t>(cap, maxgrid))), gx = 1;
        while (gx * 2 <= want) gx *= 2;
        return dim3((unsigned)gx, (unsigned)bs);
    }
    GradCtx ctx() const { return GradCtx{d_M, d_bits, d_item, plan.ns, maxgrid, arena}; }
    size_t seg_per_string() const { return (size_t)std::max(0, every - 1) * seg_stride; }
    double2 *seg(int pos) const { return d_seg + (size_t)(pos - 1) * seg_stride; }   // pos = 1 .. every-1 (slot 0)

    // forward / reverse step launches, instantiated for the step's number of coset offsets
    void fwd(const StepArgs &s, double2 *gather, size_t gstride, int write, const GradCtx &g) {
        if (s.ntq == 1) k_gr_fwd<1><<<grid_of(s), 256, 0, stream>>>(s, T, gather, gstride, write, g);
        else if (s.ntq == 2) k_gr_fwd<2><<<grid_of(s), 256, 0, stream>>>(s, T, gather, gstride, write, g);
        else k_gr_fwd<4><<<grid_of(s), 256, 0, stream>>>(s, T, gather, gstride, write, g);
    }
    void bwd(const StepArgs &s, const double2 *tk, size_t tstride, const GradCtx &g) {
        if (s.ntq == 1) k_gr_bwd<1><<<grid_of(s), 256, 0, stream>>>(s, tk, tstride, Lam, g, partials, d_counter, d_grad);
        else if (s.ntq == 2) k_gr_bwd<2><<<grid_of(s), 256, 0, stream>>>(s, tk, tstride, Lam, g, partials, d_counter, d_grad);
        else k_gr_bwd<4><<<grid_of(s), 256, 0, stream>>>(s, tk, tstride, Lam, g, partials, d_counter, d_grad);
    }

    // The sequence of one launch of bs strings (captured once as a graph).
    cudaError_t enqueue() {
        const int ns = plan.ns;
        const GradCtx g = ctx();
        const dim3 one(1, (unsigned)bs);
        k_gr_begin<<<one, 1, 0, stream>>>(T, g);
        for (int k = 0; k < ns; k++) {
            const StepArgs &s = args[(size_t)k];
            fwd(s, k % every == 0 ? d_ckpt + ckpt_off[(size_t)k] : nullptr, ckpt_n, 1, g);
        }
        k_gr_final<<<one, 1, 0, stream>>>(T, Lam, d_z, g);
        for (int c = ((ns - 1) / every) * every; c >= 0; c -= every) {
            const int e = std::min(c + every, ns);
            const StepArgs &sc = args[(size_t)c];
            k_gr_scatter<<<grid_of(sc), 256, 0, stream>>>(sc, d_ckpt + ckpt_off[(size_t)c], ckpt_n, T, g);
            for (int j = c; j < e; j++) {   // recompute: gather T_j (j > c), write T_{j+1} (j < e - 1)
                if (j == c && e - 1 == c) break;
                const StepArgs &s = args[(size_t)j];
                fwd(s, j == c ? nullptr : seg(j - c), seg_per_string(), j < e - 1 ? 1 : 0, g);
            }
            for (int j = e - 1; j >= c; j--) {
                const StepArgs &s = args[(size_t)j];
                const double2 *tk = j == c ? d_ckpt + ckpt_off[(size_t)c] : seg(j - c);
                bwd(s, tk, j == c ? ckpt_n : seg_per_string(), g);
            }
        }
        k_gr_next<<<1, 1, 0, stream>>>(d_item, bs);
        return cudaGetLastError();
    }
};

}  // namespace gsb

using namespace gsb;

#define GR_CK(x)                                                                                                  \
    do {                                                                                                          \
        cudaError_t e_ = (x);                                                                                     \
        if (e_ != cudaSuccess) return fail(GSB_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #x); \
    } while (0)

struct gsb_grad {
    GradEngine E;
};

extern "C" {

int gsb_grad_open_text(const char *text, size_t len, int device, int every, gsb_grad **out) {
    if (!text || !out) return fail(GSB_E_USAGE, "null argument");
    *out = nullptr;
    if (every < 1 || every > 64) return fail(GSB_E_USAGE, "checkpoint interval must be 1..64");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(GSB_E_CUDA, "no CUDA device is visible");
    if (device < 0 || device >= ndev) return fail(GSB_E_USAGE, "device out of range");
    gsb_grad *h = new gsb_grad();
    GradEngine &E = h->E;
    std::string err;
    int rc = parse_plan_text(text, len, E.plan, err);
    if (!rc) rc = validate_plan(E.plan, err);
    if (rc) {
        delete h;
        return fail(rc, err);
    }
    const HPlan &p = E.plan;
    if (p.ns < 1) {
        delete h;
        return fail(GSB_E_USAGE, "plan has no steps");
    }
    const HStep &lastst = p.st[(size_t)p.ns - 1];
    if (lastst.nk != 0 || lastst.m != 1) {
        delete h;
        return fail(GSB_E_USAGE, "the last step must leave a single entry (nk = 0, m = 1)");
    }
    E.dev = device;
    E.every = every;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    struct Restore {
        int p;
        ~Restore() { cudaSetDevice(p); }
    } restore{prev};
    cudaDeviceGetAttribute(&E.sms, cudaDevAttrMultiProcessorCount, device);
    E.maxgrid = std::max(1, E.sms * 8);
    E.args.resize((size_t)p.ns);
    E.ckpt_off.assign((size_t)p.ns, 0);
    size_t ck = 0, maxr = 0;
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
        a.nk = s.nk;
        a.k = k;
        a.m = s.m;
        E.args[(size_t)k] = a;
        const size_t entries = ((size_t)1 << s.nk) * (size_t)a.ntq;
        maxr = std::max(maxr, entries);
        if (k % every == 0) {
            E.ckpt_off[(size_t)k] = ck;
            ck += entries;
        }
    }
    E.seg_stride = maxr;
    E.ckpt_n = ck;
    const size_t arena = (size_t)1 << p.R;
    E.arena = arena;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    // strings per launch: a power of two up to 32, each with its own arenas, checkpoints and segment tables, within
    // half of the free device memory
    const size_t per_string = 16 * (2 * arena + ck + (size_t)std::max(0, every - 1) * maxr) +
                              (size_t)E.maxgrid * 4 * sizeof(double);
    if (per_string > free_b / 10 * 9) {
        delete h;
        return fail(GSB_E_ALLOC, "arena, checkpoints and segment tables need " + std::to_string(per_string) +
                                     " bytes; the device has " + std::to_string(free_b) + " free");
    }
    E.bs = 1;
    while (E.bs < 32 && (size_t)(2 * E.bs) * per_string <= free_b / 2) E.bs *= 2;
    const size_t bs = (size_t)E.bs;
    cudaError_t e = cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&E.T, bs * arena * 16);
    if (e == cudaSuccess) e = cudaMalloc(&E.Lam, bs * arena * 16);
    if (e == cudaSuccess) e = cudaMalloc(&E.d_ckpt, bs * std::max<size_t>(ck, 1) * 16);
    if (e == cudaSuccess) e = cudaMalloc(&E.d_seg, bs * std::max<size_t>(E.seg_per_string(), 1) * 16);
    if (e == cudaSuccess) e = cudaMalloc(&E.d_M, (size_t)p.ns * 8 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&E.partials, bs * (size_t)E.maxgrid * 4 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&E.d_grad, (size_t)E.cap * (size_t)p.ns * 4 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&E.d_z, (size_t)E.cap * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&E.d_bits, (size_t)E.cap * (size_t)p.ns);
    if (e == cudaSuccess) e = cudaMalloc(&E.d_item, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&E.d_counter, bs * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(E.d_counter, 0, bs * sizeof(unsigned int), E.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(E.T, 0, bs * arena * 16, E.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(E.Lam, 0, bs * arena * 16, E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    if (e != cudaSuccess) {
        delete h;
        return fail(GSB_E_ALLOC, std::string("device allocation: ") + cudaGetErrorString(e));
    }
    *out = h;
    return 0;
}

int gsb_grad_close(gsb_grad *h) {
    delete h;
    return 0;
}

int gsb_grad_run(gsb_grad *h, const double *M, const int8_t *bits, int64_t nstr, double *z, double *dz) {
    if (!h) return fail(GSB_E_STATE, "null handle");
    if (nstr < 0 || (nstr && (!M || !bits || !z || !dz))) return fail(GSB_E_USAGE, "null argument");
    GradEngine &E = h->E;
    const int ns = E.plan.ns;
    for (int64_t i = 0; i < nstr * ns; i++)
        if (bits[i] != 0 && bits[i] != 1) return fail(GSB_E_USAGE, "bits must be 0 or 1");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(E.dev);
    struct Restore {
        int p;
        ~Restore() { cudaSetDevice(p); }
    } restore{prev};
    GR_CK(cudaMemcpyAsync(E.d_M, M, (size_t)ns * 8 * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    if (!E.graph) {
        cudaGraph_t gr = nullptr;
        GR_CK(cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = E.enqueue();
        cudaError_t e2 = cudaStreamEndCapture(E.stream, &gr);
        if (e != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            GR_CK(e);
        }
        GR_CK(e2);
        e = cudaGraphInstantiate(&E.graph, gr, 0);
        cudaGraphDestroy(gr);
        GR_CK(e);
    }
    for (int64_t off = 0; off < nstr; off += E.cap) {
        const int64_t nb = std::min<int64_t>(E.cap, nstr - off);
        const int64_t launches = (nb + E.bs - 1) / E.bs;   // the last launch's unused slots run all-zero strings
        GR_CK(cudaMemcpyAsync(E.d_bits, bits + off * ns, (size_t)(nb * ns), cudaMemcpyHostToDevice, E.stream));
        if (launches * E.bs > nb)
            GR_CK(cudaMemsetAsync(E.d_bits + nb * ns, 0, (size_t)((launches * E.bs - nb) * ns), E.stream));
        k_gr_set_item<<<1, 1, 0, E.stream>>>(E.d_item, 0);
        GR_CK(cudaGetLastError());
        for (int64_t i = 0; i < launches; i++) GR_CK(cudaGraphLaunch(E.graph, E.stream));
        GR_CK(cudaMemcpyAsync(z + 2 * off, E.d_z, (size_t)nb * 16, cudaMemcpyDeviceToHost, E.stream));
        GR_CK(cudaMemcpyAsync(dz + off * ns * 4, E.d_grad, (size_t)(nb * ns) * 4 * sizeof(double),
                              cudaMemcpyDeviceToHost, E.stream));
        GR_CK(cudaStreamSynchronize(E.stream));
    }
    return 0;
}

int gsb_grad_info(const gsb_grad *h, int *n, int *nsteps, int *R) {
    if (!h) return fail(GSB_E_STATE, "null handle");
    if (n) *n = h->E.plan.n;
    if (nsteps) *nsteps = h->E.plan.ns;
    if (R) *R = h->E.plan.R;
    return 0;
}

}  // extern "C"
