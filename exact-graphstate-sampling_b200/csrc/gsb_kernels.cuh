// Device side of the in-place cut-rank DP executor for sm_100a.
//
// One DP step is one streaming pass over the live part of the 2^R arena (reference gsamp2.cpp:39-120, whose
// `outputs` gsamp2.cpp:32-38 is the per-coset arithmetic):
//   for every coset c < 2^nk:  base = XOR_{j in c} Tkeep[j]
//       v_i  = mem[base ^ tq_i]                                  (the 2^q slots of the coset, q <= 2)
//       S0[tau0_i] += v_i;  S1[tau1_i] += (-1)^(parity(c & rhoc) ^ par_i) v_i     (x = 0 / x = 1 terms)
//       out[b][tau] = M[b][0] S0[tau] + M[b][1] S1[tau]
//   norm pass : n_b += sum_tau |out[b][tau]|^2
//   write pass: mem[base] = sc out[bv][0];  if m = 2: mem[base ^ g] = sc out[bv][1];   nb += |written|^2
// Each coset reads and overwrites only its own slots, so the pass is race-free with one thread per coset.
//
// Layout of a launch: a block covers chunks of 2^chunk_log2 consecutive cosets; thread t handles cosets
// chunk_base + t + u * blockDim (u < U).  In planner layouts the low coset bits map to the low arena bits
// (Tkeep[j] = 2^j), so for every offset tq a warp's 32 loads fall in one aligned segment (XOR with a constant only
// permutes lanes inside it): fully coalesced 256 B (complex64) or 512 B (complex128) per warp access.
//
// Reductions are deterministic: per-thread FP64 sums in coset order, a fixed warp-shuffle and block tree, one
// partial per block, and the last block to finish sums the partials in block order.  That block also runs the
// scalar step logic of the chosen mode (bit draw, scale, conditional, log2 Pr) on the device, so a whole string
// or sample runs without a host round trip (the reference's GPU port copies an accumulator back every step,
// gsamp_cuda.cu:74-83).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gsb_step.h"

namespace gsb {

enum Driver : int {
    DRV_CHAIN = 0,   // normalised: norm pass, draw/force, write with 1/sqrt(n_b)      (gsamp2.cpp:39-55)
    DRV_CHAIN1 = 1,  // one pass, unnormalised storage, cond = nb / (2 prev)         (gsamp2.cpp:59-70)
    DRV_HYBRID = 2,  // lazily rescaled run_steps: optional norm pass, write with 1/sqrt(prev)   (gsamp2.cpp:77-98)
};

struct DevState {
    double prev;      // norm of the stored table
    double lsc;       // CHAIN1: stored amplitudes = true amplitudes * 2^-lsc
    double logscale;  // HYBRID: the reference's running logscale
    double logp;      // running log2 probability
    double sc;        // scale of the next write (CHAIN: 1/sqrt(n_b); CHAIN1: 2^-ek)
    double n0, n1;    // last branch norms of a step (norm pass, or the trailing step of a fused sampling pass)
    double aux;       // resume: log2 Pr(prefix)
    int ek;           // CHAIN1: exponent of the next write's power-of-two scale
    int bv;           // bit of the next write
    int dead;         // a zero-probability branch was taken: later passes do nothing
    int item;         // index of the string / sample being evaluated
    unsigned int counter;   // blocks finished in the current launch
    int err;                // a bounded pipeline wait gave up (reported to the host, cleared when read)
    int trx;                // n0, n1 were expanded from a trailing step's shared sums (fused sampling passes)
};

struct Ctx {
    DevState *st;
    double *partials;        // [gridDim][2]
    const int8_t *forced;    // [cap][ns] or null
    const double *unif;      // [cap][ns] or null
    int8_t *bits_out;        // [cap][ns]
    double *cond_out;        // [cap][ns]
    int ns;
    int driver;
    int k1;                  // end of the step range of this run (HYBRID zero-fill)
    int tpb_log2;            // log2 blockDim
    int chunk_log2;          // log2 cosets per chunk (= tpb_log2 + log2 U)
    unsigned int nchunks;
};

__device__ __forceinline__ void load_entry(const float2 *p, double &re, double &im) {
    const float2 v = *p;
    re = v.x;
    im = v.y;
}
__device__ __forceinline__ void load_entry(const double2 *p, double &re, double &im) {
    const double2 v = *p;
    re = v.x;
    im = v.y;
}
__device__ __forceinline__ void store_entry(float2 *p, double re, double im) { *p = make_float2((float)re, (float)im); }
__device__ __forceinline__ void store_entry(double2 *p, double re, double im) { *p = make_double2(re, im); }

// XOR of tks[j] over the set bits j of c (c may have bits up to 39)
__device__ __forceinline__ uint64_t xor_cols(const uint64_t *tks, uint64_t c) {
    uint64_t a = 0;
    while (c) {
        const int j = __ffsll((long long)c) - 1;
        a ^= tks[j];
        c &= c - 1;
    }
    return a;
}


// Block-wide sum of (a0, a1) into partials[blockIdx]; returns true in thread 0 of the last block to finish, with
// the grid totals in (t0, t1).  All threads of the block must call it.
__device__ __forceinline__ bool grid_reduce2(double a0, double a1, const Ctx &cx, double &t0, double &t1) {
    __shared__ double red[2][32];
    __shared__ int last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    if (lane == 0) { red[0][warp] = a0; red[1][warp] = a1; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0;
        for (int w = 0; w < nw; w++) { s0 += red[0][w]; s1 += red[1][w]; }
        cx.partials[2 * blockIdx.x] = s0;
        cx.partials[2 * blockIdx.x + 1] = s1;
        __threadfence();
        const unsigned int done = atomicAdd(&cx.st->counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // the last block sums the partials in block order: thread t takes blocks t, t + blockDim, ... then a fixed tree
    double s0 = 0, s1 = 0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        s0 += __ldcg(cx.partials + 2 * b);
        s1 += __ldcg(cx.partials + 2 * b + 1);
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    __syncthreads();
    if (lane == 0) { red[0][warp] = s0; red[1][warp] = s1; }
    __syncthreads();
    if (threadIdx.x != 0) return false;
    t0 = 0;
    t1 = 0;
    for (int w = 0; w < nw; w++) { t0 += red[0][w]; t1 += red[1][w]; }
    cx.st->counter = 0;
    return true;
}

// Scalar logic after a norm pass (one thread).
__device__ __forceinline__ void norm_epilogue(const Ctx &cx, int k, double n0, double n1) {
    DevState *st = cx.st;
    st->n0 = n0;
    st->n1 = n1;
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    if (cx.driver == DRV_CHAIN) {
        const double p1 = n1 / (n0 + n1);
        int bv;
        if (cx.forced) bv = cx.forced[row + k];
        else bv = cx.unif[row + k] < p1;
        const double pb = bv ? p1 : 1 - p1;
        if (pb <= 0) {
            st->dead = 1;
            st->logp = -INFINITY;
            for (int j = k; j < cx.ns; j++) cx.bits_out[row + j] = cx.forced ? cx.forced[row + j] : 0;
            return;
        }
        st->logp += log2(pb);
        cx.bits_out[row + k] = (int8_t)bv;
        st->bv = bv;
        st->sc = 1.0 / sqrt(bv ? n1 : n0);
    } else {   // DRV_HYBRID, a '?' step
        st->bv = cx.unif[row + k] < n1 / (n0 + n1);
    }
}

// Scalar logic after a write pass (one thread).
__device__ __forceinline__ void write_epilogue(const Ctx &cx, int k, int bv, double nb) {
    DevState *st = cx.st;
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    if (cx.driver == DRV_CHAIN) {
        st->prev = nb;
    } else if (cx.driver == DRV_CHAIN1) {
        // the write scaled by 2^-ek; the conditional is scale free: nb_true / (2 prev_true)
        cx.cond_out[row + k] = ldexp(nb, 2 * st->ek) / (2 * st->prev);
        st->lsc += st->ek;
        st->prev = nb;
        if (nb <= 0) {
            for (int j = k; j < cx.ns; j++) cx.cond_out[row + j] = 0;
            st->dead = 1;
            st->logp = -INFINITY;
            return;
        }
        int ex;
        frexp(nb, &ex);                      // nb = f 2^ex, f in [0.5, 1)
        st->ek = (ex - 1) >> 1;              // next write scales by 2^-ek: the stored norm stays near 1
        st->sc = ldexp(1.0, -st->ek);
    } else {   // DRV_HYBRID
        const double prev = st->prev;
        st->logscale += 0.5 * log2(prev);
        const double c = nb / 2;
        cx.cond_out[row + k] = c;
        cx.bits_out[row + k] = (int8_t)bv;
        st->prev = nb;
        if (nb <= 0) {
            for (int j = k; j < cx.k1; j++) {
                cx.cond_out[row + j] = 0;
                const int f = cx.forced[row + j];
                cx.bits_out[row + j] = (int8_t)(f < 0 ? 0 : f);
            }
            st->dead = 1;
            st->logp = -INFINITY;
            return;
        }
        st->logp += log2(c);
    }
}

template <typename E, int NTQ, int MOUT, int U, bool WRITE>
__global__ void __launch_bounds__(256) k_step(const StepArgs s, E *__restrict__ mem, const Ctx cx) {
    DevState *st = cx.st;
    if (*(volatile int *)&st->dead) return;
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    int bv = 0;
    double sc = 1.0;
    if (WRITE) {
        if (cx.driver == DRV_HYBRID) {
            const int f = cx.forced[row + s.k];
            bv = f >= 0 ? f : st->bv;
            sc = 1.0 / sqrt(st->prev);
        } else if (cx.driver == DRV_CHAIN1) {
            bv = cx.forced[row + s.k];
            sc = st->sc;
        } else {
            bv = st->bv;
            sc = st->sc;
        }
    } else if (cx.driver == DRV_HYBRID && cx.forced[row + s.k] >= 0) {
        return;   // forced step of a hybrid run: no norm pass (uniform across the grid)
    }

    __shared__ uint64_t tks[40];
    for (int j = threadIdx.x; j < 40; j += blockDim.x) tks[j] = s.tk[j];
    __syncthreads();

    const int tid = threadIdx.x;
    const int tl = cx.tpb_log2;
    uint64_t Tt = 0;
    for (int j = 0; j < tl; j++)
        if ((tid >> j) & 1) Tt ^= tks[j];
    const int pt = __popcll((unsigned long long)tid & s.rhoc) & 1;
    uint64_t Tu[U];
    int pu[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const uint64_t cu = (uint64_t)u << tl;
        Tu[u] = xor_cols(tks, cu);
        pu[u] = __popcll(cu & s.rhoc) & 1;
    }
    // M row of the written branch (write pass)
    const double m0r = bv ? s.Mr[1][0] : s.Mr[0][0], m0i = bv ? s.Mi[1][0] : s.Mi[0][0];
    const double m1r = bv ? s.Mr[1][1] : s.Mr[0][1], m1i = bv ? s.Mi[1][1] : s.Mi[0][1];

    double a0 = 0, a1 = 0;
    const bool act = (unsigned int)tid < (1u << tl);   // blocks of < 32 cosets keep a full warp; the rest idle
    for (unsigned int ch = act ? blockIdx.x : cx.nchunks; ch < cx.nchunks; ch += gridDim.x) {
        const uint64_t cb = (uint64_t)ch << cx.chunk_log2;
        const uint64_t bh = xor_cols(tks, cb) ^ Tt;
        const int ph = (__popcll(cb & s.rhoc) & 1) ^ pt;
        double vr[U][NTQ], vi[U][NTQ];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t b = bh ^ Tu[u];
#pragma unroll
            for (int i = 0; i < NTQ; i++) load_entry(mem + (b ^ s.tq[i]), vr[u][i], vi[u][i]);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int pc = ph ^ pu[u];
            // S[x][tau]
            double s00r = 0, s00i = 0, s01r = 0, s01i = 0, s10r = 0, s10i = 0, s11r = 0, s11i = 0;
#pragma unroll
            for (int i = 0; i < NTQ; i++) {
                const double xr = vr[u][i], xi = vi[u][i];
                if (MOUT == 1 || s.tau0[i] == 0) { s00r += xr; s00i += xi; }
                else { s01r += xr; s01i += xi; }
                const bool neg = (pc ^ s.par[i]) != 0;
                const double yr = neg ? -xr : xr, yi = neg ? -xi : xi;
                if (MOUT == 1 || s.tau1[i] == 0) { s10r += yr; s10i += yi; }
                else { s11r += yr; s11i += yi; }
            }
            const uint64_t b = bh ^ Tu[u];
            if (WRITE) {
                double o0r = m0r * s00r - m0i * s00i + m1r * s10r - m1i * s10i;
                double o0i = m0r * s00i + m0i * s00r + m1r * s10i + m1i * s10r;
                o0r *= sc;
                o0i *= sc;
                store_entry(mem + b, o0r, o0i);
                a0 += o0r * o0r + o0i * o0i;
                if (MOUT == 2) {
                    double o1r = m0r * s01r - m0i * s01i + m1r * s11r - m1i * s11i;
                    double o1i = m0r * s01i + m0i * s01r + m1r * s11i + m1i * s11r;
                    o1r *= sc;
                    o1i *= sc;
                    store_entry(mem + (b ^ s.g), o1r, o1i);
                    a0 += o1r * o1r + o1i * o1i;
                }
            } else {
#pragma unroll
                for (int bb = 0; bb < 2; bb++) {
                    const double p0r = s.Mr[bb][0], p0i = s.Mi[bb][0], p1r = s.Mr[bb][1], p1i = s.Mi[bb][1];
                    const double o0r = p0r * s00r - p0i * s00i + p1r * s10r - p1i * s10i;
                    const double o0i = p0r * s00i + p0i * s00r + p1r * s10i + p1i * s10r;
                    double nn = o0r * o0r + o0i * o0i;
                    if (MOUT == 2) {
                        const double o1r = p0r * s01r - p0i * s01i + p1r * s11r - p1i * s11i;
                        const double o1i = p0r * s01i + p0i * s01r + p1r * s11i + p1i * s11r;
                        nn += o1r * o1r + o1i * o1i;
                    }
                    if (bb == 0) a0 += nn;
                    else a1 += nn;
                }
            }
        }
    }
    double t0, t1;
    if (!grid_reduce2(a0, a1, cx, t0, t1)) return;
    if (WRITE) write_epilogue(cx, s.k, bv, t0);
    else norm_epilogue(cx, s.k, t0, t1);
}

// ---------------------------------------------------------------------------------------------------------------
// A run of consecutive small steps (at most 2^SMALL_NK cosets each) in one launch of one CTA.  One k_step launch
// per small step costs several microseconds of launch gap and dependent global round trips (state, partials,
// counter) for a few kilobytes of table; the two ends of a string or sample are two dozen such steps.  Here the
// CTA walks the steps itself: per step, the same coset arithmetic as k_step (FP64, in place on the arena; the
// block's threads own disjoint cosets, and a block barrier separates the steps), the norm pass first when `norm` is
// set (sampling and hybrid drivers; skipped for a forced hybrid step), a block-tree reduction in a fixed order, and
// the same scalar epilogues run by thread 0.  Step descriptors come from the device copy of the engine's StepArgs.
constexpr int SMALL_NK = 11;          // steps of up to 2^11 cosets join a run
constexpr int SMALL_THREADS = 512;    // 4 cosets per thread at most
constexpr int SMALL_U = (1 << SMALL_NK) / SMALL_THREADS;

template <typename E>
__global__ void __launch_bounds__(SMALL_THREADS) k_small_run(const StepArgs *__restrict__ sa, int k0, int k1, int norm,
                                                             E *__restrict__ mem, const Ctx cx) {
    __shared__ StepArgs s;
    __shared__ double red[2][SMALL_THREADS / 32];
    __shared__ int sh_skip, sh_bv;
    __shared__ double sh_sc;
    DevState *st = cx.st;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    for (int k = k0; k < k1; k++) {
        __syncthreads();   // the previous step's readers of s and sh_* are done
        {
            const uint64_t *src = reinterpret_cast<const uint64_t *>(sa + k);
            uint64_t *dst = reinterpret_cast<uint64_t *>(&s);
            for (int i = tid; i < (int)(sizeof(StepArgs) / 8); i += SMALL_THREADS) dst[i] = src[i];
        }
        for (int ph = norm ? 0 : 1; ph < 2; ph++) {
            const bool write = ph == 1;
            if (ph == 1 && norm) __syncthreads();   // the norm phase's readers of sh_* are done
            if (tid == 0) {
                int skip = *(volatile int *)&st->dead;
                int bv = 0;
                double sc = 1.0;
                if (!skip) {
                    if (write) {
                        if (cx.driver == DRV_HYBRID) {
                            const int f = cx.forced[row + k];
                            bv = f >= 0 ? f : st->bv;
                            sc = 1.0 / sqrt(st->prev);
                        } else if (cx.driver == DRV_CHAIN1) {
                            bv = cx.forced[row + k];
                            sc = st->sc;
                        } else {
                            bv = st->bv;
                            sc = st->sc;
                        }
                    } else if (cx.driver == DRV_HYBRID && cx.forced[row + k] >= 0) {
                        skip = 2;   // forced hybrid step: no norm pass
                    }
                }
                sh_skip = skip;
                sh_bv = bv;
                sh_sc = sc;
            }
            __syncthreads();
            if (sh_skip == 1) return;      // a zero-probability branch was taken: nothing more to do
            if (sh_skip == 2) continue;
            const int bv = sh_bv;
            const double sc = sh_sc;
            const uint64_t N = 1ULL << s.nk;
            const int ntq = s.ntq, mout = s.m;
            const double m0r = bv ? s.Mr[1][0] : s.Mr[0][0], m0i = bv ? s.Mi[1][0] : s.Mi[0][0];
            const double m1r = bv ? s.Mr[1][1] : s.Mr[0][1], m1i = bv ? s.Mi[1][1] : s.Mi[0][1];
            double a0 = 0, a1 = 0;
            double vr[SMALL_U][4], vi[SMALL_U][4];
            uint64_t base[SMALL_U];
#pragma unroll
            for (int u = 0; u < SMALL_U; u++) {
                const uint64_t c = (uint64_t)tid + (uint64_t)u * SMALL_THREADS;
                base[u] = c < N ? xor_cols(s.tk, c) : 0;
#pragma unroll
                for (int i = 0; i < 4; i++)
                    if (c < N && i < ntq) load_entry(mem + (base[u] ^ s.tq[i]), vr[u][i], vi[u][i]);
            }
#pragma unroll
            for (int u = 0; u < SMALL_U; u++) {
                const uint64_t c = (uint64_t)tid + (uint64_t)u * SMALL_THREADS;
                if (c >= N) continue;
                const int pc = __popcll(c & s.rhoc) & 1;
                double s00r = 0, s00i = 0, s01r = 0, s01i = 0, s10r = 0, s10i = 0, s11r = 0, s11i = 0;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (i >= ntq) break;
                    const double xr = vr[u][i], xi = vi[u][i];
                    if (mout == 1 || s.tau0[i] == 0) { s00r += xr; s00i += xi; }
                    else { s01r += xr; s01i += xi; }
                    const bool neg = (pc ^ s.par[i]) != 0;
                    const double yr = neg ? -xr : xr, yi = neg ? -xi : xi;
                    if (mout == 1 || s.tau1[i] == 0) { s10r += yr; s10i += yi; }
                    else { s11r += yr; s11i += yi; }
                }
                if (write) {
                    double o0r = m0r * s00r - m0i * s00i + m1r * s10r - m1i * s10i;
                    double o0i = m0r * s00i + m0i * s00r + m1r * s10i + m1i * s10r;
                    o0r *= sc;
                    o0i *= sc;
                    store_entry(mem + base[u], o0r, o0i);
                    a0 += o0r * o0r + o0i * o0i;
                    if (mout == 2) {
                        double o1r = m0r * s01r - m0i * s01i + m1r * s11r - m1i * s11i;
                        double o1i = m0r * s01i + m0i * s01r + m1r * s11i + m1i * s11r;
                        o1r *= sc;
                        o1i *= sc;
                        store_entry(mem + (base[u] ^ s.g), o1r, o1i);
                        a0 += o1r * o1r + o1i * o1i;
                    }
                } else {
#pragma unroll
                    for (int bb = 0; bb < 2; bb++) {
                        const double p0r = s.Mr[bb][0], p0i = s.Mi[bb][0], p1r = s.Mr[bb][1], p1i = s.Mi[bb][1];
                        const double o0r = p0r * s00r - p0i * s00i + p1r * s10r - p1i * s10i;
                        const double o0i = p0r * s00i + p0i * s00r + p1r * s10i + p1i * s10r;
                        double nn = o0r * o0r + o0i * o0i;
                        if (mout == 2) {
                            const double o1r = p0r * s01r - p0i * s01i + p1r * s11r - p1i * s11i;
                            const double o1i = p0r * s01i + p0i * s01r + p1r * s11i + p1i * s11r;
                            nn += o1r * o1r + o1i * o1i;
                        }
                        if (bb == 0) a0 += nn;
                        else a1 += nn;
                    }
                }
            }
            a0 = warp_sum(a0);
            a1 = warp_sum(a1);
            if (lane == 0) { red[0][warp] = a0; red[1][warp] = a1; }
            __syncthreads();   // the partial sums, and every store of this pass, are visible to the block
            if (tid == 0) {
                double t0 = 0, t1 = 0;
                for (int w = 0; w < SMALL_THREADS / 32; w++) { t0 += red[0][w]; t1 += red[1][w]; }
                if (write) write_epilogue(cx, k, bv, t0);
                else norm_epilogue(cx, k, t0, t1);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Wide-step kernels.  Steps with at least 2^11 cosets run one of these instead of k_step; both
//   * walk their block's range of chunks in Gray-code order, so consecutive chunks differ in one coset bit and the
//     chunk's base address is updated with one XOR (chunk i covers cosets gray(i) * 2^chunk_log2 + [0, 2^chunk_log2));
//   * fold the step's scale into the M row of the write pass (one uniform multiply per kernel, not per entry);
//   * prepare the write/norm decision exactly as k_step does (same prologue, same epilogues).

struct Prologue {
    int bv;
    double sc;
    bool skip;
};

__device__ __forceinline__ Prologue step_prologue(const StepArgs &s, const Ctx &cx, bool write) {
    Prologue P{0, 1.0, false};
    DevState *st = cx.st;
    if (*(volatile int *)&st->dead) { P.skip = true; return P; }
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    if (write) {
        if (cx.driver == DRV_HYBRID) {
            const int f = cx.forced[row + s.k];
            P.bv = f >= 0 ? f : st->bv;
            P.sc = 1.0 / sqrt(st->prev);
        } else if (cx.driver == DRV_CHAIN1) {
            P.bv = cx.forced[row + s.k];
            P.sc = st->sc;
        } else {
            P.bv = st->bv;
            P.sc = st->sc;
        }
    } else if (cx.driver == DRV_HYBRID && cx.forced[row + s.k] >= 0) {
        P.skip = true;
    }
    return P;
}

// chunk range of this block: [i0, i1) of gray-code indices
__device__ __forceinline__ void block_range(unsigned int nch, unsigned int &i0, unsigned int &i1) {
    const unsigned int per = (nch + gridDim.x - 1) / gridDim.x;
    i0 = min(nch, blockIdx.x * per);
    i1 = min(nch, i0 + per);
}

__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return fma(a, b, c); }

// complex64 arena, two adjacent cosets per thread and per 16-byte access.  Requires Tkeep[0] = 1 (coset bit 0 is arena
// bit 0, as the planner lays out wide steps): cosets c (even) and c + 1 have bases b and b ^ 1, so each coset offset
// tq, and the two write targets, address one aligned pair of entries; a swap flag (bit 0 of the address) says which
// half belongs to the even coset.  Norms are accumulated in FP64.
// Arithmetic type T:
//   double: the coset's pair sums of float entries are exact in FP64 (the compensated form), the rotation by M is
//           done in FP64, and the only rounding is the store to complex64 -- the arithmetic of the reference's
//           complex64 build (gsamp2.cpp:32-38, 52);
//   float : sums and rotation in FP32 (a few roundings per entry; faster on the FP32 pipe).
// Chunk = 256 threads x U pairs = 2^(9 + log2 U) cosets; pair u of thread t covers cosets 2t + 512u + {0, 1}.
template <typename T, int NTQ, int MOUT, int U, bool WRITE>
__global__ void __launch_bounds__(256) k_pair64(const StepArgs s, float2 *__restrict__ mem, const Ctx cx) {
    const Prologue P = step_prologue(s, cx, WRITE);
    if (P.skip) return;
    __shared__ uint64_t tks[40];
    for (int j = threadIdx.x; j < 40; j += blockDim.x) tks[j] = s.tk[j];
    __syncthreads();
    const int tid = threadIdx.x;
    const int cl = cx.chunk_log2;
    float4 *__restrict__ mem4 = reinterpret_cast<float4 *>(mem);
    // M rows: write pass uses sc * M[bv][x]; norm pass both rows
    T wr[2][2], wi[2][2];
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
        for (int x = 0; x < 2; x++) {
            const int bb = WRITE ? P.bv : b;
            const double f = WRITE ? P.sc : 1.0;
            // FP32 arithmetic takes the engine's float-rounded coefficients; FP64 the plan's own
            const bool f32 = sizeof(T) == 4;
            wr[b][x] = (T)(f * (f32 ? s.Mr32[bb][x] : s.Mr[bb][x]));
            wi[b][x] = (T)(f * (f32 ? s.Mi32[bb][x] : s.Mi[bb][x]));
        }
    uint64_t Tt = 0;
    for (int j = 0; j < 8; j++)
        if ((tid >> j) & 1) Tt ^= tks[j + 1];
    const int pt = __popcll((uint64_t)(2 * tid) & s.rhoc) & 1;
    uint64_t Tu[U];
    int pu[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const uint64_t cu = (uint64_t)u << 9;
        Tu[u] = xor_cols(tks, cu);
        pu[u] = __popcll(cu & s.rhoc) & 1;
    }
    const int podd = (int)(s.rhoc & 1);
    double a0 = 0, a1 = 0;
    unsigned int i0, i1;
    block_range(cx.nchunks, i0, i1);
    uint64_t bh = 0;
    int ph = 0;
    if (i0 < i1) {
        const uint64_t cb = (uint64_t)(i0 ^ (i0 >> 1)) << cl;
        bh = xor_cols(tks, cb) ^ Tt;
        ph = (__popcll(cb & s.rhoc) & 1) ^ pt;
    }
    for (unsigned int i = i0; i < i1; i++) {
        if (i > i0) {
            const int j = __ffs((int)i) - 1 + cl;   // gray(i) = gray(i - 1) ^ 2^ctz(i)
            bh ^= tks[j];
            ph ^= (int)((s.rhoc >> j) & 1);
        }
        float4 v[U][NTQ];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t be = bh ^ Tu[u];
#pragma unroll
            for (int t = 0; t < NTQ; t++) v[u][t] = mem4[(be ^ s.tq[t]) >> 1];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t be = bh ^ Tu[u];
            const int pe = ph ^ pu[u];
            T S[2][2][2][2] = {};   // [coset e/o][x][tau][re/im]
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                const bool sw = ((be ^ s.tq[t]) & 1) != 0;
                const T er = sw ? v[u][t].z : v[u][t].x, ei = sw ? v[u][t].w : v[u][t].y;
                const T orr = sw ? v[u][t].x : v[u][t].z, oi = sw ? v[u][t].y : v[u][t].w;
                const int t0 = MOUT == 1 ? 0 : s.tau0[t], t1 = MOUT == 1 ? 0 : s.tau1[t];
                const bool ne = ((pe ^ s.par[t]) & 1) != 0, no = ((pe ^ podd ^ s.par[t]) & 1) != 0;
#pragma unroll
                for (int tau = 0; tau < MOUT; tau++) {
                    if (t0 == tau) {
                        S[0][0][tau][0] += er; S[0][0][tau][1] += ei;
                        S[1][0][tau][0] += orr; S[1][0][tau][1] += oi;
                    }
                    if (t1 == tau) {
                        S[0][1][tau][0] += ne ? -er : er; S[0][1][tau][1] += ne ? -ei : ei;
                        S[1][1][tau][0] += no ? -orr : orr; S[1][1][tau][1] += no ? -oi : oi;
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < (WRITE ? 1 : 2); b++) {
                float o[2][MOUT][2];   // [eo][tau][re/im], rounded to the arena type
                T nn = 0;
#pragma unroll
                for (int eo = 0; eo < 2; eo++)
#pragma unroll
                    for (int tau = 0; tau < MOUT; tau++) {
                        const T *s0 = S[eo][0][tau], *s1 = S[eo][1][tau];
                        T r = wr[b][0] * s0[0];
                        r = fmaT(-wi[b][0], s0[1], r);
                        r = fmaT(wr[b][1], s1[0], r);
                        r = fmaT(-wi[b][1], s1[1], r);
                        T im = wr[b][0] * s0[1];
                        im = fmaT(wi[b][0], s0[0], im);
                        im = fmaT(wr[b][1], s1[1], im);
                        im = fmaT(wi[b][1], s1[0], im);
                        o[eo][tau][0] = (float)r;
                        o[eo][tau][1] = (float)im;
                        nn = fmaT(r, r, nn);
                        nn = fmaT(im, im, nn);
                    }
                if (b == 0) a0 += (double)nn;
                else a1 += (double)nn;
                if (WRITE) {
                    const bool s0w = (be & 1) != 0;
                    mem4[be >> 1] = s0w ? make_float4(o[1][0][0], o[1][0][1], o[0][0][0], o[0][0][1])
                                        : make_float4(o[0][0][0], o[0][0][1], o[1][0][0], o[1][0][1]);
                    if (MOUT == 2) {
                        const uint64_t bg = be ^ s.g;
                        const bool s1w = (bg & 1) != 0;
                        const int t1 = MOUT - 1;
                        mem4[bg >> 1] = s1w ? make_float4(o[1][t1][0], o[1][t1][1], o[0][t1][0], o[0][t1][1])
                                            : make_float4(o[0][t1][0], o[0][t1][1], o[1][t1][0], o[1][t1][1]);
                    }
                }
            }
        }
    }
    double t0, t1;
    if (!grid_reduce2(a0, a1, cx, t0, t1)) return;
    if (WRITE) write_epilogue(cx, s.k, P.bv, t0);
    else norm_epilogue(cx, s.k, t0, t1);
}

// complex128 arena, one coset per thread and per 16-byte entry; FP64 arithmetic.
// Chunk = 256 threads x U cosets = 2^(8 + log2 U) cosets; coset u of thread t is t + 256u.
template <int NTQ, int MOUT, int U, bool WRITE>
__global__ void __launch_bounds__(256) k_wide128(const StepArgs s, double2 *__restrict__ mem, const Ctx cx) {
    const Prologue P = step_prologue(s, cx, WRITE);
    if (P.skip) return;
    __shared__ uint64_t tks[40];
    for (int j = threadIdx.x; j < 40; j += blockDim.x) tks[j] = s.tk[j];
    __syncthreads();
    const int tid = threadIdx.x;
    const int cl = cx.chunk_log2;
    double wr[2][2], wi[2][2];
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
        for (int x = 0; x < 2; x++) {
            const int bb = WRITE ? P.bv : b;
            const double f = WRITE ? P.sc : 1.0;
            wr[b][x] = f * s.Mr[bb][x];
            wi[b][x] = f * s.Mi[bb][x];
        }
    uint64_t Tt = 0;
    for (int j = 0; j < 8; j++)
        if ((tid >> j) & 1) Tt ^= tks[j];
    const int pt = __popcll((uint64_t)tid & s.rhoc) & 1;
    uint64_t Tu[U];
    int pu[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const uint64_t cu = (uint64_t)u << 8;
        Tu[u] = xor_cols(tks, cu);
        pu[u] = __popcll(cu & s.rhoc) & 1;
    }
    double a0 = 0, a1 = 0;
    unsigned int i0, i1;
    block_range(cx.nchunks, i0, i1);
    uint64_t bh = 0;
    int ph = 0;
    if (i0 < i1) {
        const uint64_t cb = (uint64_t)(i0 ^ (i0 >> 1)) << cl;
        bh = xor_cols(tks, cb) ^ Tt;
        ph = (__popcll(cb & s.rhoc) & 1) ^ pt;
    }
    for (unsigned int i = i0; i < i1; i++) {
        if (i > i0) {
            const int j = __ffs((int)i) - 1 + cl;
            bh ^= tks[j];
            ph ^= (int)((s.rhoc >> j) & 1);
        }
        double2 v[U][NTQ];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t b = bh ^ Tu[u];
#pragma unroll
            for (int t = 0; t < NTQ; t++) v[u][t] = mem[b ^ s.tq[t]];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t b = bh ^ Tu[u];
            const int pc = ph ^ pu[u];
            double S[2][2][2] = {};   // [x][tau][re/im]
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                const int t0 = MOUT == 1 ? 0 : s.tau0[t], t1 = MOUT == 1 ? 0 : s.tau1[t];
                const bool ng = ((pc ^ s.par[t]) & 1) != 0;
#pragma unroll
                for (int tau = 0; tau < MOUT; tau++) {
                    if (t0 == tau) { S[0][tau][0] += v[u][t].x; S[0][tau][1] += v[u][t].y; }
                    if (t1 == tau) { S[1][tau][0] += ng ? -v[u][t].x : v[u][t].x; S[1][tau][1] += ng ? -v[u][t].y : v[u][t].y; }
                }
            }
#pragma unroll
            for (int b2 = 0; b2 < (WRITE ? 1 : 2); b2++) {
                double nn = 0;
#pragma unroll
                for (int tau = 0; tau < MOUT; tau++) {
                    const double r = wr[b2][0] * S[0][tau][0] - wi[b2][0] * S[0][tau][1] + wr[b2][1] * S[1][tau][0] - wi[b2][1] * S[1][tau][1];
                    const double im = wr[b2][0] * S[0][tau][1] + wi[b2][0] * S[0][tau][0] + wr[b2][1] * S[1][tau][1] + wi[b2][1] * S[1][tau][0];
                    nn += r * r + im * im;
                    if (WRITE) mem[tau == 0 ? b : (b ^ s.g)] = make_double2(r, im);
                }
                if (b2 == 0) a0 += nn;
                else a1 += nn;
            }
        }
    }
    double t0, t1;
    if (!grid_reduce2(a0, a1, cx, t0, t1)) return;
    if (WRITE) write_epilogue(cx, s.k, P.bv, t0);
    else norm_epilogue(cx, s.k, t0, t1);
}

// Start of a string / sample: the unit table and a fresh state.
template <typename E>
__global__ void k_begin(E *mem, DevState *st) {
    store_entry(mem, 1.0, 0.0);
    st->prev = 1.0;
    st->lsc = 0;
    st->logscale = 0;
    st->logp = 0;
    st->sc = 1.0;
    st->ek = 0;
    st->bv = 0;
    st->dead = 0;
    st->counter = 0;
    st->aux = 0;
    st->trx = 0;
}

// End of a string / sample: final log2 Pr, next item.
static __global__ void k_finish(DevState *st, double *logp_out, double *aux_out, int driver, int ns) {
    const int it = st->item;
    double lp;
    if (driver == DRV_CHAIN1) lp = st->dead ? -INFINITY : log2(st->prev) + 2.0 * st->lsc - ns;
    else lp = st->logp;
    logp_out[it] = lp;
    if (aux_out) aux_out[it] = driver == DRV_HYBRID ? st->logscale : st->aux;
    st->item = it + 1;
}

static __global__ void k_set_item(DevState *st, int item) { st->item = item; }

// Hybrid item whose first K steps are forced and ran as 'chain' passes (DRV_CHAIN1): from here on the run_steps
// conventions (gsamp2.cpp:77-98).  The stored table is the true one times 2^-lsc, which is run_steps' logscale;
// log2 Pr of the prefix is log2 |table|^2 + 2 lsc - K.  The forced bits of the prefix go to the output row.
static __global__ void k_hybrid_switch(DevState *st, const int8_t *forced, int8_t *bits_out, int ns, int K) {
    const size_t row = (size_t)st->item * (size_t)ns;
    for (int k = 0; k < K; k++) bits_out[row + k] = forced[row + k];
    if (st->dead) {   // a zero-probability prefix: the chain epilogue zeroed every conditional from there on
        for (int k = K; k < ns; k++) bits_out[row + k] = (int8_t)(forced[row + k] < 0 ? 0 : forced[row + k]);
        st->logp = -INFINITY;
        return;
    }
    st->logp = log2(st->prev) + 2.0 * st->lsc - K;
    st->logscale = st->lsc;
}

// Live table at step K in logical (c, tq) order (the reference's prefix dump, gsamp2.cpp:170-174).
template <typename E>
__global__ void k_gather(const StepArgs s, const E *__restrict__ mem, int ntq, E *__restrict__ out) {
    __shared__ uint64_t tks[40];
    for (int j = threadIdx.x; j < 40; j += blockDim.x) tks[j] = s.tk[j];
    __syncthreads();
    const uint64_t N = (1ULL << s.nk) * (uint64_t)ntq;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = i / (uint64_t)ntq;
        const int j = (int)(i % (uint64_t)ntq);
        out[i] = mem[xor_cols(tks, c) ^ s.tq[j]];
    }
}

// Resume: sum the slice dumps into the arena (gsamp2.cpp:196-205): entry (c, ti) of the sum is
// sum_s f_s * dump_s[(c ^ cshift_s) * ntq + tperm_s[ti]], rounded to the arena type; the norm of the unrounded sum
// goes to the state (prev), with logscale = L and aux = log2 Pr(prefix) = -K + log2(norm) + 2L.
struct ResumeArgs {
    const void *const *dumps;   // device array of nsl device pointers
    const double *f;            // [nsl]
    const uint64_t *cshift;     // [nsl]
    const int *tperm;           // [nsl][4]
    int nsl, ntq, K;
    double L;
};

template <typename E>
__global__ void k_resume_sum(const StepArgs s, E *__restrict__ mem, const ResumeArgs ra, const Ctx cx) {
    __shared__ uint64_t tks[40];
    for (int j = threadIdx.x; j < 40; j += blockDim.x) tks[j] = s.tk[j];
    __syncthreads();
    const uint64_t N = 1ULL << s.nk;
    const int nt = ra.ntq;
    double a0 = 0;
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < N; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = xor_cols(tks, c);
        for (int ti = 0; ti < nt; ti++) {
            double ar = 0, ai = 0;
            for (int sl = 0; sl < ra.nsl; sl++) {
                const E *d = (const E *)ra.dumps[sl];
                const uint64_t idx = (c ^ ra.cshift[sl]) * (uint64_t)nt + (uint64_t)ra.tperm[4 * sl + ti];
                double vr, vi;
                load_entry(d + idx, vr, vi);
                ar += vr * ra.f[sl];
                ai += vi * ra.f[sl];
            }
            store_entry(mem + (base ^ s.tq[ti]), ar, ai);
            a0 += ar * ar + ai * ai;
        }
    }
    double t0, t1;
    if (!grid_reduce2(a0, 0.0, cx, t0, t1)) return;
    DevState *st = cx.st;
    st->prev = t0;
    st->logscale = ra.L;
    st->logp = 0;
    st->dead = 0;
    st->aux = -ra.K + log2(t0) + 2 * ra.L;
}

}  // namespace gsb
