// Fused pass over a group of consecutive DP steps (host derivation in gsb_fuse.cpp).
//
// A CTA owns tiles of 2^L classes.  The classes of a tile have bases TB | p (p < 2^L, TB a multiple of 2^L), so for
// every stage-0 offset z the tile's inputs are one aligned block of 2^L entries at TB ^ (z & ~mask), with class p at
// position p ^ (z & mask); the same holds for the written stage's outputs.  A tile's input blocks are bulk-copied
// into shared memory (one cp.async.bulk per block, completion on an mbarrier) two tiles ahead of the computation, and
// the last step stores to the arena directly.  For each step s of the group, work items (pair of
// adjacent classes, member j) -- a warp takes 32 consecutive pairs of one member -- read the member's ntq stage-s
// values (adjacent classes are adjacent entries, so a pair is one 16-byte access for complex64), form the coset's
// sums with the sign parity(TB & lambda) ^ parity(p & lambda) ^ mpar_j, rotate by M[b_s] (the first step also
// applies the pass's scale), write the m stage-(s+1) values and add their squares to the step's norm.
// A class's outputs land only in its own input slots or in slots no class reads (checked on the host), so tiles are
// independent and the pass is race-free in place.
#pragma once
#include <type_traits>
#include "gsb_kernels.cuh"

namespace gsb {

struct GroupStepArgs {
    int nmem, ntq, m, k, kind;
    double c[2];              // analytic branch weights |M[b][0]|^2 + |M[b][1]|^2 (one-offset steps)
    int tau0[4], tau1[4], par[4];
    uint64_t lambda;
    double Mr[2][2], Mi[2][2];
    // factored written step (complex64 arena), per bit b: pivot column (-1: not factored), beta = M[b][1-piv] /
    // M[b][piv] and cp = |M[b][piv]|^2 (1 when not factored): the stored table is the true one divided by M[b][piv]
    int piv[2];
    double br[2], bi[2], cp[2];
    unsigned char in_idx[16][4], out_idx[16][2], mpar[16];
    // member j, offset t: position of its value in the stage buffer (index << L), XORed for the first step with the
    // low bits of its stage-0 offset (z0lo); a class pair's value sits at ioff ^ pc (factored complex64 passes)
    uint32_t ioff[16][4];
    uint32_t soff[16][2];   // member j, output tau: position of its stage-(s+1) value (index << L)
};

// first-bit source of a sampling pass (group_decide)
enum { GSRC_ANALYTIC = 0, GSRC_TRAILING = 1, GSRC_NORM = 2 };
// absolute accuracy assumed of a branch probability estimated from a trailing step's shared sums (FP32 sums of
// order A + B, rounded at 2^-24, over up to 2^30 entries in per-thread and per-tile partials)
constexpr double TRX_FLOOR = 1.0 / (1 << 20);

struct GroupArgs {
    int d, L, nbhi, ssz[4];
    int src;               // GSRC_*
    int withhold_loads;    // test hook (gsb_test_withhold_tile_loads): issue no tile loads, so every wait runs out
    uint64_t bhi[40];
    uint64_t blk_in[32];   // stage-0 offsets z_i, bits >= L: input block i of a tile is the arena block at TB ^ blk_in[i]
    uint64_t blk_out[32];  // written-stage offsets, bits >= L: output block i goes to the arena block at TB ^ blk_out[i]
    uint32_t z0lo[16][4];  // first step: member j, offset t -> bits < L of its stage-0 offset (position p ^ z0lo)
    uint32_t zdlo[16][2];  // last written step: member j, output tau -> bits < L of its offset
    // fold = 1 or 2 (complex64 sampling passes of two written steps whose second is a one-offset growth step, GK_1_0): the
    // second step's outputs are not kept in shared memory; the trailing step reads the stage before it and applies
    // that step's map per term: its member j, offset t reads stage-1 value fsrc[j][t], output ftau[j][t] of the
    // growth step's member fmem[j][t].  fold = 2: every trailing member reads one output of the growth step in all
    // its offsets (group_trail_fold2_pk)
    int fold;
    unsigned char fsrc[16][4], ftau[16][4], fmem[16][4];
    // last written step: member j, output tau -> its whole written-stage offset (blk_out ^ zdlo): the class pair of a
    // tile at base TB and position pc is stored at TB ^ ooff ^ pc (factored complex64 passes)
    uint64_t ooff[16][2];
    GroupStepArgs st[3];
};

template <typename T> struct CplxOf;
template <> struct CplxOf<float> { typedef float2 type; };
template <> struct CplxOf<double> { typedef double2 type; };

__device__ __forceinline__ void to_T(const float2 v, float &r, float &i) { r = v.x; i = v.y; }
__device__ __forceinline__ void to_T(const float2 v, double &r, double &i) { r = v.x; i = v.y; }
__device__ __forceinline__ void to_T(const double2 v, double &r, double &i) { r = v.x; i = v.y; }
__device__ __forceinline__ void to_T(const double2 v, float &r, float &i) { r = (float)v.x; i = (float)v.y; }
template <typename C> __device__ __forceinline__ C mkC(double r, double i);
template <> __device__ __forceinline__ float2 mkC<float2>(double r, double i) { return make_float2((float)r, (float)i); }
template <> __device__ __forceinline__ double2 mkC<double2>(double r, double i) { return make_double2(r, i); }
__device__ __forceinline__ float2 mkCf(float r, float i) { return make_float2(r, i); }

// Threads of a fused pass that run the steps: 256, the whole block, or (warp-specialised build) the first 256, with
// one load-issuing warp after them.
constexpr int GROUP_NCT = 256;

// Grid-wide deterministic sums of ND values (same scheme as grid_reduce2); true in thread 0 of the last block.
// Only the GROUP_NCT step threads contribute, so both builds sum in the same order.
template <int ND>
__device__ __forceinline__ bool grid_reduceN(double (&a)[ND], const Ctx &cx, double (&t)[ND]) {
    __shared__ double red[ND][32];
    __shared__ int last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = GROUP_NCT / 32;
#pragma unroll
    for (int i = 0; i < ND; i++) a[i] = warp_sum(a[i]);
    if (lane == 0 && warp < nw)
#pragma unroll
        for (int i = 0; i < ND; i++) red[i][warp] = a[i];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < ND; i++) {
            double s = 0;
            for (int w = 0; w < nw; w++) s += red[i][w];
            cx.partials[ND * blockIdx.x + i] = s;
        }
        __threadfence();
        const unsigned int done = atomicAdd(&cx.st->counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    if (*(volatile int *)&cx.st->err) {
        // a block of this launch gave up waiting (it counted itself and left): no totals, no epilogue
        if (threadIdx.x == 0) cx.st->counter = 0;
        return false;
    }
    double s[ND];
#pragma unroll
    for (int i = 0; i < ND; i++) s[i] = 0;
    for (unsigned int b = threadIdx.x; threadIdx.x < GROUP_NCT && b < gridDim.x; b += GROUP_NCT)
#pragma unroll
        for (int i = 0; i < ND; i++) s[i] += __ldcg(cx.partials + ND * b + i);
#pragma unroll
    for (int i = 0; i < ND; i++) s[i] = warp_sum(s[i]);
    __syncthreads();
    if (lane == 0 && warp < nw)
#pragma unroll
        for (int i = 0; i < ND; i++) red[i][warp] = s[i];
    __syncthreads();
    if (threadIdx.x != 0) return false;
#pragma unroll
    for (int i = 0; i < ND; i++) {
        t[i] = 0;
        for (int w = 0; w < nw; w++) t[i] += red[i][w];
    }
    cx.st->counter = 0;
    return true;
}

// Scalar logic after a fused chain1 pass: the conditionals of every step of the group (gsamp2.cpp:59-70).
// cp[s]: |M[b_s][piv]|^2 of a factored step (its stored norm is the true one over cp), 1 otherwise.
template <int D>
__device__ __forceinline__ void group_chain1_epilogue(const Ctx &cx, int k0, const double (&nb)[D], const double (&cp)[D]) {
    DevState *st = cx.st;
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    double prev = st->prev;
    double lcp = 0;
    for (int s = 0; s < D; s++) {
        const double c = (s == 0 ? ldexp(nb[0], 2 * st->ek) / (2 * prev) : nb[s] / (2 * nb[s - 1])) * cp[s];
        lcp += log2(cp[s]);
        cx.cond_out[row + k0 + s] = c;
        if (!(nb[s] > 0)) {
            for (int j = k0 + s; j < cx.ns; j++) cx.cond_out[row + j] = 0;
            st->dead = 1;
            st->logp = -INFINITY;
            st->prev = 0;
            return;
        }
        prev = nb[s];
    }
    st->lsc += st->ek + 0.5 * lcp;
    st->prev = nb[D - 1];
    int ex;
    frexp(nb[D - 1], &ex);
    st->ek = (ex - 1) >> 1;
    st->sc = ldexp(1.0, -st->ek);
}

// Permuted access of P adjacent classes (even p, then p + 1 when P = 2): class p + c sits at position pos ^ c of a
// block (pos = p ^ the offset's low bits), so a pair is two 8-byte accesses (no swap of the halves of one 16-byte
// access needed) and a complex128 class one 16-byte access.
template <int P>
__device__ __forceinline__ void ld_perm(const float2 *m, uint32_t pos, float (&r)[P], float (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) {
        const float2 v = m[pos ^ (uint32_t)c];
        r[c] = v.x; i[c] = v.y;
    }
}
template <int P>
__device__ __forceinline__ void ld_perm(const float2 *m, uint32_t pos, double (&r)[P], double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) {
        const float2 v = m[pos ^ (uint32_t)c];
        r[c] = v.x; i[c] = v.y;
    }
}
template <int P>
__device__ __forceinline__ void ld_perm(const double2 *m, uint32_t pos, double (&r)[P], double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) {
        const double2 v = m[pos ^ (uint32_t)c];
        r[c] = v.x; i[c] = v.y;
    }
}
template <int P>
__device__ __forceinline__ void st_perm(float2 *m, uint32_t pos, const float (&r)[P], const float (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) m[pos ^ (uint32_t)c] = make_float2(r[c], i[c]);
}
template <int P>
__device__ __forceinline__ void st_perm(float2 *m, uint32_t pos, const double (&r)[P], const double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) m[pos ^ (uint32_t)c] = make_float2((float)r[c], (float)i[c]);
}
template <int P>
__device__ __forceinline__ void st_perm(double2 *m, uint32_t pos, const double (&r)[P], const double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) m[pos ^ (uint32_t)c] = make_double2(r[c], i[c]);
}
// A class pair (even p, then p + 1) of a complex64 block as one aligned 16-byte access: the pair's two entries sit at
// pos and pos ^ 1 (pos = p ^ offset bits), i.e. in the 16 bytes at pos & ~1, swapped when bit 0 of the offset is set
// (uniform across a warp).  One access instead of two 8-byte ones at a 16-byte thread stride, which take twice the
// shared-memory wavefronts.
__device__ __forceinline__ void ld_pair16(const float2 *m, uint32_t pos, float (&r)[2], float (&i)[2]) {
    const float4 v = *reinterpret_cast<const float4 *>(m + (pos & ~1u));
    const bool sw = (pos & 1u) != 0;
    r[0] = sw ? v.z : v.x; i[0] = sw ? v.w : v.y;
    r[1] = sw ? v.x : v.z; i[1] = sw ? v.y : v.w;
}
__device__ __forceinline__ void st_pair16(float2 *m, uint32_t pos, const float (&r)[2], const float (&i)[2]) {
    float4 *q = reinterpret_cast<float4 *>(m + (pos & ~1u));
    if (pos & 1u) *q = make_float4(r[1], i[1], r[0], i[0]);   // a warp-uniform choice: one predicated store
    else *q = make_float4(r[0], i[0], r[1], i[1]);
}

// shared memory [index][class]: P consecutive values
template <int P>
__device__ __forceinline__ void lds_cls(const float2 *q, float (&r)[P], float (&i)[P]) {
    if (P >= 2) {
#pragma unroll
        for (int c = 0; c < P; c += 2) {
            const float4 v = *reinterpret_cast<const float4 *>(q + c);
            r[c] = v.x; i[c] = v.y; r[c + 1] = v.z; i[c + 1] = v.w;
        }
    } else {
        r[0] = q[0].x; i[0] = q[0].y;
    }
}
template <int P>
__device__ __forceinline__ void lds_cls(const double2 *q, double (&r)[P], double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) { r[c] = q[c].x; i[c] = q[c].y; }
}
template <int P>
__device__ __forceinline__ void sts_cls(float2 *q, const float (&r)[P], const float (&i)[P]) {
    if (P >= 2) {
#pragma unroll
        for (int c = 0; c < P; c += 2) *reinterpret_cast<float4 *>(q + c) = make_float4(r[c], i[c], r[c + 1], i[c + 1]);
    } else {
        q[0] = make_float2(r[0], i[0]);
    }
}
template <int P>
__device__ __forceinline__ void sts_cls(double2 *q, const double (&r)[P], const double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) q[c] = make_double2(r[c], i[c]);
}

// Shape of a step's coset dataflow inside a group.  The host orders each step's offsets so that the x = 0 terms of
// the first NTQ - H offsets go to output 0 and those of the last H offsets to output 1, and the x = 1 terms to the
// other output (relabelling the two outputs where that makes H <= NTQ / 2).  With (NTQ, H) known at compile time
// the coset sums need no selects; GK_ANY keeps the per-offset output tables (any m, any pattern, ntq <= 4).
enum { GK_ANY = 0, GK_1_0, GK_2_0, GK_2_1, GK_4_0, GK_4_1, GK_4_2 };

// One step of a group on one tile.  A work item is P adjacent classes (P = 2 for complex64: one 16-byte access) of
// one member j.  Threads take class groups and, when the tile has fewer class groups than threads, split the members
// too; a thread walks its members in the outer loop, so the member's tables are read once.
// Per coset: the x = 0 terms sum into their output, the x = 1 terms sum with the sign (-1)^par_t into theirs, and
// output tau = M[b][0] * x0-sum + s * M[b][1] * x1-sum with the class sign s = (-1)^(parity(base & lambda) ^ mpar_j)
// (gsamp2.cpp:32-38 with the sign parity(c & rhoc) ^ par of the reference's term list factored per class).
// NB input tables (1, or 2 when both branches of the previous step are kept) are each rotated by NR rows of M
// (1 for a written step, 2 for a trailing step's branch norms); nsum[b][r] gets the squares of table b under row r.
// FIRST reads the tile's copy of the arena blocks (type E, class p of offset z at [z index][p ^ (z & mask)]), LAST
// writes the arena (NB = NR = 1; class p of output offset z at TB ^ (z & ~mask) ^ p ^ (z & mask)), the other stages
// use buffers [value index][class] of type CplxOf<T>; STS stores every (table, row) to such a buffer.  Buffers are
// byte offsets into the dynamic shared memory.
template <typename E, typename T, int P, int NTQ, int H, bool FIRST, bool LAST, bool STS, int NB, int NR>
__device__ __forceinline__ void group_cosets(const GroupArgs &ga, const GroupStepArgs &gs, E *__restrict__ mem,
                                             const uint64_t TB, const int L, const uint32_t (&in)[NB],
                                             const uint32_t (&out)[NB][NR], const T (&w_r)[NR][2],
                                             const T (&w_i)[NR][2], T (&nsum)[NB][NR]) {
    typedef typename CplxOf<T>::type V;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr bool ANY = H < 0;
    const uint32_t NC = 1u << L;
    const int LG = L - (P == 4 ? 2 : P == 2 ? 1 : 0);  // log2 class groups per tile
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem;
    const int m = ANY ? gs.m : 2;
    const int ntq = ANY ? gs.ntq : NTQ;
    const uint32_t lam = (uint32_t)gs.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    T sgn[NTQ];
    int ta0[NTQ], ta1[NTQ];
#pragma unroll
    for (int t = 0; t < NTQ; t++) {
        sgn[t] = gs.par[t] ? (T)-1 : (T)1;
        ta0[t] = ANY ? gs.tau0[t] : (t < NTQ - H ? 0 : 1);
        ta1[t] = ANY ? gs.tau1[t] : 1 - ta0[t];
    }
    for (int j = j0; j < nm; j += jstride) {
        const int mp = tpar ^ gs.mpar[j];
        // the member's uniform addressing: value indices of its inputs and outputs in their buffers
        uint32_t zl[NTQ];
        uint32_t ib[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) {
            ib[t] = t < ntq ? (uint32_t)gs.in_idx[j][t] * NC : 0u;
            zl[t] = FIRST && t < ntq ? ga.z0lo[j][t] : 0u;
        }
        uint32_t ol[2] = {0, 0}, oidx[2] = {0, 0};
        E *ob[2] = {mem, mem};
#pragma unroll
        for (int tau = 0; tau < 2; tau++) {
            oidx[tau] = tau < m ? (uint32_t)gs.out_idx[j][tau] * NC : 0u;
            ol[tau] = LAST && tau < m ? ga.zdlo[j][tau] : 0u;
            if (LAST && tau < m) ob[tau] = mem + (TB ^ ga.blk_out[gs.out_idx[j][tau]]);
        }
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = (uint32_t)P * g;
            // x0[b][c][tau][re/im], x1[..]: the coset's x = 0 and signed x = 1 sums per output
            T x0[NB][P][2][2], x1[NB][P][2][2];
#pragma unroll
            for (int b = 0; b < NB; b++)
#pragma unroll
                for (int c = 0; c < P; c++)
#pragma unroll
                    for (int u = 0; u < 2; u++) { x0[b][c][u][0] = 0; x0[b][c][u][1] = 0; x1[b][c][u][0] = 0; x1[b][c][u][1] = 0; }
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                if (t >= ntq) continue;
#pragma unroll
                for (int b = 0; b < NB; b++) {
                    T vr[P], vi[P];
                    if (FIRST) {
                        ld_perm<P>(reinterpret_cast<const E *>(smem + in[0]) + ib[t], pc ^ zl[t], vr, vi);
                    } else {
                        lds_cls<P>(reinterpret_cast<const V *>(smem + in[b]) + (ib[t] + pc), vr, vi);
                    }
#pragma unroll
                    for (int c = 0; c < P; c++) {
                        if (ANY) {
                            if (ta0[t]) { x0[b][c][1][0] += vr[c]; x0[b][c][1][1] += vi[c]; }
                            else { x0[b][c][0][0] += vr[c]; x0[b][c][0][1] += vi[c]; }
                            if (ta1[t]) { x1[b][c][1][0] = fmaT(sgn[t], vr[c], x1[b][c][1][0]); x1[b][c][1][1] = fmaT(sgn[t], vi[c], x1[b][c][1][1]); }
                            else { x1[b][c][0][0] = fmaT(sgn[t], vr[c], x1[b][c][0][0]); x1[b][c][0][1] = fmaT(sgn[t], vi[c], x1[b][c][0][1]); }
                        } else {
                            x0[b][c][ta0[t]][0] += vr[c];
                            x0[b][c][ta0[t]][1] += vi[c];
                            x1[b][c][ta1[t]][0] = fmaT(sgn[t], vr[c], x1[b][c][ta1[t]][0]);
                            x1[b][c][ta1[t]][1] = fmaT(sgn[t], vi[c], x1[b][c][ta1[t]][1]);
                        }
                    }
                }
            }
            // the class sign folds into the x = 1 coefficient
            T w1r[NR][P], w1i[NR][P];
#pragma unroll
            for (int c = 0; c < P; c++) {
                const bool neg = ((mp ^ __popc(pc & lam) ^ __popc((uint32_t)c & lam)) & 1) != 0;   // pc: multiple of P
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    w1r[r][c] = neg ? -w_r[r][1] : w_r[r][1];
                    w1i[r][c] = neg ? -w_i[r][1] : w_i[r][1];
                }
            }
#pragma unroll
            for (int tau = 0; tau < 2; tau++) {
                if (tau >= m) continue;
                // outputs that receive no x = 0 (or no x = 1) term skip that product
                const bool h0 = ANY || (tau == 0 ? NTQ - H > 0 : H > 0);
                const bool h1 = ANY || (tau == 0 ? H > 0 : NTQ - H > 0);
#pragma unroll
                for (int b = 0; b < NB; b++)
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        T orr[P], oii[P];
#pragma unroll
                        for (int c = 0; c < P; c++) {
                            const T xr = x0[b][c][tau][0], xi = x0[b][c][tau][1];
                            const T zr = x1[b][c][tau][0], zi = x1[b][c][tau][1];
                            T re = 0, im = 0;
                            if (h0) {
                                re = w_r[r][0] * xr;
                                re = fmaT(-w_i[r][0], xi, re);
                                im = w_r[r][0] * xi;
                                im = fmaT(w_i[r][0], xr, im);
                            }
                            if (h1) {
                                re = h0 ? fmaT(w1r[r][c], zr, re) : w1r[r][c] * zr;
                                re = fmaT(-w1i[r][c], zi, re);
                                im = h0 ? fmaT(w1r[r][c], zi, im) : w1r[r][c] * zi;
                                im = fmaT(w1i[r][c], zr, im);
                            }
                            orr[c] = re;
                            oii[c] = im;
                            nsum[b][r] = fmaT(re, re, nsum[b][r]);
                            nsum[b][r] = fmaT(im, im, nsum[b][r]);
                        }
                        if (LAST) st_perm<P>(ob[tau], pc ^ ol[tau], orr, oii);
                        if (STS) sts_cls<P>(reinterpret_cast<V *>(smem + out[b][r]) + (oidx[tau] + pc), orr, oii);
                    }
            }
        }
    }
}

// Packed two-lane FP32 (sm_100 add / mul / fma .f32x2): one 64-bit register holds the same quantity for the
// thread's two adjacent classes.  Each lane rounds exactly like the scalar instruction.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float &a, float &b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// group_cosets for complex64 with FP32 arithmetic, two classes per thread in packed registers: every coset sum,
// rotation product and norm term of the class pair is one f32x2 instruction.  The stage buffers between the steps of
// a pass hold a class pair as (re0, re1, im0, im1), so they load and store as one 16-byte access with no shuffles;
// the arena tile and the arena keep (re, im) per entry.  The class sign multiplies the x = 1 sums (an exact +-1
// product), so every lane computes what the scalar form computes, in the same order; only the norm's partial sums
// split over the two lanes.
template <int NTQ, int H, bool FIRST, bool LAST, bool STS, int NR>
__device__ __forceinline__ void group_cosets_pk(const GroupArgs &ga, const GroupStepArgs &gs, float2 *__restrict__ mem,
                                                const uint64_t TB, const int L, const uint32_t (&in)[1],
                                                const uint32_t (&out)[1][NR], const float (&w_r)[NR][2],
                                                const float (&w_i)[NR][2], float (&nsum)[1][NR]) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr bool ANY = H < 0;
    const uint32_t NC = 1u << L;
    const int LG = L - 1;   // log2 class pairs per tile
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem;
    const int m = ANY ? gs.m : 2;
    const int ntq = ANY ? gs.ntq : NTQ;
    const uint32_t lam = (uint32_t)gs.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    f32x2 sg[NTQ];
    int ta0[NTQ], ta1[NTQ];
#pragma unroll
    for (int t = 0; t < NTQ; t++) {
        const float s = gs.par[t] ? -1.f : 1.f;
        sg[t] = f2_pack(s, s);
        ta0[t] = ANY ? gs.tau0[t] : (t < NTQ - H ? 0 : 1);
        ta1[t] = ANY ? gs.tau1[t] : 1 - ta0[t];
    }
    // M rows, both lanes equal: re, im and -im of M[r][0] and M[r][1]
    f32x2 W0R[NR], W0I[NR], W0N[NR], W1R[NR], W1I[NR], W1N[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) {
        W0R[r] = f2_pack(w_r[r][0], w_r[r][0]);
        W0I[r] = f2_pack(w_i[r][0], w_i[r][0]);
        W0N[r] = f2_pack(-w_i[r][0], -w_i[r][0]);
        W1R[r] = f2_pack(w_r[r][1], w_r[r][1]);
        W1I[r] = f2_pack(w_i[r][1], w_i[r][1]);
        W1N[r] = f2_pack(-w_i[r][1], -w_i[r][1]);
    }
    // class signs of a pair (p even): class p + 1 differs from class p by parity(lambda & 1)
    const float sig1 = (lam & 1u) ? -1.f : 1.f;
    const f32x2 SGP = f2_pack(1.f, sig1), SGN = f2_pack(-1.f, -sig1);
    f32x2 NS[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) NS[r] = 0ull;
    for (int j = j0; j < nm; j += jstride) {
        const int mp = tpar ^ gs.mpar[j];
        uint32_t zl[NTQ], ib[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) {
            ib[t] = t < ntq ? (uint32_t)gs.in_idx[j][t] * NC : 0u;
            zl[t] = FIRST && t < ntq ? ga.z0lo[j][t] : 0u;
        }
        uint32_t ol[2] = {0, 0}, oidx[2] = {0, 0};
        float2 *ob[2] = {mem, mem};
#pragma unroll
        for (int tau = 0; tau < 2; tau++) {
            oidx[tau] = tau < m ? (uint32_t)gs.out_idx[j][tau] * NC : 0u;
            ol[tau] = LAST && tau < m ? ga.zdlo[j][tau] : 0u;
            if (LAST && tau < m) ob[tau] = mem + (TB ^ ga.blk_out[gs.out_idx[j][tau]]);
        }
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = 2u * g;
            f32x2 X0R[2] = {0ull, 0ull}, X0I[2] = {0ull, 0ull}, X1R[2] = {0ull, 0ull}, X1I[2] = {0ull, 0ull};
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                if (t >= ntq) continue;
                f32x2 VR, VI;
                if (FIRST) {
                    const float2 *src = reinterpret_cast<const float2 *>(smem + in[0]) + ib[t];
                    const uint32_t pos = pc ^ zl[t];
                    const float2 a = src[pos], b = src[pos ^ 1u];
                    VR = f2_pack(a.x, b.x);
                    VI = f2_pack(a.y, b.y);
                } else {
                    const float4 v = *reinterpret_cast<const float4 *>(reinterpret_cast<const float2 *>(smem + in[0]) + (ib[t] + pc));
                    VR = f2_pack(v.x, v.y);
                    VI = f2_pack(v.z, v.w);
                }
                if (ANY) {
                    if (ta0[t]) { X0R[1] = f2_add(X0R[1], VR); X0I[1] = f2_add(X0I[1], VI); }
                    else { X0R[0] = f2_add(X0R[0], VR); X0I[0] = f2_add(X0I[0], VI); }
                    if (ta1[t]) { X1R[1] = f2_fma(sg[t], VR, X1R[1]); X1I[1] = f2_fma(sg[t], VI, X1I[1]); }
                    else { X1R[0] = f2_fma(sg[t], VR, X1R[0]); X1I[0] = f2_fma(sg[t], VI, X1I[0]); }
                } else {
                    X0R[ta0[t]] = f2_add(X0R[ta0[t]], VR);
                    X0I[ta0[t]] = f2_add(X0I[ta0[t]], VI);
                    X1R[ta1[t]] = f2_fma(sg[t], VR, X1R[ta1[t]]);
                    X1I[ta1[t]] = f2_fma(sg[t], VI, X1I[ta1[t]]);
                }
            }
            const f32x2 SG = ((mp ^ __popc(pc & lam)) & 1) ? SGN : SGP;
#pragma unroll
            for (int tau = 0; tau < 2; tau++) {
                if (tau >= m) continue;
                const bool h0 = ANY || (tau == 0 ? NTQ - H > 0 : H > 0);
                const bool h1 = ANY || (tau == 0 ? H > 0 : NTQ - H > 0);
                f32x2 ZR = 0ull, ZI = 0ull;
                if (h1) {
                    ZR = f2_mul(SG, X1R[tau]);
                    ZI = f2_mul(SG, X1I[tau]);
                }
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    f32x2 RE = 0ull, IM = 0ull;
                    if (h0) {
                        RE = f2_mul(W0R[r], X0R[tau]);
                        RE = f2_fma(W0N[r], X0I[tau], RE);
                        IM = f2_mul(W0R[r], X0I[tau]);
                        IM = f2_fma(W0I[r], X0R[tau], IM);
                    }
                    if (h1) {
                        RE = h0 ? f2_fma(W1R[r], ZR, RE) : f2_mul(W1R[r], ZR);
                        RE = f2_fma(W1N[r], ZI, RE);
                        IM = h0 ? f2_fma(W1R[r], ZI, IM) : f2_mul(W1R[r], ZI);
                        IM = f2_fma(W1I[r], ZR, IM);
                    }
                    NS[r] = f2_fma(RE, RE, NS[r]);
                    NS[r] = f2_fma(IM, IM, NS[r]);
                    if (LAST || STS) {
                        float r0, r1, i0, i1;
                        f2_unpack(RE, r0, r1);
                        f2_unpack(IM, i0, i1);
                        if (LAST) {
                            const uint32_t pos = pc ^ ol[tau];
                            ob[tau][pos] = make_float2(r0, i0);
                            ob[tau][pos ^ 1u] = make_float2(r1, i1);
                        }
                        if (STS)
                            *reinterpret_cast<float4 *>(reinterpret_cast<float2 *>(smem + out[0][r]) + (oidx[tau] + pc)) =
                                make_float4(r0, r1, i0, i1);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NR; r++) {
        float a, b;
        f2_unpack(NS[r], a, b);
        nsum[0][r] += a + b;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Factored written steps (complex64 arena).  A written step stores out = M[b][0] S0 + s_c M[b][1] S1 per output
// (S0 / S1: the output's x = 0 / signed x = 1 sums).  With the pivot w = M[b][PIV], the larger of the two
// coefficients, the step stores out / w instead:
//   PIV = 0:  P + beta s_c Q,  P = sc S0,             Q = S1, beta = sc M[b][1] / M[b][0]
//   PIV = 1:  P + beta Q,      P = sc s_c S1,         Q = S0, beta = sc M[b][0] / M[b][1]
// so every output costs one complex product (beta Q) instead of two, and a sum starts from its first term instead
// of from zero.  |beta| <= sc.  The complex factor w of the whole table is left out of the stored values; the
// normalised samplers depend on ratios of norms only, and the 'chain' epilogue multiplies each step's norm ratio by
// |w|^2 (GroupStepArgs::cp).  sc is the pass's scale (first step, SC = true) or 1 (later steps of the pass).
// Shapes are the compile-time GK_* shapes (m = 2): offset t's x = 0 term goes to output o0(t) = (t >= NTQ - H),
// its x = 1 term to 1 - o0(t).
template <int NTQ, int H, int PIV>
struct FShape {
    // output of offset t's P-side term / Q-side term
    __host__ __device__ static constexpr int pout(int t) { return (PIV == 0) == (t < NTQ - H) ? 0 : 1; }
    __host__ __device__ static constexpr int qout(int t) { return 1 - pout(t); }
    __host__ __device__ static constexpr int first_p(int tau) {
        for (int t = 0; t < NTQ; t++)
            if (pout(t) == tau) return t;
        return -1;
    }
    __host__ __device__ static constexpr int first_q(int tau) {
        for (int t = 0; t < NTQ; t++)
            if (qout(t) == tau) return t;
        return -1;
    }
};

template <typename E, typename T, int P, int NTQ, int H, int PIV, bool SC, bool FIRST, bool LAST, bool STS, int NM = 0>
__device__ __forceinline__ void group_cosets_f(const GroupArgs &ga, const GroupStepArgs &gs, E *__restrict__ mem,
                                               const uint64_t TB, const int L, const uint32_t in, const uint32_t out,
                                               const T sc, const T br, const T bi, T &nsum) {
    typedef typename CplxOf<T>::type V;
    typedef FShape<NTQ, H, PIV> S;
    extern __shared__ __align__(16) unsigned char smem[];
    const int LG = L - (P == 2 ? 1 : 0);
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem;
    const uint32_t lam = (uint32_t)gs.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    T sg[NTQ];
#pragma unroll
    for (int t = 0; t < NTQ; t++) sg[t] = gs.par[t] ? (T)-1 : (T)1;
    // Q sums start from their first term: PIV = 0 folds that term's sign into beta, later terms carry the relative
    // sign; PIV = 1 sums x = 0 terms, which have none.  P coefficients: sc (PIV = 0), sc * sign of the term (PIV = 1,
    // times the class sign per class).
    T qbr[2], qbi[2], rel[NTQ], pcf[NTQ];
#pragma unroll
    for (int tau = 0; tau < 2; tau++) {
        const int f = S::first_q(tau);
        const T s = (PIV == 0 && f >= 0) ? sg[f < 0 ? 0 : f] : (T)1;
        qbr[tau] = br * s;
        qbi[tau] = bi * s;
    }
#pragma unroll
    for (int t = 0; t < NTQ; t++) {
        const int f = S::first_q(S::qout(t));
        rel[t] = PIV == 0 ? sg[t] * sg[f < 0 ? 0 : f] : (T)1;
        pcf[t] = PIV == 0 ? sc : sc * sg[t];
    }
    // one member's class pair at position pc: mpp = the class sign parity of the pair's even class before the
    // member's own parity bit is applied (mp ^ parity(pc & lambda))
    auto member = [&](const uint32_t (&io)[NTQ], const uint32_t (&oidx)[2], const uint64_t (&oo)[2], const uint32_t pc,
                      const int mpp) {
            bool neg[P];
#pragma unroll
            for (int c = 0; c < P; c++) neg[c] = ((mpp ^ __popc((uint32_t)c & lam)) & 1) != 0;
            T pr[P][2], pi[P][2], qr[P][2], qi[P][2];
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                T vr[P], vi[P];
                if (FIRST) {
                    if constexpr (P == 2 && std::is_same<T, float>::value)
                        ld_pair16(reinterpret_cast<const float2 *>(smem + in), io[t] ^ pc, vr, vi);
                    else
                        ld_perm<P>(reinterpret_cast<const E *>(smem + in), io[t] ^ pc, vr, vi);
                } else {
                    lds_cls<P>(reinterpret_cast<const V *>(smem + in) + (io[t] ^ pc), vr, vi);
                }
                const int op = S::pout(t), oq = S::qout(t);
                const bool p_first = S::first_p(op) == t, q_first = S::first_q(oq) == t;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    // P side
                    if (PIV == 0 && !SC) {
                        if (p_first) { pr[c][op] = vr[c]; pi[c][op] = vi[c]; }
                        else { pr[c][op] += vr[c]; pi[c][op] += vi[c]; }
                    } else {
                        const T k = (PIV == 1 && neg[c]) ? -pcf[t] : pcf[t];
                        if (p_first) { pr[c][op] = k * vr[c]; pi[c][op] = k * vi[c]; }
                        else { pr[c][op] = fmaT(k, vr[c], pr[c][op]); pi[c][op] = fmaT(k, vi[c], pi[c][op]); }
                    }
                    // Q side
                    if (q_first) { qr[c][oq] = vr[c]; qi[c][oq] = vi[c]; }
                    else if (PIV == 1) { qr[c][oq] += vr[c]; qi[c][oq] += vi[c]; }
                    else { qr[c][oq] = fmaT(rel[t], vr[c], qr[c][oq]); qi[c][oq] = fmaT(rel[t], vi[c], qi[c][oq]); }
                }
            }
#pragma unroll
            for (int tau = 0; tau < 2; tau++) {
                const bool hp = S::first_p(tau) >= 0, hq = S::first_q(tau) >= 0;
                T orr[P], oii[P];
#pragma unroll
                for (int c = 0; c < P; c++) {
                    T bR = qbr[tau], bI = qbi[tau];
                    if (PIV == 0 && neg[c]) { bR = -bR; bI = -bI; }
                    T re, im;
                    if (hp && hq) {
                        re = fmaT(bR, qr[c][tau], fmaT(-bI, qi[c][tau], pr[c][tau]));
                        im = fmaT(bR, qi[c][tau], fmaT(bI, qr[c][tau], pi[c][tau]));
                    } else if (hp) {
                        re = pr[c][tau];
                        im = pi[c][tau];
                    } else {
                        re = fmaT(-bI, qi[c][tau], bR * qr[c][tau]);
                        im = fmaT(bI, qr[c][tau], bR * qi[c][tau]);
                    }
                    orr[c] = re;
                    oii[c] = im;
                    nsum = fmaT(re, re, nsum);
                    nsum = fmaT(im, im, nsum);
                }
                if (LAST) {
                    const uint64_t q = oo[tau] ^ pc;
                    if constexpr (P == 2 && std::is_same<T, float>::value)
                        st_pair16(reinterpret_cast<float2 *>(mem) + (q & ~(uint64_t)1), (uint32_t)q & 1u, orr, oii);
                    else
                        st_perm<P>(mem + (q & ~(uint64_t)(P - 1)), (uint32_t)q & (uint32_t)(P - 1), orr, oii);
                }
                if (STS) sts_cls<P>(reinterpret_cast<V *>(smem + out) + (oidx[tau] + pc), orr, oii);
            }
    };
    if constexpr (NM > 0) {
        // compile-time member count (warp-specialised passes, tiles of 2^9 classes or more, so NG >= GROUP_NCT and
        // every thread runs every member of its class pairs): members unrolled inside the class-pair loop, their
        // descriptors constant operands, the pair's sign parity formed once
        for (uint32_t g = threadIdx.x; g < NG; g += GROUP_NCT) {
            const uint32_t pc = (uint32_t)P * g;
            const int pp = tpar ^ __popc(pc & lam);
#pragma unroll
            for (int j = 0; j < NM; j++) {
                uint32_t io[NTQ];
#pragma unroll
                for (int t = 0; t < NTQ; t++) io[t] = gs.ioff[j][t];
                uint32_t oidx[2] = {0, 0};
                uint64_t oo[2] = {0, 0};
#pragma unroll
                for (int tau = 0; tau < 2; tau++) {
                    if (LAST) oo[tau] = TB ^ ga.ooff[j][tau];
                    else oidx[tau] = gs.soff[j][tau];
                }
                member(io, oidx, oo, pc, pp ^ gs.mpar[j]);
            }
        }
    } else {
    for (int j = j0; j < nm; j += jstride) {   // runtime member count
        const int mp = tpar ^ gs.mpar[j];
        // the member's positions come precomputed (GroupStepArgs::ioff, GroupArgs::ooff): one word per offset and
        // output instead of an index, a multiply, the stage-0 / written-stage low bits and a block-table lookup
        uint32_t io[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) io[t] = gs.ioff[j][t];
        uint32_t oidx[2] = {0, 0};
        uint64_t oo[2] = {0, 0};
#pragma unroll
        for (int tau = 0; tau < 2; tau++) {
            if (LAST) oo[tau] = TB ^ ga.ooff[j][tau];
            else oidx[tau] = gs.soff[j][tau];
        }
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = (uint32_t)P * g;
            member(io, oidx, oo, pc, mp ^ __popc(pc & lam));
        }
    }
    }
}

// The packed two-lane FP32 form of group_cosets_f (the thread's two adjacent classes in the lanes of f32x2
// registers; stages between steps as (re0, re1, im0, im1)).
template <int NTQ, int H, int PIV, bool SC, bool FIRST, bool LAST, bool STS>
__device__ __forceinline__ void group_cosets_pkf(const GroupArgs &ga, const GroupStepArgs &gs, float2 *__restrict__ mem,
                                                 const uint64_t TB, const int L, const uint32_t in, const uint32_t out,
                                                 const float sc, const float br, const float bi, float &nsum) {
    typedef FShape<NTQ, H, PIV> S;
    extern __shared__ __align__(16) unsigned char smem[];
    const int LG = L - 1;
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem;
    const uint32_t lam = (uint32_t)gs.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    float sg[NTQ];
#pragma unroll
    for (int t = 0; t < NTQ; t++) sg[t] = gs.par[t] ? -1.f : 1.f;
    f32x2 QBR[2], QBI[2], QBN[2], REL[NTQ], PCF[NTQ];
#pragma unroll
    for (int tau = 0; tau < 2; tau++) {
        const int f = S::first_q(tau);
        const float s = (PIV == 0 && f >= 0) ? sg[f < 0 ? 0 : f] : 1.f;
        QBR[tau] = f2_pack(br * s, br * s);
        QBI[tau] = f2_pack(bi * s, bi * s);
        QBN[tau] = f2_pack(-bi * s, -bi * s);
    }
#pragma unroll
    for (int t = 0; t < NTQ; t++) {
        const int f = S::first_q(S::qout(t));
        const float rl = PIV == 0 ? sg[t] * sg[f < 0 ? 0 : f] : 1.f;
        const float pk = PIV == 0 ? sc : sc * sg[t];
        REL[t] = f2_pack(rl, rl);
        PCF[t] = f2_pack(pk, pk);
    }
    const float sig1 = (lam & 1u) ? -1.f : 1.f;
    const f32x2 SGP = f2_pack(1.f, sig1), SGN = f2_pack(-1.f, -sig1);
    f32x2 NS = 0ull;
    for (int j = j0; j < nm; j += jstride) {
        const int mp = tpar ^ gs.mpar[j];
        // precomputed member positions, as in group_cosets_f
        uint32_t io[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) io[t] = gs.ioff[j][t];
        uint32_t oidx[2] = {0, 0};
        uint64_t oo[2] = {0, 0};
#pragma unroll
        for (int tau = 0; tau < 2; tau++) {
            if (STS) oidx[tau] = gs.soff[j][tau];
            if (LAST) oo[tau] = TB ^ ga.ooff[j][tau];
        }
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = 2u * g;
            const f32x2 SG = ((mp ^ __popc(pc & lam)) & 1) ? SGN : SGP;
            f32x2 PR[2], PI[2], QR[2], QI[2];
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                f32x2 VR, VI;
                if (FIRST) {
                    float r2[2], i2[2];
                    ld_pair16(reinterpret_cast<const float2 *>(smem + in), io[t] ^ pc, r2, i2);
                    VR = f2_pack(r2[0], r2[1]);
                    VI = f2_pack(i2[0], i2[1]);
                } else {
                    const float4 v = *reinterpret_cast<const float4 *>(reinterpret_cast<const float2 *>(smem + in) + (io[t] ^ pc));
                    VR = f2_pack(v.x, v.y);
                    VI = f2_pack(v.z, v.w);
                }
                const int op = S::pout(t), oq = S::qout(t);
                const bool p_first = S::first_p(op) == t, q_first = S::first_q(oq) == t;
                if (PIV == 0 && !SC) {
                    if (p_first) { PR[op] = VR; PI[op] = VI; }
                    else { PR[op] = f2_add(PR[op], VR); PI[op] = f2_add(PI[op], VI); }
                } else {
                    const f32x2 K = PIV == 1 ? f2_mul(SG, PCF[t]) : PCF[t];
                    if (p_first) { PR[op] = f2_mul(K, VR); PI[op] = f2_mul(K, VI); }
                    else { PR[op] = f2_fma(K, VR, PR[op]); PI[op] = f2_fma(K, VI, PI[op]); }
                }
                if (q_first) { QR[oq] = VR; QI[oq] = VI; }
                else if (PIV == 1) { QR[oq] = f2_add(QR[oq], VR); QI[oq] = f2_add(QI[oq], VI); }
                else { QR[oq] = f2_fma(REL[t], VR, QR[oq]); QI[oq] = f2_fma(REL[t], VI, QI[oq]); }
            }
#pragma unroll
            for (int tau = 0; tau < 2; tau++) {
                const bool hp = S::first_p(tau) >= 0, hq = S::first_q(tau) >= 0;
                f32x2 BR = QBR[tau], BI = QBI[tau], BN = QBN[tau];
                if (PIV == 0) { BR = f2_mul(SG, BR); BI = f2_mul(SG, BI); BN = f2_mul(SG, BN); }
                f32x2 RE, IM;
                if (hp && hq) {
                    RE = f2_fma(BR, QR[tau], f2_fma(BN, QI[tau], PR[tau]));
                    IM = f2_fma(BR, QI[tau], f2_fma(BI, QR[tau], PI[tau]));
                } else if (hp) {
                    RE = PR[tau];
                    IM = PI[tau];
                } else {
                    RE = f2_fma(BN, QI[tau], f2_mul(BR, QR[tau]));
                    IM = f2_fma(BI, QR[tau], f2_mul(BR, QI[tau]));
                }
                NS = f2_fma(RE, RE, NS);
                NS = f2_fma(IM, IM, NS);
                if (LAST || STS) {
                    float r0, r1, i0, i1;
                    f2_unpack(RE, r0, r1);
                    f2_unpack(IM, i0, i1);
                    if (LAST) {
                        const float rr2[2] = {r0, r1}, ii2[2] = {i0, i1};
                        const uint64_t q = oo[tau] ^ pc;
                        st_pair16(mem + (q & ~(uint64_t)1), (uint32_t)q & 1u, rr2, ii2);
                    }
                    if (STS)
                        *reinterpret_cast<float4 *>(reinterpret_cast<float2 *>(smem + out) + (oidx[tau] + pc)) =
                            make_float4(r0, r1, i0, i1);
                }
            }
        }
    }
    float a, b;
    f2_unpack(NS, a, b);
    nsum += a + b;
}

template <typename E, typename T, bool FIRST, bool LAST, bool STS, int NB, int NR, bool PK>
__device__ __forceinline__ void group_cosets_any(const GroupArgs &ga, const GroupStepArgs &gs, E *__restrict__ mem,
                                                 const uint64_t TB, const int L, const uint32_t (&in)[NB],
                                                 const uint32_t (&out)[NB][NR], const T (&w_r)[NR][2],
                                                 const T (&w_i)[NR][2], T (&ns)[NB][NR]) {
    // classes per thread: two adjacent classes for complex64 (their values sit in one 16-byte span of a block),
    // one for complex128.  Four per thread was measured slower: per-class 8-byte accesses at a 32-byte stride
    // conflict in shared memory and scatter the arena stores.
    // PK (FP32 arithmetic only): the packed form, with its stage layout, for every step of the pass.
    constexpr int P = sizeof(E) == 8 ? 2 : 1;
    if constexpr (PK) {
        static_assert(std::is_same<T, float>::value, "packed form: FP32 arithmetic");
        static_assert(NB == 1 && sizeof(E) == 8, "packed form: one complex64 table");
#define GSB_GC(NTQ_, H_) group_cosets_pk<NTQ_, H_, FIRST, LAST, STS, NR>(ga, gs, mem, TB, L, in, out, w_r, w_i, ns)
        switch (gs.kind) {   // uniform across the grid
            case GK_1_0: GSB_GC(1, 0); break;
            case GK_2_0: GSB_GC(2, 0); break;
            case GK_2_1: GSB_GC(2, 1); break;
            case GK_4_0: GSB_GC(4, 0); break;
            case GK_4_1: GSB_GC(4, 1); break;
            case GK_4_2: GSB_GC(4, 2); break;
            default: GSB_GC(4, -1); break;
        }
#undef GSB_GC
    } else {
#define GSB_GC(NTQ_, H_) group_cosets<E, T, P, NTQ_, H_, FIRST, LAST, STS, NB, NR>(ga, gs, mem, TB, L, in, out, w_r, w_i, ns)
        switch (gs.kind) {
            case GK_1_0: GSB_GC(1, 0); break;
            case GK_2_0: GSB_GC(2, 0); break;
            case GK_2_1: GSB_GC(2, 1); break;
            case GK_4_0: GSB_GC(4, 0); break;
            case GK_4_1: GSB_GC(4, 1); break;
            case GK_4_2: GSB_GC(4, 2); break;
            default: GSB_GC(4, -1); break;
        }
#undef GSB_GC
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Trailing step of a complex64 sampling pass by shared sums.  Both branch norms of the next step,
//   n(b) = sum |M[b][0] S0 + M[b][1] Z|^2 = |M[b][0]|^2 A + |M[b][1]|^2 B + 2 Re(M[b][0] conj(M[b][1]) C),
// need only A = sum |S0|^2, B = sum |Z|^2 and C = sum S0 conj(Z) (Z = s_c S1, the signed x = 1 sum), about half the
// arithmetic of rotating by both rows.  acc = (A, B, Re C, Im C).  n(b) then carries an absolute error of order
// eps (A + B) instead of a relative one; n(0) + n(1) = A + B has none (M is unitary), so the bit decision is as
// good, and the log2 Pr of the chosen branch is taken from the norm the next pass writes (group_decide / k_group).
template <typename E, typename T, int P, int NTQ, int H>
__device__ __forceinline__ void group_trail_abc(const GroupArgs &ga, const GroupStepArgs &gs, const uint64_t TB,
                                                const int L, const uint32_t in, T (&acc)[4]) {
    typedef typename CplxOf<T>::type V;
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t NC = 1u << L;
    const int LG = L - (P == 2 ? 1 : 0);
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem;
    const uint32_t lam = (uint32_t)gs.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    T sg[NTQ];
#pragma unroll
    for (int t = 0; t < NTQ; t++) sg[t] = gs.par[t] ? (T)-1 : (T)1;
    typedef FShape<NTQ, H, 0> S;   // pout = output of the x = 0 term, qout = output of the x = 1 term
    for (int j = j0; j < nm; j += jstride) {
        const int mp = tpar ^ gs.mpar[j];
        uint32_t ib[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) ib[t] = (uint32_t)gs.in_idx[j][t] * NC;
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = (uint32_t)P * g;
            T xr[P][2], xi[P][2], zr[P][2], zi[P][2];
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                T vr[P], vi[P];
                lds_cls<P>(reinterpret_cast<const V *>(smem + in) + (ib[t] + pc), vr, vi);
                const int o0 = S::pout(t), o1 = S::qout(t);
                const bool f0 = S::first_p(o0) == t, f1 = S::first_q(o1) == t;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    if (f0) { xr[c][o0] = vr[c]; xi[c][o0] = vi[c]; }
                    else { xr[c][o0] += vr[c]; xi[c][o0] += vi[c]; }
                    if (f1) { zr[c][o1] = sg[t] * vr[c]; zi[c][o1] = sg[t] * vi[c]; }
                    else { zr[c][o1] = fmaT(sg[t], vr[c], zr[c][o1]); zi[c][o1] = fmaT(sg[t], vi[c], zi[c][o1]); }
                }
            }
#pragma unroll
            for (int c = 0; c < P; c++) {
                const bool neg = ((mp ^ __popc(pc & lam) ^ __popc((uint32_t)c & lam)) & 1) != 0;
                const T s = neg ? (T)-1 : (T)1;
#pragma unroll
                for (int tau = 0; tau < 2; tau++) {
                    const bool h0 = S::first_p(tau) >= 0, h1 = S::first_q(tau) >= 0;
                    if (h0) acc[0] = fmaT(xr[c][tau], xr[c][tau], fmaT(xi[c][tau], xi[c][tau], acc[0]));
                    if (h1) acc[1] = fmaT(zr[c][tau], zr[c][tau], fmaT(zi[c][tau], zi[c][tau], acc[1]));
                    if (h0 && h1) {
                        // C += s_c (x0 conj(z1))
                        const T cr = fmaT(xr[c][tau], zr[c][tau], xi[c][tau] * zi[c][tau]);
                        const T ci = fmaT(xi[c][tau], zr[c][tau], -xr[c][tau] * zi[c][tau]);
                        acc[2] = fmaT(s, cr, acc[2]);
                        acc[3] = fmaT(s, ci, acc[3]);
                    }
                }
            }
        }
    }
}

// The packed two-lane FP32 form (stage layout (re0, re1, im0, im1)).
template <int NTQ, int H>
__device__ __forceinline__ void group_trail_abc_pk(const GroupArgs &ga, const GroupStepArgs &gs, const uint64_t TB,
                                                   const int L, const uint32_t in, float (&acc)[4]) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t NC = 1u << L;
    const int LG = L - 1;
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem;
    const uint32_t lam = (uint32_t)gs.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    typedef FShape<NTQ, H, 0> S;
    f32x2 SGT[NTQ];
#pragma unroll
    for (int t = 0; t < NTQ; t++) {
        const float v = gs.par[t] ? -1.f : 1.f;
        SGT[t] = f2_pack(v, v);
    }
    const float sig1 = (lam & 1u) ? -1.f : 1.f;
    const f32x2 SGP = f2_pack(1.f, sig1), SGN = f2_pack(-1.f, -sig1);
    f32x2 AA = 0ull, BB = 0ull, CR = 0ull, CI = 0ull;
    for (int j = j0; j < nm; j += jstride) {
        const int mp = tpar ^ gs.mpar[j];
        uint32_t ib[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) ib[t] = (uint32_t)gs.in_idx[j][t] * NC;
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = 2u * g;
            f32x2 XR[2], XI[2], ZR[2], ZI[2];
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                const float4 v = *reinterpret_cast<const float4 *>(reinterpret_cast<const float2 *>(smem + in) + (ib[t] + pc));
                const f32x2 VR = f2_pack(v.x, v.y), VI = f2_pack(v.z, v.w);
                const int o0 = S::pout(t), o1 = S::qout(t);
                const bool f0 = S::first_p(o0) == t, f1 = S::first_q(o1) == t;
                if (f0) { XR[o0] = VR; XI[o0] = VI; }
                else { XR[o0] = f2_add(XR[o0], VR); XI[o0] = f2_add(XI[o0], VI); }
                if (f1) { ZR[o1] = f2_mul(SGT[t], VR); ZI[o1] = f2_mul(SGT[t], VI); }
                else { ZR[o1] = f2_fma(SGT[t], VR, ZR[o1]); ZI[o1] = f2_fma(SGT[t], VI, ZI[o1]); }
            }
            const f32x2 SG = ((mp ^ __popc(pc & lam)) & 1) ? SGN : SGP;
#pragma unroll
            for (int tau = 0; tau < 2; tau++) {
                const bool h0 = S::first_p(tau) >= 0, h1 = S::first_q(tau) >= 0;
                if (h0) AA = f2_fma(XR[tau], XR[tau], f2_fma(XI[tau], XI[tau], AA));
                if (h1) BB = f2_fma(ZR[tau], ZR[tau], f2_fma(ZI[tau], ZI[tau], BB));
                if (h0 && h1) {
                    const f32x2 SZR = f2_mul(SG, ZR[tau]), SZI = f2_mul(SG, ZI[tau]);
                    CR = f2_fma(XR[tau], SZR, f2_fma(XI[tau], SZI, CR));
                    CI = f2_fma(XI[tau], SZR, f2_fma(f2_mul(XR[tau], f2_pack(-1.f, -1.f)), SZI, CI));
                }
            }
        }
    }
    float a, b;
    f2_unpack(AA, a, b); acc[0] += a + b;
    f2_unpack(BB, a, b); acc[1] += a + b;
    f2_unpack(CR, a, b); acc[2] += a + b;
    f2_unpack(CI, a, b); acc[3] += a + b;
}

// The shared-sum trailing step of a folded pass (GroupArgs::fold, packed FP32): the written stage is the output of a
// one-offset growth step g (GK_1_0) applied to stage `in`: its member m writes stage1[in_idx_g[m][0]] times
//   output 0: 1 (pivot 0) or beta (pivot 1),  output 1: beta s_m sgn (pivot 0) or s_m sgn (pivot 1),
// with s_m the growth step's class sign and sgn the sign of its x = 1 term.  This reads those stage-1 values and
// applies the coefficients, then accumulates A, B, C as group_trail_abc_pk does.
template <int NTQ, int H>
__device__ __forceinline__ void group_trail_fold_pk(const GroupArgs &ga, const GroupStepArgs &gg, const GroupStepArgs &gs,
                                                    const uint64_t TB, const int L, const uint32_t in, const int gpiv,
                                                    const float gbr, const float gbi, float (&acc)[4]) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t NC = 1u << L;
    const int LG = L - 1;
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1, gtpar = __popcll(TB & gg.lambda) & 1;
    const int nm = gs.nmem;
    const uint32_t lam = (uint32_t)gs.lambda, glam = (uint32_t)gg.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    typedef FShape<NTQ, H, 0> S;
    f32x2 SGT[NTQ];
#pragma unroll
    for (int t = 0; t < NTQ; t++) {
        const float v = gs.par[t] ? -1.f : 1.f;
        SGT[t] = f2_pack(v, v);
    }
    const float gsg = gg.par[0] ? -1.f : 1.f;
    // growth-step coefficients: output 0 / output 1 (before the class sign of output 1)
    const float c0r = gpiv == 0 ? 1.f : gbr, c0i = gpiv == 0 ? 0.f : gbi;
    const float c1r = gpiv == 0 ? gbr * gsg : gsg, c1i = gpiv == 0 ? gbi * gsg : 0.f;
    const float sig1 = (lam & 1u) ? -1.f : 1.f, gsig1 = (glam & 1u) ? -1.f : 1.f;
    const f32x2 SGP = f2_pack(1.f, sig1), SGN = f2_pack(-1.f, -sig1);
    const f32x2 GSP = f2_pack(1.f, gsig1), GSN = f2_pack(-1.f, -gsig1);
    const f32x2 MONE = f2_pack(-1.f, -1.f);
    f32x2 AA = 0ull, BB = 0ull, CR = 0ull, CI = 0ull;
    for (int j = j0; j < nm; j += jstride) {
        const int mp = tpar ^ gs.mpar[j];
        uint32_t ib[NTQ];
        int gm[NTQ], tt[NTQ];
#pragma unroll
        for (int t = 0; t < NTQ; t++) {
            ib[t] = (uint32_t)ga.fsrc[j][t] * NC;
            tt[t] = ga.ftau[j][t];
            gm[t] = gtpar ^ gg.mpar[ga.fmem[j][t]];
        }
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = 2u * g;
            const int gpp = __popc(pc & glam);
            f32x2 XR[2], XI[2], ZR[2], ZI[2];
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                const float4 v = *reinterpret_cast<const float4 *>(reinterpret_cast<const float2 *>(smem + in) + (ib[t] + pc));
                f32x2 VR = f2_pack(v.x, v.y), VI = f2_pack(v.z, v.w);
                // the growth step's output value: coefficient (times its class sign for output 1)
                float kr = tt[t] ? c1r : c0r, ki = tt[t] ? c1i : c0i;
                f32x2 KR = f2_pack(kr, kr), KI = f2_pack(ki, ki);
                if (tt[t]) {
                    const f32x2 GS = ((gm[t] ^ gpp) & 1) ? GSN : GSP;
                    KR = f2_mul(GS, KR);
                    KI = f2_mul(GS, KI);
                }
                // the written step's operation order (group_cosets_pkf), so the values match its stores bit for bit
                const f32x2 WR = f2_fma(f2_mul(KI, MONE), VI, f2_mul(KR, VR));
                const f32x2 WI = f2_fma(KI, VR, f2_mul(KR, VI));
                VR = WR;
                VI = WI;
                const int o0 = S::pout(t), o1 = S::qout(t);
                const bool f0 = S::first_p(o0) == t, f1 = S::first_q(o1) == t;
                if (f0) { XR[o0] = VR; XI[o0] = VI; }
                else { XR[o0] = f2_add(XR[o0], VR); XI[o0] = f2_add(XI[o0], VI); }
                if (f1) { ZR[o1] = f2_mul(SGT[t], VR); ZI[o1] = f2_mul(SGT[t], VI); }
                else { ZR[o1] = f2_fma(SGT[t], VR, ZR[o1]); ZI[o1] = f2_fma(SGT[t], VI, ZI[o1]); }
            }
            const f32x2 SG = ((mp ^ __popc(pc & lam)) & 1) ? SGN : SGP;
#pragma unroll
            for (int tau = 0; tau < 2; tau++) {
                const bool h0 = S::first_p(tau) >= 0, h1 = S::first_q(tau) >= 0;
                if (h0) AA = f2_fma(XR[tau], XR[tau], f2_fma(XI[tau], XI[tau], AA));
                if (h1) BB = f2_fma(ZR[tau], ZR[tau], f2_fma(ZI[tau], ZI[tau], BB));
                if (h0 && h1) {
                    const f32x2 SZR = f2_mul(SG, ZR[tau]), SZI = f2_mul(SG, ZI[tau]);
                    CR = f2_fma(XR[tau], SZR, f2_fma(XI[tau], SZI, CR));
                    CI = f2_fma(XI[tau], SZR, f2_fma(f2_mul(XR[tau], MONE), SZI, CI));
                }
            }
        }
    }
    float a, b;
    f2_unpack(AA, a, b); acc[0] += a + b;
    f2_unpack(BB, a, b); acc[1] += a + b;
    f2_unpack(CR, a, b); acc[2] += a + b;
    f2_unpack(CI, a, b); acc[3] += a + b;
}

// The folded trailing step when every trailing member reads one output tau of the growth step in all its offsets
// (GroupArgs::fold = 2).  Those offsets then share the coefficient K (1 or beta, and the term sign), and their class
// signs differ by the growth members' parities only (the class-dependent part is common), so
//   A_j = |K|^2 A'_j, B_j = |K|^2 B'_j, C_j = |K|^2 C'_j,
// with A', B', C' the sums over the stage-1 values times the relative signs r_t = s_t s_0: no complex products.
template <int NTQ, int H>
__device__ __forceinline__ void group_trail_fold2_pk(const GroupArgs &ga, const GroupStepArgs &gg, const GroupStepArgs &gs,
                                                     const uint64_t TB, const int L, const uint32_t in, const int gpiv,
                                                     const float gbr, const float gbi, float (&acc)[4]) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t NC = 1u << L;
    const int LG = L - 1;
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem;
    const uint32_t lam = (uint32_t)gs.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    typedef FShape<NTQ, H, 0> S;
    // |K|^2 of the growth step's outputs: output 0 carries 1 (pivot 0) or beta (pivot 1), output 1 the other
    const float bb = gbr * gbr + gbi * gbi;
    const float kk0 = gpiv == 0 ? 1.f : bb, kk1 = gpiv == 0 ? bb : 1.f;
    const float sig1 = (lam & 1u) ? -1.f : 1.f;
    const f32x2 SGP = f2_pack(1.f, sig1), SGN = f2_pack(-1.f, -sig1);
    const f32x2 MONE = f2_pack(-1.f, -1.f);
    f32x2 AA = 0ull, BB = 0ull, CR = 0ull, CI = 0ull;
    for (int j = j0; j < nm; j += jstride) {
        const int mp = tpar ^ gs.mpar[j];
        uint32_t ib[NTQ];
        f32x2 RT[NTQ], ST[NTQ];
        const int m0par = gg.mpar[ga.fmem[j][0]];
#pragma unroll
        for (int t = 0; t < NTQ; t++) {
            ib[t] = (uint32_t)ga.fsrc[j][t] * NC;
            // relative class sign of this offset's growth member (output 1 only: output 0 has no class sign)
            const float r = (ga.ftau[j][0] && ((gg.mpar[ga.fmem[j][t]] ^ m0par) & 1)) ? -1.f : 1.f;
            const float sq = gs.par[t] ? -r : r;
            RT[t] = f2_pack(r, r);
            ST[t] = f2_pack(sq, sq);
        }
        f32x2 aa = 0ull, bq = 0ull, cr = 0ull, ci = 0ull;
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = 2u * g;
            f32x2 XR[2], XI[2], ZR[2], ZI[2];
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                const float4 v = *reinterpret_cast<const float4 *>(reinterpret_cast<const float2 *>(smem + in) + (ib[t] + pc));
                const f32x2 VR = f2_pack(v.x, v.y), VI = f2_pack(v.z, v.w);
                const int o0 = S::pout(t), o1 = S::qout(t);
                const bool f0 = S::first_p(o0) == t, f1 = S::first_q(o1) == t;
                if (f0) { XR[o0] = f2_mul(RT[t], VR); XI[o0] = f2_mul(RT[t], VI); }
                else { XR[o0] = f2_fma(RT[t], VR, XR[o0]); XI[o0] = f2_fma(RT[t], VI, XI[o0]); }
                if (f1) { ZR[o1] = f2_mul(ST[t], VR); ZI[o1] = f2_mul(ST[t], VI); }
                else { ZR[o1] = f2_fma(ST[t], VR, ZR[o1]); ZI[o1] = f2_fma(ST[t], VI, ZI[o1]); }
            }
            const f32x2 SG = ((mp ^ __popc(pc & lam)) & 1) ? SGN : SGP;
#pragma unroll
            for (int tau = 0; tau < 2; tau++) {
                const bool h0 = S::first_p(tau) >= 0, h1 = S::first_q(tau) >= 0;
                if (h0) aa = f2_fma(XR[tau], XR[tau], f2_fma(XI[tau], XI[tau], aa));
                if (h1) bq = f2_fma(ZR[tau], ZR[tau], f2_fma(ZI[tau], ZI[tau], bq));
                if (h0 && h1) {
                    const f32x2 SZR = f2_mul(SG, ZR[tau]), SZI = f2_mul(SG, ZI[tau]);
                    cr = f2_fma(XR[tau], SZR, f2_fma(XI[tau], SZI, cr));
                    ci = f2_fma(XI[tau], SZR, f2_fma(f2_mul(XR[tau], MONE), SZI, ci));
                }
            }
        }
        const float k = ga.ftau[j][0] ? kk1 : kk0;
        const f32x2 KK = f2_pack(k, k);
        AA = f2_fma(KK, aa, AA);
        BB = f2_fma(KK, bq, BB);
        CR = f2_fma(KK, cr, CR);
        CI = f2_fma(KK, ci, CI);
    }
    float a, b;
    f2_unpack(AA, a, b); acc[0] += a + b;
    f2_unpack(BB, a, b); acc[1] += a + b;
    f2_unpack(CR, a, b); acc[2] += a + b;
    f2_unpack(CI, a, b); acc[3] += a + b;
}

// The shared sums of a trailing step of shape GK_2_1 (offset 0's x = 0 term to output 0, offset 1's to output 1, the
// x = 1 terms to the other output), packed FP32.  With W_t the value offset t reads:
//   X_0 = W_0, X_1 = W_1, Z_0 = sg_1 W_1, Z_1 = sg_0 W_0, so A = B = sum |W_0|^2 + |W_1|^2 and
//   C = sum SG (sg_1 P + sg_0 conj(P)), P = W_0 conj(W_1), SG the class sign:
// two squared norms and one complex product per class pair instead of the output sums.  FOLD (GroupArgs::fold): W_t
// is K_t s_t V_t, a growth output (K_t its coefficient, s_t its class sign for output 1) of the stage-1 value V_t;
// then A = sum |K_0|^2 |V_0|^2 + |K_1|^2 |V_1|^2 and P = K_0 conj(K_1) s_0 s_1 V_0 conj(V_1), and the class signs
// SG s_0 s_1 of a pair reduce to the parity of (a member constant) ^ popc(pc & msk).
template <bool FOLD>
__device__ __forceinline__ void group_trail21_pk(const GroupArgs &ga, const GroupStepArgs &gg, const GroupStepArgs &gs,
                                                 const uint64_t TB, const int L, const uint32_t in, const int gpiv,
                                                 const float gbr, const float gbi, float (&acc)[4]) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t NC = 1u << L;
    const int LG = L - 1;
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem;
    const uint32_t lam = (uint32_t)gs.lambda;
    uint32_t g0 = threadIdx.x, gstride = GROUP_NCT;
    int j0 = 0, jstride = 1;
    if (NG < GROUP_NCT) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(GROUP_NCT >> LG);
    }
    const float sg0 = gs.par[0] ? -1.f : 1.f, sg1 = gs.par[1] ? -1.f : 1.f;
    const float csum = sg0 + sg1, cdif = sg1 - sg0;
    // growth-step coefficients (FOLD): output 0 / output 1 before its class sign
    float c0r = 1.f, c0i = 0.f, c1r = 1.f, c1i = 0.f;
    uint32_t glam = 0;
    int gtpar = 0;
    if (FOLD) {
        const float gsg = gg.par[0] ? -1.f : 1.f;
        c0r = gpiv == 0 ? 1.f : gbr;
        c0i = gpiv == 0 ? 0.f : gbi;
        c1r = gpiv == 0 ? gbr * gsg : gsg;
        c1i = gpiv == 0 ? gbi * gsg : 0.f;
        glam = (uint32_t)gg.lambda;
        gtpar = __popcll(TB & gg.lambda) & 1;
    }
    const f32x2 MONE = f2_pack(-1.f, -1.f);
    f32x2 AA = 0ull, CR = 0ull, CI = 0ull;
    for (int j = j0; j < nm; j += jstride) {
        uint32_t ib0, ib1, msk = lam;
        int cst = tpar ^ gs.mpar[j];
        float k0 = 1.f, k1 = 1.f, kr = 1.f, ki = 0.f;
        if (FOLD) {
            ib0 = (uint32_t)ga.fsrc[j][0] * NC;
            ib1 = (uint32_t)ga.fsrc[j][1] * NC;
            const int t0 = ga.ftau[j][0], t1 = ga.ftau[j][1];
            if (t0) cst ^= gtpar ^ gg.mpar[ga.fmem[j][0]];
            if (t1) cst ^= gtpar ^ gg.mpar[ga.fmem[j][1]];
            if (t0 != t1) msk ^= glam;
            const float ar = t0 ? c1r : c0r, ai = t0 ? c1i : c0i, br = t1 ? c1r : c0r, bi = t1 ? c1i : c0i;
            k0 = ar * ar + ai * ai;
            k1 = br * br + bi * bi;
            kr = ar * br + ai * bi;   // K_0 conj(K_1)
            ki = ai * br - ar * bi;
        } else {
            ib0 = (uint32_t)gs.in_idx[j][0] * NC;
            ib1 = (uint32_t)gs.in_idx[j][1] * NC;
        }
        const float s1 = (msk & 1u) ? -1.f : 1.f;
        const f32x2 SGP = f2_pack(1.f, s1), SGN = f2_pack(-1.f, -s1);
        f32x2 a0 = 0ull, a1 = 0ull, qr = 0ull, qi = 0ull;
        for (uint32_t g = g0; g < NG; g += gstride) {
            const uint32_t pc = 2u * g;
            const float4 u = *reinterpret_cast<const float4 *>(reinterpret_cast<const float2 *>(smem + in) + (ib0 + pc));
            const float4 v = *reinterpret_cast<const float4 *>(reinterpret_cast<const float2 *>(smem + in) + (ib1 + pc));
            const f32x2 UR = f2_pack(u.x, u.y), UI = f2_pack(u.z, u.w), VR = f2_pack(v.x, v.y), VI = f2_pack(v.z, v.w);
            a0 = f2_fma(UR, UR, f2_fma(UI, UI, a0));
            a1 = f2_fma(VR, VR, f2_fma(VI, VI, a1));
            const f32x2 SG = ((cst ^ __popc(pc & msk)) & 1) ? SGN : SGP;
            const f32x2 PR = f2_fma(UR, VR, f2_mul(UI, VI));             // Re U conj(V)
            const f32x2 PI = f2_fma(UI, VR, f2_mul(f2_mul(UR, MONE), VI));  // Im U conj(V)
            qr = f2_fma(SG, PR, qr);
            qi = f2_fma(SG, PI, qi);
        }
        AA = f2_fma(f2_pack(k0, k0), a0, f2_fma(f2_pack(k1, k1), a1, AA));
        // C += sg_1 K Q + sg_0 conj(K Q), K = K_0 conj(K_1), Q = (qr, qi)
        const f32x2 KR = f2_pack(kr, kr), KI = f2_pack(ki, ki);
        const f32x2 QR = f2_fma(KR, qr, f2_mul(f2_mul(KI, MONE), qi)), QI = f2_fma(KR, qi, f2_mul(KI, qr));
        CR = f2_fma(f2_pack(csum, csum), QR, CR);
        CI = f2_fma(f2_pack(cdif, cdif), QI, CI);
    }
    float a, b;
    f2_unpack(AA, a, b);
    acc[0] += a + b;
    acc[1] += a + b;
    f2_unpack(CR, a, b); acc[2] += a + b;
    f2_unpack(CI, a, b); acc[3] += a + b;
}

__device__ __forceinline__ void group_trail_fold(const GroupArgs &ga, const GroupStepArgs &gg, const GroupStepArgs &gs,
                                                 const uint64_t TB, const int L, const uint32_t in, const int gpiv,
                                                 const float gbr, const float gbi, float (&acc)[4]) {
#define GSB_GT(NTQ_, H_)                                                                  \
    (ga.fold == 2 ? group_trail_fold2_pk<NTQ_, H_>(ga, gg, gs, TB, L, in, gpiv, gbr, gbi, acc) \
                  : group_trail_fold_pk<NTQ_, H_>(ga, gg, gs, TB, L, in, gpiv, gbr, gbi, acc))
    switch (gs.kind) {
        case GK_1_0: GSB_GT(1, 0); break;
        case GK_2_0: GSB_GT(2, 0); break;
        case GK_2_1: group_trail21_pk<true>(ga, gg, gs, TB, L, in, gpiv, gbr, gbi, acc); break;
        case GK_4_0: GSB_GT(4, 0); break;
        case GK_4_1: GSB_GT(4, 1); break;
        default: GSB_GT(4, 2); break;
    }
#undef GSB_GT
}

template <typename E, typename T, bool PK>
__device__ __forceinline__ void group_trail64(const GroupArgs &ga, const GroupStepArgs &gs, const uint64_t TB,
                                              const int L, const uint32_t in, T (&acc)[4]) {
    if constexpr (PK) {
#define GSB_GT(NTQ_, H_) group_trail_abc_pk<NTQ_, H_>(ga, gs, TB, L, in, acc)
        switch (gs.kind) {
            case GK_1_0: GSB_GT(1, 0); break;
            case GK_2_0: GSB_GT(2, 0); break;
            case GK_2_1: group_trail21_pk<false>(ga, gs, gs, TB, L, in, 0, 0.f, 0.f, acc); break;
            case GK_4_0: GSB_GT(4, 0); break;
            case GK_4_1: GSB_GT(4, 1); break;
            default: GSB_GT(4, 2); break;
        }
#undef GSB_GT
    } else {
#define GSB_GT(NTQ_, H_) group_trail_abc<E, T, 2, NTQ_, H_>(ga, gs, TB, L, in, acc)
        switch (gs.kind) {
            case GK_1_0: GSB_GT(1, 0); break;
            case GK_2_0: GSB_GT(2, 0); break;
            case GK_2_1: GSB_GT(2, 1); break;
            case GK_4_0: GSB_GT(4, 0); break;
            case GK_4_1: GSB_GT(4, 1); break;
            default: GSB_GT(4, 2); break;
        }
#undef GSB_GT
    }
}

// A written step of a complex64 pass: the factored form when the step has a compile-time shape and a pivot (piv >= 0,
// GroupStepArgs::piv), else the general form with the scaled M row (w_r, w_i).
template <typename T, bool SC, bool FIRST, bool LAST, bool STS, bool PK, bool UM = false>
__device__ __forceinline__ void group_written64(const GroupArgs &ga, const GroupStepArgs &gs, float2 *__restrict__ mem,
                                                const uint64_t TB, const int L, const uint32_t in, const uint32_t out,
                                                const int piv, const T sc, const T br, const T bi,
                                                const T (&w_r)[1][2], const T (&w_i)[1][2], T &nsum) {
    if (piv >= 0 && gs.kind != GK_ANY) {
        if constexpr (PK) {
            static_assert(std::is_same<T, float>::value, "packed form: FP32 arithmetic");
#define GSB_GF(NTQ_, H_, P_) group_cosets_pkf<NTQ_, H_, P_, SC, FIRST, LAST, STS>(ga, gs, mem, TB, L, in, out, sc, br, bi, nsum)
            switch (gs.kind * 2 + piv) {
                case GK_1_0 * 2: GSB_GF(1, 0, 0); break;
                case GK_1_0 * 2 + 1: GSB_GF(1, 0, 1); break;
                case GK_2_0 * 2: GSB_GF(2, 0, 0); break;
                case GK_2_0 * 2 + 1: GSB_GF(2, 0, 1); break;
                case GK_2_1 * 2: GSB_GF(2, 1, 0); break;
                case GK_2_1 * 2 + 1: GSB_GF(2, 1, 1); break;
                case GK_4_0 * 2: GSB_GF(4, 0, 0); break;
                case GK_4_0 * 2 + 1: GSB_GF(4, 0, 1); break;
                case GK_4_1 * 2: GSB_GF(4, 1, 0); break;
                case GK_4_1 * 2 + 1: GSB_GF(4, 1, 1); break;
                case GK_4_2 * 2: GSB_GF(4, 2, 0); break;
                default: GSB_GF(4, 2, 1); break;
            }
#undef GSB_GF
        } else {
// UM (warp-specialised passes): the common member counts 1, 2 and 4 at compile time
#define GSB_GFN(NTQ_, H_, P_, NM_) \
    group_cosets_f<float2, T, 2, NTQ_, H_, P_, SC, FIRST, LAST, STS, NM_>(ga, gs, mem, TB, L, in, out, sc, br, bi, nsum)
#define GSB_GF(NTQ_, H_, P_)                                             \
    do {                                                                 \
        if constexpr (UM) {                                              \
            switch (gs.nmem) {                                           \
                case 1: GSB_GFN(NTQ_, H_, P_, 1); break;                 \
                case 2: GSB_GFN(NTQ_, H_, P_, 2); break;                 \
                case 4: GSB_GFN(NTQ_, H_, P_, 4); break;                 \
                default: GSB_GFN(NTQ_, H_, P_, 0); break;                \
            }                                                            \
        } else {                                                         \
            GSB_GFN(NTQ_, H_, P_, 0);                                    \
        }                                                                \
    } while (0)
            switch (gs.kind * 2 + piv) {
                case GK_1_0 * 2: GSB_GF(1, 0, 0); break;
                case GK_1_0 * 2 + 1: GSB_GF(1, 0, 1); break;
                case GK_2_0 * 2: GSB_GF(2, 0, 0); break;
                case GK_2_0 * 2 + 1: GSB_GF(2, 0, 1); break;
                case GK_2_1 * 2: GSB_GF(2, 1, 0); break;
                case GK_2_1 * 2 + 1: GSB_GF(2, 1, 1); break;
                case GK_4_0 * 2: GSB_GF(4, 0, 0); break;
                case GK_4_0 * 2 + 1: GSB_GF(4, 0, 1); break;
                case GK_4_1 * 2: GSB_GF(4, 1, 0); break;
                case GK_4_1 * 2 + 1: GSB_GF(4, 1, 1); break;
                case GK_4_2 * 2: GSB_GF(4, 2, 0); break;
                default: GSB_GF(4, 2, 1); break;
            }
#undef GSB_GF
#undef GSB_GFN
        }
        return;
    }
    const uint32_t i1[1] = {in}, o1[1][1] = {{out}};
    T ns1[1][1] = {{0}};
    group_cosets_any<float2, T, FIRST, LAST, STS, 1, 1, PK>(ga, gs, mem, TB, L, i1, o1, w_r, w_i, ns1);
    nsum += ns1[0][0];
}

// Bits of a sampling pass ('sample' / 'prob': the normalised two-pass chain, gsamp2.cpp:39-55), decided at the start
// of the pass.  Step k's branch norms n(b) = |L_k(b) T|^2 come from
//   GSRC_TRAILING: the previous pass (it evaluated step k on the table it wrote: st->n0, st->n1);
//   GSRC_NORM:     a norm pass of step k just before this one, which already drew the bit (st->bv, st->sc);
//   GSRC_ANALYTIC: the step itself: with one coset offset and the x = 0 and x = 1 terms in different outputs, every
//                  entry v becomes M[b][0] v and +-M[b][1] v, so n(b) = (|M[b][0]|^2 + |M[b][1]|^2) |T|^2 exactly
//                  (ga.st[s].c[b]; |T|^2 is the stored table's norm for the pass's first step and 1 after it).
// The group's later steps are always analytic, so one pass writes them all.  Every block computes the same bits
// from the same inputs; block 0 records them (bits, log2 Pr).  Returns false when the item died here.
template <int D>
__device__ __forceinline__ bool group_decide(const GroupArgs &ga, const Ctx &cx, int (&bv)[3], double &scale) {
    DevState *st = cx.st;
    const bool rec = blockIdx.x == 0;
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    double lp = 0;
    scale = 1;
#pragma unroll
    for (int s = 0; s < D; s++) {
        const int k = ga.st[s].k;
        if (s == 0 && ga.src == GSRC_NORM) {
            bv[0] = st->bv;
            scale = st->sc;
            continue;
        }
        double n0, n1;
        if (s == 0 && ga.src == GSRC_TRAILING) { n0 = st->n0; n1 = st->n1; }
        else if (s == 0) { n0 = ga.st[0].c[0] * st->prev; n1 = ga.st[0].c[1] * st->prev; }   // |T|^2 as stored
        else { n0 = ga.st[s].c[0]; n1 = ga.st[s].c[1]; }
        // shared-sum estimates (st->trx) are good to about TRX_FLOOR absolute in p1: a draw never takes a branch
        // below that, and a forced branch is written with at least that estimate; the pass's written norm then
        // gives the branch probability itself (k_group's epilogue)
        const bool trx = s == 0 && ga.src == GSRC_TRAILING && st->trx;
        double p1 = n1 / (n0 + n1);
        if (trx && !cx.forced) p1 = p1 < TRX_FLOOR ? 0.0 : p1 > 1 - TRX_FLOOR ? 1.0 : p1;
        const int b = cx.forced ? cx.forced[row + k] : (cx.unif[row + k] < p1);
        double pb = b ? p1 : 1 - p1;
        if (trx && cx.forced && pb < TRX_FLOOR) pb = TRX_FLOOR;
        if (!(pb > 0)) {
            if (rec) {
                st->dead = 1;
                st->logp = -INFINITY;
                for (int j = k; j < cx.ns; j++) cx.bits_out[row + j] = cx.forced ? cx.forced[row + j] : 0;
            }
            return false;
        }
        lp += log2(pb);
        scale /= sqrt(trx ? pb * (n0 + n1) : (b ? n1 : n0));
        bv[s] = b;
        if (rec) cx.bits_out[row + k] = (int8_t)b;
    }
    if (rec) st->logp += lp;
    return true;
}

// ---------------------------------------------------------------------------------------------------------------
// Bulk-copy pipeline (sm_90+ PTX: mbarrier transaction counts, cp.async.bulk from global to shared memory).

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// global -> shared, completion counted on the mbarrier (bytes: multiple of 16, both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

constexpr long long PIPE_WAIT_CYCLES = 1ll << 31;   // about a second: a tile's loads take microseconds

// Wait for phase `parity` of the mbarrier, at most PIPE_WAIT_CYCLES; gives up early when another thread of the block
// already gave up (*abort).  Returns false on time-out.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, volatile int *abort) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > PIPE_WAIT_CYCLES) return false;
    }
    return true;
}

// Shared-memory layout of a fused pass (bytes; every buffer 16-byte aligned):
//   [0, 32)  four mbarriers: per input buffer, its loads landed; and (warp-specialised build) every step warp is done
//            reading it
//   two input tiles   ssz[0] blocks of 2^L arena entries (E), block i = arena block at TB ^ blk_in[i]
//   stages 1 .. D-1 (and D when a step trails it): [value index][class] (CplxOf<T>)
struct GroupSmem {
    uint32_t in0, in_bytes, mid[4], total;
};
template <typename E, typename T, int D, int TR>
__host__ __device__ inline GroupSmem group_smem(const int (&ssz)[4], int L, bool fold = false) {
    typedef typename CplxOf<T>::type V;
    GroupSmem g{};
    const uint32_t NC = 1u << L;
    g.in0 = 32;
    g.in_bytes = (uint32_t)ssz[0] * NC * (uint32_t)sizeof(E);
    uint32_t off = 32 + 2 * g.in_bytes;
    for (int s = 1; s <= D - 1 + TR; s++) {
        g.mid[s] = off;
        if (fold && s == D) continue;   // the written stage is not kept (GroupArgs::fold)
        off += (uint32_t)ssz[s] * NC * (uint32_t)sizeof(V);
    }
    g.total = off;
    return g;
}

// One fused pass: D written steps, then (TR = 1) the branch norms of the next step from the written stage, which
// stays in shared memory for it.  The bits: 'chain' (CHAIN1) takes the forced bits and the run's power-of-two scale;
// the sampling driver decides them per block (group_decide).
// A CTA walks its range of tiles in Gray-code order.  Thread 0 bulk-loads the input blocks of tile n into input
// buffer n & 1 (completion on that buffer's mbarrier) two tiles ahead: the loads of tile n + 2 are issued as soon as
// tile n's first step has read its buffer.  The last written step stores straight to the arena.  A tile's writes
// never reach another class's input (checked on the host), so the early loads are race-free.
// MINB CTAs per SM: 2 by default (up to 128 registers a thread: without this bound the compiler kept some
// instantiations at 64-80 registers and spilled); 3 for complex64 FP32 passes with tiles small enough for three
// CTAs' shared memory (85 registers: more resident warps to hide the dependent arithmetic), an autotuner candidate.
// WS (warp-specialised build, complex64 FP32 passes with tiles of 2^9 classes or more): 256 step threads and one
// load-issuing warp.  From 2^9 classes a step thread handles the same class pairs in every step of the pass, so the
// stages between steps are private to it and need no barrier; the input buffers are handed over by mbarriers (loads
// landed / every step warp done reading), so the step warps do not wait for one another within or between tiles.
template <typename E, typename T, int D, int TR, int MINB = 2, bool WS = false>
__global__ void __launch_bounds__(WS ? GROUP_NCT + 32 : GROUP_NCT, MINB)
    k_group(const GroupArgs ga, E *__restrict__ mem, const Ctx cx) {
    DevState *st = cx.st;
    if (*(volatile int *)&st->dead) return;
    extern __shared__ __align__(16) unsigned char smem[];
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    const int L = ga.L;
    const uint32_t NC = 1u << L;
    const uint64_t mask = ((uint64_t)1 << L) - 1;
    __shared__ int s_bv[3], s_ok;
    __shared__ double s_sc;
    __shared__ volatile int s_abort;
    if (threadIdx.x == 0) {
        s_ok = 1;
        s_abort = 0;
        if (cx.driver == DRV_CHAIN1) {
            for (int s = 0; s < D; s++) s_bv[s] = cx.forced[row + ga.st[s].k];
            s_sc = st->sc;
        } else {
            s_ok = group_decide<D>(ga, cx, s_bv, s_sc) ? 1 : 0;
        }
    }
    __syncthreads();
    if (!s_ok) return;
    const GroupSmem sm = group_smem<E, T, D, TR>(ga.ssz, L, ga.fold != 0);
    // Packed FP32 pairs pay where a trailing step evaluates both branch rows on the same coset sums (the sampling
    // passes, 3-7 % faster per pass).  A packed instruction holds the FMA pipe for two cycles, so passes without a
    // trailing step gain no throughput from it and lost up to 10 % to the extra register moves: they stay scalar.
    constexpr bool PK = std::is_same<T, float>::value && TR == 1;
    const uint32_t bar0 = smem_addr(smem);
    // per-step M row of the step's bit; the first step carries the pass's scale
    T w[D][1][2], wj[D][1][2];
#pragma unroll
    for (int s = 0; s < D; s++) {
        const int bv = s_bv[s];
        const double f = s == 0 ? s_sc : 1.0;
#pragma unroll
        for (int x = 0; x < 2; x++) {
            w[s][0][x] = (T)(f * ga.st[s].Mr[bv][x]);
            wj[s][0][x] = (T)(f * ga.st[s].Mi[bv][x]);
        }
    }
    // complex64 arena with FP32 arithmetic: the factored coefficients of each written step (pivot, beta with the
    // pass's scale, cp).  FP64 arithmetic (gsb_set_arith(64)) keeps the reference's complex64 arithmetic exactly:
    // full rotation, direct branch norms, the store the only rounding.
    constexpr bool FACT = sizeof(E) == 8 && std::is_same<T, float>::value;
    // folded sampling passes (GroupArgs::fold) exist only in the two-CTA build: the three-CTA register cap spills them
    constexpr bool FOLD = FACT && PK && D == 2 && TR == 1 && MINB == 2;
    static_assert(!WS || (FACT && MINB == 2), "warp-specialised build: complex64 FP32, two CTAs per SM");
    int fpiv[D];
    T fsc[D], fbr[D], fbi[D];
    double fcp[D];
#pragma unroll
    for (int s = 0; s < D; s++) {
        const int bv = s_bv[s];
        const double f = s == 0 ? s_sc : 1.0;
        fpiv[s] = FACT ? ga.st[s].piv[bv] : -1;
        fsc[s] = (T)f;
        fbr[s] = (T)(f * ga.st[s].br[bv]);
        fbi[s] = (T)(f * ga.st[s].bi[bv]);
        fcp[s] = FACT ? ga.st[s].cp[bv] : 1.0;
    }
    T tr_r[2][2], tr_i[2][2];   // trailing step: both rows
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
        for (int x = 0; x < 2; x++) {
            tr_r[b][x] = TR ? (T)ga.st[D].Mr[b][x] : (T)0;
            tr_i[b][x] = TR ? (T)ga.st[D].Mi[b][x] : (T)0;
        }
    // reduced sums: the written steps' norms, then (TR) the trailing step's (n0, n1, 0, 0), or its shared sums
    // (A, B, Re C, Im C) when it takes the complex64 shared-sum form
    constexpr int ND = D + 4 * TR;
    const bool trail_abc = FACT && TR == 1 && ga.st[D].kind != GK_ANY;
    double acc[ND];
#pragma unroll
    for (int s = 0; s < ND; s++) acc[s] = 0;
    const uint32_t none1[1][1] = {{0}};
    const uint32_t none2[1][2] = {{0, 0}};
    const uint32_t m1[1] = {sm.mid[1]}, m1o[1][1] = {{sm.mid[1]}};
    const uint32_t m2[1] = {sm.mid[2]}, m2o[1][1] = {{sm.mid[2]}};
    const uint32_t blk_bytes = NC * (uint32_t)sizeof(E);
    unsigned int i0, i1;
    block_range(cx.nchunks, i0, i1);
    // Gray-code tile bases: tile n covers classes gray(n) over bhi (the low L bits are the class index)
    auto tile_tb = [&](unsigned int n) {
        const uint32_t g = n ^ (n >> 1);
        uint64_t t = 0;
        for (int j = 0; j < ga.nbhi; j++)
            if ((g >> j) & 1) t ^= ga.bhi[j];
        return t & ~mask;
    };
    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        if (WS) {
            mbar_init(bar0 + 16, GROUP_NCT / 32);
            mbar_init(bar0 + 24, GROUP_NCT / 32);
        }
        mbar_init_fence();
    }
    __syncthreads();
    auto issue_loads = [&](unsigned int n, uint64_t TBn) {   // tile n (base TBn) into buffer (n - i0) & 1
        const int buf = (int)((n - i0) & 1);
        const uint32_t bar = bar0 + 8 * (uint32_t)buf;
        const uint32_t dst = bar0 + sm.in0 + (uint32_t)buf * sm.in_bytes;
        mbar_arrive_expect_tx(bar, sm.in_bytes);
        for (int i = 0; i < ga.ssz[0]; i++) bulk_load(dst + (uint32_t)i * blk_bytes, mem + (TBn ^ ga.blk_in[i]), blk_bytes, bar);
    };
    int issued = 0;   // tiles whose loads thread 0 issued
    // test hook: 1 withholds every CTA's tile loads, 2 only those of the odd CTAs (a partial failure)
    const bool withhold = ga.withhold_loads == 1 || (ga.withhold_loads == 2 && (blockIdx.x & 1u));
    if (!WS && threadIdx.x == 0 && !withhold)
        for (unsigned int n = i0; n < i1 && n < i0 + 2; n++) {
            issue_loads(n, tile_tb(n));
            issued++;
        }
    int waited = 0;   // tiles whose loads completed
    bool failed = false;
    uint64_t tb = i0 < i1 ? tile_tb(i0) : 0;
    if (WS && threadIdx.x >= GROUP_NCT) {
        // the load-issuing warp: tile n goes into buffer (n - i0) & 1 once every step warp is done with tile n - 2
        if (threadIdx.x == GROUP_NCT && !withhold) {
            uint64_t tp = tb;
            unsigned int n = i0;
            for (; n < i1; n++) {
                const uint32_t b = (n - i0) & 1;
                if (n >= i0 + 2 && !mbar_wait_bounded(bar0 + 16 + 8 * b, ((n - i0 - 2) >> 1) & 1, &s_abort)) {
                    s_abort = 1;
                    break;
                }
                issue_loads(n, tp);
                if (n + 1 < i1) tp ^= ga.bhi[__ffs((int)(n + 1)) - 1] & ~mask;
            }
            // the last tile issued into each buffer has landed before the block goes on (bounded): nothing is in
            // flight into this block's shared memory when it leaves
            volatile int never = 0;
            for (unsigned int m = n >= i0 + 2 ? n - 2 : i0; m < n; m++)
                mbar_wait_bounded(bar0 + 8 * ((m - i0) & 1), ((m - i0) >> 1) & 1, &never);
        }
    } else
    for (unsigned int it = i0; it < i1; it++) {
        const int buf = (int)((it - i0) & 1);
        const uint64_t TB = tb;
        if constexpr (WS) {
            // one decision per warp: a warp whose wait ran out stops, and the others' waits see s_abort
            if (!__all_sync(0xffffffffu, mbar_wait_bounded(bar0 + 8 * (uint32_t)buf, ((it - i0) >> 1) & 1, &s_abort))) {
                s_abort = 1;
                failed = true;
                break;
            }
        } else {
            if (!mbar_wait_bounded(bar0 + 8 * (uint32_t)buf, ((it - i0) >> 1) & 1, &s_abort)) s_abort = 1;
            __syncthreads();
            if (s_abort) {
                failed = true;
                break;
            }
        }
        waited++;
        T ns[D][1][1];
        T nt[1][2] = {{0, 0}};
#pragma unroll
        for (int s = 0; s < D; s++) ns[s][0][0] = 0;
        const uint32_t tin[1] = {sm.in0 + (uint32_t)buf * sm.in_bytes};
        // written steps: the first reads the input tile, the last writes the arena (and keeps its stage for the
        // trailing step); the input buffer is free once the first step is done: tile it + 2 goes there
        if constexpr (FACT) {
            float2 *m64 = reinterpret_cast<float2 *>(mem);
            if (D == 1)
                group_written64<T, true, true, true, TR == 1, PK, WS && !PK>(ga, ga.st[0], m64, TB, L, tin[0], sm.mid[1], fpiv[0],
                                                                 fsc[0], fbr[0], fbi[0], w[0], wj[0], ns[0][0][0]);
            else
                group_written64<T, true, true, false, true, PK, WS && !PK>(ga, ga.st[0], m64, TB, L, tin[0], sm.mid[1], fpiv[0],
                                                               fsc[0], fbr[0], fbi[0], w[0], wj[0], ns[0][0][0]);
        } else if (D == 1) {
            group_cosets_any<E, T, true, true, TR == 1, 1, 1, PK>(ga, ga.st[0], mem, TB, L, tin, m1o, w[0], wj[0], ns[0]);
        } else {
            group_cosets_any<E, T, true, false, true, 1, 1, PK>(ga, ga.st[0], mem, TB, L, tin, m1o, w[0], wj[0], ns[0]);
        }
        if constexpr (WS) {
            __syncwarp();
            if ((threadIdx.x & 31) == 0) mbar_arrive(bar0 + 16 + 8 * (uint32_t)buf);   // this warp is done with the tile
        } else {
            __syncthreads();
        }
        if (!WS && threadIdx.x == 0 && it + 2 < i1 && !withhold) {
            // tile it + 2 is two Gray-code steps from this tile (gray(n + 1) = gray(n) ^ 2^ctz(n + 1)); rebuilding its
            // base from the index, a loop over the class-base vectors, held up warp 0 and so every warp at the next
            // barrier (4-7 % of the pass)
            issue_loads(it + 2, TB ^ ((ga.bhi[__ffs((int)(it + 1)) - 1] ^ ga.bhi[__ffs((int)(it + 2)) - 1]) & ~mask));
            issued++;
        }
        if constexpr (FACT) {
            float2 *m64 = reinterpret_cast<float2 *>(mem);
            if (FOLD && ga.fold) {   // the written stage is not kept: the trailing step folds it
                group_written64<T, false, false, true, false, PK, WS && !PK>(ga, ga.st[1], m64, TB, L, sm.mid[1], 0u,
                                                                 fpiv[D > 1 ? 1 : 0], fsc[D > 1 ? 1 : 0],
                                                                 fbr[D > 1 ? 1 : 0], fbi[D > 1 ? 1 : 0],
                                                                 w[D > 1 ? 1 : 0], wj[D > 1 ? 1 : 0], ns[D > 1 ? 1 : 0][0][0]);
            } else if (D == 2) {
                group_written64<T, false, false, true, TR == 1, PK, WS && !PK>(ga, ga.st[1], m64, TB, L, sm.mid[1], sm.mid[2],
                                                                   fpiv[D > 1 ? 1 : 0], fsc[D > 1 ? 1 : 0],
                                                                   fbr[D > 1 ? 1 : 0], fbi[D > 1 ? 1 : 0],
                                                                   w[D > 1 ? 1 : 0], wj[D > 1 ? 1 : 0], ns[D > 1 ? 1 : 0][0][0]);
            } else if (D == 3) {
                group_written64<T, false, false, false, true, PK, WS && !PK>(ga, ga.st[1], m64, TB, L, sm.mid[1], sm.mid[2],
                                                                 fpiv[D > 1 ? 1 : 0], fsc[D > 1 ? 1 : 0],
                                                                 fbr[D > 1 ? 1 : 0], fbi[D > 1 ? 1 : 0],
                                                                 w[D > 1 ? 1 : 0], wj[D > 1 ? 1 : 0], ns[D > 1 ? 1 : 0][0][0]);
                if constexpr (!WS) __syncthreads();
                group_written64<T, false, false, true, false, PK, WS && !PK>(ga, ga.st[2], m64, TB, L, sm.mid[2], 0u,
                                                                 fpiv[D > 2 ? 2 : 0], fsc[D > 2 ? 2 : 0],
                                                                 fbr[D > 2 ? 2 : 0], fbi[D > 2 ? 2 : 0],
                                                                 w[D > 2 ? 2 : 0], wj[D > 2 ? 2 : 0], ns[D > 2 ? 2 : 0][0][0]);
            }
        } else if (D == 2) {
            group_cosets_any<E, T, false, true, TR == 1, 1, 1, PK>(ga, ga.st[1], mem, TB, L, m1, m2o, w[1], wj[1], ns[1]);
        } else if (D == 3) {
            group_cosets_any<E, T, false, false, true, 1, 1, PK>(ga, ga.st[1], mem, TB, L, m1, m2o, w[1], wj[1], ns[1]);
            __syncthreads();
            group_cosets_any<E, T, false, true, false, 1, 1, PK>(ga, ga.st[2], mem, TB, L, m2, none1, w[2], wj[2], ns[2]);
        }
        T tabc[4] = {0, 0, 0, 0};
        if (TR) {
            if (D > 1 && !WS) __syncthreads();
            const uint32_t(&tmid)[1] = D == 1 ? m1 : m2;
            bool done = false;
            if constexpr (FOLD) {
                if (ga.fold) {
                    group_trail_fold(ga, ga.st[1], ga.st[2], TB, L, sm.mid[1], fpiv[D > 1 ? 1 : 0], fbr[D > 1 ? 1 : 0],
                                     fbi[D > 1 ? 1 : 0], tabc);
                    done = true;
                }
            }
            if (done) {
            } else if (FACT && trail_abc)
                group_trail64<E, T, PK>(ga, ga.st[D], TB, L, tmid[0], tabc);
            else
                group_cosets_any<E, T, false, false, false, 1, 2, PK>(ga, ga.st[D], mem, TB, L, tmid, none2, tr_r, tr_i, nt);
        }
        if constexpr (!WS) __syncthreads();
#pragma unroll
        for (int s = 0; s < D; s++) acc[s] += (double)ns[s][0][0];
        if (TR) {
            if (trail_abc) {
#pragma unroll
                for (int i = 0; i < 4; i++) acc[TR ? D + i : 0] += (double)tabc[i];
            } else {
                acc[TR ? D : 0] += (double)nt[0][0];
                acc[TR ? D + 1 : 0] += (double)nt[0][1];
            }
        }
        if (it + 1 < i1) tb ^= ga.bhi[__ffs((int)(it + 1)) - 1] & ~mask;
    }
    if constexpr (WS) {
        __syncthreads();   // every warp has left its loop (each wait is bounded); the load warp has drained its loads
        failed = s_abort != 0;
    }
    if (failed) {
        // a load never completed: record it, let the loads still in flight land (bounded) and leave the item
        if (threadIdx.x == 0) {
            atomicExch(&st->err, 1);
            st->dead = 1;
            volatile int never = 0;
            if (!WS)
                for (int n = waited; n < issued; n++)
                    mbar_wait_bounded(bar0 + 8 * (uint32_t)(n & 1), (uint32_t)(n >> 1) & 1, &never);
            // count this block as finished, so the block that finishes last (a failed one or one in grid_reduceN)
            // sees every block and returns the counter to zero
            __threadfence();
            if (atomicAdd(&st->counter, 1u) == gridDim.x - 1) st->counter = 0;
        }
        __syncthreads();
        return;
    }
    double tot[ND];
    if (!grid_reduceN<ND>(acc, cx, tot)) return;
    if (cx.driver == DRV_CHAIN1) {
        group_chain1_epilogue<D>(cx, ga.st[0].k, *reinterpret_cast<const double(*)[D]>(tot), fcp);
    } else {
        if (ga.src == GSRC_TRAILING && st->trx) {
            // the first bit came from shared-sum estimates: its branch probability is the estimate used times the
            // ratio of the written norm to the one the pass's scale aimed at (1 / prod cp)
            double cpp = 1;
#pragma unroll
            for (int s = 0; s < D; s++) cpp *= fcp[s];
            const double ratio = tot[D - 1] * cpp;
            if (!(ratio > 0)) {
                const size_t row = (size_t)st->item * (size_t)cx.ns;
                st->dead = 1;
                st->logp = -INFINITY;
                for (int j = ga.st[0].k; j < cx.ns; j++) cx.bits_out[row + j] = cx.forced ? cx.forced[row + j] : 0;
                return;
            }
            st->logp += log2(ratio);
        }
        st->prev = tot[D - 1];
        st->trx = 0;
        if (TR) {
            if (trail_abc) {
                const GroupStepArgs &g = ga.st[D < 3 ? D : 0];
                const double A = tot[TR ? D : 0], B = tot[TR ? D + 1 : 0], Cr = tot[TR ? D + 2 : 0], Ci = tot[TR ? D + 3 : 0];
                double nb[2];
                for (int b = 0; b < 2; b++) {
                    const double a0 = g.Mr[b][0], b0 = g.Mi[b][0], a1 = g.Mr[b][1], b1 = g.Mi[b][1];
                    const double v = (a0 * a0 + b0 * b0) * A + (a1 * a1 + b1 * b1) * B +
                                     2 * ((a0 * a1 + b0 * b1) * Cr - (b0 * a1 - a0 * b1) * Ci);
                    nb[b] = v > 0 ? v : 0;
                }
                st->n0 = nb[0];
                st->n1 = nb[1];
                st->trx = 1;
            } else {
                st->n0 = tot[TR ? D : 0];
                st->n1 = tot[TR ? D + 1 : 0];
            }
        }
    }
}

}  // namespace gsb
