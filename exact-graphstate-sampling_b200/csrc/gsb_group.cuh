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
    unsigned char in_idx[16][4], out_idx[16][2], mpar[16];
};

// first-bit source of a sampling pass (group_decide)
enum { GSRC_ANALYTIC = 0, GSRC_TRAILING = 1, GSRC_NORM = 2 };

struct GroupArgs {
    int d, L, nbhi, ssz[4];
    int src;               // GSRC_*
    int withhold_loads;    // test hook (gsb_test_withhold_tile_loads): issue no tile loads, so every wait runs out
    uint64_t bhi[40];
    uint64_t blk_in[32];   // stage-0 offsets z_i, bits >= L: input block i of a tile is the arena block at TB ^ blk_in[i]
    uint64_t blk_out[32];  // written-stage offsets, bits >= L: output block i goes to the arena block at TB ^ blk_out[i]
    uint32_t z0lo[16][4];  // first step: member j, offset t -> bits < L of its stage-0 offset (position p ^ z0lo)
    uint32_t zdlo[16][2];  // last written step: member j, output tau -> bits < L of its offset
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

// Grid-wide deterministic sums of ND values (same scheme as grid_reduce2); true in thread 0 of the last block.
template <int ND>
__device__ __forceinline__ bool grid_reduceN(double (&a)[ND], const Ctx &cx, double (&t)[ND]) {
    __shared__ double red[ND][32];
    __shared__ int last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < ND; i++) a[i] = warp_sum(a[i]);
    if (lane == 0)
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
    double s[ND];
#pragma unroll
    for (int i = 0; i < ND; i++) s[i] = 0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int i = 0; i < ND; i++) s[i] += __ldcg(cx.partials + ND * b + i);
#pragma unroll
    for (int i = 0; i < ND; i++) s[i] = warp_sum(s[i]);
    __syncthreads();
    if (lane == 0)
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
template <int D>
__device__ __forceinline__ void group_chain1_epilogue(const Ctx &cx, int k0, const double (&nb)[D]) {
    DevState *st = cx.st;
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    double prev = st->prev;
    for (int s = 0; s < D; s++) {
        const double c = s == 0 ? ldexp(nb[0], 2 * st->ek) / (2 * prev) : nb[s] / (2 * nb[s - 1]);
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
    st->lsc += st->ek;
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
    uint32_t g0 = threadIdx.x, gstride = blockDim.x;
    int j0 = 0, jstride = 1;
    if (NG < blockDim.x) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(blockDim.x >> LG);
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
    uint32_t g0 = threadIdx.x, gstride = blockDim.x;
    int j0 = 0, jstride = 1;
    if (NG < blockDim.x) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(blockDim.x >> LG);
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
        const double p1 = n1 / (n0 + n1);
        const int b = cx.forced ? cx.forced[row + k] : (cx.unif[row + k] < p1);
        const double pb = b ? p1 : 1 - p1;
        if (!(pb > 0)) {
            if (rec) {
                st->dead = 1;
                st->logp = -INFINITY;
                for (int j = k; j < cx.ns; j++) cx.bits_out[row + j] = cx.forced ? cx.forced[row + j] : 0;
            }
            return false;
        }
        lp += log2(pb);
        scale /= sqrt(b ? n1 : n0);
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
//   [0, 16)  two mbarriers (one per input buffer)
//   two input tiles   ssz[0] blocks of 2^L arena entries (E), block i = arena block at TB ^ blk_in[i]
//   stages 1 .. D-1 (and D when a step trails it): [value index][class] (CplxOf<T>)
struct GroupSmem {
    uint32_t in0, in_bytes, mid[4], total;
};
template <typename E, typename T, int D, int TR>
__host__ __device__ inline GroupSmem group_smem(const int (&ssz)[4], int L) {
    typedef typename CplxOf<T>::type V;
    GroupSmem g{};
    const uint32_t NC = 1u << L;
    g.in0 = 16;
    g.in_bytes = (uint32_t)ssz[0] * NC * (uint32_t)sizeof(E);
    uint32_t off = 16 + 2 * g.in_bytes;
    for (int s = 1; s <= D - 1 + TR; s++) {
        g.mid[s] = off;
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
// Two CTAs per SM (the shared-memory budget allows no more), so up to 128 registers a thread: without this bound the
// compiler kept some instantiations at 64-80 registers and spilled.
template <typename E, typename T, int D, int TR>
__global__ void __launch_bounds__(256, 2) k_group(const GroupArgs ga, E *__restrict__ mem, const Ctx cx) {
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
    const GroupSmem sm = group_smem<E, T, D, TR>(ga.ssz, L);
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
    T tr_r[2][2], tr_i[2][2];   // trailing step: both rows
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
        for (int x = 0; x < 2; x++) {
            tr_r[b][x] = TR ? (T)ga.st[D].Mr[b][x] : (T)0;
            tr_i[b][x] = TR ? (T)ga.st[D].Mi[b][x] : (T)0;
        }
    constexpr int ND = D + 2 * TR;
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
    if (threadIdx.x == 0 && !ga.withhold_loads)
        for (unsigned int n = i0; n < i1 && n < i0 + 2; n++) {
            issue_loads(n, tile_tb(n));
            issued++;
        }
    int waited = 0;   // tiles whose loads completed
    bool failed = false;
    uint64_t tb = i0 < i1 ? tile_tb(i0) : 0;
    for (unsigned int it = i0; it < i1; it++) {
        const int buf = (int)((it - i0) & 1);
        const uint64_t TB = tb;
        if (!mbar_wait_bounded(bar0 + 8 * (uint32_t)buf, ((it - i0) >> 1) & 1, &s_abort)) s_abort = 1;
        __syncthreads();
        if (s_abort) {
            failed = true;
            break;
        }
        waited++;
        T ns[D][1][1];
        T nt[1][2] = {{0, 0}};
#pragma unroll
        for (int s = 0; s < D; s++) ns[s][0][0] = 0;
        const uint32_t tin[1] = {sm.in0 + (uint32_t)buf * sm.in_bytes};
        // written steps: the first reads the input tile, the last writes the arena (and keeps its stage for the
        // trailing step); the input buffer is free once the first step is done: tile it + 2 goes there
        if (D == 1) {
            group_cosets_any<E, T, true, true, TR == 1, 1, 1, PK>(ga, ga.st[0], mem, TB, L, tin, m1o, w[0], wj[0], ns[0]);
            __syncthreads();
        } else {
            group_cosets_any<E, T, true, false, true, 1, 1, PK>(ga, ga.st[0], mem, TB, L, tin, m1o, w[0], wj[0], ns[0]);
            __syncthreads();
        }
        if (threadIdx.x == 0 && it + 2 < i1 && !ga.withhold_loads) {
            // tile it + 2 is two Gray-code steps from this tile (gray(n + 1) = gray(n) ^ 2^ctz(n + 1)); rebuilding its
            // base from the index, a loop over the class-base vectors, held up warp 0 and so every warp at the next
            // barrier (4-7 % of the pass)
            issue_loads(it + 2, TB ^ ((ga.bhi[__ffs((int)(it + 1)) - 1] ^ ga.bhi[__ffs((int)(it + 2)) - 1]) & ~mask));
            issued++;
        }
        if (D == 2) {
            group_cosets_any<E, T, false, true, TR == 1, 1, 1, PK>(ga, ga.st[1], mem, TB, L, m1, m2o, w[1], wj[1], ns[1]);
        } else if (D == 3) {
            group_cosets_any<E, T, false, false, true, 1, 1, PK>(ga, ga.st[1], mem, TB, L, m1, m2o, w[1], wj[1], ns[1]);
            __syncthreads();
            group_cosets_any<E, T, false, true, false, 1, 1, PK>(ga, ga.st[2], mem, TB, L, m2, none1, w[2], wj[2], ns[2]);
        }
        if (TR) {
            if (D > 1) __syncthreads();
            const uint32_t(&tmid)[1] = D == 1 ? m1 : m2;
            group_cosets_any<E, T, false, false, false, 1, 2, PK>(ga, ga.st[D], mem, TB, L, tmid, none2, tr_r, tr_i, nt);
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < D; s++) acc[s] += (double)ns[s][0][0];
        if (TR) {
            acc[D] += (double)nt[0][0];
            acc[ND - 1] += (double)nt[0][1];
        }
        if (it + 1 < i1) tb ^= ga.bhi[__ffs((int)(it + 1)) - 1] & ~mask;
    }
    if (failed) {
        // a load never completed: record it, let the loads still in flight land (bounded) and leave the item
        if (threadIdx.x == 0) {
            atomicExch(&st->err, 1);
            st->dead = 1;
            volatile int never = 0;
            for (int n = waited; n < issued; n++) mbar_wait_bounded(bar0 + 8 * (uint32_t)(n & 1), (uint32_t)(n >> 1) & 1, &never);
        }
        __syncthreads();
        return;
    }
    double tot[ND];
    if (!grid_reduceN<ND>(acc, cx, tot)) return;
    if (cx.driver == DRV_CHAIN1) {
        group_chain1_epilogue<D>(cx, ga.st[0].k, *reinterpret_cast<const double(*)[D]>(tot));
    } else {
        st->prev = tot[D - 1];
        if (TR) {
            st->n0 = tot[D];
            st->n1 = tot[ND - 1];
        }
    }
}

}  // namespace gsb
