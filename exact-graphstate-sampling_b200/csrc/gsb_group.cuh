// Fused pass over a group of consecutive DP steps (host derivation in gsb_fuse.cpp).
//
// A CTA owns tiles of 2^L classes.  The classes of a tile have bases TB | p (p < 2^L, TB a multiple of 2^L), so for
// every stage-0 offset z the tile's inputs are one aligned block of 2^L entries at TB ^ (z & ~mask), with class p at
// position p ^ (z & mask); the same holds for the stage-d outputs.  For each step s of the group, work items
// (pair of adjacent classes, member j) -- a warp takes 32 consecutive pairs of one member -- read the member's ntq
// stage-s values (adjacent classes are adjacent entries, so a pair is one 16-byte access for complex64),
// form the coset's sums with the sign parity(TB & lambda) ^ parity(p & lambda) ^ mpar_j, rotate by M[b_s] (the first
// step also applies the run's scale), write the m stage-(s+1) values and add their squares to the step's norm.
// The first step reads the arena directly (each warp access is one contiguous segment: XOR by a constant only
// permutes lanes inside it), the last step writes the arena directly, and the stages in between stay in shared
// memory.
// A class's outputs land only in its own input slots or in slots no class reads (checked on the host), so tiles are
// independent and the pass is race-free in place.
#pragma once
#include "gsb_kernels.cuh"

namespace gsb {

struct GroupStepArgs {
    int nmem, ntq, m, k;
    int tau0[4], tau1[4], par[4];
    uint64_t lambda;
    double Mr[2][2], Mi[2][2];
    unsigned char in_idx[16][4], out_idx[16][2], mpar[16];
};

struct GroupArgs {
    int d, L, nbhi, ssz[4];
    uint64_t bhi[40];
    uint64_t z0hi[16][4];  // first step: member j, offset t -> stage-0 offset, bits >= L (read from the arena)
    uint32_t z0lo[16][4];  //                                                 bits <  L
    uint64_t zdhi[16][2];  // last step: member j, class tau -> stage-d offset, bits >= L (written to the arena)
    uint32_t zdlo[16][2];
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

// Two complex values of adjacent classes (even p, p ^ 1) at entry index a (a even): the pair is one 16-byte access
// for a complex64 arena and two for complex128.
__device__ __forceinline__ void ld_pair(const float2 *m, uint64_t a, float &er, float &ei, float &orr, float &oi) {
    const float4 v = *reinterpret_cast<const float4 *>(m + a);
    er = v.x; ei = v.y; orr = v.z; oi = v.w;
}
__device__ __forceinline__ void ld_pair(const float2 *m, uint64_t a, double &er, double &ei, double &orr, double &oi) {
    const float4 v = *reinterpret_cast<const float4 *>(m + a);
    er = v.x; ei = v.y; orr = v.z; oi = v.w;
}
__device__ __forceinline__ void ld_pair(const double2 *m, uint64_t a, double &er, double &ei, double &orr, double &oi) {
    const double2 u = m[a], v = m[a + 1];
    er = u.x; ei = u.y; orr = v.x; oi = v.y;
}
__device__ __forceinline__ void st_pair(float2 *m, uint64_t a, float er, float ei, float orr, float oi) {
    *reinterpret_cast<float4 *>(m + a) = make_float4(er, ei, orr, oi);
}
__device__ __forceinline__ void st_pair(float2 *m, uint64_t a, double er, double ei, double orr, double oi) {
    *reinterpret_cast<float4 *>(m + a) = make_float4((float)er, (float)ei, (float)orr, (float)oi);
}
__device__ __forceinline__ void st_pair(double2 *m, uint64_t a, double er, double ei, double orr, double oi) {
    m[a] = make_double2(er, ei);
    m[a + 1] = make_double2(orr, oi);
}

// Shared-memory pair access of adjacent classes: one 16-byte access for 8-byte values.
__device__ __forceinline__ void lds_pair(const float2 *q, float &er, float &ei, float &orr, float &oi) {
    const float4 v = *reinterpret_cast<const float4 *>(q);
    er = v.x; ei = v.y; orr = v.z; oi = v.w;
}
__device__ __forceinline__ void lds_pair(const double2 *q, double &er, double &ei, double &orr, double &oi) {
    const double2 u = q[0], v = q[1];
    er = u.x; ei = u.y; orr = v.x; oi = v.y;
}
__device__ __forceinline__ void sts_pair(float2 *q, float er, float ei, float orr, float oi) {
    *reinterpret_cast<float4 *>(q) = make_float4(er, ei, orr, oi);
}
__device__ __forceinline__ void sts_pair(double2 *q, double er, double ei, double orr, double oi) {
    q[0] = make_double2(er, ei);
    q[1] = make_double2(orr, oi);
}

// Arena / shared-memory access of P adjacent classes (even p, then p ^ 1 when P = 2).
template <int P>
__device__ __forceinline__ void ld_cls(const float2 *m, uint64_t a, bool sw, float (&r)[P], float (&i)[P]) {
    if (P == 2) {
        const float4 v = *reinterpret_cast<const float4 *>(m + a);
        r[0] = sw ? v.z : v.x; i[0] = sw ? v.w : v.y;
        r[P - 1] = sw ? v.x : v.z; i[P - 1] = sw ? v.y : v.w;
    } else {
        const float2 v = m[a + (sw ? 1 : 0)];
        r[0] = v.x; i[0] = v.y;
    }
}
template <int P>
__device__ __forceinline__ void ld_cls(const float2 *m, uint64_t a, bool sw, double (&r)[P], double (&i)[P]) {
    float fr[P], fi[P];
    ld_cls<P>(m, a, sw, fr, fi);
#pragma unroll
    for (int c = 0; c < P; c++) { r[c] = fr[c]; i[c] = fi[c]; }
}
template <int P>
__device__ __forceinline__ void ld_cls(const double2 *m, uint64_t a, bool sw, double (&r)[P], double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) {
        const double2 v = m[a + (uint64_t)((c ^ (sw ? 1 : 0)) & 1)];
        r[c] = v.x; i[c] = v.y;
    }
}
template <int P>
__device__ __forceinline__ void st_cls(float2 *m, uint64_t a, bool sw, const float (&r)[P], const float (&i)[P]) {
    if (P == 2) *reinterpret_cast<float4 *>(m + a) = sw ? make_float4(r[P - 1], i[P - 1], r[0], i[0]) : make_float4(r[0], i[0], r[P - 1], i[P - 1]);
    else m[a + (sw ? 1 : 0)] = make_float2(r[0], i[0]);
}
template <int P>
__device__ __forceinline__ void st_cls(float2 *m, uint64_t a, bool sw, const double (&r)[P], const double (&i)[P]) {
    float fr[P], fi[P];
#pragma unroll
    for (int c = 0; c < P; c++) { fr[c] = (float)r[c]; fi[c] = (float)i[c]; }
    st_cls<P>(m, a, sw, fr, fi);
}
template <int P>
__device__ __forceinline__ void st_cls(double2 *m, uint64_t a, bool sw, const double (&r)[P], const double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) m[a + (uint64_t)((c ^ (sw ? 1 : 0)) & 1)] = make_double2(r[c], i[c]);
}
// shared memory [index][class]: P consecutive values
template <int P>
__device__ __forceinline__ void lds_cls(const float2 *q, float (&r)[P], float (&i)[P]) {
    if (P == 2) {
        const float4 v = *reinterpret_cast<const float4 *>(q);
        r[0] = v.x; i[0] = v.y; r[P - 1] = v.z; i[P - 1] = v.w;
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
    if (P == 2) *reinterpret_cast<float4 *>(q) = make_float4(r[0], i[0], r[P - 1], i[P - 1]);
    else q[0] = make_float2(r[0], i[0]);
}
template <int P>
__device__ __forceinline__ void sts_cls(double2 *q, const double (&r)[P], const double (&i)[P]) {
#pragma unroll
    for (int c = 0; c < P; c++) q[c] = make_double2(r[c], i[c]);
}

// One step of a group on one tile.  A work item is P adjacent classes (P = 2 for complex64: one 16-byte access) of
// one member j.  Threads take class groups and, when the tile has fewer class groups than threads, split the members
// too.  Per coset: the x = 0 terms sum into their output class, the x = 1 terms sum with the sign
// (-1)^(parity(base & lambda) ^ par_t) into theirs, and each output class is rotated by the M row of the step's bit.
// FIRST reads the arena, LAST writes it; the other stages use the shared-memory buffers [index][class].
template <typename E, typename T, int P, int NTQ, bool FIRST, bool LAST>
__device__ __forceinline__ void group_step(const GroupArgs &ga, const GroupStepArgs &gs, E *__restrict__ mem,
                                           const uint64_t TB, const int L, typename CplxOf<T>::type *in_buf,
                                           typename CplxOf<T>::type *out_buf, const T (&w_r)[2], const T (&w_i)[2],
                                           double &acc) {
    const uint32_t NC = 1u << L;
    const int LG = P == 2 ? L - 1 : L;                 // log2 class groups per tile
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem, m = gs.m;
    // thread -> (first class group, first member, member stride)
    uint32_t g0 = threadIdx.x, gstride = blockDim.x;
    int j0 = 0, jstride = 1;
    if (NG < blockDim.x) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(blockDim.x >> LG);
    }
    T nsum = 0;
    for (uint32_t g = g0; g < NG; g += gstride) {
        const uint32_t pc = (uint32_t)P * g;
        int pcls[P];
#pragma unroll
        for (int c = 0; c < P; c++) pcls[c] = tpar ^ (__popc((pc + c) & (uint32_t)gs.lambda) & 1);
        for (int j = j0; j < nm; j += jstride) {
            // sums by (class c, x, tau, re/im); every index below is a compile-time constant (registers)
            T S[P][2][2][2];
#pragma unroll
            for (int c = 0; c < P; c++)
#pragma unroll
                for (int x = 0; x < 2; x++) { S[c][x][0][0] = 0; S[c][x][0][1] = 0; S[c][x][1][0] = 0; S[c][x][1][1] = 0; }
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                T vr[P], vi[P];
                if (FIRST) {
                    const uint32_t zl = ga.z0lo[j][t];
                    const uint64_t a = (TB ^ ga.z0hi[j][t]) | (uint64_t)((pc ^ zl) & ~(uint32_t)(P - 1));
                    ld_cls<P>(mem, a, P == 2 ? (zl & 1) != 0 : false, vr, vi);
                } else {
                    lds_cls<P>(in_buf + (size_t)gs.in_idx[j][t] * NC + pc, vr, vi);
                }
                const bool t0 = gs.tau0[t] != 0, t1 = gs.tau1[t] != 0;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    const T sg = ((pcls[c] ^ gs.mpar[j] ^ gs.par[t]) & 1) ? (T)-1 : (T)1;
                    if (!t0) { S[c][0][0][0] += vr[c]; S[c][0][0][1] += vi[c]; }
                    else { S[c][0][1][0] += vr[c]; S[c][0][1][1] += vi[c]; }
                    if (!t1) { S[c][1][0][0] = fmaT(sg, vr[c], S[c][1][0][0]); S[c][1][0][1] = fmaT(sg, vi[c], S[c][1][0][1]); }
                    else { S[c][1][1][0] = fmaT(sg, vr[c], S[c][1][1][0]); S[c][1][1][1] = fmaT(sg, vi[c], S[c][1][1][1]); }
                }
            }
#pragma unroll
            for (int tau = 0; tau < 2; tau++) {
                if (tau >= m) break;
                T orr[P], oi[P];
#pragma unroll
                for (int c = 0; c < P; c++) {
                    const T xr = S[c][0][tau][0], xi = S[c][0][tau][1], zr = S[c][1][tau][0], zi = S[c][1][tau][1];
                    T r = w_r[0] * xr;
                    r = fmaT(-w_i[0], xi, r);
                    r = fmaT(w_r[1], zr, r);
                    r = fmaT(-w_i[1], zi, r);
                    T im = w_r[0] * xi;
                    im = fmaT(w_i[0], xr, im);
                    im = fmaT(w_r[1], zi, im);
                    im = fmaT(w_i[1], zr, im);
                    orr[c] = r;
                    oi[c] = im;
                    nsum = fmaT(r, r, nsum);
                    nsum = fmaT(im, im, nsum);
                }
                if (LAST) {
                    const uint32_t zl = ga.zdlo[j][tau];
                    const uint64_t a = (TB ^ ga.zdhi[j][tau]) | (uint64_t)((pc ^ zl) & ~(uint32_t)(P - 1));
                    st_cls<P>(mem, a, P == 2 ? (zl & 1) != 0 : false, orr, oi);
                } else {
                    sts_cls<P>(out_buf + (size_t)gs.out_idx[j][tau] * NC + pc, orr, oi);
                }
            }
        }
    }
    acc += (double)nsum;
}

template <typename E, typename T, bool FIRST, bool LAST>
__device__ __forceinline__ void group_step_any(const GroupArgs &ga, const GroupStepArgs &gs, E *__restrict__ mem,
                                               const uint64_t TB, const int L, typename CplxOf<T>::type *in_buf,
                                               typename CplxOf<T>::type *out_buf, const T (&w_r)[2],
                                               const T (&w_i)[2], double &acc) {
    constexpr int P = sizeof(E) == 8 ? 2 : 1;          // complex64: two classes per 16-byte access
    switch (gs.ntq) {   // uniform across the grid
        case 1: group_step<E, T, P, 1, FIRST, LAST>(ga, gs, mem, TB, L, in_buf, out_buf, w_r, w_i, acc); break;
        case 2: group_step<E, T, P, 2, FIRST, LAST>(ga, gs, mem, TB, L, in_buf, out_buf, w_r, w_i, acc); break;
        default: group_step<E, T, P, 4, FIRST, LAST>(ga, gs, mem, TB, L, in_buf, out_buf, w_r, w_i, acc); break;
    }
}

// Branch norms of one step on one tile for both values of the step's bit (the look-ahead of exact sampling): the
// coset sums are formed once, rotated by both rows of M, the squares of each row's outputs summed into n[b], and, when
// out[b] is given, the outputs stored to that shared-memory stage buffer.  FIRST reads the stage from the arena.
template <typename E, typename T, int P, int NTQ, bool FIRST>
__device__ __forceinline__ void group_step_rows(const GroupArgs &ga, const GroupStepArgs &gs, E *__restrict__ mem,
                                                const uint64_t TB, const int L, typename CplxOf<T>::type *in_buf,
                                                typename CplxOf<T>::type *out0, typename CplxOf<T>::type *out1,
                                                const T (&w_r)[2][2], const T (&w_i)[2][2], double &n0, double &n1) {
    const uint32_t NC = 1u << L;
    const int LG = P == 2 ? L - 1 : L;
    const uint32_t NG = 1u << LG;
    const int tpar = __popcll(TB & gs.lambda) & 1;
    const int nm = gs.nmem, m = gs.m;
    uint32_t g0 = threadIdx.x, gstride = blockDim.x;
    int j0 = 0, jstride = 1;
    if (NG < blockDim.x) {
        g0 = threadIdx.x & (NG - 1);
        gstride = NG;
        j0 = (int)(threadIdx.x >> LG);
        jstride = (int)(blockDim.x >> LG);
    }
    T ns0 = 0, ns1 = 0;
    for (uint32_t g = g0; g < NG; g += gstride) {
        const uint32_t pc = (uint32_t)P * g;
        int pcls[P];
#pragma unroll
        for (int c = 0; c < P; c++) pcls[c] = tpar ^ (__popc((pc + c) & (uint32_t)gs.lambda) & 1);
        for (int j = j0; j < nm; j += jstride) {
            T S[P][2][2][2];
#pragma unroll
            for (int c = 0; c < P; c++)
#pragma unroll
                for (int x = 0; x < 2; x++) { S[c][x][0][0] = 0; S[c][x][0][1] = 0; S[c][x][1][0] = 0; S[c][x][1][1] = 0; }
#pragma unroll
            for (int t = 0; t < NTQ; t++) {
                T vr[P], vi[P];
                if (FIRST) {
                    const uint32_t zl = ga.z0lo[j][t];
                    const uint64_t a = (TB ^ ga.z0hi[j][t]) | (uint64_t)((pc ^ zl) & ~(uint32_t)(P - 1));
                    ld_cls<P>(mem, a, P == 2 ? (zl & 1) != 0 : false, vr, vi);
                } else {
                    lds_cls<P>(in_buf + (size_t)gs.in_idx[j][t] * NC + pc, vr, vi);
                }
                const bool t0 = gs.tau0[t] != 0, t1 = gs.tau1[t] != 0;
#pragma unroll
                for (int c = 0; c < P; c++) {
                    const T sg = ((pcls[c] ^ gs.mpar[j] ^ gs.par[t]) & 1) ? (T)-1 : (T)1;
                    if (!t0) { S[c][0][0][0] += vr[c]; S[c][0][0][1] += vi[c]; }
                    else { S[c][0][1][0] += vr[c]; S[c][0][1][1] += vi[c]; }
                    if (!t1) { S[c][1][0][0] = fmaT(sg, vr[c], S[c][1][0][0]); S[c][1][0][1] = fmaT(sg, vi[c], S[c][1][0][1]); }
                    else { S[c][1][1][0] = fmaT(sg, vr[c], S[c][1][1][0]); S[c][1][1][1] = fmaT(sg, vi[c], S[c][1][1][1]); }
                }
            }
#pragma unroll
            for (int b = 0; b < 2; b++) {
                typename CplxOf<T>::type *out = b ? out1 : out0;
#pragma unroll
                for (int tau = 0; tau < 2; tau++) {
                    if (tau >= m) break;
                    T orr[P], oi[P];
#pragma unroll
                    for (int c = 0; c < P; c++) {
                        const T xr = S[c][0][tau][0], xi = S[c][0][tau][1], zr = S[c][1][tau][0], zi = S[c][1][tau][1];
                        T r = w_r[b][0] * xr;
                        r = fmaT(-w_i[b][0], xi, r);
                        r = fmaT(w_r[b][1], zr, r);
                        r = fmaT(-w_i[b][1], zi, r);
                        T im = w_r[b][0] * xi;
                        im = fmaT(w_i[b][0], xr, im);
                        im = fmaT(w_r[b][1], zi, im);
                        im = fmaT(w_i[b][1], zr, im);
                        orr[c] = r;
                        oi[c] = im;
                        if (b) { ns1 = fmaT(r, r, ns1); ns1 = fmaT(im, im, ns1); }
                        else { ns0 = fmaT(r, r, ns0); ns0 = fmaT(im, im, ns0); }
                    }
                    if (out) sts_cls<P>(out + (size_t)gs.out_idx[j][tau] * NC + pc, orr, oi);
                }
            }
        }
    }
    n0 += (double)ns0;
    n1 += (double)ns1;
}

template <typename E, typename T, bool FIRST>
__device__ __forceinline__ void group_step_rows_any(const GroupArgs &ga, const GroupStepArgs &gs, E *__restrict__ mem,
                                                    const uint64_t TB, const int L, typename CplxOf<T>::type *in_buf,
                                                    typename CplxOf<T>::type *out0, typename CplxOf<T>::type *out1,
                                                    const T (&w_r)[2][2], const T (&w_i)[2][2], double &n0, double &n1) {
    constexpr int P = sizeof(E) == 8 ? 2 : 1;
    switch (gs.ntq) {
        case 1: group_step_rows<E, T, P, 1, FIRST>(ga, gs, mem, TB, L, in_buf, out0, out1, w_r, w_i, n0, n1); break;
        case 2: group_step_rows<E, T, P, 2, FIRST>(ga, gs, mem, TB, L, in_buf, out0, out1, w_r, w_i, n0, n1); break;
        default: group_step_rows<E, T, P, 4, FIRST>(ga, gs, mem, TB, L, in_buf, out0, out1, w_r, w_i, n0, n1); break;
    }
}

// Look-ahead norm pass of a pair of steps (k, k+1) for exact sampling ('sample' / 'prob', gsamp2.cpp:39-55): one
// read-only pass over the table before step k gives n(b) = |L_k(b) T|^2 and n(b, b') = |L_{k+1}(b') L_k(b) T|^2 for
// every b, b'.  The epilogue draws (or takes) b_k from n(.), then b_{k+1} from n(b_k, .) -- the conditionals of the
// two-pass chain, since the normalisation between the steps cancels in the ratio -- and leaves both bits and the
// pair's combined scale 1 / sqrt(n(b_k, b_{k+1})) for the fused write pass.
template <typename E, typename T>
__global__ void __launch_bounds__(256) k_group_norm2(const GroupArgs ga, E *__restrict__ mem, const Ctx cx) {
    typedef typename CplxOf<T>::type V;
    DevState *st = cx.st;
    if (*(volatile int *)&st->dead) return;
    extern __shared__ __align__(16) unsigned char smem[];
    const int L = ga.L;
    const uint64_t mask = ((uint64_t)1 << L) - 1;
    V *b0 = reinterpret_cast<V *>(smem);
    V *b1 = b0 + ((size_t)ga.ssz[1] << L);
    T w0r[2][2], w0i[2][2], w1r[2][2], w1i[2][2];
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
        for (int x = 0; x < 2; x++) {
            w0r[b][x] = (T)ga.st[0].Mr[b][x];
            w0i[b][x] = (T)ga.st[0].Mi[b][x];
            w1r[b][x] = (T)ga.st[1].Mr[b][x];
            w1i[b][x] = (T)ga.st[1].Mi[b][x];
        }
    double acc[6] = {0, 0, 0, 0, 0, 0};   // n(0), n(1), n(0,0), n(0,1), n(1,0), n(1,1)
    unsigned int i0, i1;
    block_range(cx.nchunks, i0, i1);
    uint64_t tb = 0;
    if (i0 < i1) {
        const uint32_t g = i0 ^ (i0 >> 1);
        for (int j = 0; j < ga.nbhi; j++)
            if ((g >> j) & 1) tb ^= ga.bhi[j];
    }
    for (unsigned int it = i0; it < i1; it++) {
        if (it > i0) tb ^= ga.bhi[__ffs((int)it) - 1];
        const uint64_t TB = tb & ~mask;
        group_step_rows_any<E, T, true>(ga, ga.st[0], mem, TB, L, nullptr, b0, b1, w0r, w0i, acc[0], acc[1]);
        __syncthreads();
        group_step_rows_any<E, T, false>(ga, ga.st[1], mem, TB, L, b0, nullptr, nullptr, w1r, w1i, acc[2], acc[3]);
        group_step_rows_any<E, T, false>(ga, ga.st[1], mem, TB, L, b1, nullptr, nullptr, w1r, w1i, acc[4], acc[5]);
        __syncthreads();
    }
    double n[6];
    if (!grid_reduceN<6>(acc, cx, n)) return;
    // scalar logic of the two steps (gsamp2.cpp:42-49 twice)
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    const int k = ga.st[0].k;
    const double p1 = n[1] / (n[0] + n[1]);
    const int bv0 = cx.forced ? cx.forced[row + k] : (cx.unif[row + k] < p1);
    const double pb0 = bv0 ? p1 : 1 - p1;
    if (pb0 <= 0) {
        st->dead = 1;
        st->logp = -INFINITY;
        for (int j = k; j < cx.ns; j++) cx.bits_out[row + j] = cx.forced ? cx.forced[row + j] : 0;
        return;
    }
    st->logp += log2(pb0);
    cx.bits_out[row + k] = (int8_t)bv0;
    const double q0 = n[2 + 2 * bv0], q1 = n[3 + 2 * bv0];
    const double p2 = q1 / (q0 + q1);
    const int bv1 = cx.forced ? cx.forced[row + k + 1] : (cx.unif[row + k + 1] < p2);
    const double pb1 = bv1 ? p2 : 1 - p2;
    if (pb1 <= 0) {
        st->dead = 1;
        st->logp = -INFINITY;
        for (int j = k + 1; j < cx.ns; j++) cx.bits_out[row + j] = cx.forced ? cx.forced[row + j] : 0;
        return;
    }
    st->logp += log2(pb1);
    cx.bits_out[row + k + 1] = (int8_t)bv1;
    st->gbv[0] = bv0;
    st->gbv[1] = bv1;
    st->sc = 1.0 / sqrt(bv1 ? q1 : q0);
}

template <typename E, typename T, int D>
__global__ void __launch_bounds__(256) k_group(const GroupArgs ga, E *__restrict__ mem, const Ctx cx) {
    typedef typename CplxOf<T>::type V;
    DevState *st = cx.st;
    if (*(volatile int *)&st->dead) return;
    const size_t row = (size_t)st->item * (size_t)cx.ns;
    extern __shared__ __align__(16) unsigned char smem[];
    const int L = ga.L;
    const uint64_t mask = ((uint64_t)1 << L) - 1;
    // intermediate stages 1 .. D-1 in shared memory, [value index][class]
    V *bufm[3] = {nullptr, nullptr, nullptr};
    {
        unsigned char *p = smem;
        for (int s = 1; s < D; s++) {
            bufm[s] = reinterpret_cast<V *>(p);
            p += ((size_t)ga.ssz[s] << L) * sizeof(V);
        }
    }
    // per-step M rows of the forced bits (the first step carries the run's scale)
    T wr[D][2], wi[D][2];
#pragma unroll
    for (int s = 0; s < D; s++) {
        // 'chain' takes the forced bits; the sampling driver takes the bits its look-ahead pass drew
        const int bv = cx.driver == DRV_CHAIN1 ? cx.forced[row + ga.st[s].k] : st->gbv[s];
        const double f = s == 0 ? st->sc : 1.0;
#pragma unroll
        for (int x = 0; x < 2; x++) {
            wr[s][x] = (T)(f * ga.st[s].Mr[bv][x]);
            wi[s][x] = (T)(f * ga.st[s].Mi[bv][x]);
        }
    }
    double acc[D];
#pragma unroll
    for (int s = 0; s < D; s++) acc[s] = 0;
    unsigned int i0, i1;
    block_range(cx.nchunks, i0, i1);
    uint64_t tb = 0;
    if (i0 < i1) {
        const uint32_t g = i0 ^ (i0 >> 1);
        for (int j = 0; j < ga.nbhi; j++)
            if ((g >> j) & 1) tb ^= ga.bhi[j];
    }
    for (unsigned int it = i0; it < i1; it++) {
        if (it > i0) tb ^= ga.bhi[__ffs((int)it) - 1];
        const uint64_t TB = tb & ~mask;
        if (D == 2) {
            group_step_any<E, T, true, false>(ga, ga.st[0], mem, TB, L, nullptr, bufm[1], wr[0], wi[0], acc[0]);
            __syncthreads();
            group_step_any<E, T, false, true>(ga, ga.st[1], mem, TB, L, bufm[1], nullptr, wr[1], wi[1], acc[1]);
            __syncthreads();
        } else {
            group_step_any<E, T, true, false>(ga, ga.st[0], mem, TB, L, nullptr, bufm[1], wr[0], wi[0], acc[0]);
            __syncthreads();
            group_step_any<E, T, false, false>(ga, ga.st[1], mem, TB, L, bufm[1], bufm[2], wr[1], wi[1], acc[1]);
            __syncthreads();
            group_step_any<E, T, false, true>(ga, ga.st[2], mem, TB, L, bufm[2], nullptr, wr[2], wi[2], acc[2]);
            __syncthreads();
        }
    }
    double tot[D];
    if (!grid_reduceN<D>(acc, cx, tot)) return;
    if (cx.driver == DRV_CHAIN1) group_chain1_epilogue<D>(cx, ga.st[0].k, tot);
    else st->prev = tot[D - 1];
}

}  // namespace gsb
