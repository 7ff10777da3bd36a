// Out-of-place cut-rank DP amplitude engine on the GPU: the reference's dp.cpp (dp.cpp:14-63) behind the C ABI.
//
//   Z(w) = sum_x prod_j w_j(x_j) (-1)^{sum_{i<j} A_ij x_i x_j}
//
// Plan (engine.py:5-12 writes it): "m nsteps maxr", then per step "v r rn rho pivmask nker ker...".  Each step is the
// gather  new[c'] = sum_{k in span(ker)} coef(u) old[u & (2^r - 1)],  u = pdep(c', pivmask) ^ k, with coef(u) = w_v(0)
// when bit r of u is clear and (-1)^{parity(c & rho)} w_v(1) when it is set (dp.cpp:47-56).  Two tables of 2^maxr
// entries (complex128, or complex64 storage with FP64 accumulation as the reference's -DDP_FLOAT build) alternate.
// A job is a list of slices (prefactor, weights of every vertex); the result is sum over slices of prefactor * Z.
// The per-slice step sequence is captured as a CUDA graph that reads the weights from device memory, so slices run
// back to back without host round trips; the slice results accumulate on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "gsb.h"
#include "gsb_common.h"

namespace gsb {

struct DpStep {
    int v, r, rn, nspan;
    uint64_t rho, pivmask;
    uint64_t span[4];        // the kernel span (nker <= 2 for a cut-rank plan; nspan <= 4)
    uint64_t pos[40];        // positions of the set bits of pivmask (pdep by table)
    int npos;
};

template <typename E>
__device__ __forceinline__ void dp_load(const E *p, double &re, double &im);
template <>
__device__ __forceinline__ void dp_load<double2>(const double2 *p, double &re, double &im) {
    const double2 v = *p;
    re = v.x;
    im = v.y;
}
template <>
__device__ __forceinline__ void dp_load<float2>(const float2 *p, double &re, double &im) {
    const float2 v = *p;
    re = v.x;
    im = v.y;
}
__device__ __forceinline__ void dp_store(double2 *p, double re, double im) { *p = make_double2(re, im); }
__device__ __forceinline__ void dp_store(float2 *p, double re, double im) { *p = make_float2((float)re, (float)im); }

// w: per vertex (w0re, w0im, w1re, w1im).  The grid is a power of two of threads, 2^ls: a thread takes the outputs
// c' = t | (g << ls) for the Gray codes g of the high bits, so pdep(c', pivmask) is its fixed low part XOR one
// running value (one XOR per output instead of a loop over the bits of c').
template <typename E>
__global__ void k_dp_step(const DpStep s, const E *__restrict__ old, E *__restrict__ nw, const double *__restrict__ w) {
    const uint64_t low = s.r >= 64 ? ~0ULL : ((1ULL << s.r) - 1), xbit = 1ULL << s.r;
    const double w0r = w[4 * s.v], w0i = w[4 * s.v + 1], w1r = w[4 * s.v + 2], w1i = w[4 * s.v + 3];
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const int ls = __ffsll((long long)nthreads) - 1;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s.rn < ls && t >= (1ULL << s.rn)) return;
    uint64_t lo = 0;
    for (int j = 0; j < s.npos && j < ls; j++)
        if ((t >> j) & 1) lo |= 1ULL << s.pos[j];
    const uint64_t nh = s.rn > ls ? 1ULL << (s.rn - ls) : 1;
    uint64_t hi = 0;
    for (uint64_t n = 0; n < nh; n++) {
        if (n) hi ^= 1ULL << s.pos[ls + __ffsll((long long)n) - 1];
        const uint64_t cp = t | ((n ^ (n >> 1)) << ls), u0 = lo ^ hi;
        double ar = 0, ai = 0;
        for (int q = 0; q < s.nspan; q++) {
            const uint64_t u = u0 ^ s.span[q], c = u & low;
            double vr, vi;
            dp_load(old + c, vr, vi);
            double cr, ci;
            if (u & xbit) {
                const bool neg = __popcll(c & s.rho) & 1;
                cr = neg ? -w1r : w1r;
                ci = neg ? -w1i : w1i;
            } else {
                cr = w0r;
                ci = w0i;
            }
            ar += cr * vr - ci * vi;
            ai += cr * vi + ci * vr;
        }
        dp_store(nw + cp, ar, ai);
    }
}

// A power of two of 256-thread blocks covering 2^rn outputs, at most `cap` blocks (k_dp_step's thread split).
static unsigned dp_grid(int rn, uint64_t cap) {
    const uint64_t want = std::max<uint64_t>(1, std::min<uint64_t>(((1ULL << rn) + 255) / 256, cap));
    uint64_t g = 1;
    while (g * 2 <= want) g *= 2;
    return (unsigned)g;
}

template <typename E>
__global__ void k_dp_begin(E *t) { dp_store(t, 1.0, 0.0); }

// acc += pre[slice] * t[0]; slice counter advances
template <typename E>
__global__ void k_dp_accumulate(const E *t, const double *pre, int *slice, double *acc) {
    const int s = *slice;
    double vr, vi;
    dp_load(t, vr, vi);
    const double pr = pre[2 * s], pi = pre[2 * s + 1];
    acc[0] += pr * vr - pi * vi;
    acc[1] += pr * vi + pi * vr;
    *slice = s + 1;
}

__global__ void k_dp_next_weights(double *w, const double *all, const int *slice, int m) {
    const int s = *slice;
    for (int i = threadIdx.x; i < 4 * m; i += blockDim.x) w[i] = all[(size_t)s * 4 * m + i];
}

struct DpEngine {
    int m = 0, ns = 0, maxr = 0, prec = 128, dev = 0, sms = 0;
    std::vector<DpStep> st;
    void *ta = nullptr, *tb = nullptr;
    double *d_w = nullptr, *d_wall = nullptr, *d_pre = nullptr, *d_acc = nullptr;
    int *d_slice = nullptr;
    size_t wall_cap = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    ~DpEngine() {
        if (graph) cudaGraphExecDestroy(graph);
        cudaFree(ta);
        cudaFree(tb);
        cudaFree(d_w);
        cudaFree(d_wall);
        cudaFree(d_pre);
        cudaFree(d_acc);
        cudaFree(d_slice);
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace gsb

using namespace gsb;

static int dp_fail(int code, const std::string &m) { return gsb::fail(code, m); }
#define DP_CK(x)                                                                                              \
    do {                                                                                                      \
        cudaError_t e_ = (x);                                                                                 \
        if (e_ != cudaSuccess) return dp_fail(GSB_E_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_)); \
    } while (0)

template <typename E>
static cudaError_t dp_enqueue_slice(DpEngine *D) {
    k_dp_next_weights<<<1, 256, 0, D->stream>>>(D->d_w, D->d_wall, D->d_slice, D->m);
    k_dp_begin<E><<<1, 1, 0, D->stream>>>((E *)D->ta);
    E *a = (E *)D->ta, *b = (E *)D->tb;
    for (const DpStep &s : D->st) {
        k_dp_step<E><<<dp_grid(s.rn, (uint64_t)D->sms * 8), 256, 0, D->stream>>>(s, a, b, D->d_w);
        std::swap(a, b);
    }
    k_dp_accumulate<E><<<1, 1, 0, D->stream>>>(a, D->d_pre, D->d_slice, D->d_acc);
    return cudaGetLastError();
}

extern "C" {

int gsb_dp_open_text(const char *text, size_t len, int precision, int device, gsb_dp **out) {
    if (!text || !out) return dp_fail(GSB_E_USAGE, "null argument");
    if (precision != 64 && precision != 128) return dp_fail(GSB_E_USAGE, "precision must be 64 or 128");
    *out = nullptr;
    std::string s(text, len);
    const char *p = s.c_str();
    int off = 0, m, ns, maxr;
    if (sscanf(p, "%d %d %d%n", &m, &ns, &maxr, &off) != 3 || m < 0 || ns < 0 || maxr < 0 || maxr > 40)
        return dp_fail(2, "dp plan header 'm nsteps maxr' unreadable");
    p += off;
    DpEngine *D = new DpEngine();
    D->m = m;
    D->ns = ns;
    D->maxr = maxr;
    D->prec = precision;
    D->dev = device;
    for (int k = 0; k < ns; k++) {
        DpStep st;
        memset(&st, 0, sizeof st);
        unsigned long long rho, pm;
        int nk;
        if (sscanf(p, "%d %d %d %llu %llu %d%n", &st.v, &st.r, &st.rn, &rho, &pm, &nk, &off) != 6) { delete D; return dp_fail(3, "dp plan step unreadable"); }
        p += off;
        if (st.r > 40 || st.rn > 40 || st.r > maxr || st.rn > maxr || nk < 0 || nk > 2 || st.v < 0 || st.v >= m) {
            delete D;
            return dp_fail(7, "dp plan step out of range");
        }
        st.rho = rho;
        st.pivmask = pm;
        st.span[0] = 0;
        st.nspan = 1;
        for (int i = 0; i < nk; i++) {
            unsigned long long kv;
            if (sscanf(p, "%llu%n", &kv, &off) != 1) { delete D; return dp_fail(4, "dp plan kernel vector unreadable"); }
            p += off;
            for (int t = 0; t < st.nspan; t++) st.span[st.nspan + t] = st.span[t] ^ kv;
            st.nspan *= 2;
        }
        st.npos = 0;
        for (int b = 0; b < 64; b++)
            if ((pm >> b) & 1) {
                if (st.npos >= 40 || b > st.r) { delete D; return dp_fail(7, "dp plan pivot mask out of range"); }
                st.pos[st.npos++] = (uint64_t)b;
            }
        if (st.npos != st.rn) { delete D; return dp_fail(7, "dp plan pivot mask does not have rn bits"); }
        for (int t = 0; t < st.nspan; t++)
            if (st.span[t] >> (st.r + 1)) { delete D; return dp_fail(7, "dp plan kernel vector out of range"); }
        D->st.push_back(st);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) { delete D; return dp_fail(GSB_E_CUDA, "no such CUDA device"); }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    D->sms = prop.multiProcessorCount;
    const size_t es = precision == 128 ? 16 : 8, bytes = ((size_t)1 << maxr) * es;
    cudaError_t e = cudaStreamCreateWithFlags(&D->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&D->ta, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&D->tb, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&D->d_w, (size_t)std::max(1, m) * 4 * 8);
    if (e == cudaSuccess) e = cudaMalloc(&D->d_acc, 16);
    if (e == cudaSuccess) e = cudaMalloc(&D->d_slice, sizeof(int));
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete D;
        return dp_fail(GSB_E_ALLOC, "dp table allocation failed");
    }
    *out = reinterpret_cast<gsb_dp *>(D);
    return 0;
}

int gsb_dp_close(gsb_dp *d) {
    if (!d) return dp_fail(GSB_E_STATE, "null dp engine");
    DpEngine *D = reinterpret_cast<DpEngine *>(d);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(D->dev);
    delete D;
    cudaSetDevice(prev);
    return 0;
}

int gsb_dp_info(const gsb_dp *d, int *m, int *nsteps, int *maxr) {
    if (!d) return dp_fail(GSB_E_STATE, "null dp engine");
    const DpEngine *D = reinterpret_cast<const DpEngine *>(d);
    if (m) *m = D->m;
    if (nsteps) *nsteps = D->ns;
    if (maxr) *maxr = D->maxr;
    return 0;
}

int gsb_dp_run(gsb_dp *d, int64_t nslices, const double *pre, const double *w, double *out) {
    if (!d) return dp_fail(GSB_E_STATE, "null dp engine");
    if (nslices < 0 || (nslices && (!pre || !w)) || !out) return dp_fail(GSB_E_USAGE, "bad argument");
    DpEngine *D = reinterpret_cast<DpEngine *>(d);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(D->dev);
    struct Restore {
        int p;
        ~Restore() { cudaSetDevice(p); }
    } restore{prev};
    const size_t wbytes = (size_t)nslices * (size_t)std::max(1, D->m) * 4 * 8;
    if (wbytes > D->wall_cap) {
        cudaFree(D->d_wall);
        cudaFree(D->d_pre);
        D->d_wall = nullptr;
        D->d_pre = nullptr;
        DP_CK(cudaMalloc(&D->d_wall, wbytes));
        DP_CK(cudaMalloc(&D->d_pre, (size_t)nslices * 16));
        D->wall_cap = wbytes;
        if (D->graph) { cudaGraphExecDestroy(D->graph); D->graph = nullptr; }
    }
    if (!D->graph) {
        cudaGraph_t g = nullptr;
        DP_CK(cudaStreamBeginCapture(D->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = D->prec == 128 ? dp_enqueue_slice<double2>(D) : dp_enqueue_slice<float2>(D);
        cudaError_t e2 = cudaStreamEndCapture(D->stream, &g);
        if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); DP_CK(e); }
        DP_CK(e2);
        e = cudaGraphInstantiate(&D->graph, g, 0);
        cudaGraphDestroy(g);
        DP_CK(e);
    }
    const double zero[2] = {0, 0};
    const int zi = 0;
    if (nslices) {
        DP_CK(cudaMemcpyAsync(D->d_wall, w, wbytes, cudaMemcpyHostToDevice, D->stream));
        DP_CK(cudaMemcpyAsync(D->d_pre, pre, (size_t)nslices * 16, cudaMemcpyHostToDevice, D->stream));
    }
    DP_CK(cudaMemcpyAsync(D->d_acc, zero, 16, cudaMemcpyHostToDevice, D->stream));
    DP_CK(cudaMemcpyAsync(D->d_slice, &zi, sizeof zi, cudaMemcpyHostToDevice, D->stream));
    for (int64_t s = 0; s < nslices; s++) DP_CK(cudaGraphLaunch(D->graph, D->stream));
    DP_CK(cudaMemcpyAsync(out, D->d_acc, 16, cudaMemcpyDeviceToHost, D->stream));
    DP_CK(cudaStreamSynchronize(D->stream));
    return 0;
}

}  // extern "C"

// Step descriptor of gsb_dp_extend / gsb_dp_extend_static from the caller's arguments (arguments already checked).
static int extend_step(int r, int rn, uint64_t rho, uint64_t pivmask, int nker, const uint64_t *ker, DpStep &st) {
    memset(&st, 0, sizeof st);
    st.v = 0;
    st.r = r;
    st.rn = rn;
    st.rho = rho;
    st.pivmask = pivmask;
    st.span[0] = 0;
    st.nspan = 1;
    for (int i = 0; i < nker; i++) {
        for (int t = 0; t < st.nspan; t++) st.span[st.nspan + t] = st.span[t] ^ ker[i];
        st.nspan *= 2;
    }
    for (int b = 0; b < 64; b++)
        if ((pivmask >> b) & 1) {
            if (st.npos >= 40 || b > r) return dp_fail(GSB_E_USAGE, "pivot mask out of range");
            st.pos[st.npos++] = (uint64_t)b;
        }
    if (st.npos != rn) return dp_fail(GSB_E_USAGE, "pivot mask must have rn bits");
    return 0;
}

// Scratch of gsb_dp_extend_static, in the library's static device memory (every GPU that loads the library holds it
// until the process exits): the old table, the new table (2^EXTEND_STATIC_LOG2 complex128 entries each) and the
// weights.  Calls share it; each call overwrites what it uses (the kernel writes every entry of the new table, so
// nothing has to start at zero).
constexpr int EXTEND_STATIC_LOG2 = 16;
constexpr size_t EXTEND_STATIC_N = (size_t)1 << EXTEND_STATIC_LOG2;
static __device__ __align__(256) double2 g_extend_scratch[2 * EXTEND_STATIC_N + 2];   // 2 MiB + 32 B

// Device address of the scratch on `device` (current), looked up once per device and kept.
static int extend_scratch(int device, double2 **out) {
    static std::mutex mu;
    static std::vector<double2 *> addr;
    std::lock_guard<std::mutex> lock(mu);
    if ((size_t)device >= addr.size()) addr.resize((size_t)device + 1, nullptr);
    if (!addr[(size_t)device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_extend_scratch);
        if (e != cudaSuccess) return dp_fail(GSB_E_CUDA, std::string("static scratch lookup: ") + cudaGetErrorString(e));
        addr[(size_t)device] = static_cast<double2 *>(p);
    }
    *out = addr[(size_t)device];
    return 0;
}

extern "C" {

// One out-of-place step on a caller table (complex128, host memory): the reference's sampler_ref.extend
// (sampler_ref.py:8-23) and ref.run's inner step (ref.py:18-31).
int gsb_dp_extend(int r, int rn, uint64_t rho, uint64_t pivmask, int nker, const uint64_t *ker, const double *wv,
                  const double *old, double *out, int device) {
    if (r < 0 || rn < 0 || r > 30 || rn > 30 || nker < 0 || nker > 2 || (nker && !ker) || !wv || !old || !out)
        return dp_fail(GSB_E_USAGE, "bad argument");
    DpStep st;
    if (int rc = extend_step(r, rn, rho, pivmask, nker, ker, st)) return rc;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    struct Restore {
        int p;
        ~Restore() { cudaSetDevice(p); }
    } restore{prev};
    struct Buffers {   // freed on every return path (cudaFree of a null pointer does nothing)
        double2 *a = nullptr, *b = nullptr;
        double *w = nullptr;
        ~Buffers() {
            cudaFree(a);
            cudaFree(b);
            cudaFree(w);
        }
    } m;
    const size_t na = (size_t)1 << r, nb = (size_t)1 << rn;
    DP_CK(cudaMalloc(&m.a, na * 16));
    DP_CK(cudaMalloc(&m.b, nb * 16));
    DP_CK(cudaMalloc(&m.w, 32));
    DP_CK(cudaMemcpy(m.a, old, na * 16, cudaMemcpyHostToDevice));
    DP_CK(cudaMemcpy(m.w, wv, 32, cudaMemcpyHostToDevice));
    k_dp_step<double2><<<dp_grid(rn, 4096), 256>>>(st, m.a, m.b, m.w);
    DP_CK(cudaGetLastError());
    DP_CK(cudaMemcpy(out, m.b, nb * 16, cudaMemcpyDeviceToHost));
    return 0;
}

// gsb_dp_extend without any device allocation: the tables and weights go through the static scratch above, so
// r and rn are limited to EXTEND_STATIC_LOG2.  The first call on a device looks up the scratch's address.
int gsb_dp_extend_static(int r, int rn, uint64_t rho, uint64_t pivmask, int nker, const uint64_t *ker,
                         const double *wv, const double *old, double *out, int device) {
    if (r < 0 || rn < 0 || nker < 0 || nker > 2 || (nker && !ker) || !wv || !old || !out)
        return dp_fail(GSB_E_USAGE, "bad argument");
    if (r > EXTEND_STATIC_LOG2 || rn > EXTEND_STATIC_LOG2)
        return dp_fail(GSB_E_USAGE, "table too large for the static scratch: r and rn must be at most " +
                                        std::to_string(EXTEND_STATIC_LOG2));
    DpStep st;
    if (int rc = extend_step(r, rn, rho, pivmask, nker, ker, st)) return rc;
    int prev = 0;
    cudaGetDevice(&prev);
    DP_CK(cudaSetDevice(device));
    struct Restore {
        int p;
        ~Restore() { cudaSetDevice(p); }
    } restore{prev};
    double2 *scratch = nullptr;
    if (int rc = extend_scratch(device, &scratch)) return rc;
    double2 *a = scratch, *b = scratch + EXTEND_STATIC_N;
    double *w = reinterpret_cast<double *>(scratch + 2 * EXTEND_STATIC_N);
    const size_t na = (size_t)1 << r, nb = (size_t)1 << rn;
    DP_CK(cudaMemcpy(a, old, na * 16, cudaMemcpyHostToDevice));
    DP_CK(cudaMemcpy(w, wv, 32, cudaMemcpyHostToDevice));
    k_dp_step<double2><<<dp_grid(rn, 4096), 256>>>(st, a, b, w);
    DP_CK(cudaGetLastError());
    DP_CK(cudaMemcpy(out, b, nb * 16, cudaMemcpyDeviceToHost));
    return 0;
}

}  // extern "C"
