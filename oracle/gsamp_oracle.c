/*
 * CPU oracle for the in-place cut-rank DP executor.  TEST INFRASTRUCTURE ONLY: this file is the checker that the
 * CUDA path is compared against (tests, smoke check, the CPU-baseline leg of the benchmark).  Nothing in the
 * product links it.
 *
 * It restates, in plain C99 with OpenMP, the executor of the reference's gsamp2.cpp:
 *   plan text format           gsamp2.cpp:2, parse gsamp2.cpp:128-139
 *   base_of (5 byte tables)    gsamp2.cpp:29-31
 *   outputs (coset gather)     gsamp2.cpp:32-38
 *   chain  (norm + write)      gsamp2.cpp:39-55   (modes 'sample', 'sample2', 'prob')
 *   chain1 (one pass/step)     gsamp2.cpp:56-70   (mode 'chain')
 *   run_steps / hybrid         gsamp2.cpp:71-120  (modes 'hybrid', 'prefix', 'resume')
 *   coset_offsets              gsamp2.cpp:121-125
 *   prefix dump / resume sum   gsamp2.cpp:162-208 (including the twist translation)
 * and the random streams those modes draw from:
 *   std::mt19937_64 (Matsumoto-Nishimura MT19937-64, as specified for the C++ standard library),
 *   std::uniform_real_distribution<double>(0,1) over it as libstdc++ implements it (generate_canonical with one
 *   64-bit draw: U = double(x) / 2^64, clamped below 1), and std::seed_seq::generate as the C++ standard specifies
 *   it (used by 'sample2', gsamp2.cpp:153-161).
 * The arena element is complex64 (prec 64) or complex128 (prec 128, the reference's -DGS_DOUBLE build); all
 * arithmetic is in double, as in the reference.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define ORC_MAXT 16

typedef struct { uint64_t tq; int x, tau, par; } orc_term;
typedef struct {
    int v, nk, m, nt;
    uint64_t g, rhoc;
    uint64_t *tk;
    orc_term t[ORC_MAXT];
    double Mr[2][2], Mi[2][2];        /* M[b][x] */
    uint64_t tab[5][256];
} orc_step;

typedef struct {
    int n, ns, R, prec;
    orc_step *st;
    void *mem;                        /* 2^R entries of float[2] or double[2] */
} orc_plan;

static char orc_err[256];
const char *orc_last_error(void) { return orc_err; }

/* ------------------------------------------------------------------ random streams */
typedef struct { uint64_t mt[312]; int mti; } orc_mt64;

static void mt64_seed(orc_mt64 *r, uint64_t s) {
    r->mt[0] = s;
    for (int i = 1; i < 312; i++) r->mt[i] = 6364136223846793005ULL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 62)) + (uint64_t)i;
    r->mti = 312;
}

static uint64_t mt64_next(orc_mt64 *r) {
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL, A = 0xB5026F5AA96619E9ULL;
    if (r->mti >= 312) {
        for (int i = 0; i < 312; i++) {
            uint64_t y = (r->mt[i] & UM) | (r->mt[(i + 1) % 312] & LM);
            r->mt[i] = r->mt[(i + 156) % 312] ^ (y >> 1) ^ ((y & 1) ? A : 0);
        }
        r->mti = 0;
    }
    uint64_t x = r->mt[r->mti++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

static double mt64_uniform(orc_mt64 *r) {
    double u = (double)mt64_next(r) / 18446744073709551616.0;
    if (u >= 1.0) u = nextafter(1.0, 0.0);
    return u;
}

/* std::seed_seq{v[0..s-1]}.generate(out, out + n) as the C++ standard specifies it, all arithmetic mod 2^32 */
static void seed_seq_generate(const uint32_t *v, int s, uint32_t *out, int n) {
    for (int i = 0; i < n; i++) out[i] = 0x8b8b8b8bu;
    int t = n >= 623 ? 11 : n >= 68 ? 7 : n >= 39 ? 5 : n >= 7 ? 3 : (n - 1) / 2;
    int p = (n - t) / 2, q = p + t, m = (s + 1 > n) ? s + 1 : n;
#define SST(x) ((x) ^ ((x) >> 27))
    for (int k = 0; k < m; k++) {
        uint32_t a = out[k % n] ^ out[(k + p) % n] ^ out[(k + n - 1) % n];
        uint32_t r1 = 1664525u * SST(a);
        uint32_t r2 = r1 + (k == 0 ? (uint32_t)s : (k <= s ? (uint32_t)(k % n) + v[k - 1] : (uint32_t)(k % n)));
        out[(k + p) % n] += r1;
        out[(k + q) % n] += r2;
        out[k % n] = r2;
    }
    for (int k = m; k < m + n; k++) {
        uint32_t a = out[k % n] + out[(k + p) % n] + out[(k + n - 1) % n];
        uint32_t r3 = 1566083941u * SST(a);
        uint32_t r4 = r3 - (uint32_t)(k % n);
        out[(k + p) % n] ^= r3;
        out[(k + q) % n] ^= r4;
        out[k % n] = r4;
    }
#undef SST
}

/* std::mt19937_64 constructed from a seed_seq: 624 32-bit words, two per 64-bit state word (low word first) */
static void mt64_seed_seq(orc_mt64 *r, const uint32_t *v, int s) {
    uint32_t a[624];
    seed_seq_generate(v, s, a, 624);
    for (int i = 0; i < 312; i++) r->mt[i] = (uint64_t)a[2 * i] | ((uint64_t)a[2 * i + 1] << 32);
    int zero = (r->mt[0] & 0xFFFFFFFF80000000ULL) == 0;
    for (int i = 1; i < 312 && zero; i++) zero = r->mt[i] == 0;
    if (zero) r->mt[0] = 1ULL << 63;
    r->mti = 312;
}

/* 'sample' seeds sample i with the integer seed+i; 'sample2' with seed_seq{seed_lo, seed_hi, i_lo, i_hi, 0x9E3779B9} */
static void orc_rng_for(orc_mt64 *r, int mode, uint64_t seed, uint64_t i) {
    if (mode == 0) { mt64_seed(r, seed + i); return; }
    uint32_t v[5] = {(uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32), (uint32_t)(i & 0xffffffffu), (uint32_t)(i >> 32),
                     0x9E3779B9u};
    mt64_seed_seq(r, v, 5);
}

/* First `count` uniforms of the stream a given mode/seed/index uses (for tests of the stream itself). */
void orc_uniforms(int mode, uint64_t seed, uint64_t i, int count, double *out) {
    orc_mt64 r;
    orc_rng_for(&r, mode, seed, i);
    for (int k = 0; k < count; k++) out[k] = mt64_uniform(&r);
}

/* ------------------------------------------------------------------ plan */
void orc_free(orc_plan *p) {
    if (!p) return;
    if (p->st) for (int k = 0; k < p->ns; k++) free(p->st[k].tk);
    free(p->st);
    free(p->mem);
    free(p);
}

orc_plan *orc_load(const char *path, int prec) {
    orc_plan *p = (orc_plan *)calloc(1, sizeof *p);
    FILE *f = fopen(path, "r");
    if (!f) { snprintf(orc_err, sizeof orc_err, "cannot open %s", path); free(p); return NULL; }
    p->prec = prec;
    if (fscanf(f, "%d %d %d", &p->n, &p->ns, &p->R) != 3) { snprintf(orc_err, sizeof orc_err, "bad header"); goto fail; }
    p->st = (orc_step *)calloc((size_t)p->ns, sizeof(orc_step));
    for (int k = 0; k < p->ns; k++) {
        orc_step *s = &p->st[k];
        unsigned long long g, rc;
        if (fscanf(f, "%d %d %d %llu %llu %d", &s->v, &s->nk, &s->m, &g, &rc, &s->nt) != 6) { snprintf(orc_err, sizeof orc_err, "bad step %d", k); goto fail; }
        s->g = g; s->rhoc = rc;
        if (s->nk > 40 || s->nt > ORC_MAXT || s->nk < 0 || s->nt < 1) { snprintf(orc_err, sizeof orc_err, "step %d out of range", k); goto fail; }
        s->tk = (uint64_t *)calloc((size_t)(s->nk + 1), 8);
        for (int j = 0; j < s->nk; j++) { unsigned long long y; if (fscanf(f, "%llu", &y) != 1) { snprintf(orc_err, sizeof orc_err, "bad Tkeep %d", k); goto fail; } s->tk[j] = y; }
        for (int i = 0; i < s->nt; i++) {
            unsigned long long y;
            if (fscanf(f, "%llu %d %d %d", &y, &s->t[i].x, &s->t[i].tau, &s->t[i].par) != 4) { snprintf(orc_err, sizeof orc_err, "bad term %d", k); goto fail; }
            s->t[i].tq = y;
        }
        for (int b = 0; b < 2; b++)
            for (int x = 0; x < 2; x++)
                if (fscanf(f, "%lf %lf", &s->Mr[b][x], &s->Mi[b][x]) != 2) { snprintf(orc_err, sizeof orc_err, "bad M %d", k); goto fail; }
        for (int t = 0; t < 5; t++)
            for (int v = 0; v < 256; v++) {
                uint64_t a = 0;
                for (int j = 0; j < 8; j++) if (((v >> j) & 1) && 8 * t + j < s->nk) a ^= s->tk[8 * t + j];
                s->tab[t][v] = a;
            }
    }
    fclose(f);
    f = NULL;
    {
        size_t es = prec == 128 ? 16 : 8;
        p->mem = calloc((size_t)1 << p->R, es);
        if (!p->mem) { snprintf(orc_err, sizeof orc_err, "arena allocation failed"); goto fail; }
    }
    return p;
fail:
    if (f) fclose(f);
    orc_free(p);
    return NULL;
}

int orc_n(const orc_plan *p) { return p->n; }
int orc_ns(const orc_plan *p) { return p->ns; }
int orc_R(const orc_plan *p) { return p->R; }

static inline uint64_t base_of(const orc_step *s, uint64_t c) {
    return s->tab[0][c & 255] ^ s->tab[1][(c >> 8) & 255] ^ s->tab[2][(c >> 16) & 255] ^ s->tab[3][(c >> 24) & 255] ^
           s->tab[4][(c >> 32) & 255];
}

/* element access: the arena is float[2] (prec 64) or double[2] (prec 128) */
static inline void ld(const orc_plan *p, uint64_t a, double *re, double *im) {
    if (p->prec == 128) { const double *m = (const double *)p->mem; *re = m[2 * a]; *im = m[2 * a + 1]; }
    else { const float *m = (const float *)p->mem; *re = m[2 * a]; *im = m[2 * a + 1]; }
}
static inline void st(const orc_plan *p, uint64_t a, double re, double im) {
    if (p->prec == 128) { double *m = (double *)p->mem; m[2 * a] = re; m[2 * a + 1] = im; }
    else { float *m = (float *)p->mem; m[2 * a] = (float)re; m[2 * a + 1] = (float)im; }
}

/* out[b][tau] = sum over terms of M[b][x] * (+-) mem[base ^ tq]  (gsamp2.cpp:32-38) */
static inline void outputs(const orc_plan *p, const orc_step *s, uint64_t c, uint64_t base, double orr[2][2], double oi[2][2]) {
    orr[0][0] = orr[0][1] = orr[1][0] = orr[1][1] = 0;
    oi[0][0] = oi[0][1] = oi[1][0] = oi[1][1] = 0;
    const int pc = __builtin_parityll(c & s->rhoc);
    for (int i = 0; i < s->nt; i++) {
        const orc_term *t = &s->t[i];
        double vr, vi;
        ld(p, base ^ t->tq, &vr, &vi);
        if (t->x && (pc ^ t->par)) { vr = -vr; vi = -vi; }
        for (int b = 0; b < 2; b++) {
            double mr = s->Mr[b][t->x], mi = s->Mi[b][t->x];
            orr[b][t->tau] += mr * vr - mi * vi;
            oi[b][t->tau] += mr * vi + mi * vr;
        }
    }
}

static void norms(orc_plan *p, int k, double *n0o, double *n1o) {
    const orc_step *s = &p->st[k];
    const int64_t N = (int64_t)1 << s->nk;
    double n0 = 0, n1 = 0;
#pragma omp parallel for schedule(static) reduction(+ : n0, n1)
    for (int64_t c = 0; c < N; c++) {
        double orr[2][2], oi[2][2];
        uint64_t b = base_of(s, (uint64_t)c);
        outputs(p, s, (uint64_t)c, b, orr, oi);
        n0 += orr[0][0] * orr[0][0] + oi[0][0] * oi[0][0] + orr[0][1] * orr[0][1] + oi[0][1] * oi[0][1];
        n1 += orr[1][0] * orr[1][0] + oi[1][0] * oi[1][0] + orr[1][1] * orr[1][1] + oi[1][1] * oi[1][1];
    }
    *n0o = n0; *n1o = n1;
}

/* write branch bv scaled by sc into the coset's own slots; returns the norm of what was written */
static double write_pass(orc_plan *p, int k, int bv, double sc) {
    const orc_step *s = &p->st[k];
    const int64_t N = (int64_t)1 << s->nk;
    double nb = 0;
#pragma omp parallel for schedule(static) reduction(+ : nb)
    for (int64_t c = 0; c < N; c++) {
        double orr[2][2], oi[2][2];
        uint64_t b = base_of(s, (uint64_t)c);
        outputs(p, s, (uint64_t)c, b, orr, oi);
        double v0r = orr[bv][0] * sc, v0i = oi[bv][0] * sc, v1r = orr[bv][1] * sc, v1i = oi[bv][1] * sc;
        st(p, b, v0r, v0i);
        if (s->m == 2) st(p, b ^ s->g, v1r, v1i);
        nb += v0r * v0r + v0i * v0i + v1r * v1r + v1i * v1i;
    }
    return nb;
}

static void set_one(orc_plan *p) { st(p, 0, 1.0, 0.0); }

/* chain: normalised, two passes per step; forced == NULL draws from rng (gsamp2.cpp:39-55) */
static double chain(orc_plan *p, const int *forced, int *bits, orc_mt64 *rng) {
    set_one(p);
    double logp = 0;
    for (int k = 0; k < p->ns; k++) {
        double n0, n1;
        norms(p, k, &n0, &n1);
        double p1 = n1 / (n0 + n1);
        int bv = forced ? forced[k] : (mt64_uniform(rng) < p1);
        double pb = bv ? p1 : 1 - p1;
        if (pb <= 0) { for (; k < p->ns; k++) bits[k] = forced ? forced[k] : 0; return -INFINITY; }
        logp += log2(pb);
        bits[k] = bv;
        write_pass(p, k, bv, 1.0 / sqrt(bv ? n1 : n0));
    }
    return logp;
}

/* 'prob' mode on one string (step order) */
double orc_prob(orc_plan *p, const int *forced) {
    int *bits = (int *)malloc(sizeof(int) * (size_t)p->ns);
    double lp = chain(p, forced, bits, NULL);
    free(bits);
    return lp;
}

/* 'sample'/'sample2' mode: bits[ns] and log2 Pr of sample i of stream (mode, seed) */
double orc_sample(orc_plan *p, int mode, uint64_t seed, uint64_t i, int *bits) {
    orc_mt64 r;
    orc_rng_for(&r, mode, seed, i);
    return chain(p, NULL, bits, &r);
}

/* chain1: one pass per step, unnormalised storage; cond[k] = nb / (2 prev) (gsamp2.cpp:56-70) */
double orc_chain1(orc_plan *p, const int *forced, double *cond) {
    set_one(p);
    double prev = 1;
    for (int k = 0; k < p->ns; k++) {
        double nb = write_pass(p, k, forced[k], 1.0);
        cond[k] = nb / (2 * prev);
        prev = nb;
        if (nb <= 0) { for (; k < p->ns; k++) cond[k] = 0; return -INFINITY; }
    }
    return log2(prev) - p->ns;
}

/* run_steps: hybrid loop with lazy rescaling by 1/sqrt(prev) (gsamp2.cpp:71-98) */
static double run_steps(orc_plan *p, int k0, int k1, const int *forced, int *bits, double *cond, orc_mt64 *rng, double *prev,
                        double *logscale) {
    double logp = 0;
    for (int k = k0; k < k1; k++) {
        int bv = forced[k];
        const double sc = 1.0 / sqrt(*prev);
        if (bv < 0) {
            double n0, n1;
            norms(p, k, &n0, &n1);
            bv = mt64_uniform(rng) < n1 / (n0 + n1);
        }
        double nb = write_pass(p, k, bv, sc);
        *logscale += 0.5 * log2(*prev);
        cond[k] = nb / 2;
        bits[k] = bv;
        *prev = nb;
        if (nb <= 0) {
            for (; k < k1; k++) { cond[k] = 0; bits[k] = forced[k] < 0 ? 0 : forced[k]; }
            return -INFINITY;
        }
        logp += log2(cond[k]);
    }
    return logp;
}

/* 'hybrid' mode on one line: forced[k] in {0,1,-1}; line index li seeds mt19937_64(seed + li) (gsamp2.cpp:209-216) */
double orc_hybrid(orc_plan *p, const int *forced, uint64_t seed, uint64_t li, int *bits, double *cond) {
    orc_mt64 r;
    mt64_seed(&r, seed + li);
    set_one(p);
    double prev = 1, logscale = 0;
    return run_steps(p, 0, p->ns, forced, bits, cond, &r, &prev, &logscale);
}

/* distinct coset offsets of step K, sorted; {0} past the end (gsamp2.cpp:121-125); returns their count */
static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}
int orc_coset_offsets(const orc_plan *p, int K, uint64_t *out) {
    if (K >= p->ns) { out[0] = 0; return 1; }
    const orc_step *s = &p->st[K];
    uint64_t v[ORC_MAXT];
    for (int i = 0; i < s->nt; i++) v[i] = s->t[i].tq;
    qsort(v, (size_t)s->nt, 8, cmp_u64);
    int n = 0;
    for (int i = 0; i < s->nt; i++) if (n == 0 || v[i] != out[n - 1]) out[n++] = v[i];
    return n;
}
int orc_dump_nk(const orc_plan *p, int K) { return K < p->ns ? p->st[K].nk : 0; }

/* 'prefix' on one line: forced steps 0..K-1, then the live table at logical index (c, tq) in c-major order, each
 * entry as two doubles (the reference writes its arena type; callers convert). Returns log2 Pr(prefix) and sets
 * *logscale (gsamp2.cpp:162-175). */
double orc_prefix(orc_plan *p, const int *forced, int K, double *dump, double *logscale) {
    int *bits = (int *)calloc((size_t)p->ns + 1, sizeof(int));
    double *cond = (double *)calloc((size_t)p->ns + 1, sizeof(double));
    set_one(p);
    double prev = 1;
    *logscale = 0;
    double lp = run_steps(p, 0, K, forced, bits, cond, NULL, &prev, logscale);
    uint64_t tqs[ORC_MAXT];
    int ntq = orc_coset_offsets(p, K, tqs), nk = orc_dump_nk(p, K);
    for (int64_t c = 0; c < ((int64_t)1 << nk); c++)
        for (int j = 0; j < ntq; j++) {
            uint64_t a = K < p->ns ? (base_of(&p->st[K], (uint64_t)c) ^ tqs[j]) : 0;
            ld(p, a, &dump[2 * (c * ntq + j)], &dump[2 * (c * ntq + j) + 1]);
        }
    free(bits);
    free(cond);
    return lp;
}

/* 'resume' on one line: sum the nsl dumped tables (each scaled by 2^(ls[s]-L), read through the twist translation
 * (cshift, tqshift) when given), continue steps K..ns-1 with '?' drawn from mt19937_64(seed + li).
 * Returns 0 or a reference exit code (14 for a bad twist) (gsamp2.cpp:176-208). */
int orc_resume(orc_plan *p, const int *forced, int K, uint64_t seed, uint64_t li, int nsl, const double *const *tabs, const double *ls,
               const uint64_t *cshift, const uint64_t *tqshift, int *bits, double *cond, double *lp_full, double *lp_prefix) {
    uint64_t tqs[ORC_MAXT];
    int ntq = orc_coset_offsets(p, K, tqs), nk = orc_dump_nk(p, K);
    int tperm[64][ORC_MAXT];
    if (nsl > 64) return 13;
    for (int s = 0; s < nsl; s++)
        for (int t = 0; t < ntq; t++) {
            tperm[s][t] = t;
            if (cshift || tqshift) {
                if (cshift && (cshift[s] >> nk)) return 14;
                uint64_t want = tqs[t] ^ (tqshift ? tqshift[s] : 0);
                int pos = -1;
                for (int u = 0; u < ntq; u++) if (tqs[u] == want) pos = u;
                if (pos < 0) return 14;
                tperm[s][t] = pos;
            }
        }
    double L = -1e300;
    for (int s = 0; s < nsl; s++) if (ls[s] > L) L = ls[s];
    double norm = 0;
    for (int64_t c = 0; c < ((int64_t)1 << nk); c++)
        for (int ti = 0; ti < ntq; ti++) {
            double ar = 0, ai = 0;
            for (int s = 0; s < nsl; s++) {
                int64_t idx = (int64_t)((uint64_t)c ^ (cshift ? cshift[s] : 0)) * ntq + tperm[s][ti];
                double f = exp2(ls[s] - L);
                ar += tabs[s][2 * idx] * f;
                ai += tabs[s][2 * idx + 1] * f;
            }
            /* the reference rounds the summed entry to its arena type before storing and measures the unrounded norm */
            st(p, K < p->ns ? (base_of(&p->st[K], (uint64_t)c) ^ tqs[ti]) : 0, ar, ai);
            norm += ar * ar + ai * ai;
        }
    *lp_prefix = -K + log2(norm) + 2 * L;
    double prev = norm, logscale = L;
    orc_mt64 r;
    mt64_seed(&r, seed + li);
    for (int k = 0; k < K; k++) bits[k] = forced[k];
    double lps = run_steps(p, K, p->ns, forced, bits, cond, &r, &prev, &logscale);
    *lp_full = *lp_prefix + lps;
    return 0;
}
