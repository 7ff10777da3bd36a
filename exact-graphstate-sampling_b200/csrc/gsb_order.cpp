// Host-side linear order search for the cut-rank DP (no GPU involved).
//
// The DP table at step k has 2^{r_k} entries, r_k = rank over GF(2) of A[prefix_k, suffix_k] (reference
// order.py:14-20, plan.py:1-9).  An order is scored, as the reference's order search scores it (order2.py:27-28),
// by the key (max r_k, number of steps at the max, log2 sum_k 2^{r_k}), compared lexicographically.
// The search is the reference's strategy (order2.py:16-25, frontier_instance.py:29-37) restated natively:
//   * randomised greedy construction: append the vertex whose cut rank after appending is smallest, ties broken by
//     uniform noise;
//   * local search from the best greedy order: move one vertex a short distance, swap two, or reverse a segment;
//     keep a move when the key does not get worse (and, rarely, when it does), remembering the best order seen.
// Only the cuts between the two moved positions change, so a move re-ranks just those cuts.
// Vertices are bits of 128-bit words (n <= 128).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

#include "gsb.h"

namespace {

typedef unsigned __int128 u128;

int lead(u128 x) {
    const uint64_t hi = (uint64_t)(x >> 64);
    if (hi) return 127 - __builtin_clzll(hi);
    return 63 - __builtin_clzll((uint64_t)x);
}

// rank of the rows (each restricted to mask)
int rank_rows(const u128 *nb, const int *rows, int nrows, u128 mask) {
    u128 piv[128];
    bool has[128] = {false};
    int r = 0;
    for (int i = 0; i < nrows; i++) {
        u128 x = nb[rows[i]] & mask;
        while (x) {
            const int b = lead(x);
            if (!has[b]) { has[b] = true; piv[b] = x; r++; break; }
            x ^= piv[b];
        }
    }
    return r;
}

struct Key {
    int w = 0, cnt = 0;
    double cost = 0;
    bool operator<(const Key &o) const {
        if (w != o.w) return w < o.w;
        if (cnt != o.cnt) return cnt < o.cnt;
        return cost < o.cost - 1e-12;
    }
    bool operator<=(const Key &o) const { return !(o < *this); }
};

Key key_of(const std::vector<int> &prof) {
    Key k;
    double s = 0;
    for (int r : prof) k.w = std::max(k.w, r);
    for (int r : prof) {
        if (r == k.w) k.cnt++;
        s += std::ldexp(1.0, r);
    }
    k.cost = s > 0 ? std::log2(s) : 0;
    return k;
}

struct Graph {
    int n;
    std::vector<u128> nb;
    u128 full;
    // cut rank after the first k vertices of order (1 <= k <= n-1)
    int cut(const std::vector<int> &order, int k) const {
        u128 F = full;
        for (int i = 0; i < k; i++) F &= ~((u128)1 << order[(size_t)i]);
        return rank_rows(nb.data(), order.data(), k, F);
    }
    void profile(const std::vector<int> &order, std::vector<int> &prof) const {
        prof.assign((size_t)std::max(0, n - 1), 0);
        for (int k = 1; k < n; k++) prof[(size_t)k - 1] = cut(order, k);
    }
};

std::vector<int> greedy(const Graph &G, std::mt19937_64 &rng, double noise) {
    const int n = G.n;
    std::vector<int> P;
    std::vector<char> used((size_t)n, 0);
    std::uniform_real_distribution<double> U(0, 1);
    u128 Pm = 0;
    for (int k = 0; k < n; k++) {
        std::vector<int> cand;
        for (int v = 0; v < n; v++)
            if (!used[(size_t)v]) cand.push_back(v);
        std::shuffle(cand.begin(), cand.end(), rng);
        double best = 1e300;
        int bv = cand[0];
        for (int v : cand) {
            P.push_back(v);
            const u128 F = G.full & ~(Pm | ((u128)1 << v));
            const double c = rank_rows(G.nb.data(), P.data(), (int)P.size(), F) + noise * U(rng);
            P.pop_back();
            if (c < best) { best = c; bv = v; }
        }
        P.push_back(bv);
        used[(size_t)bv] = 1;
        Pm |= (u128)1 << bv;
    }
    return P;
}

}  // namespace

extern "C" {

int gsb_cut_profile(int n, const uint8_t *A, const int *order, int *prof) {
    if (n < 1 || n > 128 || !A || !order || !prof) return GSB_E_USAGE;
    Graph G;
    G.n = n;
    G.nb.assign((size_t)n, 0);
    G.full = n == 128 ? ~(u128)0 : (((u128)1 << n) - 1);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            if (A[(size_t)i * n + j] & 1) G.nb[(size_t)i] |= (u128)1 << j;
    std::vector<int> o(order, order + n), p;
    G.profile(o, p);
    for (int k = 0; k + 1 < n; k++) prof[k] = p[(size_t)k];
    return GSB_OK;
}

int gsb_order_search(int n, const uint8_t *A, uint64_t seed, int ngreedy, int64_t iters, int *order_out, int *width_out) {
    if (n < 1 || n > 128 || !A || !order_out || ngreedy < 1 || iters < 0) return GSB_E_USAGE;
    Graph G;
    G.n = n;
    G.nb.assign((size_t)n, 0);
    G.full = n == 128 ? ~(u128)0 : (((u128)1 << n) - 1);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            if (A[(size_t)i * n + j] & 1) G.nb[(size_t)i] |= (u128)1 << j;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(0, 1);
    std::vector<int> cur, prof;
    Key ck;
    for (int g = 0; g < ngreedy; g++) {
        std::vector<int> o = greedy(G, rng, 0.9);
        G.profile(o, prof);
        const Key k = key_of(prof);
        if (g == 0 || k < ck) { ck = k; cur = o; }
    }
    G.profile(cur, prof);
    std::vector<int> best = cur, bprof = prof, nprof;
    Key bk = ck;
    std::vector<int> nw;
    for (int64_t it = 0; it < iters && n > 2; it++) {
        int a = (int)(rng() % (uint64_t)n), b = (int)(rng() % (uint64_t)n);
        if (a == b) continue;
        if (a > b) std::swap(a, b);
        if (b - a > 12 && U(rng) < 0.7) b = a + 1 + (int)(rng() % 12ULL);
        nw = cur;
        const double u = U(rng);
        if (u < 0.35) std::swap(nw[(size_t)a], nw[(size_t)b]);
        else if (u < 0.7) {
            const int x = nw[(size_t)a];
            nw.erase(nw.begin() + a);
            nw.insert(nw.begin() + b, x);
        } else std::reverse(nw.begin() + a, nw.begin() + b + 1);
        // cuts k with a < k <= b change (k = number of vertices before the cut)
        nprof = prof;
        for (int k = a + 1; k <= b && k < n; k++) nprof[(size_t)k - 1] = G.cut(nw, k);
        const Key nk = key_of(nprof);
        if (nk <= ck || U(rng) < 0.002) {
            cur.swap(nw);
            prof.swap(nprof);
            ck = nk;
            if (ck < bk) { bk = ck; best = cur; bprof = prof; }
        }
    }
    for (int i = 0; i < n; i++) order_out[i] = best[(size_t)i];
    if (width_out) *width_out = bk.w;
    return GSB_OK;
}

}  // extern "C"
