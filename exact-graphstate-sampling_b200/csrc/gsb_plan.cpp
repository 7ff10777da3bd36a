// Plan text parsing and structural validation (see gsb_plan.h).
#include "gsb_plan.h"

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace gsb {

namespace {

struct Tok {
    const char *p, *end;
    void skip() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\f' || *p == '\v')) p++;
    }
    // next token copied into a small buffer (numbers are short); false at end of text
    bool next(char *buf, size_t cap) {
        skip();
        if (p >= end) return false;
        size_t n = 0;
        while (p < end && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\f' || *p == '\v')) {
            if (n + 1 >= cap) return false;
            buf[n++] = *p++;
        }
        buf[n] = 0;
        return true;
    }
    bool i32(int &out) {
        char b[64];
        if (!next(b, sizeof b)) return false;
        char *e = nullptr;
        errno = 0;
        long v = strtol(b, &e, 10);
        if (*e || errno || v < -2147483647L || v > 2147483647L) return false;
        out = (int)v;
        return true;
    }
    bool u64(uint64_t &out) {
        char b[64];
        if (!next(b, sizeof b)) return false;
        if (b[0] == '-') return false;
        char *e = nullptr;
        errno = 0;
        unsigned long long v = strtoull(b, &e, 10);
        if (*e || errno) return false;
        out = (uint64_t)v;
        return true;
    }
    bool f64(double &out) {
        char b[64];
        if (!next(b, sizeof b)) return false;
        char *e = nullptr;
        out = strtod(b, &e);
        return *e == 0;
    }
};

std::string fmt(const char *f, int a, int b = 0) {
    char buf[256];
    snprintf(buf, sizeof buf, f, a, b);
    return buf;
}

}  // namespace

int gf2_rank(const std::vector<uint64_t> &v) {
    uint64_t piv[64] = {0};
    int r = 0;
    for (uint64_t x : v) {
        for (int b = 63; b >= 0 && x; b--) {
            if (!((x >> b) & 1)) continue;
            if (!piv[b]) { piv[b] = x; r++; x = 0; break; }
            x ^= piv[b];
        }
    }
    return r;
}

bool gf2_in_span(const std::vector<uint64_t> &basis, uint64_t x) {
    std::vector<uint64_t> v(basis);
    int r = gf2_rank(v);
    v.push_back(x);
    return gf2_rank(v) == r;
}

int parse_plan_text(const char *text, size_t len, HPlan &p, std::string &err) {
    Tok t{text, text + len};
    if (!t.i32(p.n) || !t.i32(p.ns) || !t.i32(p.R) || p.ns < 0 || p.R < 0) { err = "plan header 'n nsteps R' unreadable"; return 2; }
    if (p.R > 40) { err = fmt("arena exponent R = %d exceeds 40", p.R); return 7; }
    p.st.assign((size_t)p.ns, HStep());
    for (int k = 0; k < p.ns; k++) {
        HStep &s = p.st[(size_t)k];
        int nt = 0;
        if (!t.i32(s.v) || !t.i32(s.nk) || !t.i32(s.m) || !t.u64(s.g) || !t.u64(s.rhoc) || !t.i32(nt)) {
            err = fmt("plan step %d: 'v nk m g rhoc nterms' unreadable", k);
            return 3;
        }
        if (s.nk < 0 || s.nk > 40) { err = fmt("plan step %d: nk = %d outside 0..40", k, s.nk); return 7; }
        if (nt < 1 || nt > 16) { err = fmt("plan step %d: nterms = %d outside 1..16", k, nt); return 7; }
        s.tk.resize((size_t)s.nk);
        for (int j = 0; j < s.nk; j++)
            if (!t.u64(s.tk[(size_t)j])) { err = fmt("plan step %d: Tkeep entry %d unreadable", k, j); return 4; }
        s.t.resize((size_t)nt);
        for (int i = 0; i < nt; i++) {
            HTerm &h = s.t[(size_t)i];
            if (!t.u64(h.tq) || !t.i32(h.x) || !t.i32(h.tau) || !t.i32(h.par)) { err = fmt("plan step %d: term %d unreadable", k, i); return 5; }
        }
        for (int b = 0; b < 2; b++)
            for (int x = 0; x < 2; x++)
                if (!t.f64(s.Mr[b][x]) || !t.f64(s.Mi[b][x])) { err = fmt("plan step %d: M[%d][.] unreadable", k, b); return 6; }
    }
    return 0;
}

int validate_plan(HPlan &p, std::string &err) {
    const uint64_t lim = p.R >= 64 ? ~0ULL : (1ULL << p.R);
    std::vector<uint64_t> live{};   // basis of the live address space before the step; {0} = empty basis
    for (int k = 0; k < p.ns; k++) {
        HStep &s = p.st[(size_t)k];
        if (s.m != 1 && s.m != 2) { err = fmt("plan step %d: m = %d (must be 1 or 2)", k, s.m); return 7; }
        for (uint64_t a : s.tk)
            if (a >= lim) { err = fmt("plan step %d: Tkeep address outside the 2^R arena", k); return 15; }
        if (s.m == 2 && s.g >= lim) { err = fmt("plan step %d: g outside the 2^R arena", k); return 15; }
        // distinct offsets, sorted
        std::vector<uint64_t> d;
        for (const HTerm &h : s.t) {
            if (h.tq >= lim) { err = fmt("plan step %d: term offset outside the 2^R arena", k); return 15; }
            if (h.x != 0 && h.x != 1) { err = fmt("plan step %d: term x must be 0 or 1", k); return 7; }
            if (h.tau < 0 || h.tau >= s.m) { err = fmt("plan step %d: term class outside 0..m-1", k); return 7; }
            d.push_back(h.tq);
        }
        std::sort(d.begin(), d.end());
        d.erase(std::unique(d.begin(), d.end()), d.end());
        if (d.size() != 1 && d.size() != 2 && d.size() != 4) { err = fmt("plan step %d: %d distinct coset offsets (1, 2 or 4 expected)", k, (int)d.size()); return 7; }
        if (d[0] != 0) { err = fmt("plan step %d: coset offsets do not contain 0", k); return 15; }
        for (uint64_t a : d)
            for (uint64_t b : d)
                if (!std::binary_search(d.begin(), d.end(), a ^ b)) { err = fmt("plan step %d: coset offsets are not a subspace", k); return 15; }
        if (s.t.size() != 2 * d.size()) { err = fmt("plan step %d: expected two terms (x = 0, 1) per coset offset", k); return 7; }
        s.tqs = d;
        for (size_t i = 0; i < d.size(); i++) {
            int seen0 = 0, seen1 = 0;
            for (const HTerm &h : s.t) {
                if (h.tq != d[i]) continue;
                if (h.x == 0) { seen0++; s.tau0[i] = h.tau; }
                else { seen1++; s.tau1[i] = h.tau; s.par[i] = h.par & 1; }
            }
            if (seen0 != 1 || seen1 != 1) { err = fmt("plan step %d: offset %d lacks exactly one x=0 and one x=1 term", k, (int)i); return 7; }
        }
        // read layout: Tkeep u basis(D) independent
        std::vector<uint64_t> rd(s.tk);
        std::vector<uint64_t> dbasis;
        for (uint64_t a : d)
            if (a && !gf2_in_span(dbasis, a)) dbasis.push_back(a);
        rd.insert(rd.end(), dbasis.begin(), dbasis.end());
        if (gf2_rank(rd) != (int)rd.size()) { err = fmt("plan step %d: coset slots are not disjoint (Tkeep and offsets dependent)", k); return 15; }
        // the slots read must be exactly the live slots left by the previous step
        if (rd.size() != live.size()) {
            err = fmt("plan step %d reads a table of 2^%d entries", k, (int)rd.size()) + fmt("; the previous step left 2^%d", (int)live.size());
            return 15;
        }
        for (uint64_t a : rd)
            if (!gf2_in_span(live, a)) { err = fmt("plan step %d reads slots the previous step did not write", k); return 15; }
        // write layout
        std::vector<uint64_t> nl(s.tk);
        if (s.m == 2) {
            if (s.g == 0) { err = fmt("plan step %d: m = 2 with g = 0", k); return 15; }
            if (d.size() > 1) {
                if (!std::binary_search(d.begin(), d.end(), s.g)) { err = fmt("plan step %d: second output outside the coset's own slots", k); return 15; }
            } else if (gf2_in_span(s.tk, s.g)) {
                err = fmt("plan step %d: growth slot g collides with a live slot", k);
                return 15;
            }
            nl.push_back(s.g);
        }
        live = nl;
    }
    if (!live.empty()) { err = "the plan does not end with a single entry"; return 15; }
    return 0;
}

}  // namespace gsb
