// Host derivation of fused step groups (see gsb_fuse.h).
#include "gsb_fuse.h"

#include <algorithm>
#include <map>

namespace gsb {

namespace {

// Subspace of GF(2)^64 with a pivot basis (pivot = leading bit).
struct Sp {
    uint64_t piv[64] = {0};
    std::vector<uint64_t> basis;   // insertion order (elements() enumerates by doubling over it)
    uint64_t reduce(uint64_t x) const {
        for (int i = 63; i >= 0 && x; i--)
            if (((x >> i) & 1) && piv[i]) x ^= piv[i];
        return x;
    }
    bool add(uint64_t x) {
        const uint64_t r = reduce(x);
        if (!r) return false;
        piv[63 - __builtin_clzll(r)] = r;
        basis.push_back(x);
        return true;
    }
    bool contains(uint64_t x) const { return reduce(x) == 0; }
    int dim() const { return (int)basis.size(); }
    std::vector<uint64_t> elements() const {
        std::vector<uint64_t> e{0};
        for (uint64_t b : basis) {
            const size_t n = e.size();
            for (size_t i = 0; i < n; i++) e.push_back(e[i] ^ b);
        }
        return e;
    }
};

// lambda with parity(v_i & lambda) = t_i for independent v_i
uint64_t solve_parity(const std::vector<uint64_t> &v, const std::vector<int> &t) {
    struct Row {
        uint64_t v;
        int t;
        int p;
    };
    std::vector<Row> rows;
    for (size_t i = 0; i < v.size(); i++) {
        Row r{v[i], t[i] & 1, -1};
        for (const Row &q : rows)
            if ((r.v >> q.p) & 1) { r.v ^= q.v; r.t ^= q.t; }
        if (!r.v) continue;   // dependent (cannot happen for a validated plan)
        r.p = 63 - __builtin_clzll(r.v);
        for (Row &q : rows)
            if ((q.v >> r.p) & 1) { q.v ^= r.v; q.t ^= r.t; }
        rows.push_back(r);
    }
    uint64_t lam = 0;
    for (const Row &q : rows)
        if (q.t) lam |= 1ULL << q.p;
    return lam;
}

}  // namespace

bool plan_group(const HPlan &p, int k0, int d, int min_L, int max_L, GroupPlan &gp, int write_stage) {
    if (d < 1 || d > FUSE_MAX_STEPS || k0 < 0 || k0 + d > p.ns) return false;
    const int ws = write_stage < 0 ? d : write_stage;
    if (ws < 1 || ws > d) return false;
    gp = GroupPlan();
    gp.k0 = k0;
    gp.d = d;
    gp.ws = ws;
    std::vector<Sp> T((size_t)d), D((size_t)d);
    for (int s = 0; s < d; s++) {
        const HStep &st = p.st[(size_t)(k0 + s)];
        for (uint64_t a : st.tk) T[(size_t)s].add(a);
        for (uint64_t a : st.tqs)
            if (a) D[(size_t)s].add(a);
    }
    auto g_of = [&](int s) -> uint64_t {
        const HStep &st = p.st[(size_t)(k0 + s)];
        return st.m == 2 ? st.g : 0;
    };
    // projection of a stage-(s+1) address onto span(Tkeep_s) along G_s
    auto proj = [&](int s, uint64_t z) -> uint64_t {
        if (T[(size_t)s].contains(z)) return z;
        return z ^ g_of(s);
    };
    std::vector<Sp> Z((size_t)d + 1);
    for (int s = 0; s < d; s++) Z[(size_t)s] = D[(size_t)s];
    bool changed = true;
    int iter = 0;
    while (changed && iter++ < 64) {
        changed = false;
        for (int s = 0; s < d; s++) {
            for (uint64_t y : Z[(size_t)s].elements())
                if (T[(size_t)s].contains(y)) {
                    changed |= Z[(size_t)s + 1].add(y);
                    if (g_of(s)) changed |= Z[(size_t)s + 1].add(y ^ g_of(s));
                }
            if (s + 1 < d)
                for (uint64_t t : D[(size_t)s + 1].basis) changed |= Z[(size_t)s + 1].add(t);
        }
        for (int s = d - 1; s >= 0; s--)
            for (uint64_t z : std::vector<uint64_t>(Z[(size_t)s + 1].basis)) changed |= Z[(size_t)s].add(proj(s, z));
        for (int s = 0; s <= d; s++)
            if (Z[(size_t)s].dim() > 5) return false;   // FUSE_MAX_STAGE = 32 values per class and stage
    }
    if (changed) return false;
    // dataflow tables
    for (int s = 0; s <= d; s++) gp.stage_size[s] = 1 << Z[(size_t)s].dim();
    std::vector<std::map<uint64_t, int>> index((size_t)d + 1);
    std::vector<std::vector<uint64_t>> elems((size_t)d + 1);
    for (int s = 0; s <= d; s++) {
        elems[(size_t)s] = Z[(size_t)s].elements();
        for (size_t i = 0; i < elems[(size_t)s].size(); i++) index[(size_t)s][elems[(size_t)s][i]] = (int)i;
    }
    for (int s = 0; s < d; s++) {
        const HStep &st = p.st[(size_t)(k0 + s)];
        GroupPlan::Step &gs = gp.step[s];
        gs.ntq = (int)st.tqs.size();
        gs.m = st.m;
        std::vector<uint64_t> members;
        for (uint64_t y : elems[(size_t)s])
            if (T[(size_t)s].contains(y)) members.push_back(y);
        gs.nmem = (int)members.size();
        if (gs.nmem > FUSE_MAX_MEMBERS) return false;
        if ((size_t)gs.nmem * st.tqs.size() != elems[(size_t)s].size()) return false;
        if ((size_t)gs.nmem * (size_t)st.m != elems[(size_t)s + 1].size()) return false;
        std::vector<int> seen_in(elems[(size_t)s].size(), 0), seen_out(elems[(size_t)s + 1].size(), 0);
        // parity mask: parity(Tkeep[j] & lambda) = rhoc bit j, parity(offset basis & lambda) = 0
        std::vector<uint64_t> vv(st.tk);
        std::vector<int> tt;
        for (int j = 0; j < st.nk; j++) tt.push_back((int)((st.rhoc >> j) & 1));
        for (uint64_t a : D[(size_t)s].basis) { vv.push_back(a); tt.push_back(0); }
        gs.lambda = solve_parity(vv, tt);
        for (int j = 0; j < gs.nmem; j++) {
            const uint64_t y = members[(size_t)j];
            gs.mpar[j] = __builtin_popcountll(y & gs.lambda) & 1;
            for (int t = 0; t < gs.ntq; t++) {
                auto it = index[(size_t)s].find(y ^ st.tqs[(size_t)t]);
                if (it == index[(size_t)s].end()) return false;
                gs.in_idx[j][t] = it->second;
                seen_in[(size_t)it->second]++;
            }
            for (int tau = 0; tau < st.m; tau++) {
                auto it = index[(size_t)s + 1].find(tau ? (y ^ st.g) : y);
                if (it == index[(size_t)s + 1].end()) return false;
                gs.out_idx[j][tau] = it->second;
                seen_out[(size_t)it->second]++;
            }
        }
        for (int c : seen_in)
            if (c != 1) return false;
        for (int c : seen_out)
            if (c != 1) return false;
    }
    // in-place safety: (Z_0 + Z_ws) n L_0 = Z_0
    Sp L0;
    for (uint64_t a : T[0].basis) L0.add(a);
    for (uint64_t a : D[0].basis) L0.add(a);
    Sp both = Z[0];
    for (uint64_t z : Z[(size_t)ws].basis) both.add(z);
    Sp inter;
    for (uint64_t e : both.elements())
        if (L0.contains(e)) inter.add(e);
    if (inter.dim() != Z[0].dim()) return false;
    // class-base space: columns every step of the group keeps, low unit vectors first
    std::vector<uint64_t> common;
    for (uint64_t a : p.st[(size_t)k0].tk) {
        bool all = true;
        for (int s = 1; s < d && all; s++) {
            const auto &tk = p.st[(size_t)(k0 + s)].tk;
            all = std::find(tk.begin(), tk.end(), a) != tk.end();
        }
        if (all) common.push_back(a);
    }
    Sp acc = Z[0];
    int L = 0;
    while (L < max_L) {
        const uint64_t e = 1ULL << L;
        if (std::find(common.begin(), common.end(), e) == common.end() || !acc.add(e)) break;
        L++;
    }
    if (L < min_L) return false;
    for (uint64_t a : common) {
        if (a < (1ULL << L) && __builtin_popcountll(a) == 1) continue;   // already taken as a low unit vector
        if (acc.add(a)) gp.bhi.push_back(a);
    }
    if (acc.dim() != L0.dim()) return false;
    gp.L = L;
    gp.nb = L + (int)gp.bhi.size();
    gp.z_in = elems[0];
    gp.z_out = elems[(size_t)ws];
    gp.entries_moved = (double)(gp.stage_size[0] + gp.stage_size[ws]) * (double)(1ULL << gp.nb);
    return true;
}

}  // namespace gsb
