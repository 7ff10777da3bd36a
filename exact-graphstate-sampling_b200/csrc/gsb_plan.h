// Host-side plan of the in-place cut-rank DP: parsing of the plan text and structural validation.
// The text format is the reference's (inplace.py:143-159 writes it, gsamp2.cpp:2,128-139 reads it):
//   n nsteps R
//   per step: v nk m g rhoc nterms   Tkeep[nk]   nterms x (Tq x tau par)   M[b][x] re im for b,x in (0,1)^2
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace gsb {

struct HTerm {
    uint64_t tq;
    int x, tau, par;
};

struct HStep {
    int v = 0, nk = 0, m = 0;
    uint64_t g = 0, rhoc = 0;
    std::vector<uint64_t> tk;   // physical address of kept coordinate j (bit j of the coset index c)
    std::vector<HTerm> t;
    double Mr[2][2] = {{0, 0}, {0, 0}}, Mi[2][2] = {{0, 0}, {0, 0}};
    // derived by validate_plan: the distinct coset offsets (a GF(2) subspace, sorted ascending as the reference's
    // coset_offsets, gsamp2.cpp:122-125) and, per offset, the output class of its x=0 and x=1 terms and the sign
    // parity of its x=1 term.
    std::vector<uint64_t> tqs;
    int tau0[4] = {0, 0, 0, 0}, tau1[4] = {0, 0, 0, 0}, par[4] = {0, 0, 0, 0};
};

struct HPlan {
    int n = 0, ns = 0, R = 0;
    std::vector<HStep> st;
};

// Returns 0 or the reference's exit code for the failure (2..7); err gets a message.
int parse_plan_text(const char *text, size_t len, HPlan &p, std::string &err);

// Structural checks of the in-place invariants (reference asserts them while planning, inplace.py:85-88, and while
// executing, inplace.py:126-137):
//   * every address < 2^R;
//   * the coset offsets of a step form a subspace D of dimension q <= 2 and {Tkeep} u basis(D) is independent, so
//     the coset slots base(c) ^ D are pairwise disjoint across c;
//   * each offset carries exactly one x=0 and one x=1 term with classes < m;
//   * m = 2 writes base ^ g inside the coset's own slots (g in D \ {0}) or, for q = 0, into a fresh slot
//     (g not in span Tkeep);
//   * the live addresses after a step equal the addresses the next step reads (span), starting from {0}.
// Returns 0, GSB_E_PLAN_RANGE (7) or GSB_E_PLAN_LAYOUT (15).
int validate_plan(HPlan &p, std::string &err);

// GF(2) helpers on address vectors
int gf2_rank(const std::vector<uint64_t> &v);
bool gf2_in_span(const std::vector<uint64_t> &basis, uint64_t x);

}  // namespace gsb
