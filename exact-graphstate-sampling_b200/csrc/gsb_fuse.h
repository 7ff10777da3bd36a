// Fusing consecutive DP steps into one pass over the arena (host side).
//
// A group is a run of d consecutive steps.  One pass reads the table before the group and writes the table after
// it; the steps in between run on shared-memory tiles.  The group's classes are cosets of small subspaces:
//   stage s (s = 0 .. d) holds the table before step k0 + s;
//   class b at stage s = { b ^ z : z in Z_s },
// where b ranges over a class-base space B.  B is spanned by address columns that every step of the group keeps,
// so b is a coset base of every step and the same address names the class at every stage.
// The zero class is the least family of subspaces closed under the steps:
//   Z_s contains the step's coset offsets D_s;
//   step s maps each of its cosets y ^ D_s (y in Y_s = Z_s n span(Tkeep_s)) to y ^ G_s (G_s = {0, g_s});
//   projecting stage s+1 back along G_s stays in Z_s.
// Within a class, step s is a fixed dataflow over the class's values:
//   member y_j reads stage-s values y_j ^ tq_t and writes stage-(s+1) values y_j ^ G_s[tau];
//   its sign parity is parity(b & lambda_s) ^ parity(y_j & lambda_s).
// lambda_s is a physical mask with parity(base(c) & lambda_s) = parity(c & rhoc_s).
// A group is safe in place when a class's writes never meet another class's reads: (Z_0 + Z_d) n L_0 = Z_0, where
// L_0 is the live space before the group.
#pragma once
#include <cstdint>
#include <vector>

#include "gsb_plan.h"

namespace gsb {

constexpr int FUSE_MAX_STEPS = 3;
constexpr int FUSE_MAX_MEMBERS = 16;   // step cosets per class and step
constexpr int FUSE_MAX_STAGE = 32;     // values per class and stage

struct GroupPlan {
    int k0 = 0, d = 0;
    int L = 0;                          // log2 classes per tile (class-base bits 0..L-1 are address bits 0..L-1)
    int nb = 0;                         // dim B
    std::vector<uint64_t> bhi;          // class-base basis vectors beyond the L low unit vectors (nb - L of them)
    int ws = 0;                         // stage written to the arena (d, or d - 1 when the last step only feeds norms)
    int stage_size[FUSE_MAX_STEPS + 1] = {0};
    std::vector<uint64_t> z_in;         // elements of Z_0 (stage-0 offsets), index order
    std::vector<uint64_t> z_out;        // elements of Z_ws (offsets of the written stage), index order
    struct Step {
        int nmem = 0, ntq = 0, m = 0;
        uint64_t lambda = 0;
        int in_idx[FUSE_MAX_MEMBERS][4];    // member j, offset t -> stage-s index
        int out_idx[FUSE_MAX_MEMBERS][2];   // member j, class tau -> stage-(s+1) index
        int mpar[FUSE_MAX_MEMBERS];         // parity(y_j & lambda)
    } step[FUSE_MAX_STEPS];
    // algorithmic bytes per element size: entries read + written by the pass
    double entries_moved = 0;
};

// Try to fuse steps k0 .. k0 + d - 1 of a validated plan.  Returns true and fills gp when the group is safe and fits
// the kernel's limits (stage sizes <= FUSE_MAX_STAGE, at least min_L low unit vectors among the class-base bits).
// write_stage (default d) is the stage the pass stores; with write_stage = d - 1 the last step is evaluated from the
// stored stage in shared memory only (its branch norms), and safety is checked for the stored stage.
bool plan_group(const HPlan &p, int k0, int d, int min_L, int max_L, GroupPlan &gp, int write_stage = -1);

}  // namespace gsb
