/*
 * gsb.h -- C ABI of the B200 executor for the in-place cut-rank dynamic program (libgsb.so).
 *
 * The reference has no in-process interface for this path: its seam is the executor process `gsamp2 <plan> <mode>`
 * (gsamp2.cpp:1-6, 149-225), chosen by path through `doped_sampler.py --bin` (doped_sampler.py:28) and run by the
 * cloud scripts and tests.  Each mode of that command line becomes one entry point here, with the same inputs
 * (plan text, strings in step order, seeds, dump tables) and the same numbers out (bits, log2 Pr, conditionals,
 * dump tables), so a ctypes / C / C++ caller can replace the subprocess call.  `gsb2` (the command line built on
 * this library) keeps the reference's argv and stdout formats for callers that stay process based.
 *
 * Conventions
 *   - Every function returns a status: 0 = GSB_OK, otherwise one of the codes below.  Codes 1-14 are the reference
 *     executor's exit codes for the same failures.  Nothing calls exit(); gsb_last_error() gives a message
 *     (thread-local, valid until the next call on this thread).
 *   - Strings / bits are int8 arrays in STEP order (character k of a reference strings-file line is element k):
 *     0, 1, or -1 for '?' where a mode allows it.  Multi-string arguments are row-major [nstr][nsteps].
 *   - An engine owns one arena (2^R entries of complex64 or complex128) and one CUDA stream on one device.  Calls on
 *     one engine must not overlap (one engine per host thread); different engines are independent.
 *   - Host-buffer entry points are synchronous: they copy inputs in, run, and copy results out before returning.
 */
#ifndef GSB_H
#define GSB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSB_OK 0
#define GSB_E_USAGE 1          /* bad argument (reference: exit 1, usage) */
#define GSB_E_PLAN_HEADER 2    /* plan header "n nsteps R" unreadable (gsamp2.cpp:128) */
#define GSB_E_PLAN_STEP 3      /* step line "v nk m g rhoc nterms" unreadable (gsamp2.cpp:131) */
#define GSB_E_PLAN_TKEEP 4     /* Tkeep list unreadable (gsamp2.cpp:132) */
#define GSB_E_PLAN_TERM 5      /* term "Tq x tau par" unreadable (gsamp2.cpp:133) */
#define GSB_E_PLAN_M 6         /* M matrix unreadable (gsamp2.cpp:134) */
#define GSB_E_PLAN_RANGE 7     /* nk > 40 or a term list outside what the plan format allows (gsamp2.cpp:135) */
#define GSB_E_PREFIX_FREE 8    /* '?' before step K in prefix mode (gsamp2.cpp:168) */
#define GSB_E_DUMP_MISSING 9   /* a dump table is missing (gsamp2.cpp:199) */
#define GSB_E_DUMP_BAD 10      /* a dump table has the wrong shape (gsamp2.cpp:200) */
#define GSB_E_ALLOC 11         /* arena allocation failed (gsamp2.cpp:142) */
#define GSB_E_TWIST_MISSING 12 /* twist file missing (gsamp2.cpp:190) */
#define GSB_E_TWIST_LINE 13    /* twist line unreadable (gsamp2.cpp:191) */
#define GSB_E_TWIST_RANGE 14   /* twist shift outside the kept coordinates / coset offsets (gsamp2.cpp:192-194) */
#define GSB_E_PLAN_LAYOUT 15   /* the plan breaks an in-place invariant (reference asserts inplace.py:85-88,131-137) */
#define GSB_E_CUDA 20          /* CUDA runtime error (reference GPU port: exit 99, gsamp_cuda.cu:23) */
#define GSB_E_STATE 21         /* invalid engine handle */

#define GSB_C64 64             /* complex64 arena, FP64 arithmetic (the reference's default build) */
#define GSB_C128 128           /* complex128 arena (the reference's -DGS_DOUBLE build, gsamp2.cpp:19-23) */

#define GSB_SEED_INT 0         /* sample i uses std::mt19937_64(seed + i)                  ('sample', gsamp2.cpp:151) */
#define GSB_SEED_SEQ 1         /* std::seed_seq{seed_lo, seed_hi, i_lo, i_hi, 0x9E3779B9}   ('sample2', gsamp2.cpp:159) */

typedef struct gsb_engine gsb_engine;

const char *gsb_version(void);
const char *gsb_last_error(void);

/* Load a plan (file path, or text in memory) and allocate the arena on `device`.
 * Replaces the plan parse + arena set-up of gsamp2.cpp:128-147 / gsamp_cuda.cu:125-142.  The plan is also checked
 * for the in-place invariants (independent addresses, writes inside the coset's own slots, addresses < 2^R). */
int gsb_open_file(const char *plan_path, int precision, int device, gsb_engine **out);
int gsb_open_text(const char *plan_text, size_t len, int precision, int device, gsb_engine **out);
int gsb_close(gsb_engine *e);
int gsb_info(const gsb_engine *e, int *n, int *nsteps, int *R, int *precision);
/* qubit (vertex) of each step, nsteps entries */
int gsb_step_vertices(const gsb_engine *e, int *out);

/* 'prob': log2 Pr of each string, normalised two-pass chain (gsamp2.cpp:39-55, 217-223). */
int gsb_prob(gsb_engine *e, const int8_t *bits, int64_t nstr, double *log2p);

/* 'chain': one pass per step; log2 Pr and every conditional Pr(b_k | b_1..b_{k-1}) (gsamp2.cpp:56-70, 217-222).
 * cond is [nstr][nsteps]; may be NULL. */
int gsb_chain(gsb_engine *e, const int8_t *bits, int64_t nstr, double *log2p, double *cond);

/* 'sample' / 'sample2': samples first .. first+count-1 of stream (seeding, seed): bits [count][nsteps] and log2 Pr
 * (gsamp2.cpp:149-161).  The sample printed by the reference as "<bits> lp seed+i" is sample i here. */
int gsb_sample(gsb_engine *e, int seeding, uint64_t seed, int64_t first, int64_t count, int8_t *bits, double *log2p);

/* Exact chain-rule samples driven by caller-supplied uniforms u [count][nsteps] (bit k = u[k] < Pr(b_k = 1 | prefix)),
 * the same draw rule as gsamp2.cpp:46-47. */
int gsb_sample_uniform(gsb_engine *e, const double *u, int64_t count, int8_t *bits, double *log2p);

/* 'hybrid': forced [nstr][nsteps] in {0,1,-1}; line i draws its '?' bits from std::mt19937_64(seed + first_line + i);
 * bits, log2 Pr and all conditionals out (gsamp2.cpp:71-120, 209-216).  cond may be NULL. */
int gsb_hybrid(gsb_engine *e, const int8_t *forced, int64_t nstr, uint64_t seed, int64_t first_line, int8_t *bits,
               double *log2p, double *cond);

/* Shape of the live table dumped at step K: 2^nk cosets x ntq offsets (gsamp2.cpp:121-125, 171). */
int gsb_dump_shape(const gsb_engine *e, int K, int *nk, int *ntq);

/* 'prefix': run the forced steps 0..K-1 of one string and copy out the live table in logical (c, tq) order, entries
 * of the arena type (complex64 = 2 floats, complex128 = 2 doubles); *logscale and log2 Pr(prefix) as the reference
 * prints them (gsamp2.cpp:162-175).  dump may be NULL when only log2 Pr(prefix) (a marginal) is wanted. */
int gsb_prefix(gsb_engine *e, const int8_t *forced, int K, void *dump, double *logscale, double *log2p_prefix);

/* 'resume': sum nslices dump tables (scaled by 2^(logscale_s - max)), read through the optional twist translation
 * (cshift, tqshift per slice; both NULL for none), then run steps K..nsteps-1 drawing '?' bits from
 * std::mt19937_64(seed + line) (gsamp2.cpp:176-208).  bits are full-length (forced prefix copied); cond [nsteps],
 * entries K.. are written.  Dump entries are of the arena type. */
int gsb_resume(gsb_engine *e, const int8_t *forced, int K, uint64_t seed, int64_t line, int nslices,
               const void *const *dumps, const double *logscales, const uint64_t *cshift, const uint64_t *tqshift,
               int8_t *bits, double *log2p_full, double *log2p_prefix, double *cond);

/* Device-resident batches: all pointers are device memory on the engine's GPU.  Work is queued on the engine's
 * stream; call gsb_synchronize before reading results. */
int gsb_chain_device(gsb_engine *e, const int8_t *d_bits, int64_t nstr, double *d_log2p, double *d_cond);
int gsb_sample_device(gsb_engine *e, const double *d_u, int64_t count, int8_t *d_bits, double *d_log2p);
int gsb_synchronize(gsb_engine *e);
/* Queue the engine's work on `cuda_stream` (a cudaStream_t of the engine's device; NULL = the engine's own stream),
 * e.g. a framework's current stream, so events recorded there bracket the engine's kernels. */
int gsb_set_stream(gsb_engine *e, void *cuda_stream);
/* 'chain' mode fuses runs of up to `depth` consecutive wide steps (tables of >= 2^12 entries) into one pass over
 * the arena: the intermediate tables of a group live in shared-memory tiles only.  depth 1 disables fusion;
 * default 2.  Results are those of the unfused steps up to rounding. */
int gsb_set_fusion(gsb_engine *e, int depth);
/* Autotune the pass lists on this device: every candidate pass (one step; 2 or 3 fused steps; for sampling with or
 * without the next step's branch norms; tiles of up to 2^8, 2^9 or 2^10 classes) is timed alone with CUDA events,
 * and the covers of the steps with the least measured time replace the byte-model choice (mode 0: 'chain' passes,
 * 1: 'prob' / 'sample' passes, 2: both) -- if a whole item, replayed, gets faster; otherwise the previous list
 * stays.  The choice survives gsb_set_matrices; gsb_set_fusion discards it.  ms_before / ms_after (may be NULL):
 * device time of one item of each tuned list before and after (summed for mode 2).  No counterpart in the
 * reference. */
int gsb_autotune(gsb_engine *e, int mode, int reps, float *ms_before, float *ms_after);
/* Pass structure of 'chain' mode: group_len[k] = number of steps of the pass starting at step k (0 inside a pass);
 * entries[k] (may be NULL) = table entries the pass reads plus writes. */
int gsb_fusion_groups(const gsb_engine *e, int *group_len, double *entries);
/* The same for the sampling passes ('prob' / 'sample'): group_len[k] = steps written by the pass starting at step k;
 * entries[k] = table entries it reads plus writes, including the norm pass launched before it where it has one. */
int gsb_sample_groups(const gsb_engine *e, int *group_len, double *entries);
/* The passes of one mode (0 'chain', 1 'prob' / 'sample') in launch order: pass i starts at step k0[i], writes d[i]
 * steps, also evaluates the branch norms of step k0[i] + d[i] when tr[i] = 1, and is a fused k_group pass when
 * fused[i] = 1 (otherwise a single-step pass, after its own norm pass in sampling mode).  *count receives the number
 * of passes; at most cap entries are written (the arrays may be NULL when cap = 0).  No counterpart in the reference:
 * it shows this executor's pass lists (as built, autotuned or set by gsb_set_fusion). */
int gsb_pass_list(const gsb_engine *e, int mode, int cap, int *k0, int *d, int *tr, int *fused, int *count);
/* L2 copy bandwidth of a device in GB/s (bytes read + written): one launch copies an L2-resident buffer of `bytes`
 * (1-64 MiB, a multiple of 16) onto another `reps` times.  The denominator of the L2 roofline reported for the
 * batched launch, whose team tables stay in L2.  No counterpart in the reference (a measurement aid). */
int gsb_probe_l2_copy(int device, uint64_t bytes, int reps, float *gbs);
/* Replace every step's rotation matrix: M is [nsteps][2][2] complex (re, im), M[k][b][x] as the plan text lists
 * it.  The layout stays; this is how one engine (one arena) serves all slice plans of make_sliced_plans, which
 * share the layout and differ only in M (sliced_plans.py:1-14). */
int gsb_set_matrices(gsb_engine *e, const double *M);
/* Arithmetic of a complex64 engine's wide-step kernels (steps of >= 2^11 cosets): 32 (default) sums a coset's
 * entries and rotates them by M in FP32 (norms and scales stay FP64); 64 sums exactly and rotates in FP64, rounding
 * only when storing, which is the reference's complex64 arithmetic (slower: the FP64 pipe becomes the limit).
 * Either way the stored table is complex64.  No effect on a complex128 engine. */
int gsb_set_arith(gsb_engine *e, int bits);

/* Hybrid strings whose first K steps are forced (no counterpart in the reference; K = 0, the default, undoes it).
 * gsb_hybrid then runs those K steps as fused 'chain' passes, the way gsb_chain runs them, and the sampled steps
 * K.. as the reference's run_steps does (gsamp2.cpp:77-98): the same bits, log2 Pr and conditionals, in about the
 * time of one 'chain' string instead of one single-step sweep.  The hybrid driver's proposals have this form (first
 * ND - m data steps drawn on the host, the last m sampled, doped_sampler.py:58-76).  A string with a '?' before
 * step K is refused with GSB_E_PREFIX_FREE.  gsb_prefix and gsb_resume are unchanged. */
int gsb_set_hybrid_prefix(gsb_engine *e, int K);

/* Complex128 re-evaluation of unlikely strings (no counterpart in the reference).  A complex64 log2 Pr carries a
 * rounding error that grows like 1 / sqrt(x), x = Pr * 2^nsteps: the stored table's rounding is absolute in units
 * of its norm, and an unlikely string's amplitude is a small remainder of it.  With a complex128 engine `g` of the
 * same plan (same steps and matrices) attached to the complex64 engine `e`, every string of gsb_chain, gsb_prob,
 * gsb_chain_device, gsb_sample, gsb_sample_uniform and gsb_sample_device whose complex64 result has
 * log2 Pr + nsteps < log2_xmin (or is -inf) is evaluated again on `g`, and that result replaces it (a sample keeps
 * its bits; its log2 Pr is re-evaluated).  Both engines must stay open while attached (closing either detaches);
 * g = NULL detaches.  Errors: GSB_E_USAGE when e is not complex64, g not complex128, on another device, already
 * guarding another engine, or of another plan. */
int gsb_set_guard(gsb_engine *e, gsb_engine *g, double log2_xmin);
/* Strings the guard of e re-evaluated since it was set. */
int gsb_guard_evaluations(const gsb_engine *e, int64_t *count);

/* Per-step kernel timing for one forced string: ms_write[k] and ms_norm[k] (0 when a pass does not run) from CUDA
 * events on the engine's stream, mode 0 = 'chain' (one pass per step), 1 = 'prob' (norm + write per step). */
int gsb_profile_steps(gsb_engine *e, const int8_t *bits, int mode, float *ms_write, float *ms_norm);

/* Number of kernel launches one string / sample makes in the given mode (0 chain, 1 prob/sample, 2 hybrid). */
int gsb_launches_per_item(const gsb_engine *e, int mode, int64_t *launches);

/* ---- out-of-place amplitude engine (the reference's dp.cpp, dp.cpp:14-63) ----
 * Plan text as engine.py:5-12 writes it ("m nsteps maxr", then "v r rn rho pivmask nker ker..." per step).  Two
 * tables of 2^maxr entries, complex128 (precision 128) or complex64 storage with FP64 arithmetic (64, the reference's
 * -DDP_FLOAT build). */
typedef struct gsb_dp gsb_dp;
int gsb_dp_open_text(const char *plan_text, size_t len, int precision, int device, gsb_dp **out);
int gsb_dp_close(gsb_dp *d);
int gsb_dp_info(const gsb_dp *d, int *m, int *nsteps, int *maxr);
/* One job (dp.cpp:35-61): out = sum over slices of pre[s] * Z(w[s]); pre is [nslices] complex (re, im), w is
 * [nslices][m] x (w0 re, w0 im, w1 re, w1 im); out is one complex (re, im). */
int gsb_dp_run(gsb_dp *d, int64_t nslices, const double *pre, const double *w, double *out);
/* One out-of-place step on a host table (complex128): new[c'] for c' < 2^rn from old[2^r] with weights
 * wv = (w0 re, w0 im, w1 re, w1 im) (sampler_ref.py:8-23 `extend`, ref.py:18-31). */
int gsb_dp_extend(int r, int rn, uint64_t rho, uint64_t pivmask, int nker, const uint64_t *ker, const double *wv,
                  const double *old_table, double *new_table, int device);
/* gsb_dp_extend for callers that cannot allocate device memory (no counterpart in the reference): it calls no
 * cudaMalloc / cudaFree (which synchronise the device, and fail when another allocator, e.g. a framework's caching
 * allocator, already holds the free HBM).  The old table, the new table and the weights go through a static
 * scratch array in the library's device memory, 2 MiB + 32 B per GPU that loads the library, held until the process
 * exits, so r and rn must be at most 16 (larger tables return GSB_E_USAGE).  The first call on a device looks up the
 * scratch's address (cudaGetSymbolAddress); make that first call before any stream capture.  All calls share the
 * scratch: calls that overlap in time on one device (from several host threads) race and must be serialised by the
 * caller. */
int gsb_dp_extend_static(int r, int rn, uint64_t rho, uint64_t pivmask, int nker, const uint64_t *ker,
                         const double *wv, const double *old_table, double *new_table, int device);

/* ---- adjoint sweep: gradients of log Pr(b) with respect to the step matrices (complex128) ----
 * No counterpart in the reference (it has no differentiation).  The plan text is the in-place plan (its own M
 * values are ignored: every run takes the matrices).  `every` is the checkpoint interval in steps; the segment
 * between two checkpoints is recomputed once during the reverse sweep. */
typedef struct gsb_grad gsb_grad;
int gsb_grad_open_text(const char *plan_text, size_t len, int device, int every, gsb_grad **out);
int gsb_grad_close(gsb_grad *g);
int gsb_grad_info(const gsb_grad *g, int *n, int *nsteps, int *R);
/* M [nsteps][2][2] complex (re, im), step order; bits [nstr][nsteps] in step order.  Outputs: z [nstr] complex, the
 * sweep's final value Z(b) (Pr(b) = 2^-n |Z(b)|^2), and dz [nstr][nsteps][2] complex, dZ/dM_k[b_k][x]. */
int gsb_grad_run(gsb_grad *g, const double *M, const int8_t *bits, int64_t nstr, double *z, double *dz);

/* ---- batched instances: one persistent launch over many plans of uneven width ----
 * No counterpart in the reference (its executor runs one plan per process).  Each instance is an in-place plan
 * (width <= 24); strings are npre prefixes of K[i] bits per instance, each followed by nsuf suffixes of
 * ns_i - K[i] bits (step order): the prefix is evaluated once and every suffix resumes from its table.
 * precision: GSB_C64 (complex64 arena, FP32 sums, FP64 norms and scales) or GSB_C128. */
typedef struct gsb_batch gsb_batch;
int gsb_batch_open(const char *const *plan_texts, const size_t *lens, int ninst, int precision, int device,
                   gsb_batch **out);
int gsb_batch_close(gsb_batch *b);
/* prefix_bits: concatenation over instances of [npre][K[i]]; suffix_bits: of [npre][nsuf][ns_i - K[i]]. */
int gsb_batch_set_strings(gsb_batch *b, const int *K, int npre, int nsuf, const int8_t *prefix_bits,
                          const int8_t *suffix_bits);
/* log2p: concatenation over instances of [npre][nsuf]; ms (may be NULL): device time of the launch. */
int gsb_batch_run(gsb_batch *b, double *log2p, float *ms);
/* Launch shape: threads per CTA, widest instance run by a single warp (narrower ones too), CTAs per SM. */
int gsb_batch_set_shape(gsb_batch *b, int block, int small_R, int per_sm);
int gsb_batch_get_shape(const gsb_batch *b, int *block, int *small_R, int *per_sm);
/* Autotuner: times the candidate shapes on the current strings (reps timed runs each, arenas <= max_bytes) and
 * keeps the fastest; returns it and its mean time. */
int gsb_batch_tune(gsb_batch *b, int reps, size_t max_bytes, int *block, int *small_R, int *per_sm, float *best_ms);

/* Test hook for the fused passes' failure path (no counterpart in the reference): with on = 1 the passes issue no
 * tile loads, so every CTA's bounded wait runs out (about one second); with on = 2 only the odd CTAs are starved
 * (a partial failure: the other CTAs finish their tiles).  A starved CTA records the failure, marks the item dead,
 * counts itself as finished and returns, and the call reports GSB_E_CUDA.  Nothing faults or hangs and the engine
 * stays usable; with on = 0 the passes run normally again.  Other values: GSB_E_USAGE. */
int gsb_test_withhold_tile_loads(gsb_engine *e, int on);

/* ---- host-side helpers (no GPU needed) ---- */

/* Parse and validate a plan without allocating anything on a device: the same checks gsb_open_* makes
 * (reference parse gsamp2.cpp:128-139; layout invariants inplace.py:85-88, 131-137). */
int gsb_validate_text(const char *plan_text, size_t len, int *n, int *nsteps, int *R);

/* Cut-rank profile of a linear order of the graph A (n x n 0/1, row-major, n <= 128): prof[k-1] = rank over GF(2) of
 * A[order[0..k-1], order[k..n-1]] for k = 1..n-1 (reference order.py:14-20). */
int gsb_cut_profile(int n, const uint8_t *A, const int *order, int *prof);

/* Heuristic order search (randomised greedy + local search on the key (max cut rank, steps at the max, log2 sum
 * 2^r), as the reference's order2.py:16-28 / frontier_instance.py:29-37): best order found and its width. */
int gsb_order_search(int n, const uint8_t *A, uint64_t seed, int ngreedy, int64_t iters, int *order_out, int *width_out);

#ifdef __cplusplus
}
#endif
#endif
