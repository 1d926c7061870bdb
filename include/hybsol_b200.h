/*
 * hybsol_b200.h - C ABI of the B200-native block-sparse LU (decompose + solve).
 *
 * A drop-in for the hot path of j4nr0th/hybridized-solver: the reference's
 * `BlockSystem.decompose()` / `BlockSystem.solve()` (src/block_system.c:1143-1335),
 * whose core is the hidden-visibility "block_system interface" of src/blocks.h:65-131.
 * That interface is not exported by the reference (MODULE_INTERNAL, src/module.h:3-5);
 * the entry points below are the exported equivalents a binding calls instead. The
 * package's CPython extension `hybsol._mod` binds exactly these.
 *
 * Conventions
 *  - Plain C types only: no CUDA or torch types cross this boundary.
 *  - Block-CSR patterns: `row_ptr[n+1]`, `cols[row_ptr[n]]`, columns strictly ascending in
 *    each row, every row holding its diagonal block. Block (r, c) is `sizes[r] x sizes[c]`
 *    and its values are row-major; a value array holds the blocks in CSR order.
 *  - Dense vectors are `dof x nrhs`, row-major (C-contiguous `(dof, nrhs)`; nrhs = 1 is the
 *    reference's 1-D vector).
 *  - Every call returns a `hyb_status` (0 = success). The first four codes are the
 *    reference's `result_t` (src/module.h:67-73) with the same values.
 *  - One handle is used by one host thread at a time (the reference has no per-object
 *    lock either, src/block_system.c); its device work is ordered on the handle's stream.
 */
#ifndef HYBSOL_B200_H
#define HYBSOL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HYB_API __attribute__((visibility("default")))

typedef enum
{
    HYB_SUCCESS = 0,             /* RESULT_SUCCESS */
    HYB_BLOCK_NOT_IN_SYSTEM = 1, /* RESULT_BLOCK_NOT_IN_SYSTEM */
    HYB_FAILED_ALLOC = 2,        /* RESULT_FAILED_ALLOC (host or device memory) */
    HYB_MAX_COLORS = 3,          /* RESULT_MAX_COLORS */
    HYB_INVALID_ARGUMENT = 16,   /* bad index, size, pattern or pointer */
    HYB_MISSING_DIAGONAL = 17,   /* a row has no diagonal block */
    HYB_NOT_DECOMPOSED = 18,     /* solve/factor access before decompose */
    HYB_CUDA_ERROR = 19,         /* a CUDA runtime call failed (see hyb_last_cuda_error) */
    HYB_NO_DEVICE = 20,          /* no usable sm_100 device */
    HYB_ZERO_PIVOT = 21,         /* a diagonal-block pivot was exactly zero */
    HYB_NON_FINITE = 22,         /* a pivot or factor entry is inf/nan */
    HYB_NOT_CONVERGED = 23,      /* iterative refinement missed its tolerance */
    HYB_TOO_LARGE = 24,          /* request beyond a documented size limit */
    HYB_DEVICE_TIMEOUT = 25      /* a bounded device-side wait ran out (the work was abandoned;
                                    the context stays usable) */
} hyb_status;

typedef enum
{
    HYB_PRECISION_FP64 = 0, /* plain form: FP64 factors and solves (the drop-in) */
    HYB_PRECISION_MIXED = 1 /* FP32 factors (BF16x3 tensor-core updates) + FP64 refinement */
} hyb_precision;

typedef enum
{
    HYB_ORDERING_FIRST = 0, /* src/blocks.c:918 block_system_compute_ordering_first */
    HYB_ORDERING_GREEDY = 1, /* src/blocks.c:966 block_system_compute_ordering_greedy */
    HYB_ORDERING_BALANCED = 2 /* src/blocks.c:1054 block_system_compute_ordering_balanced */
} hyb_ordering_strategy;

typedef enum
{
    HYB_MEMORY_HOST = 0,  /* pointer is host memory (pageable or pinned) */
    HYB_MEMORY_DEVICE = 1 /* pointer is device memory of the handle's device */
} hyb_memory;

typedef struct hyb_system hyb_system;

typedef struct
{
    uint64_t n_levels;         /* stages of the dependency schedule */
    uint64_t filled_blocks;    /* stored blocks after fill */
    uint64_t factor_values;    /* scalars in the factors (unpadded) */
    double factor_flops;       /* exact algorithmic flops of the factorization */
    uint64_t zero_pivots;      /* diagonal pivots that were exactly zero */
    uint64_t non_finite;       /* diagonal pivots that came out inf/nan */
    int64_t first_bad_pivot;   /* lowest block row with a bad pivot, -1 if none */
    uint64_t growth_fp64;      /* mixed form: pivots whose FP32 LU grew past HYB_OPTION_GROWTH_LIMIT and were
                                  refactored (LU and row solve) in FP64 */
    uint64_t growth_kept;      /* mixed form: pivots past the limit whose size has no FP64 path (more than 64
                                  rows, or too large for shared memory), kept in FP32 */
} hyb_decompose_info;

typedef struct
{
    uint32_t iterations;         /* refinement steps taken: corrections applied (0 for the plain form) */
    double relative_residual;    /* max over columns (and segments) of ||b - A x||_2 / ||b||_2 (FP64), -1 if not computed */
    uint32_t krylov_iterations;  /* of `iterations`, the FGMRES steps (see HYB_OPTION_REFINEMENT) */
} hyb_solve_info;

/* Library ----------------------------------------------------------------------- */

HYB_API const char *hyb_status_string(int status);
HYB_API const char *hyb_last_cuda_error(void);
HYB_API int hyb_version(void);
/* Non-zero when a device of compute capability 10.x is visible. */
HYB_API int hyb_device_available(void);

/* Ordering (host, integer, bit-exact) -------------------------------------------- */

/* Coloring ordering of a block-CSR pattern: `ordering[i]` is the new index of block i.
 * Replaces block_system_compute_ordering_{first,greedy,balanced} + order_from_colors
 * (src/blocks.c:802-1141) as called by compute_reordering (src/block_system.c:1693-1788).
 * `max_colors` = 0 means "the largest row length" (src/block_system.c:1725-1733). */
HYB_API int hyb_compute_ordering(uint64_t n, const uint64_t *row_ptr, const uint64_t *cols, int strategy,
                                 uint64_t max_colors, uint64_t *ordering);

/* Host-only symbolic analysis ---------------------------------------------------- */

typedef struct
{
    uint64_t filled_blocks;   /* blocks after fill */
    uint64_t factor_values;   /* scalars after fill (unpadded) */
    uint64_t n_levels;        /* stages of the dependency schedule */
    uint64_t nops;            /* operations() entries: lower blocks + block rows */
    uint64_t slab_bytes_fp64; /* device bytes of the FP64 factor slab (blocks padded to 256 B) */
    double factor_flops;      /* exact algorithmic flops of the factorization */
    uint64_t pair_levels;     /* pairs of consecutive single-pivot, uniform-64 levels the mixed form can
                                 apply in one two-pivot pass (HYB_OPTION_PAIR_PASSES) */
} hyb_analysis;

/* Runs the symbolic phase on the host alone (no GPU needed): the fill the reference's
 * elimination creates (src/blocks.c:557-727 in the order of src/blocks.c:360-514), the
 * schedule statistics, and optionally the filled pattern (`filled_row_ptr[n+1]`,
 * `filled_cols[filled_blocks]`) and the operation list in the reference's single-thread
 * order (`ops[2*nops]`, as hyb_operations). Pass NULL arrays to query the sizes first. */
HYB_API int hyb_analyze(uint64_t n, const uint64_t *block_sizes, const uint64_t *row_ptr, const uint64_t *cols,
                        hyb_analysis *out, uint64_t *filled_row_ptr, uint64_t *filled_cols, int64_t *ops);

/* System lifecycle ---------------------------------------------------------------- */

/* Creates a system on the current CUDA device with a fixed block pattern and runs the
 * symbolic phase: the fill of the reference's elimination (src/blocks.c:557-727 applied
 * in the order of src/blocks.c:360-514), the dependency levels and the per-level work
 * lists. Replaces BlockSystem(*sizes) + add_block pattern building
 * (src/block_system.c:59-134, src/blocks.c:3-75). Values start at zero. */
HYB_API int hyb_system_create(uint64_t n, const uint64_t *block_sizes, const uint64_t *row_ptr,
                              const uint64_t *cols, hyb_system **out);
HYB_API int hyb_system_destroy(hyb_system *sys);
/* Deep copy (pattern, values, factors, op list): BlockSystem.copy (src/block_system.c:1343-1444). */
HYB_API int hyb_system_copy(const hyb_system *sys, hyb_system **out);

/* Loads the values of the original pattern (CSR order). Clears any decomposition, so
 * the same handle can be factored again with new values (a refactorization). */
HYB_API int hyb_system_set_values(hyb_system *sys, const double *values, int memory);
/* Size of the value array hyb_system_set_values expects (scalars). */
HYB_API uint64_t hyb_system_value_count(const hyb_system *sys);
/* Total unknowns (sum of block sizes). */
HYB_API uint64_t hyb_system_dof(const hyb_system *sys);
/* The handle's CUDA stream (a cudaStream_t as void*), for callers that time or order work. */
HYB_API void *hyb_system_stream(const hyb_system *sys);

typedef enum
{
    /* 1 (default): between consecutive single-pivot stages, factor the next pivot on a
     * second stream while the current stage's update finishes; 0: strictly in order.
     * Both give the same factors. */
    HYB_OPTION_LOOKAHEAD = 0,
    /* 1 (default): in the mixed form, the 64x64 Schur updates run on the tcgen05 tensor
     * cores as three BF16 products of a hi/lo split; 0: FP32 CUDA-core updates. */
    HYB_OPTION_TENSOR_CORE_MIXED = 1,
    /* 1 (default): hyb_solve substitutes in one cooperative launch per direction, each
     * pivot proceeding as soon as its sources are final; 0: one launch per elimination
     * stage. Both give the same solution. */
    HYB_OPTION_DATAFLOW_SOLVE = 2,
    /* Time limit, in nanoseconds, of each wait of the dataflow solve for a source row
     * (default 1e9). A wait that runs out abandons the solve, which then returns
     * HYB_DEVICE_TIMEOUT. Values below 1e5 are raised to 1e5. */
    HYB_OPTION_WAIT_LIMIT_NS = 3,
    /* Fault injection on the host, for testing the timeout path (-1, the default, turns it
     * off): in the next dataflow solves the partial sums of block row `value` are never
     * released, so the waits for that row run out. The row must have at least two blocks
     * left of its diagonal. */
    HYB_OPTION_WITHHOLD_ROW = 4,
    /* How hyb_solve refines (mixed form, or the plain form with HYB_OPTION_FP64_REFINEMENT):
     * 0 (default) iterative refinement x += LU^{-1} (b - A x) while each step shrinks the
     * FP64 residual at least tenfold, then -- from the best iterate -- restarted FGMRES in
     * FP64 preconditioned by the factors, which converges where plain refinement stalls
     * (condition number x growth x factor precision near or above 1); 1 refinement only;
     * 2 FGMRES from the first correction. Every step (a refinement step or an FGMRES
     * iteration) costs one substitution with the factors. */
    HYB_OPTION_REFINEMENT = 5,
    /* 1: the plain FP64 form refines too (with its FP64 factors, as above), for systems
     * whose plain FP64 solve misses the tolerance; 0 (default): the drop-in plain solve. */
    HYB_OPTION_FP64_REFINEMENT = 6,
    /* FGMRES restart length (Krylov vectors kept, 1..200, default 30). */
    HYB_OPTION_KRYLOV_RESTART = 7,
    /* Mixed form: growth limit of a diagonal pivot block, max|U_d| / max|D| of its FP32 LU
     * (default 1024; 0 turns the check off). A pivot above it is refactored in FP64 -- its
     * LU and the solves of its row's upper blocks, stored back in FP32 -- so the elimination
     * steps that amplify rounding most are the ones kept in FP64. Pivots of at most 32 rows
     * and of 33-64 rows have this path; larger ones are counted in growth_kept. */
    HYB_OPTION_GROWTH_LIMIT = 8,
    /* Mixed form: 1 (default) factors the block-diagonally scaled S A S, s_k = 1 /
     * sqrt(max |A_kk|) for every unknown of block row k, so each diagonal block enters the
     * FP32 / BF16-split factorization with entries of order one; the solves apply S on both
     * sides and the refinement's residual stays that of the unscaled FP64 A. hyb_get_block
     * then returns the scaled factors. 0: the factors of A itself. */
    HYB_OPTION_BLOCK_SCALING = 9,
    /* 1 (default): the Schur updates of 64-blocks walk their targets backwards on every
     * other level, so each level starts on the targets the previous one wrote last (still in
     * L2); 0: always forwards. Both give the same factors. */
    HYB_OPTION_ALTERNATE_WALK = 10,
    /* Schur updates of levels whose blocks are not all 64 wide (uneven orders): -1
     * (default) tunes the kernel per size bucket (pivot size and largest target dimension,
     * each rounded up to 8, 16, ..., 256) at the first factorization that meets the bucket,
     * timing every kernel that fits on the bucket's largest level, and keeps the fastest;
     * 0: 32x32 SIMT tiles; 1: 64x64 SIMT tiles; 2: the FP64 tensor pipe (DMMA, pivots up
     * to 128 rows, FP64 products also for FP32 factors). A kernel that does not fit a level
     * falls back to the tuned or default choice. */
    HYB_OPTION_UPDATE_KERNEL = 11,
    /* Pivots of 33-64 rows: 1 factors each diagonal block once and then solves its row's
     * upper blocks from the stored factors (two launches); 0: one fused launch in which every
     * CTA of a pivot factors the block itself before its strip; -1 (default): 1 for the FP64
     * form (its LU is costly and the redundant copies slow the concurrent update), 0 for the
     * mixed form (its FP32 LU is cheap and the extra launch lengthens the pivot chain). All
     * give the same factors. */
    HYB_OPTION_PIVOT_LU_ONCE = 12,
    /* FP64 MMA instruction shape of the FP64 form's 64-block Schur update: 0 m8n8k4,
     * 1 (default) m16n8k8, 2 m16n8k16. The same products, summed in different groups inside
     * an instruction (FP64 factors agree to rounding). */
    HYB_OPTION_FP64_MMA_SHAPE = 13,
    /* Mixed form: 1 (default) applies consecutive single pivots in pairs where the pattern allows
     * (the second pivot lies in the first one's lower column and upper row, and the first
     * one's other lower rows and upper columns are among the second one's): the first
     * pivot's update of the second one's row and column runs on the pivot chain, and one
     * tensor-core pass then applies both pivots to the second one's targets (K = 128), so
     * each target is read and written once for two pivots; on the inverse-and-products path
     * (HYB_OPTION_ROW_PIVOTS 2) the first pivot's update of the second one's row and column
     * is applied by the products launch. 2: the same with that update as its own launch.
     * 0: one pass per pivot. The factors differ
     * only by FP32 rounding (the two products are summed in the accumulator before they are
     * subtracted). */
    HYB_OPTION_PAIR_PASSES = 14,
    /* Levels whose pivots and upper blocks are all 64x64: 1 factors each diagonal block
     * with a blocked LU (eight-column panels by one warp, rank-8 updates by the CTA) and
     * solves the upper blocks in 8x8 blocks, writing the mixed form's operand splits beside
     * it (the same operations in the same order as 0: the same factors); 0: the 256-thread
     * unblocked kernels (HYB_OPTION_PIVOT_LU_ONCE); 2 (mixed form, tensor-core levels):
     * each pivot is factored once and inverted (blocked triangular inverses), and its
     * upper blocks are taken as products with the inverse, so the pivot's critical path
     * holds no substitution (FP32 factors that differ from 0 and 1 by rounding); -1
     * (default): 2 for the mixed form, 0 for the FP64 form. */
    HYB_OPTION_ROW_PIVOTS = 15,
    /* Mixed form, two-pivot passes: SMs the main update launch leaves free for the next
     * unit's pivot work, which runs beside it (default 4, at most 64). The pivot chain is
     * latency-bound; beside an update CTA it runs about twice as slowly as on a free SM.
     * Measured at 128x128 p=8 on one B200: factorization 1,561 ms with 0, 1,350 ms with 4,
     * 1,364 ms with 8, 1,383 ms with 16. The factors do not depend on it. */
    HYB_OPTION_UPDATE_SM_RESERVE = 16
} hyb_option;

/* Sets a schedule option of the handle (takes effect at the next decomposition). */
HYB_API int hyb_system_set_option(hyb_system *sys, int option, int64_t value);

/* The tuned generic update kernel per size bucket (HYB_OPTION_UPDATE_KERNEL) of the given
 * precision: `kinds[bucket]` for the 49 buckets (pivot class x 7 + target class, classes
 * 8, 16, 32, 64, 128, 256, larger), -1 where no level of that bucket was tuned. */
HYB_API int hyb_tuned_kernels(const hyb_system *sys, int precision, int32_t kinds[49]);

/* Declares the system to be `nseg` independent systems stacked block-diagonally, segment s
 * holding the unknowns [offsets[s], offsets[s+1]) (offsets[0] = 0, ascending, offsets[nseg]
 * = dof). No counterpart in the reference. Refinement (mixed form, or the plain form with
 * HYB_OPTION_FP64_REFINEMENT) then measures every segment's residual against its own
 * right-hand side and iterates until each segment of each column meets the tolerance, so
 * one badly scaled or ill-conditioned member of a batch is not declared converged by the
 * norm of the whole stack. nseg = 0 removes the segmentation. */
HYB_API int hyb_system_set_segments(hyb_system *sys, uint64_t nseg, const uint64_t *offsets);

/* After hyb_solve on a segmented system, per segment and column (nseg x nrhs, row-major):
 * the refinement steps after which its relative residual was first measured at or below
 * the tolerance (UINT32_MAX if never) and its final relative residual ||b_s - (A x)_s|| /
 * ||b_s|| (FP64). Either array may be NULL. */
HYB_API int hyb_segment_results(const hyb_system *sys, uint32_t *iterations, double *relative_residual);

/* Decomposition and solve -------------------------------------------------------- */

/* Factors the system in the given precision: replaces block_system_decompose
 * (src/blocks.c:360-514; binding src/block_system.c:1143-1187). The plain form computes
 * the reference's factors (unpivoted; U with identity diagonal blocks, diagonal blocks
 * holding their own Doolittle LU, lower blocks the Schur-complemented A) to rounding.
 * A zero pivot is not an error, as in the reference (the factor gets inf/nan); it is
 * counted in `info`. `info` may be NULL. */
HYB_API int hyb_decompose(hyb_system *sys, int precision, hyb_decompose_info *info);

/* Solves A x = b for `nrhs` right-hand sides: replaces block_system_apply_operations +
 * block_system_solve_u (src/blocks.c:729-800; binding src/block_system.c:1259-1335).
 * `b` and `x` may alias. In the mixed form the solve iterates refinement until
 * ||b - A x|| / ||b|| <= tol (FP64 residual against the original A) or `max_iter` steps;
 * tol <= 0 selects 1e-12. In the plain form tol/max_iter are ignored and the residual is
 * only computed when `info` is non-NULL and `tol` > 0. Returns HYB_NOT_CONVERGED (with
 * x holding the last iterate) when refinement misses the tolerance. */
HYB_API int hyb_solve(hyb_system *sys, const double *b, double *x, uint64_t nrhs, int memory, double tol,
                      uint32_t max_iter, hyb_solve_info *info);

/* FP64 residual r = b - A x against the original values (device or host vectors). */
HYB_API int hyb_residual(hyb_system *sys, const double *b, const double *x, double *r, uint64_t nrhs, int memory);

/* Solves A^T x = b with the FP64 factors (HYB_PRECISION_FP64; HYB_NOT_DECOMPOSED otherwise).
 * No counterpart in the reference, whose factors only solve with A: with A = L U, A^T =
 * U^T L^T, a forward pass with the transposed upper blocks (unit diagonal blocks) and a
 * backward pass with the transposed lower blocks and diagonal-block LUs, level by level.
 * `b` and `x` may alias. */
HYB_API int hyb_solve_transpose(hyb_system *sys, const double *b, double *x, uint64_t nrhs, int memory);

typedef struct
{
    double kappa1;    /* norm1 * inv_norm1: estimate of the 1-norm condition number */
    double norm1;     /* ||A||_1 of the original values (exact: largest column sum of |a|) */
    double inv_norm1; /* estimate of ||A^{-1}||_1 (a lower bound, usually within a small factor) */
    uint32_t solves;  /* solves with A and A^T the estimate took */
} hyb_condition;

/* 1-norm condition estimate of the original matrix from its FP64 factors: Hager's method
 * with Higham's refinements (the scheme of LAPACK's xLACN2: at most five sign-vector
 * iterations, each a solve with A and one with A^T, plus one alternating test vector).
 * No counterpart in the reference. Requires HYB_PRECISION_FP64 factors. */
HYB_API int hyb_condition_estimate(hyb_system *sys, hyb_condition *out);

/* Allocation-free FP64 solve. No counterpart in the reference: it exists for callers that
 * must not allocate device memory when they solve -- for example a host application
 * whose own memory pool already holds the device memory it may use (a cudaMalloc there
 * fails or breaks its budget), or a time-stepping loop that cannot afford the device-wide
 * synchronization cudaMalloc/cudaFree imply. Such a caller creates and factors the
 * handle (HYB_PRECISION_FP64) up front and then calls this entry point, which performs
 * no allocation of any kind: `b` and `x` are the caller's device buffers (dof x nrhs,
 * row-major; they may alias) and the solve's scratch for partial block products lives in
 * a fixed array inside this library, HYB_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB) that every
 * GPU which loads the library keeps until the process exits. Requests whose scratch would
 * exceed it (per stage: pivot rows x lower blocks x nrhs) are rejected with HYB_TOO_LARGE.
 * The first call on a device looks up that array's device address (once per device, with
 * the device current); make that first call before any stream capture. All calls share
 * the one array: calls that overlap on the GPU -- from two threads, or on two handles of
 * the same device -- race on it. `x` either is `b` or does not overlap it at all (a partial
 * overlap returns HYB_INVALID_ARGUMENT). The looked-up address belongs to the device's
 * current context: after cudaDeviceReset the library must be reloaded before this entry
 * point is used again on that device. The call returns after the solve has finished on the
 * handle's stream. The results equal hyb_solve's bit for bit for the same factors. */
#define HYB_NOALLOC_SCRATCH_DOUBLES (1u << 20)
HYB_API int hyb_solve_fp64_noalloc(hyb_system *sys, const double *b, double *x, uint64_t nrhs);

/* Access after decomposition ------------------------------------------------------ */

/* Number of blocks in row `row` of the filled pattern (before decomposition: original). */
HYB_API int hyb_row_count(const hyb_system *sys, uint64_t row, uint64_t *count);
/* Column indices of row `row` (get_row_block_indices, src/block_system.c:312-349). */
HYB_API int hyb_row_cols(const hyb_system *sys, uint64_t row, uint64_t *cols);
/* Copies block (row, col) to host memory as FP64 (get_block, src/block_system.c:364-396):
 * the factor after decomposition, the loaded value before. */
HYB_API int hyb_get_block(const hyb_system *sys, uint64_t row, uint64_t col, double *out);
/* Operation list in the reference's single-thread order (operations(),
 * src/block_system.c:1198-1254; order of src/blocks.c:360-514 with one thread):
 * ops[2i] = row, ops[2i+1] = source column or -1 for INVDIA. Call with ops = NULL to get
 * the count. */
HYB_API int hyb_operations(const hyb_system *sys, uint64_t *nops, int64_t *ops);
/* Kernel launches issued by the last hyb_decompose / hyb_solve call (counted on the host). */
HYB_API uint64_t hyb_last_launch_count(const hyb_system *sys);

/* Profiling (no counterpart in the reference, which has no tracing) ------------- */

typedef struct
{
    uint64_t launches; /* update passes whose Schur-update kernels were timed (one level, or a
                          pair of levels applied in one two-pivot pass, HYB_OPTION_PAIR_PASSES) */
    double total_ms;   /* sum of their device durations (CUDA events on the handle's stream) */
    double flops;      /* algorithmic flops they performed */
    double c_elems;    /* target scalars each read and written once */
    double ab_elems;   /* operand scalars (lower-column and upper-row blocks) */
    uint64_t levels;   /* levels of the decomposition that have a Schur update, timed or not */
    uint64_t passes;   /* update passes of the decomposition, timed or not (a pair counts once) */
    uint64_t pivots_timed; /* levels covered by the timed passes */
    double pivot_ms;       /* device time of the timed units' pivot work: LU, row solves, operand
                              splits and, for a pair, the first pivot's update of the second one's
                              row and column (CUDA events on the stream that runs it) */
    uint64_t pivot_units;  /* units whose pivot work was timed */
    uint64_t pivot_levels; /* levels they cover */
} hyb_kernel_profile;

/* With stride n >= 1, later decompositions record CUDA events around the Schur-update
 * kernels of every n-th level that has an update (n = 1: all of them) inside the
 * factorization graph; 0 turns this off. Each event pair adds a few microseconds to the
 * stage it brackets, so a stride of 16 or more keeps a timed run within about 1% of an
 * untimed one. hyb_profile_read returns the totals of the timed levels of the last
 * decomposition. */
HYB_API int hyb_profile_enable(hyb_system *sys, int stride);
HYB_API int hyb_profile_read(const hyb_system *sys, hyb_kernel_profile *update);

/* Dense single-block kernels on device (the fine-grained surface of
 * src/block_system.c:938-1141) -------------------------------------------------- */

/* In-place unpivoted LU of an m x m row-major block (matrix_lu_decompose, src/blocks.c:254-283). */
HYB_API int hyb_block_lu(uint64_t m, double *a, int memory);
/* out = LU^{-1} b for an m x ncols block (matrix_lu_solve, src/blocks.c:285-316); b may alias out. */
HYB_API int hyb_block_lu_solve(uint64_t m, const double *lu, uint64_t ncols, const double *b, double *out,
                               int memory);
/* Row-major block product: c = a * b (subtract = 0, matrix_multiply, src/blocks.c:200-222) or
 * c -= a * b (subtract = 1, matrix_multiply_sub_inplace, src/blocks.c:224-244); a is m x k,
 * b is k x n, c is m x n and must not alias a or b. */
HYB_API int hyb_block_gemm(uint64_t m, uint64_t k, uint64_t n, const double *a, const double *b, double *c,
                           int subtract, int memory);

/* The products of one row elimination (block_system_eliminate_row, src/blocks.c:557-727)
 * in one call: c[i] = a * b[i] or c[i] -= a * b[i] for i < count, a m x k, b[i] k x n[i],
 * c[i] m x n[i], all row-major; every c[i] distinct from a and the b's. With host memory
 * the operands travel in one copy each way. */
HYB_API int hyb_block_gemm_batched(uint64_t count, uint64_t m, uint64_t k, const uint64_t *n, const double *a,
                                   const double *const *b, double *const *c, int subtract, int memory);
/* The solves of one row's upper blocks with its factored diagonal block
 * (block_system_apply_diagonal_inverse, src/blocks.c:516-539): b[i] <- LU^{-1} b[i] in place,
 * b[i] m x n[i]. */
HYB_API int hyb_block_lu_solve_batched(uint64_t m, const double *lu, uint64_t count, const uint64_t *n,
                                       double *const *b, int memory);
/* The hyb_block_* calls above stage host operands in a device workspace of the current
 * device that is grown to the largest request and kept until the process exits, so
 * repeated calls allocate nothing; calls from several host threads take turns on it. */

/* Bulk assembly on the device: adds `count` blocks to the handle's values, block i at
 * (rows[i], cols[i]) with its row-major values next in `values` (blocks concatenated in
 * input order; `values` host or device memory). Blocks repeated in the input are summed in
 * input order, as repeated add_block calls (src/blocks.c:36-45) would. Every block must be
 * in the handle's pattern (HYB_BLOCK_NOT_IN_SYSTEM otherwise, and nothing is added). Clears
 * any decomposition, as hyb_system_set_values does. */
HYB_API int hyb_system_add_blocks(hyb_system *sys, uint64_t count, const uint64_t *rows, const uint64_t *cols,
                                  const double *values, int memory);

#ifdef __cplusplus
}
#endif

#endif /* HYBSOL_B200_H */
