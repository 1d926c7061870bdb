/*
 * hyb_oracle.h - CPU restatement of the reference's block-sparse LU, used as the
 * parity ORACLE for the B200 implementation.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the CPU
 * legs of bench.py load this library, and only to check or time against it. The
 * product never links it.
 *
 * Every function restates one piece of j4nr0th/hybridized-solver's C core
 * (`src/blocks.c`, `src/block_system.c`) in plain C with the same arithmetic
 * order, so that (built with -ffp-contract=off) its factors and solutions agree
 * bit-for-bit with the reference compiled on x86-64; the tests pin that against
 * the reference itself (oracle/_ref) and against the committed golden vectors.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Result codes: the reference's result_t (src/module.h:67-73) plus oracle-only ones. */
enum
{
    ORC_SUCCESS = 0,
    ORC_BLOCK_NOT_IN_SYSTEM = 1,
    ORC_FAILED_ALLOC = 2,
    ORC_MAX_COLORS = 3,
    ORC_BAD_ARGUMENT = 100,
    ORC_ALREADY_DECOMPOSED = 101,
    ORC_NOT_DECOMPOSED = 102,
};

/* Ordering strategies of src/blocks.h:58-63. */
enum
{
    ORC_ORDERING_FIRST = 0,
    ORC_ORDERING_GREEDY = 1,
    ORC_ORDERING_BALANCED = 2,
};

typedef struct orc_system orc_system;

orc_system *orc_create(uint64_t n, const uint64_t *block_sizes);
void orc_destroy(orc_system *sys);
orc_system *orc_copy(const orc_system *sys);

uint64_t orc_n_blocks(const orc_system *sys);
uint64_t orc_block_size(const orc_system *sys, uint64_t idx);
uint64_t orc_row_count(const orc_system *sys, uint64_t row);
void orc_row_cols(const orc_system *sys, uint64_t row, uint64_t *cols);
int orc_add_block(orc_system *sys, uint64_t row, uint64_t col, const double *vals);
int orc_get_block(const orc_system *sys, uint64_t row, uint64_t col, double *out);
uint64_t orc_total_blocks(const orc_system *sys);
/* Block-CSR export in row order: row_ptr[n+1], cols[nnz], values concatenated row-major. */
void orc_export(const orc_system *sys, uint64_t *row_ptr, uint64_t *cols, double *values);
uint64_t orc_export_value_count(const orc_system *sys);

/* Dense kernels on row-major buffers. */
void orc_lu_decompose(uint64_t m, double *a);
void orc_lu_solve(uint64_t m, const double *lu, uint64_t ncols, const double *b, double *out);
void orc_matmul(uint64_t m, uint64_t k, uint64_t n, const double *a, const double *b, double *out);

/* Row elimination T <- T - S * R_src for columns > src, with fill (src/blocks.c:557-727). */
int orc_eliminate_row(orc_system *sys, uint64_t tgt, uint64_t src, const double *scale);
void orc_decompose_diagonal(orc_system *sys, uint64_t row);
void orc_apply_diagonal_inverse(orc_system *sys, uint64_t row);

/* Full decomposition with the reference's serial schedule (src/blocks.c:360-514). */
int orc_decompose(orc_system *sys);
uint64_t orc_nops(const orc_system *sys);
/* ops[2*i] = row, ops[2*i+1] = source column, or -1 for an INVDIA operation. */
void orc_get_ops(const orc_system *sys, int64_t *ops);
/* In-place solve of one right-hand side: op replay then back substitution. */
int orc_solve(const orc_system *sys, double *vec);

/* Coloring orderings on a block-CSR pattern (src/blocks.c:802-1141). */
int orc_compute_ordering(uint64_t n, const uint64_t *row_ptr, const uint64_t *cols, int strategy, uint64_t max_colors,
                         uint64_t *ordering);
/* Symmetric permutation of the stored system (src/block_system.c:1449-1644). */
int orc_reorder_blocks(orc_system *sys, const uint64_t *order);

#ifdef __cplusplus
}
#endif
