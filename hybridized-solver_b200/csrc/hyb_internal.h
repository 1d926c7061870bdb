// hyb_internal.h - data structures shared by the host symbolic phase (hyb_symbolic.cpp),
// the orderings (hyb_ordering.cpp) and the device side (hyb_api.cu, hyb_kernels.cuh).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace hyb
{

// Scalars of each block are padded to a multiple of this many elements in the factor
// slab, so every block starts 256-byte aligned in FP64 and 128-byte aligned in FP32.
constexpr int64_t kBlockAlign = 32;

// Result of the symbolic phase: the reference's elimination replayed on the block
// pattern alone. Everything the device schedule needs is precomputed here.
struct Symbolic
{
    int64_t n = 0;                 // block rows/columns
    std::vector<int32_t> size;     // [n] block sizes
    std::vector<int64_t> dof_off;  // [n+1] scalar offsets of block rows

    // Original pattern (block-CSR) and where each original block lands after fill.
    std::vector<int64_t> a_row_ptr; // [n+1]
    std::vector<int32_t> a_cols;    // [nnzA]
    std::vector<int64_t> a_val_off; // [nnzA+1] unpadded value offsets (CSR order)
    std::vector<int32_t> a_to_f;    // [nnzA] filled block index of each original block

    // Filled pattern: rows hold their original blocks plus the fill of the elimination.
    std::vector<int64_t> row_ptr;  // [n+1]
    std::vector<int32_t> cols;     // [nnzF] ascending within a row
    std::vector<int64_t> diag_pos; // [n] index (into cols) of the diagonal block of each row
    std::vector<int64_t> blk_off;  // [nnzF+1] padded element offset of each block in the slab

    // Strictly lower part by column: lcol_row[j], lcol_blk[j] for j in
    // [lcol_ptr[k], lcol_ptr[k+1]) are the rows t > k holding block (t, k), ascending.
    std::vector<int64_t> lcol_ptr; // [n+1]
    std::vector<int32_t> lcol_row;
    std::vector<int32_t> lcol_blk;

    // Dependency levels: the pivots of level l are piv[lvl_ptr[l] .. lvl_ptr[l+1]), ascending.
    // A pivot depends on every earlier pivot whose row or column reaches it, so within a
    // level no pivot reads or writes another's row or column.
    int64_t n_levels = 0;
    std::vector<int32_t> level;     // [n] level of each block row
    std::vector<int64_t> lvl_ptr;   // [L+1]
    std::vector<int32_t> piv;       // [n]
    std::vector<int64_t> trsm_pref; // [n+1] prefix (in piv order) of upper-block counts
    std::vector<int64_t> lu_pref;   // [n+1] prefix of max(1, upper-block count): fused LU+solve units
    std::vector<int64_t> upd_pref;  // [n+1] prefix of |lower column| * |upper row|
    std::vector<int64_t> upd2_pref; // [n+1] prefix of ceil(|lower column| / 2) * |upper row| (row pairs)
    std::vector<int64_t> split_pref; // [n+1] prefix of n_lc + n_up: blocks whose BF16 split a tensor-core level stages
    std::vector<int64_t> tc_pref;    // [n+1] prefix of n_lc * ceil(n_up / 2): tensor-core update tiles
    std::vector<int64_t> fwd_pref;  // [n+1] prefix of lower-row block counts
    std::vector<int64_t> fwdu_pref; // [n+1] prefix of max(1, lower-row block count): forward solve units
    std::vector<int32_t> fwd_item_p; // [fwdu_pref[n]] pivot slot of each forward dataflow item
    std::vector<int32_t> bwd_item_p; // backward dataflow items (levels descending, max(1, n_up) per pivot)
    std::vector<int64_t> bwd_first;  // [n] first backward item of each pivot slot
    std::vector<int64_t> fwd_rows;  // [n+1] prefix of lower-row block count * pivot size, padded to 4 (scratch rows)
    std::vector<int64_t> bwd_rows;  // [n+1] prefix of upper-row block count * pivot size, padded to 4
    std::vector<int32_t> inv_idx;   // [n] slot of a 64-row block row's FP32 diagonal inverse (-1: other sizes)
    std::vector<int32_t> inv_row;   // [n_inv] block row of each inverse slot
    int64_t n_inv = 0;              // block rows of 64

    // Levels whose pivots share target rows get explicit target lists, each target's
    // sources in ascending pivot order (a fixed order, no atomics).
    std::vector<uint8_t> lvl_listed; // [L] 1 if the level's update is listed
    std::vector<int64_t> mt_lvl_ptr; // [L+1] into the target list
    std::vector<int32_t> mt_tgt;     // filled block index of each target
    std::vector<int32_t> mt_row;     // target block row
    std::vector<int32_t> mt_col;     // target block column
    std::vector<int64_t> mt_src_ptr; // [targets+1]
    std::vector<int32_t> mt_src_k;   // pivot of each source
    std::vector<int32_t> mt_src_l;   // filled block (t, k)
    std::vector<int32_t> mt_src_u;   // filled block (k, c)

    // Per-level shape summary used to pick kernels and launch sizes.
    struct LevelShape
    {
        int32_t max_piv = 0;  // largest pivot block
        int32_t max_row = 0;  // largest target row block
        int32_t max_col = 0;  // largest target column block
        int32_t max_up = 0;   // largest upper-block column size of a pivot row
        bool uniform64 = false; // every pivot, target row and column block is 64
        bool piv64 = false;     // every pivot and every upper block of its row is 64 wide
        double upd_flops = 0;   // algorithmic flops of the level's Schur updates
        double upd_c_elems = 0; // scalars of the update targets (each read and written once)
        double upd_ab_elems = 0; // scalars of the lower-column and upper-row operand blocks
        // Lookahead: when this level and the next each have one pivot and this level's
        // update reaches the next pivot's row or column, the update is split into the
        // targets in that row/column (la_i0: position of the next pivot in this pivot's
        // lower column, la_j0: in its upper row; -1 if absent) and the rest, so the next
        // pivot can be factored while the rest runs.
        bool lookahead = false;
        int32_t la_i0 = -1;
        int32_t la_j0 = -1;
        int64_t la_prio_units = 0;
        int64_t la_rest_units = 0;
        int64_t la_prio_pairs = 0; // units of the two-row kernels: row i0 one row at a time, column j0 in pairs
        int64_t la_rest_pairs = 0; // row-pair units of the rest (kernels that take two target rows)
        int64_t la_prio_tiles = 0; // tensor-core tiles (one target row x two columns): row i0, then column j0
        int64_t la_rest_tiles = 0; // tensor-core tiles of the rest
    };
    std::vector<LevelShape> shape;

    // Two pivots per update pass (mixed form, tensor-core levels). Levels l and l+1 form a
    // pair when each has one pivot (a, then b), both are uniform-64 and unlisted, b lies in
    // a's lower column and upper row, and a's other lower rows and upper columns are among
    // b's. The pair's targets are then exactly b's (every one receives b's product, and
    // a's where a reaches it), so one pass over b's targets applies both pivots with
    // K = 128. a's update of b's own row and column is done first, on the pivot chain.
    struct PairShape
    {
        // lookahead into the next unit (the level after the pair, and the one after that
        // when those two form a pair too): positions of its pivots c, d in b's lower column
        // (i0, i1) and upper row (j0, j1), ascending, -1 where absent
        bool lookahead = false;
        int32_t i0 = -1, i1 = -1, j0 = -1, j1 = -1;
        int64_t all_tiles = 0;  // one target row x two columns, every target of b
        int64_t prio_tiles = 0; // rows i0, i1 x column pairs, then columns (j0, j1) for every other row
        int64_t rest_tiles = 0; // the other rows x column pairs of the other columns
        double flops = 0;       // algorithmic flops of the pass (a's products on b's targets and b's)
        double c_elems = 0;     // target scalars, each read and written once
        double ab_elems = 0;    // operand scalars of both pivots
    };
    std::vector<uint8_t> pair_first; // [L] 1: levels l and l+1 form a pair
    std::vector<PairShape> pair;     // [L] valid where pair_first
    // For the second pivot b (slot p) of a pair, at split_pref[p] + i: the index in a's
    // lower column of b's i-th lower row, and at split_pref[p] + n_lc(b) + j: the index in
    // a's upper row of b's j-th upper column; -1 where a has no such block (and everywhere
    // outside pairs).
    std::vector<int32_t> pair_map;
    int64_t n_pairs = 0;

    int64_t max_split_blocks = 0;    // max over uniform-64 levels of the split_pref span
    int64_t max_tc_targets = 0;       // max over uniform-64 levels of the upd_pref span (target table)
    int64_t max_fwd_scratch_rows = 0; // max over levels of fwd_rows span
    int64_t max_bwd_scratch_rows = 0;
    double factor_flops = 0;          // exact algorithmic flops of the factorization
    int64_t factor_values = 0;        // unpadded scalars in the filled pattern

    int64_t nnz_a() const { return (int64_t)a_cols.size(); }
    int64_t nnz_f() const { return (int64_t)cols.size(); }
    int64_t slab_elems() const { return blk_off.empty() ? 0 : blk_off.back(); }
};

// Runs the symbolic phase. Returns a hyb_status code.
int symbolic_build(int64_t n, const uint64_t *sizes, const uint64_t *row_ptr, const uint64_t *cols, Symbolic &out,
                   std::string &err);

// Operation list in the reference's single-thread order (pairs row, src|-1).
void symbolic_operations(const Symbolic &s, std::vector<int64_t> &ops);

// Filled block index of (r, c), or -1.
int64_t find_block(const Symbolic &s, int64_t r, int64_t c);

int compute_ordering(uint64_t n, const uint64_t *row_ptr, const uint64_t *cols, int strategy, uint64_t max_colors,
                     uint64_t *ordering);

} // namespace hyb
