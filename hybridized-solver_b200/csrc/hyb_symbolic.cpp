// hyb_symbolic.cpp - host symbolic phase of the block LU.
//
// The reference discovers its fill while it factors: block_system_eliminate_row
// (src/blocks.c:557-727) merges the source row's upper blocks into the target row, and
// block_system_decompose (src/blocks.c:360-514) walks each target's lower columns in
// ascending order, including columns the fill just created. Replaying exactly that on
// the pattern gives the final (filled) block structure before any arithmetic, so the
// device factors into preallocated slabs and never allocates per block.
#include "hyb_internal.h"

#include "hybsol_b200.h"

#include <algorithm>
#include <functional>
#include <numeric>
#include <queue>

namespace hyb
{

static int64_t round_up(int64_t v, int64_t a)
{
    return (v + a - 1) / a * a;
}

int64_t find_block(const Symbolic &s, int64_t r, int64_t c)
{
    if (r < 0 || r >= s.n || c < 0 || c >= s.n)
        return -1;
    const int32_t *b = s.cols.data() + s.row_ptr[r];
    const int32_t *e = s.cols.data() + s.row_ptr[r + 1];
    const int32_t *p = std::lower_bound(b, e, (int32_t)c);
    if (p == e || *p != c)
        return -1;
    return p - s.cols.data();
}

namespace
{

using Span = std::pair<const int32_t *, const int32_t *>; // sorted block indices

// Position of v in a sorted span, -1 if absent.
int32_t span_pos(Span s, int64_t v)
{
    const int32_t *q = std::lower_bound(s.first, s.second, (int32_t)v);
    return (q != s.second && *q == v) ? (int32_t)(q - s.first) : -1;
}

// Whether every entry of a other than `skip` is in b (both sorted).
bool span_covered(Span a, Span b, int64_t skip)
{
    const int32_t *q = b.first;
    for (const int32_t *p = a.first; p != a.second; ++p)
    {
        if (*p == skip)
            continue;
        while (q != b.second && *q < *p)
            ++q;
        if (q == b.second || *q != *p)
            return false;
    }
    return true;
}

// The present ones of two positions, ascending, then -1s.
void order_pair(int32_t &x, int32_t &y)
{
    if (x < 0)
        std::swap(x, y);
    if (y >= 0 && y < x)
        std::swap(x, y);
}

// Pairs consecutive single-pivot levels for two-pivot tensor-core passes (PairShape), from
// the first level of each chain on, and records each pair's operand maps, tile counts and
// lookahead into the next unit.
void pair_levels(Symbolic &S)
{
    const int64_t L = S.n_levels;
    S.pair_first.assign(L, 0);
    S.pair.assign(L, {});
    S.pair_map.assign(S.split_pref[S.n], -1);
    S.n_pairs = 0;
    auto single = [&](int64_t l) { return l < L && S.lvl_ptr[l + 1] - S.lvl_ptr[l] == 1; };
    auto lower = [&](int64_t k) {
        return Span(S.lcol_row.data() + S.lcol_ptr[k], S.lcol_row.data() + S.lcol_ptr[k + 1]);
    };
    auto upper = [&](int64_t k) { return Span(S.cols.data() + S.diag_pos[k] + 1, S.cols.data() + S.row_ptr[k + 1]); };
    for (int64_t l = 0; l + 1 < L; ++l)
    {
        if (!single(l) || !single(l + 1) || S.lvl_listed[l] || S.lvl_listed[l + 1] || !S.shape[l].uniform64 ||
            !S.shape[l + 1].uniform64)
            continue;
        const int64_t pa = S.lvl_ptr[l], pb = S.lvl_ptr[l + 1];
        const int64_t a = S.piv[pa], b = S.piv[pb];
        const Span ra = lower(a), ca = upper(a), rb = lower(b), cb = upper(b);
        if (rb.first == rb.second || cb.first == cb.second || span_pos(ra, b) < 0 || span_pos(ca, b) < 0 ||
            !span_covered(ra, rb, b) || !span_covered(ca, cb, b))
            continue;
        S.pair_first[l] = 1;
        ++S.n_pairs;
        const int64_t n_lc = rb.second - rb.first, n_up = cb.second - cb.first;
        int64_t rows_a = 0, cols_a = 0;
        for (int64_t i = 0; i < n_lc; ++i)
        {
            const int32_t x = span_pos(ra, rb.first[i]);
            S.pair_map[S.split_pref[pb] + i] = x;
            rows_a += x >= 0;
        }
        for (int64_t j = 0; j < n_up; ++j)
        {
            const int32_t x = span_pos(ca, cb.first[j]);
            S.pair_map[S.split_pref[pb] + n_lc + j] = x;
            cols_a += x >= 0;
        }
        Symbolic::PairShape &ps = S.pair[l];
        ps.all_tiles = n_lc * ((n_up + 1) / 2);
        ps.flops = 2.0 * 64 * 64 * 64 * (double)(n_lc * n_up + rows_a * cols_a);
        ps.c_elems = 4096.0 * (double)(n_lc * n_up);
        ps.ab_elems = 4096.0 * (double)((ra.second - ra.first) + (ca.second - ca.first) + n_lc + n_up);
        ++l; // b's level belongs to the pair
    }
    for (int64_t l = 0; l + 1 < L; ++l)
    {
        if (!S.pair_first[l])
            continue;
        Symbolic::PairShape &ps = S.pair[l];
        const int64_t m = l + 2;
        if (!single(m))
            continue;
        const int64_t b = S.piv[S.lvl_ptr[l + 1]];
        const Span rb = lower(b), cb = upper(b);
        const int64_t n_lc = rb.second - rb.first, n_up = cb.second - cb.first;
        const int64_t c = S.piv[S.lvl_ptr[m]], d = S.pair_first[m] ? S.piv[S.lvl_ptr[m + 1]] : -1;
        ps.lookahead = true;
        ps.i0 = span_pos(rb, c);
        ps.i1 = d >= 0 ? span_pos(rb, d) : -1;
        ps.j0 = span_pos(cb, c);
        ps.j1 = d >= 0 ? span_pos(cb, d) : -1;
        order_pair(ps.i0, ps.i1);
        order_pair(ps.j0, ps.j1);
        const int64_t nri = (ps.i0 >= 0) + (ps.i1 >= 0), ncj = (ps.j0 >= 0) + (ps.j1 >= 0);
        ps.prio_tiles = nri * ((n_up + 1) / 2) + (ncj > 0 ? n_lc - nri : 0);
        ps.rest_tiles = (n_lc - nri) * ((n_up - ncj + 1) / 2);
    }
}

} // namespace

int symbolic_build(int64_t n, const uint64_t *sizes, const uint64_t *row_ptr, const uint64_t *cols, Symbolic &S,
                   std::string &err)
{
    if (n <= 0 || n >= INT32_MAX)
    {
        err = "number of blocks must be in [1, 2^31)";
        return HYB_INVALID_ARGUMENT;
    }
    S = Symbolic();
    S.n = n;
    S.size.resize(n);
    S.dof_off.resize(n + 1);
    S.dof_off[0] = 0;
    for (int64_t i = 0; i < n; ++i)
    {
        if (sizes[i] == 0 || sizes[i] > (1u << 20))
        {
            err = "block size " + std::to_string(sizes[i]) + " of block " + std::to_string(i) + " is out of range";
            return HYB_INVALID_ARGUMENT;
        }
        S.size[i] = (int32_t)sizes[i];
        S.dof_off[i + 1] = S.dof_off[i] + (int64_t)sizes[i];
    }
    if (row_ptr[0] != 0)
    {
        err = "row_ptr[0] must be 0";
        return HYB_INVALID_ARGUMENT;
    }
    const int64_t nnz_a = (int64_t)row_ptr[n];
    if (nnz_a >= INT32_MAX)
    {
        err = "too many blocks";
        return HYB_TOO_LARGE;
    }
    S.a_row_ptr.assign(row_ptr, row_ptr + n + 1);
    S.a_cols.resize(nnz_a);
    S.a_val_off.resize(nnz_a + 1);
    S.a_val_off[0] = 0;
    for (int64_t r = 0; r < n; ++r)
    {
        if (row_ptr[r + 1] < row_ptr[r])
        {
            err = "row_ptr must be non-decreasing";
            return HYB_INVALID_ARGUMENT;
        }
        bool has_diag = false;
        for (uint64_t j = row_ptr[r]; j < row_ptr[r + 1]; ++j)
        {
            if (cols[j] >= (uint64_t)n || (j > row_ptr[r] && cols[j] <= cols[j - 1]))
            {
                err = "columns of row " + std::to_string(r) + " must be in range and strictly ascending";
                return HYB_INVALID_ARGUMENT;
            }
            has_diag |= cols[j] == (uint64_t)r;
            S.a_cols[j] = (int32_t)cols[j];
            S.a_val_off[j + 1] = S.a_val_off[j] + (int64_t)S.size[r] * S.size[cols[j]];
        }
        if (!has_diag)
        {
            err = "row " + std::to_string(r) + " has no diagonal block";
            return HYB_MISSING_DIAGONAL;
        }
    }

    // ---- Fill: row t absorbs the upper part of every source s < t in its row, taken in
    // ascending order; new columns below t become further sources (src/blocks.c:473-507).
    S.row_ptr.assign(n + 1, 0);
    S.diag_pos.resize(n);
    S.cols.reserve((size_t)nnz_a * 2);
    std::vector<int32_t> marker(n, -1);
    std::vector<int32_t> row;
    std::vector<int32_t> heap;
    for (int64_t t = 0; t < n; ++t)
    {
        row.clear();
        heap.clear();
        for (int64_t j = S.a_row_ptr[t]; j < S.a_row_ptr[t + 1]; ++j)
        {
            const int32_t c = S.a_cols[j];
            marker[c] = (int32_t)t;
            row.push_back(c);
            if (c < t)
                heap.push_back(c);
        }
        std::make_heap(heap.begin(), heap.end(), std::greater<int32_t>());
        while (!heap.empty())
        {
            std::pop_heap(heap.begin(), heap.end(), std::greater<int32_t>());
            const int32_t s = heap.back();
            heap.pop_back();
            for (int64_t j = S.diag_pos[s] + 1; j < S.row_ptr[s + 1]; ++j)
            {
                const int32_t c = S.cols[j];
                if (marker[c] != (int32_t)t)
                {
                    marker[c] = (int32_t)t;
                    row.push_back(c);
                    if (c < t)
                    {
                        heap.push_back(c);
                        std::push_heap(heap.begin(), heap.end(), std::greater<int32_t>());
                    }
                }
            }
        }
        std::sort(row.begin(), row.end());
        S.diag_pos[t] = S.row_ptr[t] + (std::lower_bound(row.begin(), row.end(), (int32_t)t) - row.begin());
        S.cols.insert(S.cols.end(), row.begin(), row.end());
        // Row t's extent must be final before row t + 1 reads its upper part.
        S.row_ptr[t + 1] = (int64_t)S.cols.size();
        if ((int64_t)S.cols.size() >= INT32_MAX)
        {
            err = "filled pattern has too many blocks";
            return HYB_TOO_LARGE;
        }
    }
    const int64_t nnz_f = S.nnz_f();

    // ---- Slab layout and the original blocks' places in it.
    S.blk_off.resize(nnz_f + 1);
    S.blk_off[0] = 0;
    S.factor_values = 0;
    for (int64_t r = 0; r < n; ++r)
    {
        for (int64_t j = S.row_ptr[r]; j < S.row_ptr[r + 1]; ++j)
        {
            const int64_t elems = (int64_t)S.size[r] * S.size[S.cols[j]];
            S.factor_values += elems;
            S.blk_off[j + 1] = S.blk_off[j] + round_up(elems, kBlockAlign);
        }
    }
    S.a_to_f.resize(nnz_a);
    for (int64_t r = 0; r < n; ++r)
    {
        int64_t f = S.row_ptr[r];
        for (int64_t j = S.a_row_ptr[r]; j < S.a_row_ptr[r + 1]; ++j)
        {
            while (S.cols[f] != S.a_cols[j])
                ++f;
            S.a_to_f[j] = (int32_t)f;
        }
    }

    // ---- Strictly lower part by column.
    S.lcol_ptr.assign(n + 1, 0);
    for (int64_t t = 0; t < n; ++t)
        for (int64_t j = S.row_ptr[t]; j < S.diag_pos[t]; ++j)
            S.lcol_ptr[S.cols[j] + 1] += 1;
    for (int64_t k = 0; k < n; ++k)
        S.lcol_ptr[k + 1] += S.lcol_ptr[k];
    S.lcol_row.resize(S.lcol_ptr[n]);
    S.lcol_blk.resize(S.lcol_ptr[n]);
    {
        std::vector<int64_t> fillp(S.lcol_ptr.begin(), S.lcol_ptr.end() - 1);
        for (int64_t t = 0; t < n; ++t)
            for (int64_t j = S.row_ptr[t]; j < S.diag_pos[t]; ++j)
            {
                const int64_t p = fillp[S.cols[j]]++;
                S.lcol_row[p] = (int32_t)t;
                S.lcol_blk[p] = (int32_t)j;
            }
    }

    // ---- Levels: k waits for every j < k with block (k, j) or (j, k).
    S.level.assign(n, 0);
    int32_t max_level = 0;
    for (int64_t k = 0; k < n; ++k)
    {
        int32_t lv = S.level[k];
        for (int64_t j = S.row_ptr[k]; j < S.diag_pos[k]; ++j)
            lv = std::max(lv, S.level[S.cols[j]] + 1);
        S.level[k] = lv;
        for (int64_t j = S.diag_pos[k] + 1; j < S.row_ptr[k + 1]; ++j)
            S.level[S.cols[j]] = std::max(S.level[S.cols[j]], lv + 1);
        max_level = std::max(max_level, lv);
    }
    S.n_levels = max_level + 1;
    S.lvl_ptr.assign(S.n_levels + 1, 0);
    for (int64_t k = 0; k < n; ++k)
        S.lvl_ptr[S.level[k] + 1] += 1;
    for (int64_t l = 0; l < S.n_levels; ++l)
        S.lvl_ptr[l + 1] += S.lvl_ptr[l];
    S.piv.resize(n);
    {
        std::vector<int64_t> fillp(S.lvl_ptr.begin(), S.lvl_ptr.end() - 1);
        for (int64_t k = 0; k < n; ++k)
            S.piv[fillp[S.level[k]]++] = (int32_t)k;
    }

    // ---- Per-pivot work prefixes (piv order) and flop count.
    S.trsm_pref.assign(n + 1, 0);
    S.lu_pref.assign(n + 1, 0);
    S.upd_pref.assign(n + 1, 0);
    S.upd2_pref.assign(n + 1, 0);
    S.split_pref.assign(n + 1, 0);
    S.tc_pref.assign(n + 1, 0);
    S.fwd_pref.assign(n + 1, 0);
    S.fwdu_pref.assign(n + 1, 0);
    S.fwd_rows.assign(n + 1, 0);
    S.bwd_rows.assign(n + 1, 0);
    S.inv_idx.assign(n, -1);
    S.inv_row.clear();
    for (int64_t k = 0; k < n; ++k)
        if (S.size[k] == 64)
        {
            S.inv_idx[k] = (int32_t)S.inv_row.size();
            S.inv_row.push_back((int32_t)k);
        }
    S.n_inv = (int64_t)S.inv_row.size();
    double flops = 0;
    std::vector<double> piv_upd_flops(n), piv_upd_c(n), piv_upd_ab(n);
    for (int64_t p = 0; p < n; ++p)
    {
        const int64_t k = S.piv[p];
        const int64_t n_up = S.row_ptr[k + 1] - S.diag_pos[k] - 1;
        const int64_t n_lc = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
        const int64_t n_lr = S.diag_pos[k] - S.row_ptr[k];
        const double m = S.size[k];
        S.trsm_pref[p + 1] = S.trsm_pref[p] + n_up;
        S.lu_pref[p + 1] = S.lu_pref[p] + std::max<int64_t>(1, n_up);
        S.upd_pref[p + 1] = S.upd_pref[p] + n_lc * n_up;
        S.upd2_pref[p + 1] = S.upd2_pref[p] + (n_lc + 1) / 2 * n_up;
        S.split_pref[p + 1] = S.split_pref[p] + n_lc + n_up;
        S.tc_pref[p + 1] = S.tc_pref[p] + n_lc * ((n_up + 1) / 2);
        S.fwd_pref[p + 1] = S.fwd_pref[p] + n_lr;
        S.fwdu_pref[p + 1] = S.fwdu_pref[p] + std::max<int64_t>(1, n_lr);
        // partial-product spans padded to 4 values, so every pivot's partials start on a
        // 16-byte boundary in the staged (per-stage) and the dataflow (global) layouts alike
        S.fwd_rows[p + 1] = S.fwd_rows[p] + (n_lr * S.size[k] + 3) / 4 * 4;
        S.bwd_rows[p + 1] = S.bwd_rows[p] + (n_up * S.size[k] + 3) / 4 * 4;
        double up_cols = 0, lc_rows = 0;
        for (int64_t j = S.diag_pos[k] + 1; j < S.row_ptr[k + 1]; ++j)
            up_cols += S.size[S.cols[j]];
        for (int64_t j = S.lcol_ptr[k]; j < S.lcol_ptr[k + 1]; ++j)
            lc_rows += S.size[S.lcol_row[j]];
        flops += 2.0 / 3.0 * m * m * m + 2.0 * m * m * up_cols + 2.0 * lc_rows * m * up_cols;
        piv_upd_flops[p] = 2.0 * lc_rows * m * up_cols;
        piv_upd_c[p] = lc_rows * up_cols;
        piv_upd_ab[p] = m * (lc_rows + up_cols);
    }
    S.factor_flops = flops;

    // ---- Dataflow solve items: forward in pivot order, backward by levels descending.
    S.fwd_item_p.resize(S.fwdu_pref[n]);
    for (int64_t p = 0; p < n; ++p)
        for (int64_t j = S.fwdu_pref[p]; j < S.fwdu_pref[p + 1]; ++j)
            S.fwd_item_p[j] = (int32_t)p;
    S.bwd_item_p.clear();
    S.bwd_item_p.reserve(S.trsm_pref[n] + n);
    S.bwd_first.assign(n, 0);
    for (int64_t l = S.n_levels - 1; l >= 0; --l)
        for (int64_t p = S.lvl_ptr[l]; p < S.lvl_ptr[l + 1]; ++p)
        {
            const int64_t k = S.piv[p];
            const int64_t n_up = S.row_ptr[k + 1] - S.diag_pos[k] - 1;
            S.bwd_first[p] = (int64_t)S.bwd_item_p.size();
            for (int64_t j = 0; j < std::max<int64_t>(1, n_up); ++j)
                S.bwd_item_p.push_back((int32_t)p);
        }

    // ---- Level shapes, scratch spans and listed (conflicting) update levels.
    S.shape.assign(S.n_levels, {});
    S.lvl_listed.assign(S.n_levels, 0);
    S.mt_lvl_ptr.assign(S.n_levels + 1, 0);
    S.mt_src_ptr.assign(1, 0);
    std::vector<int32_t> rowmark(n, -1);
    struct Upd
    {
        int32_t tgt, k, l, u, row, col;
    };
    std::vector<Upd> ups;
    for (int64_t l = 0; l < S.n_levels; ++l)
    {
        Symbolic::LevelShape &sh = S.shape[l];
        bool uniform = true, piv64 = true;
        bool conflict = false;
        for (int64_t p = S.lvl_ptr[l]; p < S.lvl_ptr[l + 1]; ++p)
        {
            const int64_t k = S.piv[p];
            sh.upd_flops += piv_upd_flops[p];
            sh.upd_c_elems += piv_upd_c[p];
            sh.upd_ab_elems += piv_upd_ab[p];
            sh.max_piv = std::max(sh.max_piv, S.size[k]);
            uniform &= S.size[k] == 64;
            piv64 &= S.size[k] == 64;
            for (int64_t j = S.diag_pos[k] + 1; j < S.row_ptr[k + 1]; ++j)
            {
                sh.max_up = std::max(sh.max_up, S.size[S.cols[j]]);
                uniform &= S.size[S.cols[j]] == 64;
                piv64 &= S.size[S.cols[j]] == 64;
            }
            const bool has_up = S.row_ptr[k + 1] > S.diag_pos[k] + 1;
            for (int64_t j = S.lcol_ptr[k]; j < S.lcol_ptr[k + 1]; ++j)
            {
                const int32_t t = S.lcol_row[j];
                sh.max_row = std::max(sh.max_row, S.size[t]);
                uniform &= S.size[t] == 64;
                if (has_up)
                {
                    if (rowmark[t] == (int32_t)l)
                        conflict = true;
                    rowmark[t] = (int32_t)l;
                }
            }
        }
        sh.max_col = sh.max_up;
        sh.uniform64 = uniform;
        sh.piv64 = piv64;
        if (uniform)
        {
            S.max_split_blocks =
                std::max(S.max_split_blocks, S.split_pref[S.lvl_ptr[l + 1]] - S.split_pref[S.lvl_ptr[l]]);
            S.max_tc_targets = std::max(S.max_tc_targets, S.upd_pref[S.lvl_ptr[l + 1]] - S.upd_pref[S.lvl_ptr[l]]);
        }
        S.max_fwd_scratch_rows =
            std::max(S.max_fwd_scratch_rows, S.fwd_rows[S.lvl_ptr[l + 1]] - S.fwd_rows[S.lvl_ptr[l]]);
        S.max_bwd_scratch_rows =
            std::max(S.max_bwd_scratch_rows, S.bwd_rows[S.lvl_ptr[l + 1]] - S.bwd_rows[S.lvl_ptr[l]]);
        if (conflict)
        {
            S.lvl_listed[l] = 1;
            ups.clear();
            for (int64_t p = S.lvl_ptr[l]; p < S.lvl_ptr[l + 1]; ++p)
            {
                const int64_t k = S.piv[p];
                for (int64_t a = S.lcol_ptr[k]; a < S.lcol_ptr[k + 1]; ++a)
                {
                    const int32_t t = S.lcol_row[a];
                    const int32_t *rb = S.cols.data() + S.row_ptr[t];
                    const int32_t *re = S.cols.data() + S.row_ptr[t + 1];
                    for (int64_t j = S.diag_pos[k] + 1; j < S.row_ptr[k + 1]; ++j)
                    {
                        const int32_t c = S.cols[j];
                        const int32_t *q = std::lower_bound(rb, re, c);
                        ups.push_back({(int32_t)(q - S.cols.data()), (int32_t)k, S.lcol_blk[a], (int32_t)j, t, c});
                    }
                }
            }
            std::sort(ups.begin(), ups.end(),
                      [](const Upd &x, const Upd &y) { return x.tgt != y.tgt ? x.tgt < y.tgt : x.k < y.k; });
            for (size_t i = 0; i < ups.size(); ++i)
            {
                if (i == 0 || ups[i].tgt != ups[i - 1].tgt)
                {
                    if (i > 0)
                        S.mt_src_ptr.push_back((int64_t)S.mt_src_k.size());
                    S.mt_tgt.push_back(ups[i].tgt);
                    S.mt_row.push_back(ups[i].row);
                    S.mt_col.push_back(ups[i].col);
                }
                S.mt_src_k.push_back(ups[i].k);
                S.mt_src_l.push_back(ups[i].l);
                S.mt_src_u.push_back(ups[i].u);
            }
            if (!ups.empty())
                S.mt_src_ptr.push_back((int64_t)S.mt_src_k.size());
        }
        S.mt_lvl_ptr[l + 1] = (int64_t)S.mt_tgt.size();
    }

    // ---- Lookahead between consecutive single-pivot levels.
    for (int64_t l = 0; l + 1 < S.n_levels; ++l)
    {
        Symbolic::LevelShape &sh = S.shape[l];
        if (S.lvl_listed[l] || S.lvl_ptr[l + 1] - S.lvl_ptr[l] != 1 || S.lvl_ptr[l + 2] - S.lvl_ptr[l + 1] != 1)
            continue;
        const int64_t k = S.piv[S.lvl_ptr[l]], kn = S.piv[S.lvl_ptr[l + 1]];
        const int64_t n_lc = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
        const int64_t n_up = S.row_ptr[k + 1] - S.diag_pos[k] - 1;
        if (n_lc == 0 || n_up == 0)
            continue;
        int32_t i0 = -1, j0 = -1;
        for (int64_t a = 0; a < n_lc; ++a)
            if (S.lcol_row[S.lcol_ptr[k] + a] == kn)
                i0 = (int32_t)a;
        for (int64_t b = 0; b < n_up; ++b)
            if (S.cols[S.diag_pos[k] + 1 + b] == kn)
                j0 = (int32_t)b;
        if (i0 < 0 && j0 < 0)
            continue;
        sh.lookahead = true;
        sh.la_i0 = i0;
        sh.la_j0 = j0;
        sh.la_prio_units = (i0 >= 0 ? n_up : 0) + (j0 >= 0 ? n_lc : 0) - (i0 >= 0 && j0 >= 0 ? 1 : 0);
        sh.la_rest_units = (n_lc - (i0 >= 0)) * (n_up - (j0 >= 0));
        sh.la_rest_pairs = (n_lc - (i0 >= 0) + 1) / 2 * (n_up - (j0 >= 0));
        sh.la_prio_pairs = (i0 >= 0 ? n_up : 0) + (j0 >= 0 ? (n_lc - (i0 >= 0) + 1) / 2 : 0);
        sh.la_prio_tiles = (i0 >= 0 ? (n_up + 1) / 2 : 0) + (j0 >= 0 ? n_lc - (i0 >= 0) : 0);
        sh.la_rest_tiles = (n_lc - (i0 >= 0)) * ((n_up - (j0 >= 0) + 1) / 2);
    }
    pair_levels(S);
    return HYB_SUCCESS;
}

// Replays the reference's serial scheduler (src/blocks.c:373-508 with one thread) on the
// filled pattern: phase 1 records INVDIA for rows without lower blocks in index order;
// phase 2 always takes the lowest-index row whose next needed source is finished,
// records ELIMIN(row, source), and records INVDIA(row) after its last source.
void symbolic_operations(const Symbolic &S, std::vector<int64_t> &ops)
{
    const int64_t n = S.n;
    ops.clear();
    ops.reserve(2 * (size_t)(S.nnz_f() + n));
    std::vector<uint8_t> done(n, 0);
    std::vector<int64_t> pos(n, 0); // next lower position within the row
    std::vector<std::vector<int32_t>> waiting(n);
    std::priority_queue<int32_t, std::vector<int32_t>, std::greater<int32_t>> ready;
    for (int64_t i = 0; i < n; ++i)
    {
        if (S.diag_pos[i] == S.row_ptr[i])
        {
            ops.push_back(i);
            ops.push_back(-1);
            done[i] = 1;
        }
        pos[i] = S.row_ptr[i];
    }
    for (int64_t i = 0; i < n; ++i)
    {
        if (done[i])
            continue;
        const int32_t need = S.cols[pos[i]];
        if (done[need])
            ready.push((int32_t)i);
        else
            waiting[need].push_back((int32_t)i);
    }
    while (!ready.empty())
    {
        const int32_t t = ready.top();
        ready.pop();
        const int32_t src = S.cols[pos[t]];
        ops.push_back(t);
        ops.push_back(src);
        pos[t] += 1;
        if (pos[t] == S.diag_pos[t])
        {
            ops.push_back(t);
            ops.push_back(-1);
            done[t] = 1;
            for (int32_t w : waiting[t])
                ready.push(w);
            std::vector<int32_t>().swap(waiting[t]);
        }
        else
        {
            const int32_t need = S.cols[pos[t]];
            if (done[need])
                ready.push(t);
            else
                waiting[need].push_back(t);
        }
    }
}

} // namespace hyb
