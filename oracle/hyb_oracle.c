/*
 * hyb_oracle.c - CPU restatement of j4nr0th/hybridized-solver's block LU.
 *
 * TEST INFRASTRUCTURE ONLY (the parity oracle). See hyb_oracle.h for who may use
 * it. Each function names the reference function and lines it restates. The
 * arithmetic order is kept: products are accumulated left to right over k from
 * zero into a scratch block and only then subtracted (or negated for fill), the
 * Doolittle LU computes a row of U then a column of L, and a target row applies
 * its sources in ascending column order.
 */
#include "hyb_oracle.h"

#include <stdlib.h>
#include <string.h>

typedef struct
{
    uint64_t col;
    double *vals;
} orc_entry;

typedef struct
{
    uint64_t count;
    uint64_t capacity;
    orc_entry *entries; /* sorted by col, unique */
} orc_row;

struct orc_system
{
    uint64_t n;
    uint64_t *offsets; /* n + 1 prefix sums of block sizes */
    orc_row *rows;
    uint64_t nops;
    int64_t *ops; /* pairs (row, col|-1); NULL until decomposed */
};

static uint64_t bsize(const orc_system *s, uint64_t i)
{
    return s->offsets[i + 1] - s->offsets[i];
}

/* First position whose column is >= val (row_array_find_first_geq, src/blocks.c:112-155). */
static uint64_t find_geq(const orc_row *row, uint64_t val)
{
    uint64_t lo = 0, hi = row->count;
    while (lo < hi)
    {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (row->entries[mid].col < val)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

static double *find_block(const orc_system *s, uint64_t r, uint64_t c)
{
    const orc_row *row = s->rows + r;
    const uint64_t p = find_geq(row, c);
    if (p == row->count || row->entries[p].col != c)
        return NULL;
    return row->entries[p].vals;
}

orc_system *orc_create(uint64_t n, const uint64_t *block_sizes)
{
    if (n == 0)
        return NULL;
    orc_system *s = calloc(1, sizeof(*s));
    if (!s)
        return NULL;
    s->n = n;
    s->offsets = malloc((n + 1) * sizeof(uint64_t));
    s->rows = calloc(n, sizeof(orc_row));
    if (!s->offsets || !s->rows)
    {
        orc_destroy(s);
        return NULL;
    }
    s->offsets[0] = 0;
    for (uint64_t i = 0; i < n; ++i)
    {
        if (block_sizes[i] == 0)
        {
            orc_destroy(s);
            return NULL;
        }
        s->offsets[i + 1] = s->offsets[i] + block_sizes[i];
    }
    return s;
}

void orc_destroy(orc_system *s)
{
    if (!s)
        return;
    if (s->rows)
    {
        for (uint64_t i = 0; i < s->n; ++i)
        {
            for (uint64_t j = 0; j < s->rows[i].count; ++j)
                free(s->rows[i].entries[j].vals);
            free(s->rows[i].entries);
        }
    }
    free(s->rows);
    free(s->offsets);
    free(s->ops);
    free(s);
}

orc_system *orc_copy(const orc_system *src)
{
    uint64_t *sizes = malloc(src->n * sizeof(uint64_t));
    if (!sizes)
        return NULL;
    for (uint64_t i = 0; i < src->n; ++i)
        sizes[i] = bsize(src, i);
    orc_system *s = orc_create(src->n, sizes);
    free(sizes);
    if (!s)
        return NULL;
    for (uint64_t i = 0; i < src->n; ++i)
    {
        for (uint64_t j = 0; j < src->rows[i].count; ++j)
        {
            const orc_entry *e = src->rows[i].entries + j;
            if (orc_add_block(s, i, e->col, e->vals) != ORC_SUCCESS)
            {
                orc_destroy(s);
                return NULL;
            }
        }
    }
    if (src->ops)
    {
        s->ops = malloc((2 * src->nops + 1) * sizeof(int64_t));
        if (!s->ops)
        {
            orc_destroy(s);
            return NULL;
        }
        memcpy(s->ops, src->ops, 2 * src->nops * sizeof(int64_t));
        s->nops = src->nops;
    }
    return s;
}

uint64_t orc_n_blocks(const orc_system *s)
{
    return s->n;
}

uint64_t orc_block_size(const orc_system *s, uint64_t idx)
{
    return bsize(s, idx);
}

uint64_t orc_row_count(const orc_system *s, uint64_t row)
{
    return s->rows[row].count;
}

void orc_row_cols(const orc_system *s, uint64_t row, uint64_t *cols)
{
    for (uint64_t j = 0; j < s->rows[row].count; ++j)
        cols[j] = s->rows[row].entries[j].col;
}

static int row_reserve(orc_row *row, uint64_t need)
{
    if (row->capacity >= need)
        return 0;
    uint64_t cap = row->capacity ? row->capacity : 8;
    while (cap < need)
        cap *= 2;
    orc_entry *p = realloc(row->entries, cap * sizeof(orc_entry));
    if (!p)
        return -1;
    row->entries = p;
    row->capacity = cap;
    return 0;
}

/* block_system_add_block (src/blocks.c:3-75): a block already present is summed into. */
int orc_add_block(orc_system *s, uint64_t r, uint64_t c, const double *vals)
{
    if (r >= s->n || c >= s->n)
        return ORC_BAD_ARGUMENT;
    if (s->ops)
        return ORC_ALREADY_DECOMPOSED;
    orc_row *row = s->rows + r;
    const uint64_t nv = bsize(s, r) * bsize(s, c);
    const uint64_t p = find_geq(row, c);
    if (p < row->count && row->entries[p].col == c)
    {
        double *dst = row->entries[p].vals;
        for (uint64_t i = 0; i < nv; ++i)
            dst[i] += vals[i];
        return ORC_SUCCESS;
    }
    if (row_reserve(row, row->count + 1) < 0)
        return ORC_FAILED_ALLOC;
    double *block = malloc(nv * sizeof(double));
    if (!block)
        return ORC_FAILED_ALLOC;
    memcpy(block, vals, nv * sizeof(double));
    memmove(row->entries + p + 1, row->entries + p, (row->count - p) * sizeof(orc_entry));
    row->entries[p] = (orc_entry){.col = c, .vals = block};
    row->count += 1;
    return ORC_SUCCESS;
}

int orc_get_block(const orc_system *s, uint64_t r, uint64_t c, double *out)
{
    if (r >= s->n || c >= s->n)
        return ORC_BAD_ARGUMENT;
    const double *b = find_block(s, r, c);
    if (!b)
        return ORC_BLOCK_NOT_IN_SYSTEM;
    memcpy(out, b, bsize(s, r) * bsize(s, c) * sizeof(double));
    return ORC_SUCCESS;
}

uint64_t orc_total_blocks(const orc_system *s)
{
    uint64_t t = 0;
    for (uint64_t i = 0; i < s->n; ++i)
        t += s->rows[i].count;
    return t;
}

uint64_t orc_export_value_count(const orc_system *s)
{
    uint64_t t = 0;
    for (uint64_t i = 0; i < s->n; ++i)
        for (uint64_t j = 0; j < s->rows[i].count; ++j)
            t += bsize(s, i) * bsize(s, s->rows[i].entries[j].col);
    return t;
}

void orc_export(const orc_system *s, uint64_t *row_ptr, uint64_t *cols, double *values)
{
    uint64_t nb = 0, nv = 0;
    for (uint64_t i = 0; i < s->n; ++i)
    {
        if (row_ptr)
            row_ptr[i] = nb;
        for (uint64_t j = 0; j < s->rows[i].count; ++j, ++nb)
        {
            const orc_entry *e = s->rows[i].entries + j;
            const uint64_t cnt = bsize(s, i) * bsize(s, e->col);
            if (cols)
                cols[nb] = e->col;
            if (values)
                memcpy(values + nv, e->vals, cnt * sizeof(double));
            nv += cnt;
        }
    }
    if (row_ptr)
        row_ptr[s->n] = nb;
}

/* matrix_multiply (src/blocks.c:200-222): out = a * b, each entry summed over k in order from 0. */
void orc_matmul(uint64_t m, uint64_t k, uint64_t n, const double *a, const double *b, double *out)
{
    for (uint64_t i = 0; i < m; ++i)
    {
        for (uint64_t j = 0; j < n; ++j)
        {
            double v = 0;
            for (uint64_t q = 0; q < k; ++q)
                v += a[i * k + q] * b[q * n + j];
            out[i * n + j] = v;
        }
    }
}

/* matrix_lu_decompose (src/blocks.c:254-283): unpivoted Doolittle; unit L below the
 * diagonal, U on and above it. A zero pivot divides by zero, as in the reference. */
void orc_lu_decompose(uint64_t m, double *a)
{
    for (uint64_t i = 0; i < m; ++i)
    {
        for (uint64_t j = i; j < m; ++j)
        {
            double u = a[i * m + j];
            for (uint64_t k = 0; k < i; ++k)
                u -= a[i * m + k] * a[k * m + j];
            a[i * m + j] = u;
        }
        for (uint64_t j = i + 1; j < m; ++j)
        {
            double l = a[j * m + i];
            for (uint64_t k = 0; k < i; ++k)
                l -= a[k * m + i] * a[j * m + k];
            a[j * m + i] = l / a[i * m + i];
        }
    }
}

/* matrix_lu_solve (src/blocks.c:285-316): column by column, forward with unit L then
 * backward with U. `b` and `out` may be the same buffer. */
void orc_lu_solve(uint64_t m, const double *lu, uint64_t ncols, const double *b, double *out)
{
    for (uint64_t c = 0; c < ncols; ++c)
    {
        for (uint64_t i = 0; i < m; ++i)
        {
            double v = b[i * ncols + c];
            for (uint64_t j = 0; j < i; ++j)
                v -= lu[i * m + j] * out[j * ncols + c];
            out[i * ncols + c] = v;
        }
        for (uint64_t i = m; i > 0; --i)
        {
            double v = out[(i - 1) * ncols + c];
            for (uint64_t j = i; j < m; ++j)
                v -= lu[(i - 1) * m + j] * out[j * ncols + c];
            out[(i - 1) * ncols + c] = v / lu[(i - 1) * m + (i - 1)];
        }
    }
}

/* block_system_decompose_diagonal (src/blocks.c:541-555). */
void orc_decompose_diagonal(orc_system *s, uint64_t row)
{
    double *d = find_block(s, row, row);
    if (d)
        orc_lu_decompose(bsize(s, row), d);
}

/* block_system_apply_diagonal_inverse (src/blocks.c:516-539): every block right of
 * the diagonal is replaced by D^{-1} B using the factored diagonal. */
void orc_apply_diagonal_inverse(orc_system *s, uint64_t row)
{
    orc_row *r = s->rows + row;
    const uint64_t p = find_geq(r, row);
    if (p == r->count || r->entries[p].col != row)
        return;
    const uint64_t m = bsize(s, row);
    const double *d = r->entries[p].vals;
    for (uint64_t j = p + 1; j < r->count; ++j)
    {
        double *b = r->entries[j].vals;
        orc_lu_solve(m, d, bsize(s, r->entries[j].col), b, b);
    }
}

/* block_system_eliminate_row (src/blocks.c:557-727) and the binding's variant with a
 * caller-given multiplier (src/block_system.c:552-766): for every column c > src in
 * the union of both rows, T[c] -= S * R[c] where R has c, and a new fill block
 * T[c] = -(S * R[c]) where T lacked it; columns <= src are untouched. */
int orc_eliminate_row(orc_system *s, uint64_t tgt, uint64_t src, const double *scale)
{
    if (tgt >= s->n || src >= s->n)
        return ORC_BAD_ARGUMENT;
    orc_row *rt = s->rows + tgt;
    const orc_row *rs = s->rows + src;
    const uint64_t mt = bsize(s, tgt), ms = bsize(s, src);
    uint64_t pt = find_geq(rt, src + 1), ps = find_geq(rs, src + 1);
    /* Count the merged columns above src. */
    uint64_t extra = 0, max_cols = 0;
    for (uint64_t a = pt, b = ps; a < rt->count || b < rs->count;)
    {
        const uint64_t ca = a < rt->count ? rt->entries[a].col : UINT64_MAX;
        const uint64_t cb = b < rs->count ? rs->entries[b].col : UINT64_MAX;
        if (cb < ca)
        {
            extra += 1;
            ++b;
            if (bsize(s, cb) > max_cols)
                max_cols = bsize(s, cb);
        }
        else
        {
            if (ca == cb)
                ++b;
            ++a;
            if (ca == cb && bsize(s, cb) > max_cols)
                max_cols = bsize(s, cb);
        }
    }
    double *buf = malloc((mt * max_cols + 1) * sizeof(double));
    if (!buf)
        return ORC_FAILED_ALLOC;
    if (row_reserve(rt, rt->count + extra) < 0)
    {
        free(buf);
        return ORC_FAILED_ALLOC;
    }
    /* Merge from the back so that existing entries move in place. */
    uint64_t a = rt->count, b = rs->count, k = rt->count + extra;
    while (b > ps)
    {
        const orc_entry *es = rs->entries + (b - 1);
        if (a > pt && rt->entries[a - 1].col > es->col)
        {
            rt->entries[--k] = rt->entries[--a];
            continue;
        }
        const uint64_t nc = bsize(s, es->col);
        orc_matmul(mt, ms, nc, scale, es->vals, buf);
        if (a > pt && rt->entries[a - 1].col == es->col)
        {
            orc_entry e = rt->entries[--a];
            for (uint64_t i = 0; i < mt * nc; ++i) /* matrix_subtract_inplace, src/blocks.c:246-252 */
                e.vals[i] -= buf[i];
            rt->entries[--k] = e;
        }
        else
        {
            double *fill = malloc(mt * nc * sizeof(double));
            if (!fill)
            {
                free(buf);
                return ORC_FAILED_ALLOC;
            }
            for (uint64_t i = 0; i < mt * nc; ++i)
                fill[i] = -buf[i];
            rt->entries[--k] = (orc_entry){.col = es->col, .vals = fill};
        }
        --b;
    }
    rt->count += extra;
    free(buf);
    return ORC_SUCCESS;
}

static int ops_push(uint64_t *count, uint64_t *cap, int64_t **ops, int64_t row, int64_t col)
{
    if (*count == *cap)
    {
        const uint64_t nc = *cap ? 2 * *cap : 64;
        int64_t *p = realloc(*ops, 2 * nc * sizeof(int64_t));
        if (!p)
            return -1;
        *ops = p;
        *cap = nc;
    }
    (*ops)[2 * *count] = row;
    (*ops)[2 * *count + 1] = col;
    *count += 1;
    return 0;
}

/* block_system_decompose (src/blocks.c:360-514) with one thread: phase 1 factors, in
 * index order, every row whose first entry is its diagonal; phase 2 repeatedly takes
 * the lowest-index row whose next needed source row is finished, eliminates that one
 * source, and finishes the row (LU + diagonal inverse) once its next column is the
 * diagonal. The op list records INVDIA(row) and ELIMIN(row, src) in that order. */
int orc_decompose(orc_system *s)
{
    if (s->ops)
        return ORC_ALREADY_DECOMPOSED;
    const uint64_t n = s->n;
    for (uint64_t i = 0; i < n; ++i)
        if (!find_block(s, i, i))
            return ORC_BLOCK_NOT_IN_SYSTEM;
    unsigned char *done = calloc(n, 1);
    uint64_t *needed = calloc(n, sizeof(uint64_t));
    uint64_t count = 0, cap = 0;
    int64_t *ops = NULL;
    int rc = ORC_SUCCESS;
    if (!done || !needed)
    {
        rc = ORC_FAILED_ALLOC;
        goto out;
    }
    uint64_t n_tgt = 0;
    for (uint64_t i = 0; i < n; ++i)
    {
        if (s->rows[i].entries[0].col == i)
        {
            if (ops_push(&count, &cap, &ops, (int64_t)i, -1) < 0)
            {
                rc = ORC_FAILED_ALLOC;
                goto out;
            }
            orc_decompose_diagonal(s, i);
            orc_apply_diagonal_inverse(s, i);
            done[i] = 1;
        }
        else
        {
            needed[i] = s->rows[i].entries[0].col;
            n_tgt += 1;
        }
    }
    uint64_t first = 0;
    while (first < n && done[first])
        first += 1;
    while (n_tgt)
    {
        uint64_t t = first;
        while (t < n && (done[t] || !done[needed[t]]))
            ++t;
        if (t == n)
        {
            rc = ORC_BAD_ARGUMENT; /* no progress possible: malformed pattern */
            goto out;
        }
        const uint64_t src = needed[t];
        const double *mult = find_block(s, t, src);
        /* The multiplier block is left of every column the elimination writes, so it
         * stays valid while the row's entry array is rebuilt. */
        rc = orc_eliminate_row(s, t, src, mult);
        if (rc != ORC_SUCCESS)
            goto out;
        if (ops_push(&count, &cap, &ops, (int64_t)t, (int64_t)src) < 0)
        {
            rc = ORC_FAILED_ALLOC;
            goto out;
        }
        const orc_row *row = s->rows + t;
        const uint64_t next = row->entries[find_geq(row, src + 1)].col;
        if (next == t)
        {
            orc_decompose_diagonal(s, t);
            orc_apply_diagonal_inverse(s, t);
            done[t] = 1;
            if (ops_push(&count, &cap, &ops, (int64_t)t, -1) < 0)
            {
                rc = ORC_FAILED_ALLOC;
                goto out;
            }
            n_tgt -= 1;
            while (first < n && done[first])
                first += 1;
        }
        else
        {
            needed[t] = next;
        }
    }
out:
    free(done);
    free(needed);
    if (rc != ORC_SUCCESS)
    {
        free(ops);
        return rc;
    }
    if (!ops)
        ops = malloc(sizeof(int64_t) * 2);
    s->ops = ops;
    s->nops = count;
    return ORC_SUCCESS;
}

uint64_t orc_nops(const orc_system *s)
{
    return s->nops;
}

void orc_get_ops(const orc_system *s, int64_t *ops)
{
    memcpy(ops, s->ops, 2 * s->nops * sizeof(int64_t));
}

/* block_system_apply_operations (src/blocks.c:729-769) followed by
 * block_system_solve_u (src/blocks.c:771-800). */
int orc_solve(const orc_system *s, double *vec)
{
    if (!s->ops)
        return ORC_NOT_DECOMPOSED;
    uint64_t max_size = 0;
    for (uint64_t i = 0; i < s->n; ++i)
        if (bsize(s, i) > max_size)
            max_size = bsize(s, i);
    double *buf = malloc((max_size + 1) * sizeof(double));
    if (!buf)
        return ORC_FAILED_ALLOC;
    for (uint64_t o = 0; o < s->nops; ++o)
    {
        const int64_t r = s->ops[2 * o], c = s->ops[2 * o + 1];
        double *y = vec + s->offsets[r];
        const uint64_t m = bsize(s, (uint64_t)r);
        if (c < 0)
        {
            orc_lu_solve(m, find_block(s, (uint64_t)r, (uint64_t)r), 1, y, y);
        }
        else
        {
            /* matrix_multiply_sub_inplace (src/blocks.c:224-244) */
            const uint64_t k = bsize(s, (uint64_t)c);
            orc_matmul(m, k, 1, find_block(s, (uint64_t)r, (uint64_t)c), vec + s->offsets[c], buf);
            for (uint64_t i = 0; i < m; ++i)
                y[i] -= buf[i];
        }
    }
    for (uint64_t i = s->n; i > 0; --i)
    {
        const uint64_t r = i - 1;
        const orc_row *row = s->rows + r;
        const uint64_t m = bsize(s, r);
        double *y = vec + s->offsets[r];
        for (uint64_t j = row->count; j > 0 && row->entries[j - 1].col > r; --j)
        {
            const orc_entry *e = row->entries + (j - 1);
            const uint64_t k = bsize(s, e->col);
            orc_matmul(m, k, 1, e->vals, vec + s->offsets[e->col], buf);
            for (uint64_t q = 0; q < m; ++q)
                y[q] -= buf[q];
        }
    }
    free(buf);
    return ORC_SUCCESS;
}

/* order_from_colors (src/blocks.c:802-894): colors are laid out by decreasing count
 * (the reference's exchange sort, whose tie behaviour is kept), indices keep their
 * relative order inside a color. `ordering` holds colors on entry, new indices on exit. */
static void order_from_colors(uint64_t n, uint64_t *ordering, uint64_t *scratch, uint64_t color_count,
                              uint64_t *counts)
{
    uint64_t *which = scratch;
    for (uint64_t i = 0; i < color_count; ++i)
        which[i] = i;
    for (uint64_t i = 0; i + 1 < color_count; ++i)
        for (uint64_t j = i; j < color_count; ++j)
            if (counts[i] < counts[j])
            {
                uint64_t t = counts[i];
                counts[i] = counts[j];
                counts[j] = t;
                t = which[i];
                which[i] = which[j];
                which[j] = t;
            }
    uint64_t total = 0;
    for (uint64_t i = 0; i < color_count; ++i)
    {
        const uint64_t c = counts[i];
        counts[i] = total;
        total += c;
    }
    for (uint64_t i = 0; i + 1 < color_count; ++i)
        for (uint64_t j = i; j < color_count; ++j)
            if (which[i] > which[j])
            {
                uint64_t t = counts[i];
                counts[i] = counts[j];
                counts[j] = t;
                t = which[i];
                which[i] = which[j];
                which[j] = t;
            }
    for (uint64_t i = 0; i < color_count; ++i)
        which[i] = 0;
    for (uint64_t i = 0; i < n; ++i)
    {
        const uint64_t c = ordering[i];
        ordering[i] = counts[c] + which[c]++;
    }
}

/* First admissible color in `rank` order: the reference restarts its scan of the row
 * from the first entry each time a neighbour holds the candidate (goto color_check,
 * src/blocks.c:938-951, 995-1009, 1084-1098). Returns the position in `rank`. */
static uint64_t pick_color(const uint64_t *row_cols, uint64_t cnt, const uint64_t *colors, const uint64_t *rank,
                           uint64_t color_count)
{
    uint64_t pos = 0;
restart:
    for (uint64_t j = 0; j < cnt && pos < color_count; ++j)
    {
        if (colors[row_cols[j]] == (rank ? rank[pos] : pos))
        {
            pos += 1;
            goto restart;
        }
    }
    return pos;
}

/* block_system_compute_ordering_first / _greedy / _balanced (src/blocks.c:918-1141)
 * with update_color_counts (src/blocks.c:896-916). */
int orc_compute_ordering(uint64_t n, const uint64_t *row_ptr, const uint64_t *cols, int strategy, uint64_t max_colors,
                         uint64_t *ordering)
{
    if (max_colors == 0)
        return ORC_BAD_ARGUMENT;
    uint64_t *counts = calloc(max_colors + 1, sizeof(uint64_t));
    uint64_t *rank = malloc((max_colors + 1) * sizeof(uint64_t));
    if (!counts || !rank)
    {
        free(counts);
        free(rank);
        return ORC_FAILED_ALLOC;
    }
    for (uint64_t i = 0; i <= max_colors; ++i)
        rank[i] = i;
    for (uint64_t i = 0; i < n; ++i)
        ordering[i] = UINT64_MAX;
    uint64_t color_count = 0;
    int rc = ORC_SUCCESS;
    for (uint64_t i = 0; i < n; ++i)
    {
        const uint64_t *rc_cols = cols + row_ptr[i];
        const uint64_t cnt = row_ptr[i + 1] - row_ptr[i];
        const uint64_t pos =
            pick_color(rc_cols, cnt, ordering, strategy == ORC_ORDERING_FIRST ? NULL : rank, color_count);
        if (pos == color_count && color_count == max_colors)
        {
            rc = ORC_MAX_COLORS;
            break;
        }
        const uint64_t color = strategy == ORC_ORDERING_FIRST ? pos : rank[pos];
        ordering[i] = color;
        if (color == color_count)
            counts[color_count++] = 1;
        else
            counts[color] += 1;
        if (strategy == ORC_ORDERING_GREEDY)
        {
            /* Move the color towards the front while it is used more than its predecessor. */
            for (uint64_t j = pos; j > 0; --j)
            {
                if (counts[rank[j]] > counts[rank[j - 1]])
                {
                    const uint64_t t = rank[j];
                    rank[j] = rank[j - 1];
                    rank[j - 1] = t;
                }
                else
                    break;
            }
        }
        else if (strategy == ORC_ORDERING_BALANCED)
        {
            /* Move the color towards the back while its successor is used less. */
            for (uint64_t j = pos + 1; j < color_count; ++j)
            {
                if (counts[rank[j]] < counts[rank[j - 1]])
                {
                    const uint64_t t = rank[j];
                    rank[j] = rank[j - 1];
                    rank[j - 1] = t;
                }
                else
                    break;
            }
        }
    }
    if (rc == ORC_SUCCESS)
        order_from_colors(n, ordering, rank, color_count, counts);
    free(counts);
    free(rank);
    return rc;
}

static int cmp_entry(const void *a, const void *b)
{
    const uint64_t x = ((const orc_entry *)a)->col, y = ((const orc_entry *)b)->col;
    return x < y ? -1 : (x > y);
}

/* block_system_object_reorder_blocks (src/block_system.c:1449-1644): row i moves to
 * order[i], every column index c becomes order[c], rows are re-sorted by column. */
int orc_reorder_blocks(orc_system *s, const uint64_t *order)
{
    if (s->ops)
        return ORC_ALREADY_DECOMPOSED;
    const uint64_t n = s->n;
    unsigned char *seen = calloc(n, 1);
    orc_row *rows = malloc(n * sizeof(orc_row));
    uint64_t *sizes = malloc(n * sizeof(uint64_t));
    if (!seen || !rows || !sizes)
    {
        free(seen);
        free(rows);
        free(sizes);
        return ORC_FAILED_ALLOC;
    }
    for (uint64_t i = 0; i < n; ++i)
    {
        if (order[i] >= n || seen[order[i]])
        {
            free(seen);
            free(rows);
            free(sizes);
            return ORC_BAD_ARGUMENT;
        }
        seen[order[i]] = 1;
    }
    for (uint64_t i = 0; i < n; ++i)
    {
        orc_row *r = s->rows + i;
        for (uint64_t j = 0; j < r->count; ++j)
            r->entries[j].col = order[r->entries[j].col];
        qsort(r->entries, r->count, sizeof(orc_entry), cmp_entry);
        rows[order[i]] = *r;
        sizes[order[i]] = bsize(s, i);
    }
    memcpy(s->rows, rows, n * sizeof(orc_row));
    for (uint64_t i = 0; i < n; ++i)
        s->offsets[i + 1] = s->offsets[i] + sizes[i];
    free(seen);
    free(rows);
    free(sizes);
    return ORC_SUCCESS;
}
