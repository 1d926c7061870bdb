// hyb_ordering.cpp - graph-coloring orderings, integer and bit-exact with the reference.
//
// The reference colors block rows first-fit over their row entries and then lays the
// colors out by decreasing size (src/blocks.c:802-1141). The result decides which rows
// the factorization eliminates first, so every tie-break is kept: the candidate scan
// restarts from the row's first entry whenever a neighbour holds the candidate color
// (the `goto color_check` loops), "greedy" and "balanced" reorder their color ranking
// by one adjacent exchange pass after every assignment, and the final layout uses the
// reference's exchange sort of the color counts (not a stable sort).
#include "hyb_internal.h"

#include "hybsol_b200.h"

#include <vector>

namespace hyb
{

namespace
{

// Position (in `rank`, or the identity when rank is null) of the first candidate color
// no neighbour of the row holds.
uint64_t first_free(const uint64_t *row, uint64_t cnt, const std::vector<uint64_t> &color, const uint64_t *rank,
                    uint64_t n_colors)
{
    uint64_t pos = 0;
    bool clash = true;
    while (clash && pos < n_colors)
    {
        clash = false;
        const uint64_t candidate = rank ? rank[pos] : pos;
        for (uint64_t j = 0; j < cnt; ++j)
        {
            if (color[row[j]] == candidate)
            {
                clash = true;
                ++pos;
                break;
            }
        }
    }
    return pos;
}

// Turns colors into new indices: colors are placed in decreasing order of their counts
// using the reference's exchange sort (src/blocks.c:820-835), then every block gets the
// offset of its color plus its rank among earlier blocks of that color.
void layout_colors(uint64_t n, std::vector<uint64_t> &color, std::vector<uint64_t> counts, uint64_t n_colors,
                   uint64_t *ordering)
{
    std::vector<uint64_t> id(n_colors);
    for (uint64_t i = 0; i < n_colors; ++i)
        id[i] = i;
    for (uint64_t i = 0; i + 1 < n_colors; ++i)
        for (uint64_t j = i; j < n_colors; ++j)
            if (counts[i] < counts[j])
            {
                std::swap(counts[i], counts[j]);
                std::swap(id[i], id[j]);
            }
    std::vector<uint64_t> start(n_colors);
    uint64_t total = 0;
    for (uint64_t i = 0; i < n_colors; ++i)
    {
        start[id[i]] = total;
        total += counts[i];
    }
    std::vector<uint64_t> seen(n_colors, 0);
    for (uint64_t i = 0; i < n; ++i)
    {
        const uint64_t c = color[i];
        ordering[i] = start[c] + seen[c]++;
    }
}

} // namespace

int compute_ordering(uint64_t n, const uint64_t *row_ptr, const uint64_t *cols, int strategy, uint64_t max_colors,
                     uint64_t *ordering)
{
    if (strategy < HYB_ORDERING_FIRST || strategy > HYB_ORDERING_BALANCED)
        return HYB_INVALID_ARGUMENT;
    if (n == 0)
        return HYB_SUCCESS;
    if (max_colors == 0)
    {
        for (uint64_t i = 0; i < n; ++i)
            max_colors = std::max<uint64_t>(max_colors, row_ptr[i + 1] - row_ptr[i]);
        if (max_colors == 0)
            return HYB_MAX_COLORS;
    }
    for (uint64_t j = 0; j < row_ptr[n]; ++j)
        if (cols[j] >= n)
            return HYB_INVALID_ARGUMENT;
    const uint64_t unset = ~0ull;
    std::vector<uint64_t> color(n, unset);
    std::vector<uint64_t> counts(max_colors + 1, 0);
    std::vector<uint64_t> rank(max_colors + 1);
    for (uint64_t i = 0; i <= max_colors; ++i)
        rank[i] = i;
    const bool ranked = strategy != HYB_ORDERING_FIRST;
    uint64_t n_colors = 0;
    for (uint64_t i = 0; i < n; ++i)
    {
        const uint64_t pos =
            first_free(cols + row_ptr[i], row_ptr[i + 1] - row_ptr[i], color, ranked ? rank.data() : nullptr, n_colors);
        if (pos == n_colors && n_colors == max_colors)
            return HYB_MAX_COLORS; // update_color_counts, src/blocks.c:896-916
        const uint64_t c = ranked ? rank[pos] : pos;
        color[i] = c;
        if (c == n_colors)
            counts[n_colors++] = 1;
        else
            counts[c] += 1;
        if (strategy == HYB_ORDERING_GREEDY)
        {
            // most used first: src/blocks.c:1020-1033
            for (uint64_t j = pos; j > 0 && counts[rank[j]] > counts[rank[j - 1]]; --j)
                std::swap(rank[j], rank[j - 1]);
        }
        else if (strategy == HYB_ORDERING_BALANCED)
        {
            // least used first: src/blocks.c:1109-1122
            for (uint64_t j = pos + 1; j < n_colors && counts[rank[j]] < counts[rank[j - 1]]; ++j)
                std::swap(rank[j], rank[j - 1]);
        }
    }
    counts.resize(n_colors);
    layout_colors(n, color, counts, n_colors, ordering);
    return HYB_SUCCESS;
}

} // namespace hyb
