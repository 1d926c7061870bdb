// hyb_pivot.cuh - pivot work of levels whose pivots and upper blocks are all 64x64: the LU
// of each diagonal block and its row's upper blocks U(k, c) = D_k^{-1} A(k, c), plus (mixed
// form) the BF16 splits of the pivot's upper-row blocks for the tensor-core update.
//
// The work of one pivot lies on the elimination's critical path (the next pivot waits for
// it), so it is organised for latency, in CTAs of 256 threads:
//  - lu64_blocked: the 64x64 LU in eight panels of eight columns; one warp factors a panel
//    with shuffles (no CTA barrier per pivot step), then the CTA solves the panel's row
//    block and applies the rank-8 trailing update;
//  - solve64_blocked: a row solve in 8x8 blocks, four threads per column, a block's values
//    shuffled from the thread that owns it;
//  - k_piv64 (HYB_OPTION_ROW_PIVOTS 1): one CTA per upper block, each factoring the block
//    itself and solving its upper block; every element receives the operations of the
//    unblocked kernels in the same order, so the factors are the same bits;
//  - k_piv64_inv + k_strips64_inv (mixed form default): one CTA per pivot factors the block
//    once and forms its inverse, and the upper blocks become independent products with it
//    (plus, for the first pivot of a two-pivot pass, that pivot's update of the second one's
//    row and column, and the second one's LU and inverse in the CTA that forms its diagonal
//    block).
#pragma once

#include "hyb_umma.cuh"

namespace hyb
{

constexpr int kPivThreads = 256; // threads of every pivot kernel's CTA
constexpr int kLdD = 65; // row stride of the diagonal block in shared memory
constexpr int kLdQ = 80; // column stride of the transposed factors (four 16-row quarters, 20 apart)
constexpr int kLdI = 68; // row stride of the inverses and product operands (16-byte rows)

// Dynamic shared memory of k_piv64 (PivLayout below, plus reduction slots); the FP32
// kernel's FP64 fallback reuses it for a 64 x 65 FP64 block, which fits.
template <typename T> constexpr int piv64_smem()
{
    return (64 * kLdD + 2 * 64 * kLdQ + 64) * (int)sizeof(T);
}
static_assert(64 * 65 * 8 <= piv64_smem<float>(), "the FP64 fallback's block fits the FP32 layout");

// Vector of 16 bytes of T (four floats or two doubles).
template <typename T> struct Vec16;
template <> struct Vec16<float>
{
    using type = float4;
    static constexpr int n = 4;
};
template <> struct Vec16<double>
{
    using type = double2;
    static constexpr int n = 2;
};

template <typename T> __device__ __forceinline__ void load16(T *dst, const T *src)
{
    const typename Vec16<T>::type v = *reinterpret_cast<const typename Vec16<T>::type *>(src);
    if constexpr (std::is_same_v<T, float>)
    {
        dst[0] = v.x;
        dst[1] = v.y;
        dst[2] = v.z;
        dst[3] = v.w;
    }
    else
    {
        dst[0] = v.x;
        dst[1] = v.y;
    }
}

// Copies a 64x64 block from global memory into shared memory (row stride kLdD), every
// thread's 16-byte loads issued before any is stored, and returns the thread's largest
// |entry|; ends with a barrier.
template <typename T> __device__ __forceinline__ T load_block64(const T *g, T *d)
{
    constexpr int n = Vec16<T>::n, per = 64 * 64 / n / kPivThreads; // vectors per thread
    T v[per][n];
#pragma unroll
    for (int q = 0; q < per; ++q)
        load16(v[q], g + (threadIdx.x + q * kPivThreads) * n);
    T amax = T(0);
#pragma unroll
    for (int q = 0; q < per; ++q)
    {
        const int i = (threadIdx.x + q * kPivThreads) * n;
#pragma unroll
        for (int e = 0; e < n; ++e)
        {
            d[((i + e) >> 6) * kLdD + ((i + e) & 63)] = v[q][e];
            amax = fmax(amax, fabs(v[q][e]));
        }
    }
    __syncthreads();
    return amax;
}

// Shared memory of one CTA (T elements):
//   d[r * kLdD + c]           the diagonal block, factored in place (row-major, odd stride)
//   tl[tq_idx(c, r)] = L[r][c] for r > c, 0 elsewhere  (transposed, masked lower factor)
//   tu[tq_idx(c, r)] = U[r][c] for r < c, 0 elsewhere  (transposed, masked upper factor)
//   dg[c] = U[c][c]
// In the transposed factors each column's four 16-row quarters start 16-byte aligned and
// in distinct bank groups (quarter q at 20 q), so the four threads of a column read their
// quarters with 16-byte loads without conflicts.
__host__ __device__ constexpr int tq_idx(int c, int r)
{
    return c * kLdQ + r + 4 * (r >> 4);
}

template <typename T> struct PivLayout
{
    T *d, *tl, *tu, *dg;
    __device__ explicit PivLayout(unsigned char *base)
    {
        d = reinterpret_cast<T *>(base);
        tl = d + 64 * kLdD; // 16-byte aligned: 64 * 65 is a multiple of 4
        tu = tl + 64 * kLdQ;
        dg = tu + 64 * kLdQ;
    }
};

// Blocked LU of the 64x64 block in shared memory d (unit L below the diagonal, U on and
// above), 256 threads, in eight panels of eight columns. Panel p (columns c0 = 8p ..):
//  1. warp 0 factors the panel rows c0 .. 63 x columns c0 .. c0+7 in registers (lane l holds
//     rows c0 + l and c0 + l + 32), the pivot rows broadcast by shuffles -- no CTA barrier;
//  2. one thread per column of the panel's row block c0 .. c0+7 right of the panel applies
//     the unit-lower 8x8 factor (the rows of U);
//  3. the trailing block takes the rank-8 update, 4x4 register tiles per thread.
// Every element receives the updates of the unblocked right-looking elimination in the same
// order (multiplier = entry * reciprocal of the pivot; then entry -= multiplier * pivot-row
// entry for each earlier pivot in ascending order), so the factors are those of lu64_shared.
template <typename T> __device__ void lu64_blocked(T *d, int *status, int row_id)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll 1
    for (int p = 0; p < 8; ++p)
    {
        const int c0 = 8 * p;
        if (warp == 0)
        {
            const int r1 = c0 + lane, r2 = c0 + lane + 32;
            const bool has2 = r2 < 64;
            T a1[8], a2[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj)
            {
                a1[jj] = r1 < 64 ? d[r1 * kLdD + c0 + jj] : T(0);
                a2[jj] = has2 ? d[r2 * kLdD + c0 + jj] : T(0);
            }
#pragma unroll
            for (int kk = 0; kk < 8; ++kk)
            {
                const T piv = __shfl_sync(0xffffffffu, a1[kk], kk);
                if (status != nullptr && lane == 0 && (piv == T(0) || !finite_val(piv)))
                {
                    atomicAdd(status + (piv == T(0) ? ST_ZERO_PIVOTS : ST_NON_FINITE), 1);
                    atomicMin(status + ST_FIRST_BAD, row_id);
                }
                const T rp = T(1) / piv;
                T u[8];
#pragma unroll
                for (int jj = kk + 1; jj < 8; ++jj)
                    u[jj] = __shfl_sync(0xffffffffu, a1[jj], kk);
                if (lane > kk && r1 < 64)
                {
                    const T l1 = a1[kk] * rp;
                    a1[kk] = l1;
#pragma unroll
                    for (int jj = kk + 1; jj < 8; ++jj)
                        a1[jj] -= l1 * u[jj];
                }
                if (has2)
                {
                    const T l2 = a2[kk] * rp;
                    a2[kk] = l2;
#pragma unroll
                    for (int jj = kk + 1; jj < 8; ++jj)
                        a2[jj] -= l2 * u[jj];
                }
            }
#pragma unroll
            for (int jj = 0; jj < 8; ++jj)
            {
                if (r1 < 64)
                    d[r1 * kLdD + c0 + jj] = a1[jj];
                if (has2)
                    d[r2 * kLdD + c0 + jj] = a2[jj];
            }
        }
        __syncthreads();
        const int n2 = 56 - c0; // columns (and rows) right of (below) the panel
        if (tid < n2)
        {
            const int j = c0 + 8 + tid;
            T v[8];
#pragma unroll
            for (int rr = 0; rr < 8; ++rr)
                v[rr] = d[(c0 + rr) * kLdD + j];
#pragma unroll
            for (int kk = 0; kk < 7; ++kk)
#pragma unroll
                for (int rr = kk + 1; rr < 8; ++rr)
                    v[rr] -= d[(c0 + rr) * kLdD + c0 + kk] * v[kk];
#pragma unroll
            for (int rr = 1; rr < 8; ++rr)
                d[(c0 + rr) * kLdD + j] = v[rr];
        }
        __syncthreads();
        const int nt = n2 / 4;
        if (tid < nt * nt)
        {
            const int R = c0 + 8 + 4 * (tid / nt), C = c0 + 8 + 4 * (tid % nt);
            T acc[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    acc[a][b] = d[(R + a) * kLdD + C + b];
#pragma unroll
            for (int kk = 0; kk < 8; ++kk)
            {
                T lr[4], uc[4];
#pragma unroll
                for (int a = 0; a < 4; ++a)
                    lr[a] = d[(R + a) * kLdD + c0 + kk];
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    uc[b] = d[(c0 + kk) * kLdD + C + b];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        acc[a][b] -= lr[a] * uc[b];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    d[(R + a) * kLdD + C + b] = acc[a][b];
        }
        __syncthreads();
    }
}

// The factored block d as the transposed, masked factors tl, tu and the pivots dg.
template <typename T> __device__ __forceinline__ void piv_transpose(const PivLayout<T> &f)
{
    for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x)
    {
        const int c = i >> 6, r = i & 63;
        const T v = f.d[r * kLdD + c];
        f.tl[tq_idx(c, r)] = r > c ? v : T(0);
        f.tu[tq_idx(c, r)] = r < c ? v : T(0);
        if (r == c)
            f.dg[c] = v;
    }
    __syncthreads();
}

// x[j] -= c[j] * s for the thread's rows j in [J0, J1), c read 16 bytes at a time.
template <typename T, int J0, int J1> __device__ __forceinline__ void axpy_rows(T (&x)[16], const T *c, T s)
{
    constexpr int n = Vec16<T>::n;
#pragma unroll
    for (int j0 = J0; j0 < J1; j0 += n)
    {
        T dv[n];
        load16(dv, c + j0);
#pragma unroll
        for (int e = 0; e < n; ++e)
            x[j0 + e] -= dv[e] * s;
    }
}

// X = U^{-1} L^{-1} B for a 64x64 block B, 256 threads: the four threads 4c .. 4c+3 of a
// warp's lanes share column (tid >> 2), thread q of them holding rows 16q .. 16q+15 in x[].
// Both substitutions run in 8x8 blocks: the owner of a block (quarter qb) substitutes
// within it, shuffles its eight values to the column's other threads, and every thread
// applies them to its rows outside the block. Each element receives the operations of the
// unblocked column substitution (trsm64_columns) in the same order.
template <typename T> __device__ __forceinline__ void solve64_blocked(T (&x)[16], const PivLayout<T> &f)
{
    const int tid = threadIdx.x, lane = tid & 31, q = tid & 3, base = lane & ~3;
    constexpr int n = Vec16<T>::n;
    // forward, blocks 0 .. 7 (two per quarter)
#pragma unroll 1
    for (int qb = 0; qb < 4; ++qb)
    {
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            const int h0 = 8 * half, r0 = 16 * qb + h0; // the block's first row
            if (q == qb)
            {
#pragma unroll
                for (int kk = 0; kk < 7; ++kk)
                {
                    const T xk = x[h0 + kk];
#pragma unroll
                    for (int rr = kk + 1; rr < 8; ++rr)
                        x[h0 + rr] -= f.tl[tq_idx(r0 + kk, r0 + rr)] * xk;
                }
            }
            // rows below the block: all rows of the later quarters, and the second half of
            // quarter qb after its first block; each of the block's values is shuffled from
            // its owner as it is applied
#pragma unroll
            for (int kk = 0; kk < 8; ++kk)
            {
                const T sk = __shfl_sync(0xffffffffu, x[h0 + kk], base + qb);
                const T *lc = f.tl + tq_idx(r0 + kk, 16 * q);
                if (q > qb)
                    axpy_rows<T, 0, 16>(x, lc, sk);
                else if (q == qb && half == 0)
                    axpy_rows<T, 8, 16>(x, lc, sk);
            }
        }
    }
    // backward, blocks 7 .. 0
#pragma unroll 1
    for (int qb = 3; qb >= 0; --qb)
    {
#pragma unroll
        for (int half = 1; half >= 0; --half)
        {
            const int h0 = 8 * half, r0 = 16 * qb + h0;
            if (q == qb)
            {
#pragma unroll
                for (int kk = 7; kk >= 0; --kk)
                {
                    const T xk = x[h0 + kk] / f.dg[r0 + kk];
                    x[h0 + kk] = xk;
#pragma unroll
                    for (int rr = 0; rr < kk; ++rr)
                        x[h0 + rr] -= f.tu[tq_idx(r0 + kk, r0 + rr)] * xk;
                }
            }
            // rows above the block: all rows of the earlier quarters, and the first half of
            // quarter qb above its second block; the block's columns in descending order
#pragma unroll
            for (int kk = 7; kk >= 0; --kk)
            {
                const T sk = __shfl_sync(0xffffffffu, x[h0 + kk], base + qb);
                const T *uc = f.tu + tq_idx(r0 + kk, 16 * q);
                if (q < qb)
                    axpy_rows<T, 0, 16>(x, uc, sk);
                else if (q == qb && half == 1)
                    axpy_rows<T, 0, 8>(x, uc, sk);
            }
        }
    }
}
// ----------------------------------------------------------------------------------
// Mixed form: the diagonal block's inverse, once per pivot, and the row solves as products.
// In the mixed form the FP32 factors only have to approximate A (the FP64 refinement sets
// the accuracy), so the upper blocks U(k,c) = D^{-1} A(k,c) are taken as products with an
// explicit inverse: one CTA per pivot factors D and forms D^{-1} (k_piv64_inv), and the row
// solves become independent 64x64x64 products (k_strips64_inv). The pivot's critical path
// is then one LU and two short triangular inversions instead of every upper block's
// 127-step substitution, and a pivot occupies one CTA instead of one per upper block.

// Inverses of the unit-lower L and the upper U of an LU held in d (stride kLdD): li = L^{-1}
// (unit lower), ui = U^{-1} (upper), both stride kLdD, in 8x8 blocks. The diagonal blocks
// are inverted by substitution, one thread per column; then, for distance s = 1 .. 7 from
// the diagonal, every block (i, j) at that distance is
//   Li_ij = -Li_ii (sum_{k=j}^{i-1} L_ik Li_kj),   Ui_ij = -Ui_ii (sum_{k=i+1}^{j} U_ik Ui_kj)
// (two products per phase, the partial sums staged in `tmp`, 2 x 7 x 64 values).
template <typename T> __device__ void tri_inv64_blocked(const T *d, T *li, T *ui, T *tmp)
{
    const int tid = threadIdx.x;
    // zero the triangles that stay zero
    for (int e = tid; e < 64 * 64; e += blockDim.x)
    {
        const int r = e >> 6, c = e & 63;
        if (c > r)
            li[r * kLdI + c] = T(0);
        if (c < r)
            ui[r * kLdI + c] = T(0);
    }
    // diagonal blocks: thread t < 64 takes column t & 7 of block t >> 3 of L^{-1};
    // threads 64 .. 127 the same of U^{-1}
    if (tid < 128)
    {
        const int b = (tid & 63) >> 3, jj = tid & 7, o = 8 * b;
        T y[8];
        if (tid < 64)
        {
#pragma unroll
            for (int r = 0; r < 8; ++r)
            {
                T v = r == jj ? T(1) : T(0);
#pragma unroll
                for (int c = 0; c < r; ++c)
                    v -= d[(o + r) * kLdD + o + c] * y[c];
                y[r] = v;
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
                li[(o + r) * kLdI + o + jj] = y[r];
        }
        else
        {
#pragma unroll
            for (int r = 7; r >= 0; --r)
            {
                T v = r == jj ? T(1) : T(0);
#pragma unroll
                for (int c = r + 1; c < 8; ++c)
                    v -= d[(o + r) * kLdD + o + c] * y[c];
                y[r] = v / d[(o + r) * kLdD + o + r];
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
                ui[(o + r) * kLdI + o + jj] = y[r];
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int s = 1; s < 8; ++s)
    {
        const int nb = 8 - s;     // blocks at distance s
        const int outs = nb * 64; // values per triangle
        // partial sums: L side for block (i, j) = (j + s, j), U side for (i, i + s); each
        // an eight-term product per block of the sum, eight independent accumulators
        for (int e = tid; e < 2 * outs; e += blockDim.x)
        {
            const bool up = e >= outs;
            const int f = up ? e - outs : e;
            const int blk = f >> 6, r = (f >> 3) & 7, c = f & 7;
            const int i = up ? blk : blk + s, j = up ? blk + s : blk; // block (i, j)
            const int m0 = up ? 8 * i + 8 : 8 * j, m1 = up ? 8 * j + 8 : 8 * i;
            const T *row = d + (8 * i + r) * kLdD;
            const T *inv = (up ? ui : li) + 8 * j + c;
            T acc[8] = {};
            for (int m = m0; m < m1; m += 8)
            {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    acc[q] += row[m + q] * inv[(m + q) * kLdI];
            }
            tmp[e] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
        }
        __syncthreads();
        for (int e = tid; e < 2 * outs; e += blockDim.x)
        {
            const bool up = e >= outs;
            const int f = up ? e - outs : e;
            const int blk = f >> 6, r = (f >> 3) & 7, c = f & 7;
            const int i = up ? blk : blk + s, j = up ? blk + s : blk;
            const T *t = tmp + (up ? outs : 0) + blk * 64;
            const T *dgi = (up ? ui : li) + (8 * i + r) * kLdI + 8 * i; // row r of the diagonal block's inverse
            T acc = T(0);
#pragma unroll
            for (int m = 0; m < 8; ++m)
                acc -= dgi[m] * t[m * 8 + c];
            (up ? ui : li)[(8 * i + r) * kLdI + 8 * j + c] = acc;
        }
        __syncthreads();
    }
}

// acc = X B for this thread's 4x4 tile (rows R .., columns C ..) of a 64x64 product, with
// X transposed (xs[m * kLdI + r] = X[r][m]) and B row-major (bs[m * kLdI + c]) in shared
// memory. Every caller uses this one loop, so a block formed in two places is the same bits.
__device__ __forceinline__ void prod64_tile(const float *xs, const float *bs, int R, int C, float (&acc)[4][4])
{
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e)
            acc[q][e] = 0.f;
#pragma unroll 8
    for (int m = 0; m < 64; ++m)
    {
        const float4 a4 = *reinterpret_cast<const float4 *>(xs + m * kLdI + R);
        const float4 b4 = *reinterpret_cast<const float4 *>(bs + m * kLdI + C);
        const float av[4] = {a4.x, a4.y, a4.z, a4.w}, bv[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                acc[q][e] += av[q] * bv[e];
    }
}

// The same in FP64 with X row-major in global memory (x64[r * 64 + m], a high-growth
// pivot's FP64 inverse) and B in FP32 shared memory, rounded to FP32.
__device__ __forceinline__ void prod64_tile_fp64(const double *x64, const float *bs, int R, int C, float (&acc)[4][4])
{
    double ad[4][4] = {};
#pragma unroll 1
    for (int m = 0; m < 64; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                ad[q][e] += x64[(R + q) * 64 + m] * (double)bs[m * kLdI + C + e];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int e = 0; e < 4; ++e)
            acc[q][e] = (float)ad[q][e];
}

// Copies a row-major 64x64 FP32 block from global memory into shared memory with row stride
// kLdI (16-byte loads, all issued before any is stored).
__device__ __forceinline__ void load_block64_ldi(const float *g, float *s)
{
    float4 v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
        v[q] = *reinterpret_cast<const float4 *>(g + (threadIdx.x + q * kPivThreads) * 4);
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        const int i = (threadIdx.x + q * kPivThreads) * 4;
        *reinterpret_cast<float4 *>(s + (i >> 6) * kLdI + (i & 63)) = v[q];
    }
}

// the FP32 working set (LU, two triangular inverses, partial sums); the FP64 fallback's LU
// (64 x 65 doubles) fits in it, its inverse goes straight to the FP64 slot in global memory
constexpr int kInvSmem = (64 * kLdD + 2 * 64 * kLdI + 2 * 7 * 64) * 4;
static_assert(64 * 65 * 8 <= kInvSmem, "the FP64 fallback's LU fits the FP32 working set");

// One CTA per pivot of the level: the blocked LU of the 64x64 diagonal block (stored back
// in the slab), then X = U^{-1} L^{-1} into the pivot's slot of `dinv` (transposed:
// dinv[slot * 4096 + c * 64 + r] = X[r][c], the layout the forward solve reads). Growth
// check (growth_limit > 0): past the limit the pivot is factored and inverted in FP64 from
// its original values (rolled loops in shared memory), the FP64 inverse goes to `inv64`
// (slot p - p0) for the products, and hg[k] is set.
//
// First pivot c of a pair (j0 >= 0: the second pivot d's position in c's upper row): the CTA
// also forms U(c,d) = X A(c,d) into `ucd` (row-major), with the loop k_strips64_inv uses
// for the same block, so the column updates of the pair's second pivot can read it while
// that block is being overwritten in place.
// The work of k_piv64_inv for pivot slot p, by the calling CTA (256 threads) in the
// kInvSmem bytes at smem_raw, the FP64 inverse (if any) in `x64` (4096 doubles).
__device__ __noinline__ void piv64_inv_body(const DevSym &S, float *__restrict__ slab, int64_t p, int *status,
                                            float growth_limit, float *__restrict__ dinv, double *__restrict__ x64,
                                            int *__restrict__ hg, int32_t j0, float *__restrict__ ucd,
                                            unsigned char *smem_raw)
{
    float *d = reinterpret_cast<float *>(smem_raw);
    float *li = d + 64 * kLdD, *ui = li + 64 * kLdI, *tmp = ui + 64 * kLdI; // li 16-byte aligned
    const int tid = threadIdx.x;
    const int64_t k = S.piv[p];
    float *gd = slab + S.blk_off[S.diag_pos[k]];
    float *xt = dinv + (int64_t)S.inv_idx[k] * 4096;
    float amax = load_block64(gd, d);
    const bool check = growth_limit > 0;
    if (check)
        amax = cta_max(amax);
    lu64_blocked(d, status, (int)k);
    if (check)
    {
        float umax = 0.f;
        for (int i = tid; i < 64 * 64; i += kPivThreads)
        {
            const int r = i >> 6, c = i & 63;
            if (c >= r)
                umax = fmaxf(umax, fabsf(d[r * kLdD + c]));
        }
        umax = cta_max(umax);
        if (umax / amax > growth_limit)
        {
            // FP64: a = LU (64 x 65, shared memory), b = the inverse, row-major in the
            // pivot's FP64 slot (each thread works on its own column)
            double *a = reinterpret_cast<double *>(smem_raw);
            double *b = x64;
            __syncthreads();
            for (int i = tid; i < 64 * 64; i += kPivThreads)
                a[(i >> 6) * 65 + (i & 63)] = (double)gd[i];
#pragma unroll 1
            for (int kk = 0; kk < 64; ++kk)
            {
                __syncthreads(); // row kk is final
                if (tid > kk && tid < 64)
                {
                    const double l = a[tid * 65 + kk] * (1.0 / a[kk * 65 + kk]);
                    a[tid * 65 + kk] = l;
#pragma unroll 1
                    for (int j = kk + 1; j < 64; ++j)
                        a[tid * 65 + j] -= l * a[kk * 65 + j];
                }
            }
            __syncthreads();
            if (tid < 64) // column tid of the inverse: U^{-1} (L^{-1} e_tid)
            {
#pragma unroll 1
                for (int r = 0; r < 64; ++r)
                {
                    double v = r == tid ? 1.0 : 0.0;
#pragma unroll 1
                    for (int c = 0; c < r; ++c)
                        v -= a[r * 65 + c] * b[c * 64 + tid];
                    b[r * 64 + tid] = v;
                }
#pragma unroll 1
                for (int r = 63; r >= 0; --r)
                {
                    double v = b[r * 64 + tid];
#pragma unroll 1
                    for (int c = r + 1; c < 64; ++c)
                        v -= a[r * 65 + c] * b[c * 64 + tid];
                    b[r * 64 + tid] = v / a[r * 65 + r];
                }
            }
            __syncthreads();
            __threadfence_block(); // the inverse columns, written by other threads, are read below
            for (int i = tid; i < 64 * 64; i += kPivThreads)
            {
                const int r = i >> 6, c = i & 63;
                gd[i] = (float)a[r * 65 + c];
                xt[c * 64 + r] = (float)b[i];
            }
            if (tid == 0)
            {
                hg[k] = 1;
                atomicAdd(status + ST_GROWTH_FP64, 1);
            }
            if (j0 >= 0)
            {
                // U(c,d) in FP64 with the FP64 inverse, A(c,d) past the FP64 LU
                float *bsm = reinterpret_cast<float *>(smem_raw + 64 * 65 * 8);
                load_block64_ldi(slab + S.blk_off[S.diag_pos[k] + 1 + j0], bsm);
                __syncthreads();
                const int R = 4 * (tid >> 4), C = 4 * (tid & 15);
                float acc[4][4];
                prod64_tile_fp64(b, bsm, R, C, acc);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    *reinterpret_cast<float4 *>(ucd + (R + q) * 64 + C) =
                        make_float4(acc[q][0], acc[q][1], acc[q][2], acc[q][3]);
            }
            return;
        }
    }
    for (int i = tid; i < 64 * 64; i += kPivThreads)
        gd[i] = d[(i >> 6) * kLdD + (i & 63)];
    tri_inv64_blocked(d, li, ui, tmp);
    // X = Ui Li, 4x4 tiles: X[r][c] = sum over m >= max(r, c) of Ui[r][m] Li[m][c]
    {
        const int R = 4 * (tid >> 4), C = 4 * (tid & 15);
        float acc[4][4] = {};
        for (int m = max(R, C); m < 64; ++m)
        {
            float a4[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                a4[q] = ui[(R + q) * kLdI + m];
            const float4 b = *reinterpret_cast<const float4 *>(li + m * kLdI + C);
            const float b4[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    acc[q][e] += a4[q] * b4[e];
        }
#pragma unroll
        for (int e = 0; e < 4; ++e)
            *reinterpret_cast<float4 *>(xt + (C + e) * 64 + R) = make_float4(acc[0][e], acc[1][e], acc[2][e], acc[3][e]);
        if (j0 >= 0)
        {
            // X (transposed, stride kLdI) over L^{-1}, A(c,d) over U^{-1}, then U(c,d)
            __syncthreads(); // every thread is done reading li and ui
#pragma unroll
            for (int e = 0; e < 4; ++e)
                *reinterpret_cast<float4 *>(li + (C + e) * kLdI + R) =
                    make_float4(acc[0][e], acc[1][e], acc[2][e], acc[3][e]);
            load_block64_ldi(slab + S.blk_off[S.diag_pos[k] + 1 + j0], ui);
            __syncthreads();
            prod64_tile(li, ui, R, C, acc);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                *reinterpret_cast<float4 *>(ucd + (R + q) * 64 + C) =
                    make_float4(acc[q][0], acc[q][1], acc[q][2], acc[q][3]);
        }
    }
}

__global__ void __launch_bounds__(kPivThreads, 1)
    k_piv64_inv(DevSym S, float *__restrict__ slab, int64_t p0, int *status, float growth_limit,
                float *__restrict__ dinv, double *__restrict__ inv64, int *__restrict__ hg, int32_t j0,
                float *__restrict__ ucd)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t p = p0 + blockIdx.x;
    piv64_inv_body(S, slab, p, status, growth_limit, dinv, inv64 + (p - p0) * 4096, hg, j0, ucd, smem_raw);
}


// T -= L U for a 64x64 target T (global, row-major), L row-major in global memory, U in
// shared memory (row-major, stride kLdI); ls is shared scratch for L transposed. Ends with
// a barrier before ls is written, so callers may pass a buffer they just read.
__device__ __forceinline__ void sub_lu64(float *T, const float *L, const float *us, float *ls)
{
    const int tid = threadIdx.x;
    float4 v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
        v[q] = *reinterpret_cast<const float4 *>(L + (tid + q * kPivThreads) * 4);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        const int i = (tid + q * kPivThreads) * 4, r = i >> 6, c = i & 63;
        ls[(c + 0) * kLdI + r] = v[q].x;
        ls[(c + 1) * kLdI + r] = v[q].y;
        ls[(c + 2) * kLdI + r] = v[q].z;
        ls[(c + 3) * kLdI + r] = v[q].w;
    }
    __syncthreads();
    const int R = 4 * (tid >> 4), C = 4 * (tid & 15);
    float acc[4][4];
    prod64_tile(ls, us, R, C, acc);
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        float4 *t = reinterpret_cast<float4 *>(T + (R + q) * 64 + C);
        float4 o = *t;
        o.x -= acc[q][0];
        o.y -= acc[q][1];
        o.z -= acc[q][2];
        o.w -= acc[q][3];
        *t = o;
    }
}

// The upper blocks of the level's pivots as products with the pivots' inverses: CTA u of
// the level's upper blocks (trsm_pref) computes U(k, c) = X A(k, c), X = D_k^{-1} from
// `dinv` (or, for a pivot flagged in hg, the FP64 inverse in `inv64`, in FP64), stores it
// and writes its BF16 split (transposed K-major) to `ops` at its split unit.
//
// First pivot k of a pair (i0 >= 0: the second pivot d at position i0 of k's lower column
// and j0 of its upper row; the level has this one pivot): each upper-block CTA then also
// applies k's update to d's row, T(d, c) -= L(d, k) U(k, c), and CTAs past the upper blocks
// apply it to d's column, T(t, d) -= L(t, k) U(k, d) for the other rows t of k's lower
// column, with U(k, d) from `ucd` (formed by k_piv64_inv with the same loop).
//
// With pd >= 0 (the pair's second pivot, slot pd), the CTA of the upper block in d's column
// -- which forms d's diagonal block T(d, d) -- goes on to factor and invert it
// (piv64_inv_body, in the launch's dynamic shared memory, FP64 inverse in x64_d), while the
// launch's other CTAs finish: d's pivot work then needs only its products launch.
// growth_limit > 0: hg flags pivots whose products run in FP64 (and d's check may set it).
__global__ void __launch_bounds__(kPivThreads, 2)
    k_strips64_inv(DevSym S, float *__restrict__ slab, int64_t p0, int64_t p1, float *__restrict__ dinv,
                   const double *__restrict__ inv64, int *__restrict__ hg, unsigned char *__restrict__ ops,
                   int32_t i0, int32_t j0, const float *__restrict__ ucd, int64_t pd, double *__restrict__ x64_d,
                   float growth_limit, int *status)
{
    __shared__ __align__(16) float xs[64 * kLdI]; // X transposed: xs[c * kLdI + r] = X[r][c]
    __shared__ __align__(16) float as[64 * kLdI]; // A(k, c), then the product, row-major
    const int tid = threadIdx.x;
    const int64_t n_trsm = S.trsm_pref[p1] - S.trsm_pref[p0];
    if ((int64_t)blockIdx.x >= n_trsm)
    {
        // pair: a target in the second pivot's column
        const int64_t k = S.piv[p0];
        const int32_t ci = (int32_t)((int64_t)blockIdx.x - n_trsm);
        const int32_t i = ci < i0 ? ci : ci + 1; // skip d's own row
        const int32_t t = S.lcol_row[S.lcol_ptr[k] + i];
        const int32_t dcol = S.cols[S.diag_pos[k] + 1 + j0];
        float *T = slab + S.blk_off[find_col(S.cols, S.row_ptr[t], S.row_ptr[t + 1], dcol)];
        const float *L = slab + S.blk_off[S.lcol_blk[S.lcol_ptr[k] + i]];
        load_block64_ldi(ucd, as);
        sub_lu64(T, L, as, xs);
        return;
    }
    const int64_t u = S.trsm_pref[p0] + blockIdx.x;
    const int64_t p = find_owner(S.trsm_pref, p0, p1, u);
    const int64_t k = S.piv[p];
    const int64_t j = u - S.trsm_pref[p];
    float *gb = slab + S.blk_off[S.diag_pos[k] + 1 + j];
    const float *xt = dinv + (int64_t)S.inv_idx[k] * 4096;
    load_block64_ldi(xt, xs);
    load_block64_ldi(gb, as);
    __syncthreads();
    const int R = 4 * (tid >> 4), C = 4 * (tid & 15);
    float acc[4][4];
    if (growth_limit > 0 && hg[k])
        prod64_tile_fp64(inv64 + (p - p0) * 4096, as, R, C, acc);
    else
        prod64_tile(xs, as, R, C, acc);
    __syncthreads(); // every thread is done reading A
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        const float4 v = make_float4(acc[q][0], acc[q][1], acc[q][2], acc[q][3]);
        *reinterpret_cast<float4 *>(gb + (R + q) * 64 + C) = v;
        *reinterpret_cast<float4 *>(as + (R + q) * kLdI + C) = v;
    }
    __syncthreads();
    // split: row n of the transposed tile is column n of U, K = its row index
    const int64_t n_lc = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
    unsigned char *dst = ops + (S.split_pref[p] - S.split_pref[p0] + n_lc + j) * (int64_t)kSplitBytes;
    for (int ch = tid; ch < 512; ch += kPivThreads)
    {
        const int nn = ch & 63, q = ch >> 6; // a warp reads 32 consecutive columns: no conflicts
        float x[8];
#pragma unroll
        for (int e = 0; e < 8; ++e)
            x[e] = as[(q * 8 + e) * kLdI + nn];
        uint4 hi, lo;
        split8(x, hi, lo);
        const uint32_t off = sw128_offset(nn, q * 8);
        *reinterpret_cast<uint4 *>(dst + off) = hi;
        *reinterpret_cast<uint4 *>(dst + kSplitHalf + off) = lo;
    }
    if (i0 >= 0)
    {
        // pair: the target in the second pivot's row, T(d, c) -= L(d, k) U(k, c)
        const int32_t drow = S.lcol_row[S.lcol_ptr[k] + i0];
        const int32_t col = S.cols[S.diag_pos[k] + 1 + j];
        float *T = slab + S.blk_off[find_col(S.cols, S.row_ptr[drow], S.row_ptr[drow + 1], col)];
        sub_lu64(T, slab + S.blk_off[S.lcol_blk[S.lcol_ptr[k] + i0]], as, xs);
        if (pd >= 0 && j == j0)
        {
            // this CTA formed T(d, d): the second pivot's LU and inverse follow here
            extern __shared__ __align__(16) unsigned char smem_dyn[];
            __syncthreads(); // T(d, d) written by every thread of the CTA
            piv64_inv_body(S, slab, pd, status, growth_limit, dinv, x64_d, hg, -1, nullptr, smem_dyn);
        }
    }
}

// Mixed form, a pivot whose FP32 LU grew past the limit: every CTA of the pivot re-reads
// the original block, factors it in FP64, solves its upper block in FP64 and stores it (and
// its split) in FP32; the pivot's ticket (not taken on the FP32 path, which none of them
// finished) picks the CTA that stores the FP64 LU rounded to FP32. A rare path: the FP64 LU
// lives in shared memory (row-major, stride 65, reusing the FP32 layout's space), threads
// 0-63 each hold one row (LU) and then one column of the upper block (in local memory),
// with rolled loops, so it adds neither registers nor shared memory to the kernel.
__device__ __noinline__ void piv64_fp64(float *gd, float *gb, unsigned char *split, int *lu_tickets, int64_t p,
                                        int total, int *status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *a = reinterpret_cast<double *>(smem_raw); // a[r * 65 + c]
    __shared__ int s_last;
    const int tid = threadIdx.x;
    const bool act = tid < 64;
    __syncthreads(); // every thread is done with the FP32 working set
    if (act)
    {
#pragma unroll 1
        for (int c = 0; c < 64; ++c)
            a[tid * 65 + c] = (double)gd[tid * 64 + c];
    }
#pragma unroll 1
    for (int k = 0; k < 64; ++k)
    {
        __syncthreads(); // row k is final
        if (act && tid > k)
        {
            const double rp = 1.0 / a[k * 65 + k];
            const double l = a[tid * 65 + k] * rp;
            a[tid * 65 + k] = l;
#pragma unroll 1
            for (int j = k + 1; j < 64; ++j)
                a[tid * 65 + j] -= l * a[k * 65 + j];
        }
    }
    __syncthreads();
    if (tid == 0)
    {
        __threadfence();
        s_last = atomicAdd(lu_tickets + p, 1) == total - 1;
    }
    __syncthreads();
    if (s_last && act)
    {
#pragma unroll 1
        for (int c = 0; c < 64; ++c)
            gd[tid * 64 + c] = (float)a[tid * 65 + c];
    }
    if (s_last && tid == 0)
        lu_tickets[p] = 0;
    if (gb != nullptr && act)
    {
        const int j = tid;
        double x[64];
#pragma unroll 1
        for (int r = 0; r < 64; ++r)
            x[r] = (double)gb[r * 64 + j];
#pragma unroll 1
        for (int i = 0; i < 63; ++i)
        {
            const double xi = x[i];
#pragma unroll 1
            for (int r = i + 1; r < 64; ++r)
                x[r] -= a[r * 65 + i] * xi;
        }
#pragma unroll 1
        for (int i = 63; i >= 0; --i)
        {
            const double xi = x[i] / a[i * 65 + i];
            x[i] = xi;
#pragma unroll 1
            for (int r = 0; r < i; ++r)
                x[r] -= a[r * 65 + i] * xi;
        }
#pragma unroll 1
        for (int r = 0; r < 64; ++r)
            gb[r * 64 + j] = (float)x[r];
        if (split != nullptr)
        {
#pragma unroll 1
            for (int q = 0; q < 8; ++q)
            {
                float v[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    v[e] = (float)x[8 * q + e];
                uint4 hi, lo;
                split8(v, hi, lo);
                const uint32_t off = sw128_offset(j, q * 8);
                *reinterpret_cast<uint4 *>(split + off) = hi;
                *reinterpret_cast<uint4 *>(split + kSplitHalf + off) = lo;
            }
        }
    }
    if (status != nullptr && tid == 0)
        atomicAdd(status + ST_GROWTH_FP64, 1);
}

// Pivot work of the level's pivots p0 .. p1 (pivots and upper blocks all 64 wide), 256
// threads per CTA. CTA u - lu_pref[p0] is unit u of pivot p (lu_pref: one per upper block,
// one for a pivot without any): it factors the pivot's diagonal block (lu64_blocked) and
// solves upper block u - lu_pref[p] (solve64_blocked); the last CTA of the pivot to have
// read the unfactored block writes the factors (per-pivot ticket). With kSplit (mixed form,
// the level's update on the tensor cores) the solved block's BF16 split goes to `ops` at
// its split unit (k_split64 with lower_only writes the lower blocks'). Mixed form,
// growth_limit > 0: a pivot whose FP32 LU grew past it takes the FP64 path (piv64_fp64).
template <typename T, bool kSplit>
__global__ void __launch_bounds__(kPivThreads, 3)
    k_piv64(DevSym S, T *__restrict__ slab, int64_t p0, int64_t p1, int *__restrict__ lu_tickets, int *status,
            float growth_limit, unsigned char *__restrict__ ops)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const PivLayout<T> f(smem_raw);
    __shared__ int s_writer;
    const int64_t u = S.lu_pref[p0] + blockIdx.x;
    const int64_t p = find_owner(S.lu_pref, p0, p1, u);
    const int64_t k = S.piv[p];
    const int64_t j = u - S.lu_pref[p];
    const int total = (int)(S.lu_pref[p + 1] - S.lu_pref[p]);
    const bool owner = j == 0; // reports zero and non-finite pivots
    T *gd = slab + S.blk_off[S.diag_pos[k]];
    const int64_t blk = S.diag_pos[k] + 1 + j;
    T *gb = blk < S.row_ptr[k + 1] ? slab + S.blk_off[blk] : nullptr;
    const int64_t n_lc = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
    unsigned char *split =
        kSplit && gb != nullptr ? ops + (S.split_pref[p] - S.split_pref[p0] + n_lc + j) * (int64_t)kSplitBytes : nullptr;
    const bool check = std::is_same_v<T, float> && growth_limit > 0;
    T amax = load_block64(gd, f.d);
    if (check)
        amax = cta_max(amax);
    lu64_blocked(f.d, owner ? status : nullptr, (int)k);
    if (check)
    {
        T umax = T(0);
        for (int i = tid; i < 64 * 64; i += kPivThreads)
        {
            const int r = i >> 6, c = i & 63;
            if (c >= r)
                umax = fmax(umax, fabs(f.d[r * kLdD + c]));
        }
        umax = cta_max(umax);
        if (umax / amax > (T)growth_limit) // the same decision in every CTA of the pivot
        {
            if constexpr (std::is_same_v<T, float>)
                piv64_fp64(gd, gb, split, lu_tickets, p, total, owner ? status : nullptr);
            return;
        }
    }
    // the last CTA of the pivot to take a ticket -- after every other one has read the block
    // and finished its LU -- writes the factors
    if (tid == 0)
    {
        __threadfence();
        s_writer = atomicAdd(lu_tickets + p, 1) == total - 1;
    }
    piv_transpose(f); // ends with a barrier, after which s_writer is visible
    if (s_writer)
    {
        for (int i = tid; i < 64 * 64; i += kPivThreads)
            gd[i] = f.d[(i >> 6) * kLdD + (i & 63)];
        if (tid == 0)
            lu_tickets[p] = 0; // ready for the next factorization
    }
    if (gb == nullptr)
        return;
    // this thread's quarter of column `col` of the upper block
    const int col = tid >> 2, q = tid & 3;
    T x[16];
#pragma unroll
    for (int jj = 0; jj < 16; ++jj)
        x[jj] = gb[(16 * q + jj) * 64 + col];
    solve64_blocked(x, f);
#pragma unroll
    for (int jj = 0; jj < 16; ++jj)
        gb[(16 * q + jj) * 64 + col] = x[jj];
    if constexpr (kSplit && std::is_same_v<T, float>)
    {
        // row `col` of the transposed K-major tile: K = 16 q .. 16 q + 15, two 8-value chunks
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            float v[8];
#pragma unroll
            for (int e = 0; e < 8; ++e)
                v[e] = x[8 * h + e];
            uint4 hi, lo;
            split8(v, hi, lo);
            const uint32_t off = sw128_offset(col, 16 * q + 8 * h);
            *reinterpret_cast<uint4 *>(split + off) = hi;
            *reinterpret_cast<uint4 *>(split + kSplitHalf + off) = lo;
        }
    }
}

} // namespace hyb
