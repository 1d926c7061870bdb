// hyb_krylov.cuh - device side of the solves with A^T and of the Krylov refinement.
//
// * Solves with the transpose of the factored matrix: the block factors are A = L U with
//   L holding the Schur-complemented lower blocks and the diagonal blocks' LU (D = L_d U_d),
//   and U unit block-upper with the blocks D^{-1} A(k,c). So A^T = U^T L^T: forward with
//   U^T (identity diagonal blocks, blocks U(k,c)^T), then backward with L^T (blocks
//   L(t,k)^T and the diagonal D^T = U_d^T L_d^T). Both run level by level like the staged
//   solve (one launch per level and direction, partial products summed in a fixed order by
//   the CTA that takes a pivot's last ticket). They serve the 1-norm condition estimate
//   (Hager's method needs products with A^{-1} and with A^{-T}).
// * Column sums of |A| for ||A||_1, one CTA per block column over the column view of the
//   original pattern (no atomics).
// * Vector kernels of the FGMRES refinement: per-column dot products (deterministic two
//   passes), scaled updates with coefficients held in device memory, linear combinations.
//   Vectors are dof x nrhs row-major, each column an independent Krylov process.
#pragma once

#include "hyb_kernels.cuh"

namespace hyb
{

// Column view of the factors and of the original pattern, for the transposed solve and the
// column sums (built on the host at first use).
struct DevTrans
{
    const int64_t *ucol_ptr; // [n+1] upper blocks (k, c), k < c, of column c
    const int32_t *ucol_row; // row k of each, ascending
    const int32_t *ucol_blk; // filled block index of each
    const int64_t *fu_pref;  // [n+1] piv order: max(1, |upper column|) work units of the forward pass
    const int64_t *fu_rows;  // [n+1] piv order: partial-product rows (|upper column| * size, padded to 4)
    const int64_t *bu_pref;  // [n+1] piv order: max(1, |lower column|) units of the backward pass
    const int64_t *bu_rows;  // [n+1] piv order: partial rows (|lower column| * size, padded to 4)
    const int64_t *acol_ptr; // [n+1] original blocks (r, c) of block column c
    const int32_t *acol_row; // row r of each, ascending
    const int32_t *acol_blk; // index of the block in the original CSR order
};

// out[i][r] = sum_q blk[q][i] y[q][r] for a K x m row-major block (the product with its
// transpose). Threads take the columns i; when m < blockDim, G = blockDim / m groups split
// the rows q (group g: q = g, g + G, ...) and the group sums are added in group order.
// `red` is shared scratch of blockDim values. Every thread of the CTA calls it.
template <typename T, typename V>
__device__ void block_gemv_t(const T *__restrict__ blk, int K, int m, const V *__restrict__ y, V *__restrict__ out,
                             int nrhs, V *red)
{
    const int nt = blockDim.x, tid = threadIdx.x;
    for (int i0 = 0; i0 < m; i0 += nt)
    {
        const int mc = min(m - i0, nt);
        const int G = nt / mc;
        const int i = tid % mc, g = tid / mc;
        for (int r = 0; r < nrhs; ++r)
        {
            V s = V(0);
            if (g < G)
                for (int q = g; q < K; q += G)
                    s += (V)blk[(int64_t)q * m + i0 + i] * y[(int64_t)q * nrhs + r];
            __syncthreads(); // red is free
            if (g < G)
                red[g * mc + i] = s;
            __syncthreads();
            if (tid < mc)
            {
                V t = red[tid];
                for (int gg = 1; gg < G; ++gg)
                    t += red[gg * mc + tid];
                out[(int64_t)(i0 + tid) * nrhs + r] = t;
            }
        }
    }
    __syncthreads();
}

// x <- D^{-T} x for column r of acc (m x nrhs, shared memory), D = L_d U_d factored in
// place (row stride ldd): U_d^T z = x forward (U_d^T is lower triangular with U_d's
// diagonal), then L_d^T y = z backward (unit upper). One warp; the rows of U_d and of the
// multipliers L_d are read contiguously.
template <typename T, typename V> __device__ void warp_lu_solve_t(const T *d, int ldd, int m, V *acc, int r, int nrhs)
{
    const int lane = threadIdx.x & 31;
    for (int i = 0; i < m; ++i)
    {
        const V zi = acc[i * nrhs + r] / (V)d[(int64_t)i * ldd + i];
        __syncwarp();
        if (lane == 0)
            acc[i * nrhs + r] = zi;
        for (int q = i + 1 + lane; q < m; q += 32)
            acc[q * nrhs + r] -= (V)d[(int64_t)i * ldd + q] * zi;
        __syncwarp();
    }
    for (int i = m - 1; i >= 0; --i)
    {
        const V yi = acc[i * nrhs + r];
        __syncwarp();
        for (int q = lane; q < i; q += 32)
            acc[q * nrhs + r] -= (V)d[(int64_t)i * ldd + q] * yi;
        __syncwarp();
    }
}

// Forward pass with U^T for the level's pivots: y_c <- y_c - sum_k U(k,c)^T y_k over the
// upper blocks (k, c) of column c (rows k of earlier levels). Units: fu_pref, one per block.
template <typename T, typename V>
__global__ void __launch_bounds__(kThreads)
    k_fwdT_stage(DevSym S, DevTrans TS, const T *__restrict__ slab, V *__restrict__ y, V *__restrict__ scratch,
                 int *__restrict__ tickets, int64_t p0, int64_t p1, int nrhs)
{
    __shared__ __align__(16) V red[kThreads * 16 / sizeof(V)];
    const int64_t u = TS.fu_pref[p0] + blockIdx.x;
    const int64_t p = find_owner(TS.fu_pref, p0, p1, u);
    const int64_t c = S.piv[p];
    const int m = S.size[c];
    const int64_t nparts = TS.ucol_ptr[c + 1] - TS.ucol_ptr[c];
    if (nparts == 0)
        return; // nothing above column c: y_c is final as it is
    const int E = m * nrhs;
    V *part = scratch + (TS.fu_rows[p] - TS.fu_rows[p0]) * nrhs;
    const int64_t j = u - TS.fu_pref[p];
    const int64_t e = TS.ucol_ptr[c] + j;
    const int32_t k = TS.ucol_row[e];
    block_gemv_t(slab + S.blk_off[TS.ucol_blk[e]], S.size[k], m, y + S.dof_off[k] * nrhs, part + j * E, nrhs, red);
    if (!last_ticket(tickets, p, nparts))
        return;
    sum_partials(part, nparts, E, part, red);
    __syncthreads();
    V *yc = y + S.dof_off[c] * nrhs;
    for (int i = threadIdx.x; i < E; i += blockDim.x)
        yc[i] -= __ldcg(part + i);
}

// Backward pass with L^T: y_k <- D_k^{-T} (y_k - sum_t L(t,k)^T y_t) over the lower blocks
// (t, k) of column k (rows t of later levels). Units: bu_pref. Dynamic shared memory:
// m x nrhs values of the type V.
template <typename T, typename V>
__global__ void __launch_bounds__(kThreads)
    k_bwdT_stage(DevSym S, DevTrans TS, const T *__restrict__ slab, V *__restrict__ y, V *__restrict__ scratch,
                 int *__restrict__ tickets, int64_t p0, int64_t p1, int nrhs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) V red[kThreads * 16 / sizeof(V)];
    const int64_t u = TS.bu_pref[p0] + blockIdx.x;
    const int64_t p = find_owner(TS.bu_pref, p0, p1, u);
    const int64_t k = S.piv[p];
    const int m = S.size[k];
    const int E = m * nrhs;
    const int64_t nparts = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
    V *part = scratch + (TS.bu_rows[p] - TS.bu_rows[p0]) * nrhs;
    if (nparts > 0)
    {
        const int64_t j = u - TS.bu_pref[p];
        const int64_t e = S.lcol_ptr[k] + j;
        const int32_t t = S.lcol_row[e];
        block_gemv_t(slab + S.blk_off[S.lcol_blk[e]], S.size[t], m, y + S.dof_off[t] * nrhs, part + j * E, nrhs,
                     red);
        if (!last_ticket(tickets, p, nparts))
            return;
        sum_partials(part, nparts, E, part, red);
        __syncthreads();
    }
    V *acc = reinterpret_cast<V *>(smem_raw);
    V *yk = y + S.dof_off[k] * nrhs;
    for (int i = threadIdx.x; i < E; i += blockDim.x)
        acc[i] = nparts > 0 ? yk[i] - __ldcg(part + i) : yk[i];
    __syncthreads();
    const T *gd = slab + S.blk_off[S.diag_pos[k]];
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = warp; r < nrhs; r += nw)
        warp_lu_solve_t(gd, m, m, acc, r, nrhs);
    __syncthreads();
    for (int i = threadIdx.x; i < E; i += blockDim.x)
        yk[i] = acc[i];
}

// colsum[dof_off[c] + j] = sum over the original blocks (r, c) and their rows i of
// |a(r, c)[i][j]|: one CTA per block column c, threads over its columns j, blocks in
// ascending row order.
__global__ void __launch_bounds__(kThreads)
    k_col_abs_sums(DevSym S, DevTrans TS, const double *__restrict__ a, double *__restrict__ colsum)
{
    const int64_t c = blockIdx.x;
    const int nc = S.size[c];
    for (int j = threadIdx.x; j < nc; j += blockDim.x)
    {
        double s = 0;
        for (int64_t e = TS.acol_ptr[c]; e < TS.acol_ptr[c + 1]; ++e)
        {
            const int32_t r = TS.acol_row[e];
            const double *blk = a + S.a_val_off[TS.acol_blk[e]];
            const int nr = S.size[r];
            for (int i = 0; i < nr; ++i)
                s += fabs(blk[(int64_t)i * nc + j]);
        }
        colsum[S.dof_off[c] + j] = s;
    }
}

// ---------------------------------------------------------------------------------
// FGMRES vectors (dof x nrhs row-major, FP64).

// Per-column partial dot products of one CTA: partial[blockIdx.x * nrhs + r] (pass 1 of 2;
// k_sumsq_final adds the partials in CTA order).
__global__ void __launch_bounds__(kThreads)
    k_dot_partial(const double *__restrict__ a, const double *__restrict__ b, int64_t rows, int nrhs,
                  double *__restrict__ partial)
{
    __shared__ double red[kThreads];
    for (int r = 0; r < nrhs; ++r)
    {
        double s = 0;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x)
            s += a[i * nrhs + r] * b[i * nrhs + r];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1)
        {
            if ((int)threadIdx.x < o)
                red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            partial[(int64_t)blockIdx.x * nrhs + r] = red[0];
        __syncthreads();
    }
}

// Squared 2-norms of the segments of every column: out[s * nrhs + r] = sum over rows
// [off[s], off[s+1]) of v[i][r]^2. One CTA per segment, a fixed-order reduction.
__global__ void __launch_bounds__(kThreads)
    k_sumsq_segments(const double *__restrict__ v, const int64_t *__restrict__ off, int nrhs, double *__restrict__ out)
{
    __shared__ double red[kThreads];
    const int64_t seg = blockIdx.x, b = off[seg], e = off[seg + 1];
    for (int r = 0; r < nrhs; ++r)
    {
        double s = 0;
        for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x)
        {
            const double x = v[i * nrhs + r];
            s += x * x;
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1)
        {
            if ((int)threadIdx.x < o)
                red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            out[seg * nrhs + r] = red[0];
        __syncthreads();
    }
}

// dst[i][r] = (B)(src[i][r] * dscale[i]): the conversions around a substitution with
// factors of the scaled matrix S A S (dscale: S's diagonal, one value per unknown).
template <typename A, typename B>
__global__ void k_convert_scaled(const A *__restrict__ src, B *__restrict__ dst, const double *__restrict__ dscale,
                                 int64_t rows, int nrhs)
{
    const int64_t n = rows * nrhs;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (B)((double)src[i] * dscale[i / nrhs]);
}

// y[i][r] -= coef[r] * x[i][r] (the coefficients stay on the device between launches).
__global__ void k_sub_scaled(double *__restrict__ y, const double *__restrict__ x, const double *__restrict__ coef,
                             int64_t rows, int nrhs)
{
    const int64_t n = rows * nrhs;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] -= coef[i % nrhs] * x[i];
}

// y[i][r] = x[i][r] / sqrt(sumsq[r]), or 0 where sumsq[r] is 0 (a column whose Krylov
// space is exhausted contributes nothing further).
__global__ void k_normalize(double *__restrict__ y, const double *__restrict__ x, const double *__restrict__ sumsq,
                            int64_t rows, int nrhs)
{
    const int64_t n = rows * nrhs;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        const double s = sumsq[i % nrhs];
        y[i] = s > 0 ? x[i] / sqrt(s) : 0.0;
    }
}

// x[i][r] += sum_{j < k} coef[j * nrhs + r] * Z_j[i][r], Z_j = z + j * stride (ascending j).
__global__ void k_add_combination(double *__restrict__ x, const double *__restrict__ z, int64_t stride,
                                  const double *__restrict__ coef, int k, int64_t rows, int nrhs)
{
    const int64_t n = rows * nrhs;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        const int r = (int)(i % nrhs);
        double s = 0;
        for (int j = 0; j < k; ++j)
            s += coef[j * nrhs + r] * z[j * stride + i];
        x[i] += s;
    }
}

} // namespace hyb
