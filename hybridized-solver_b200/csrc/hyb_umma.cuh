// hyb_umma.cuh - 5th-generation tensor-core (tcgen05 / UMMA) Schur update for the mixed
// form: FP32 blocks, products formed from a two-term BF16 split on the tensor cores.
//
// Every FP32 operand x is split into hi = bf16(x) and lo = bf16(x - hi); a product is taken
// as hi_a*hi_b + hi_a*lo_b + lo_a*hi_b (three BF16 MMAs, FP32 accumulation in tensor memory),
// which keeps about 16 significant bits per term -- the FP32 factorization is then brought
// to full FP64 accuracy by iterative refinement against the original FP64 matrix.
#pragma once

#include "hyb_kernels.cuh"

#include <cuda_bf16.h>

namespace hyb
{

constexpr int kUmmaThreads = 128;
// A (128 x 64) and B (64 x 64) as hi/lo BF16 tiles, each in the K-major 128-byte-swizzled
// layout the MMA reads: 16 + 16 + 8 + 8 KB, then the mbarrier and the tensor-memory address.
constexpr int kUmmaTileA = 128 * 64 * 2;
constexpr int kUmmaTileB = 64 * 64 * 2;
constexpr int kUmmaSmem = 2 * kUmmaTileA + 2 * kUmmaTileB + 64 + 1024; // + alignment slack

// Byte offset of element (row, k) of a K-major tile with 64 BF16 per row (one 128-byte
// swizzle row): rows come in groups of 8 (1024 bytes), the 16-byte chunks of a row are
// permuted by XOR with the row's index in its group.
__device__ __forceinline__ uint32_t sw128_offset(int row, int k)
{
    return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 3) ^ (row & 7))) << 4) + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start address, leading offset 16 B (unused by the
// swizzled K-major layout), stride 1024 B between 8-row groups, descriptor version 1,
// 128-byte swizzle.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tmem_load32(uint32_t addr, uint32_t (&v)[32])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                   "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                   "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                   "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                 : "r"(addr));
}

// Splits 4 consecutive FP32 values into hi and lo BF16 and stores them at byte offset `off`
// of the hi and lo tiles (the 4 values share one 16-byte chunk).
__device__ __forceinline__ void split_store4(unsigned char *hi, unsigned char *lo, uint32_t off, float4 x)
{
    const float v[4] = {x.x, x.y, x.z, x.w};
    __nv_bfloat16 h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        h[i] = __float2bfloat16_rn(v[i]);
        l[i] = __float2bfloat16_rn(v[i] - __bfloat162float(h[i]));
    }
    *reinterpret_cast<uint2 *>(hi + off) =
        make_uint2(((uint32_t)__bfloat16_as_ushort(h[1]) << 16) | __bfloat16_as_ushort(h[0]),
                   ((uint32_t)__bfloat16_as_ushort(h[3]) << 16) | __bfloat16_as_ushort(h[2]));
    *reinterpret_cast<uint2 *>(lo + off) =
        make_uint2(((uint32_t)__bfloat16_as_ushort(l[1]) << 16) | __bfloat16_as_ushort(l[0]),
                   ((uint32_t)__bfloat16_as_ushort(l[3]) << 16) | __bfloat16_as_ushort(l[2]));
}

// Uniform-64 FP32 update on the tensor cores. One CTA owns two target blocks of the same
// column block c and consecutive rows t_a, t_b of the pivot's lower column (M = 128 rows,
// N = 64): C(t,c) -= A(t,k) * U(k,c). Units: mode 0 enumerates row pairs of every pivot
// of the level through upd2_pref; with one pivot and lookahead, mode 1 takes row i0
// (one row per unit, every column) and then column j0 (row pairs of the other rows), and
// mode 2 the row pairs and columns other than (i0, j0). Each target row's arithmetic is
// the same whichever rows share its tile, so all modes give identical results.
__global__ void __launch_bounds__(kUmmaThreads)
    k_update64_umma(DevSym S, float *__restrict__ slab, int64_t p0, int64_t p1, int mode, int i0, int j0,
                    int *status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char *a_hi = base;
    unsigned char *a_lo = a_hi + kUmmaTileA;
    unsigned char *b_hi = a_lo + kUmmaTileA;
    unsigned char *b_lo = b_hi + kUmmaTileB;
    uint64_t *bar = reinterpret_cast<uint64_t *>(b_lo + kUmmaTileB);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);

    // ---- work unit: pivot k, lower-column rows (ia, ib), upper column j
    int64_t p = p0, local = blockIdx.x;
    if (mode == 0)
    {
        const int64_t u = S.upd2_pref[p0] + blockIdx.x;
        p = find_owner(S.upd2_pref, p0, p1, u);
        local = u - S.upd2_pref[p];
    }
    const int64_t k = S.piv[p];
    const int64_t n_lc = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
    const int64_t n_up = S.row_ptr[k + 1] - S.diag_pos[k] - 1;
    int64_t ia, ib, jj;
    bool has_b;
    if (mode == 1 && i0 >= 0 && local < n_up)
    {
        ia = i0; // the next pivot's row, alone
        ib = i0;
        jj = local;
        has_b = false;
    }
    else if (mode == 1)
    {
        // the next pivot's column: row pairs of every row except i0
        const int64_t pr = local - (i0 >= 0 ? n_up : 0);
        const int64_t rows = n_lc - (i0 >= 0 ? 1 : 0);
        ia = 2 * pr;
        ib = 2 * pr + 1;
        has_b = ib < rows;
        if (i0 >= 0)
        {
            ia += ia >= i0;
            ib += ib >= i0;
        }
        jj = j0;
    }
    else
    {
        const int64_t rows = n_lc - (mode == 2 && i0 >= 0 ? 1 : 0);
        const int64_t cols = n_up - (mode == 2 && j0 >= 0 ? 1 : 0);
        const int64_t pr = local / cols;
        jj = local % cols;
        ia = 2 * pr;
        ib = 2 * pr + 1;
        has_b = ib < rows;
        if (mode == 2)
        {
            if (i0 >= 0)
            {
                ia += ia >= i0;
                ib += ib >= i0;
            }
            if (j0 >= 0)
                jj += jj >= j0;
        }
    }
    const int64_t la = S.lcol_ptr[k] + ia, lb = S.lcol_ptr[k] + ib;
    const int64_t bu = S.diag_pos[k] + 1 + jj;
    const int32_t c = S.cols[bu];
    const float *ga = slab + S.blk_off[S.lcol_blk[la]];
    const float *gb2 = has_b ? slab + S.blk_off[S.lcol_blk[lb]] : nullptr;
    const float *gu = slab + S.blk_off[bu];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(64));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0)
        mbar_init(bar, 1);

    // ---- operands: FP32 -> (hi, lo) BF16 in the swizzled K-major layouts
    for (int i = tid; i < 128 * 16; i += kUmmaThreads)
    {
        const int r = i >> 4, q = (i & 15) * 4;
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        if (r < 64)
            x = *reinterpret_cast<const float4 *>(ga + r * 64 + q);
        else if (has_b)
            x = *reinterpret_cast<const float4 *>(gb2 + (r - 64) * 64 + q);
        split_store4(a_hi, a_lo, sw128_offset(r, q), x);
    }
    for (int i = tid; i < 64 * 64; i += kUmmaThreads)
    {
        // U is row-major [k][n]; the MMA wants it K-major (rows = n, K contiguous)
        const int kk = i >> 6, nn = i & 63;
        const float x = gu[i];
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
        *reinterpret_cast<__nv_bfloat16 *>(b_hi + sw128_offset(nn, kk)) = h;
        *reinterpret_cast<__nv_bfloat16 *>(b_lo + sw128_offset(nn, kk)) = l;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    // ---- 4 K-steps of 16, three split products each, one issuing thread
    if (tid == 0)
    {
        constexpr uint32_t idesc = umma_idesc_bf16(128, 64);
        const uint64_t dah = umma_smem_desc(smem_u32(a_hi)), dal = umma_smem_desc(smem_u32(a_lo));
        const uint64_t dbh = umma_smem_desc(smem_u32(b_hi)), dbl = umma_smem_desc(smem_u32(b_lo));
#pragma unroll
        for (int s = 0; s < 4; ++s)
        {
            const uint64_t off = (uint64_t)((s * 32) >> 4); // 16 BF16 = 32 bytes along K
            umma_bf16(tmem, dah + off, dbh + off, idesc, s > 0);
            umma_bf16(tmem, dah + off, dbl + off, idesc, 1);
            umma_bf16(tmem, dal + off, dbh + off, idesc, 1);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(bar))
                     : "memory");
    }
    const bool ok = mbar_wait(bar, 0);
    if (!ok && lane == 0)
        atomicOr(status + ST_TIMEOUT, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // ---- epilogue: row r of the product is tensor-memory lane r; C -= P in FP32
    const int r = warp * 32 + lane;
    float *gc = nullptr;
    if (ok && (r < 64 || has_b))
    {
        const int32_t t = S.lcol_row[r < 64 ? la : lb];
        const int64_t tgt = find_col(S.cols, S.row_ptr[t], S.row_ptr[t + 1], c);
        gc = slab + S.blk_off[tgt] + (r & 63) * 64;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
        uint32_t v[32];
        tmem_load32(tmem + ((uint32_t)(warp * 32) << 16) + h * 32, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (gc != nullptr)
        {
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                float4 cv = *reinterpret_cast<float4 *>(gc + h * 32 + q * 4);
                cv.x -= __uint_as_float(v[q * 4 + 0]);
                cv.y -= __uint_as_float(v[q * 4 + 1]);
                cv.z -= __uint_as_float(v[q * 4 + 2]);
                cv.w -= __uint_as_float(v[q * 4 + 3]);
                *reinterpret_cast<float4 *>(gc + h * 32 + q * 4) = cv;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64));
}

} // namespace hyb
