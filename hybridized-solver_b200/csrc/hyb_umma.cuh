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

// One 64x64 FP32 block as its BF16 split: hi (8 KB) then lo (8 KB), each a K-major tile of
// 64 rows x 64 K in the 128-byte-swizzled layout the MMA reads.
constexpr int kSplitBytes = 16384;
constexpr int kSplitHalf = 8192;

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

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Packs the BF16 split of 8 FP32 values into one 16-byte chunk of hi and one of lo.
__device__ __forceinline__ void split8(const float (&x)[8], uint4 &hi, uint4 &lo)
{
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const __nv_bfloat16 h0 = __float2bfloat16_rn(x[2 * i]), h1 = __float2bfloat16_rn(x[2 * i + 1]);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(x[2 * i] - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(x[2 * i + 1] - __bfloat162float(h1));
        h[i] = ((uint32_t)__bfloat16_as_ushort(h1) << 16) | __bfloat16_as_ushort(h0);
        l[i] = ((uint32_t)__bfloat16_as_ushort(l1) << 16) | __bfloat16_as_ushort(l0);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// ----------------------------------------------------------------------------------
// Operand staging of a tensor-core level: every lower-column block L(t,k) and upper-row
// block U(k,c) of the level's pivots, split once into BF16 hi/lo in the layout the MMA
// reads, so the update kernel only copies them into shared memory. Layout in `ops`: the
// level's pivots in order, each with its n_lc lower blocks then its n_up upper blocks,
// kSplitBytes apiece. L(t,k) is stored as it is (rows m, K = k contiguous); U(k,c) is
// stored transposed (rows = its columns n, K = k contiguous). The CTA of lower block i
// also writes the slab offsets of the targets (t_i, c_j) of its row for every upper
// column j into `tgt` (per pivot n_lc x n_up, at upd_pref[p] - upd_pref[p0]), so the
// update kernel finds a tile's C blocks with one load. With lower_only, only the lower
// blocks (and the target table) are written.
constexpr int kSplitThreads = 128;

__global__ void __launch_bounds__(kSplitThreads)
    k_split64(DevSym S, const float *__restrict__ slab, unsigned char *__restrict__ ops, int64_t *__restrict__ tgt,
              int64_t p0, int64_t p1, int lower_only)
{
    __shared__ float tr[64 * 65];
    const int64_t u = S.split_pref[p0] + blockIdx.x;
    const int64_t p = find_owner(S.split_pref, p0, p1, u);
    const int64_t k = S.piv[p];
    const int64_t local = u - S.split_pref[p];
    const int64_t n_lc = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
    unsigned char *dst = ops + (u - S.split_pref[p0]) * (int64_t)kSplitBytes;
    const int tid = threadIdx.x;
    if (local < n_lc)
    {
        const float *src = slab + S.blk_off[S.lcol_blk[S.lcol_ptr[k] + local]];
        for (int ch = tid; ch < 512; ch += kSplitThreads)
        {
            const int row = ch >> 3, q = ch & 7;
            const float4 a = *reinterpret_cast<const float4 *>(src + row * 64 + q * 8);
            const float4 b = *reinterpret_cast<const float4 *>(src + row * 64 + q * 8 + 4);
            const float x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            uint4 hi, lo;
            split8(x, hi, lo);
            const uint32_t off = sw128_offset(row, q * 8);
            *reinterpret_cast<uint4 *>(dst + off) = hi;
            *reinterpret_cast<uint4 *>(dst + kSplitHalf + off) = lo;
        }
        const int64_t n_up = S.row_ptr[k + 1] - S.diag_pos[k] - 1;
        const int32_t t = S.lcol_row[S.lcol_ptr[k] + local];
        int64_t *row_tgt = tgt + (S.upd_pref[p] - S.upd_pref[p0]) + local * n_up;
        for (int64_t j = tid; j < n_up; j += kSplitThreads)
        {
            const int32_t c = S.cols[S.diag_pos[k] + 1 + j];
            row_tgt[j] = S.blk_off[find_col(S.cols, S.row_ptr[t], S.row_ptr[t + 1], c)];
        }
        return;
    }
    if (lower_only) // the upper blocks' splits are written by the pivot kernel's row solves
        return;
    const float *src = slab + S.blk_off[S.diag_pos[k] + 1 + (local - n_lc)];
    for (int i = tid; i < 64 * 16; i += kSplitThreads)
    {
        const float4 v = *reinterpret_cast<const float4 *>(src + i * 4);
        const int r = i >> 4, c = (i & 15) * 4;
        tr[r * 65 + c] = v.x;
        tr[r * 65 + c + 1] = v.y;
        tr[r * 65 + c + 2] = v.z;
        tr[r * 65 + c + 3] = v.w;
    }
    __syncthreads();
    for (int ch = tid; ch < 512; ch += kSplitThreads)
    {
        const int n = ch >> 3, q = ch & 7;
        float x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
            x[i] = tr[(q * 8 + i) * 65 + n];
        uint4 hi, lo;
        split8(x, hi, lo);
        const uint32_t off = sw128_offset(n, q * 8);
        *reinterpret_cast<uint4 *>(dst + off) = hi;
        *reinterpret_cast<uint4 *>(dst + kSplitHalf + off) = lo;
    }
}

__device__ __forceinline__ void bulk_s2g(void *dst, const void *src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}

// ----------------------------------------------------------------------------------
// Uniform-64 FP32 Schur update on the tensor cores, C(t,c) -= L(t,k) U(k,c), computed
// transposed: one tile is D = U(k, [c0 c1])^T L(t,k)^T (M = 128: the 2 x 64 columns of two
// upper blocks, N = 64: the rows of one target row t, K = 64), so tensor-memory lane i holds
// column i of the tile. Each product takes three BF16 MMAs (hi*hi + hi*lo + lo*hi)
// accumulated in FP32.
//
// One persistent CTA per SM walks a contiguous range of tiles ordered column pair major,
// so the U pair stays in shared memory across its rows. All global traffic goes through
// the bulk-copy engine: warp 8 (one lane) copies the U pair, the L(t,k) splits (2-stage
// ring) and the tile's C blocks (3-slot ring, target offsets from the split kernel's
// table); warp 9 (one lane) issues the MMAs into one of two tensor-memory accumulators;
// warps 0-7 (warp w: lanes 32 (w & 3).., rows 32 (w >> 2)..) subtract the accumulator from
// C in shared memory, and one of them bulk-stores the blocks back. At about 160 KB of
// shared memory and few registers the CTA leaves room on its SM for the next pivot's
// LU/solve CTA. Every wait is bounded in time; on expiry the CTA sets ST_TIMEOUT, drains its
// copies and MMAs and returns.
//
// Tiles: mode 0 enumerates every pivot of the level through tc_pref (n_lc x column pairs);
// with one pivot and lookahead, mode 1 takes row i0 (column pairs) and then column j0 alone
// for every other row, and mode 2 the other rows x column pairs of the other columns.
// An element's value does not depend on which columns share its tile, so all modes give
// identical results.
constexpr int kTcThreads = 320;
constexpr int kTcEpiWarps = 8;
constexpr int kTcStages = 2; // L(t,k) operand ring
constexpr int kTcCSlots = 3; // C tile ring (two 16 KB blocks each)
constexpr int kTcCBytes = 2 * 16384;
constexpr int kTcSmem = 2 * kSplitBytes + kTcStages * kSplitBytes + kTcCSlots * kTcCBytes + 256 + 1024;

struct TcTile
{
    int64_t p;   // pivot slot
    int64_t row; // index in the pivot's lower column
    int32_t ja;  // index in the pivot's upper row of the tile's first column block
    int32_t jb;  // second column block, -1 if the tile has one
};

__device__ __forceinline__ TcTile tc_tile(const DevSym &S, int64_t p0, int64_t p1, int mode, int i0, int j0,
                                          int64_t t)
{
    TcTile x;
    int64_t p = p0, local = t;
    if (mode == 0)
    {
        const int64_t u = S.tc_pref[p0] + t;
        p = find_owner(S.tc_pref, p0, p1, u);
        local = u - S.tc_pref[p];
    }
    const int64_t k = S.piv[p];
    const int64_t n_lc = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
    const int32_t n_up = (int32_t)(S.row_ptr[k + 1] - S.diag_pos[k] - 1);
    x.p = p;
    if (mode == 0)
    {
        const int64_t cp = local / n_lc;
        x.row = local - cp * n_lc;
        x.ja = (int32_t)(2 * cp);
        x.jb = x.ja + 1 < n_up ? x.ja + 1 : -1;
    }
    else if (mode == 1)
    {
        const int64_t ncp = i0 >= 0 ? (n_up + 1) / 2 : 0;
        if (local < ncp)
        {
            x.row = i0;
            x.ja = (int32_t)(2 * local);
            x.jb = x.ja + 1 < n_up ? x.ja + 1 : -1;
        }
        else
        {
            const int64_t r = local - ncp;
            x.row = r + (i0 >= 0 && r >= i0);
            x.ja = j0;
            x.jb = -1;
        }
    }
    else
    {
        const int64_t nr = n_lc - (i0 >= 0);
        const int32_t nc = n_up - (j0 >= 0);
        const int64_t cp = local / nr;
        const int64_t r = local - cp * nr;
        x.row = r + (i0 >= 0 && r >= i0);
        const int32_t a = (int32_t)(2 * cp), b = a + 1;
        x.ja = a + (j0 >= 0 && a >= j0);
        x.jb = b < nc ? b + (j0 >= 0 && b >= j0) : -1;
    }
    return x;
}

__global__ void __launch_bounds__(kTcThreads, 1)
    k_update64_tc(DevSym S, float *__restrict__ slab, const unsigned char *__restrict__ ops,
                  const int64_t *__restrict__ tgt, int64_t p0, int64_t p1, int mode, int i0, int j0, int64_t n_tiles,
                  int *status, int reverse)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char *u_hi = base;                           // M = 128 rows: column block ja, then jb
    unsigned char *u_lo = u_hi + kSplitBytes;             //
    unsigned char *ring = u_lo + kSplitBytes;             // kTcStages x (hi 8 KB, lo 8 KB) of L(t,k)
    unsigned char *cbuf = ring + kTcStages * kSplitBytes; // kTcCSlots x (C(t, c_ja), C(t, c_jb)) FP32
    uint64_t *bars = reinterpret_cast<uint64_t *>(cbuf + kTcCSlots * kTcCBytes);
    uint64_t *full = bars;                // [kTcStages] operand landed
    uint64_t *empty = full + kTcStages;   // [kTcStages] operand consumed by the MMAs
    uint64_t *cfull = empty + kTcStages;  // [kTcCSlots] C blocks landed
    uint64_t *cempty = cfull + kTcCSlots; // [kTcCSlots] C blocks stored back (slot free)
    uint64_t *ufull = cempty + kTcCSlots; // U pair landed
    uint64_t *uempty = ufull + 1;         // MMAs on the previous U pair done
    uint64_t *tfull = ufull + 2;          // [2] accumulator ready
    uint64_t *tempty = ufull + 4;         // [2] accumulator drained (one arrival per epilogue warp)
    uint64_t *done = ufull + 6;           // all MMAs of the CTA done
    int64_t *coff = reinterpret_cast<int64_t *>(ufull + 7); // [kTcCSlots][2] target offsets of a slot
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(coff + 2 * kTcCSlots);
    __shared__ int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t t0 = n_tiles * blockIdx.x / gridDim.x, t1 = n_tiles * (blockIdx.x + 1) / gridDim.x;
    // With `reverse` the CTA walks its range from the end: on alternate levels every CTA
    // starts on the targets it wrote last (consecutive levels update nearly the same
    // targets), which are still in L2; column-pair-major order, and with it the reuse of
    // the U pair, is kept. Every target's arithmetic is the same either way.
    auto tix = [&](int64_t t) { return reverse ? t0 + t1 - 1 - t : t; };
    if (tid == 0)
    {
        for (int i = 0; i < kTcStages; ++i)
        {
            mbar_init(full + i, 1);
            mbar_init(empty + i, 1);
        }
        for (int i = 0; i < kTcCSlots; ++i)
        {
            mbar_init(cfull + i, 1);
            mbar_init(cempty + i, 1);
        }
        mbar_init(ufull, 1);
        mbar_init(uempty, 1);
        mbar_init(tfull, 1);
        mbar_init(tfull + 1, 1);
        mbar_init(tempty, kTcEpiWarps);
        mbar_init(tempty + 1, kTcEpiWarps);
        mbar_init(done, 1);
        s_fail = schedule_aborted(status);
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(128));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int64_t lvl_base = S.split_pref[p0];
    const int64_t tgt_base = S.upd_pref[p0];
    const bool run = s_fail == 0; // read by every thread before any role can change it
    __syncthreads();

    if (!run)
    {
    }
    else if (warp == kTcEpiWarps)
    {
        // ---- producer: U pair on change, one L(t,k) split and the C blocks per tile
        if (lane == 0)
        {
            // target offsets of a tile (loads issued one tile ahead of their use)
            auto targets = [&](const TcTile &x, int64_t &oa, int64_t &ob) {
                const int64_t k = S.piv[x.p];
                const int64_t n_up = S.row_ptr[k + 1] - S.diag_pos[k] - 1;
                const int64_t *row_tgt = tgt + (S.upd_pref[x.p] - tgt_base) + x.row * n_up;
                oa = row_tgt[x.ja];
                ob = x.jb >= 0 ? row_tgt[x.jb] : -1;
            };
            int64_t cur_p = -1;
            int32_t cur_a = -2, cur_b = -2;
            uint32_t uloads = 0;
            TcTile xn{};
            int64_t na = -1, nb = -1;
            if (t0 < t1)
            {
                xn = tc_tile(S, p0, p1, mode, i0, j0, tix(t0));
                targets(xn, na, nb);
            }
            int64_t i = 0;
            for (int64_t t = t0; t < t1; ++t, ++i)
            {
                const TcTile x = xn;
                const int64_t off_a = na, off_b = nb;
                if (t + 1 < t1)
                {
                    xn = tc_tile(S, p0, p1, mode, i0, j0, tix(t + 1));
                    targets(xn, na, nb);
                }
                const int64_t k = S.piv[x.p];
                const int64_t n_lc = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
                const unsigned char *pb = ops + (S.split_pref[x.p] - lvl_base) * (int64_t)kSplitBytes;
                if (x.p != cur_p || x.ja != cur_a || x.jb != cur_b)
                {
                    if (uloads > 0 && !mbar_wait(uempty, (uloads - 1) & 1))
                    {
                        s_fail = 1;
                        break;
                    }
                    mbar_expect_tx(ufull, x.jb >= 0 ? 2 * kSplitBytes : kSplitBytes);
                    const unsigned char *sa = pb + (n_lc + x.ja) * (int64_t)kSplitBytes;
                    bulk_g2s(u_hi, sa, kSplitHalf, ufull);
                    bulk_g2s(u_lo, sa + kSplitHalf, kSplitHalf, ufull);
                    if (x.jb >= 0)
                    {
                        const unsigned char *sb = pb + (n_lc + x.jb) * (int64_t)kSplitBytes;
                        bulk_g2s(u_hi + kSplitHalf, sb, kSplitHalf, ufull);
                        bulk_g2s(u_lo + kSplitHalf, sb + kSplitHalf, kSplitHalf, ufull);
                    }
                    ++uloads;
                    cur_p = x.p;
                    cur_a = x.ja;
                    cur_b = x.jb;
                }
                const int s = (int)(i % kTcStages);
                if (i >= kTcStages && !mbar_wait(empty + s, (uint32_t)((i / kTcStages - 1) & 1)))
                {
                    s_fail = 1;
                    break;
                }
                mbar_expect_tx(full + s, kSplitBytes);
                bulk_g2s(ring + s * kSplitBytes, pb + x.row * (int64_t)kSplitBytes, kSplitBytes, full + s);
                const int cs = (int)(i % kTcCSlots);
                if (i >= kTcCSlots && !mbar_wait(cempty + cs, (uint32_t)((i / kTcCSlots - 1) & 1)))
                {
                    s_fail = 1;
                    break;
                }
                coff[2 * cs] = off_a;
                coff[2 * cs + 1] = off_b;
                unsigned char *cb = cbuf + cs * kTcCBytes;
                // the arrive releases coff to the epilogue together with the copies
                mbar_expect_tx(cfull + cs, off_b >= 0 ? 2 * 16384 : 16384);
                bulk_g2s(cb, slab + off_a, 16384, cfull + cs);
                if (off_b >= 0)
                    bulk_g2s(cb + 16384, slab + off_b, 16384, cfull + cs);
            }
            // drain: every copy issued lands before the CTA can leave
            const int64_t issued = i;
            for (int64_t j = issued > kTcStages ? issued - kTcStages : 0; j < issued; ++j)
                if (!mbar_wait(full + (j % kTcStages), (uint32_t)((j / kTcStages) & 1)))
                    s_fail = 1;
            for (int64_t j = issued > kTcCSlots ? issued - kTcCSlots : 0; j < issued; ++j)
                if (!mbar_wait(cfull + (j % kTcCSlots), (uint32_t)((j / kTcCSlots) & 1)))
                    s_fail = 1;
            if (uloads > 0 && !mbar_wait(ufull, (uloads - 1) & 1))
                s_fail = 1;
        }
    }
    else if (warp == kTcEpiWarps + 1)
    {
        // ---- MMA issuer
        if (lane == 0)
        {
            constexpr uint32_t idesc = umma_idesc_bf16(128, 64);
            const uint64_t duh = umma_smem_desc(smem_u32(u_hi)), dul = umma_smem_desc(smem_u32(u_lo));
            int64_t cur_p = -1;
            int32_t cur_a = -2, cur_b = -2;
            uint32_t uloads = 0;
            int64_t i = 0;
            for (int64_t t = t0; t < t1; ++t, ++i)
            {
                const TcTile x = tc_tile(S, p0, p1, mode, i0, j0, tix(t));
                if (x.p != cur_p || x.ja != cur_a || x.jb != cur_b)
                {
                    if (uloads > 0)
                        umma_commit(uempty);
                    if (!mbar_wait(ufull, uloads & 1))
                    {
                        s_fail = 1;
                        break;
                    }
                    ++uloads;
                    cur_p = x.p;
                    cur_a = x.ja;
                    cur_b = x.jb;
                }
                const int s = (int)(i % kTcStages);
                const int a = (int)(i & 1);
                if (!mbar_wait(full + s, (uint32_t)((i / kTcStages) & 1)) ||
                    (i >= 2 && !mbar_wait(tempty + a, (uint32_t)(((i >> 1) - 1) & 1))))
                {
                    s_fail = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t lh = smem_u32(ring + s * kSplitBytes);
                const uint64_t dlh = umma_smem_desc(lh), dll = umma_smem_desc(lh + kSplitHalf);
                const uint32_t acc = tmem + (uint32_t)(a * 64);
#pragma unroll
                for (int ks = 0; ks < 4; ++ks)
                {
                    const uint64_t off = (uint64_t)((ks * 32) >> 4); // 16 BF16 = 32 bytes along K
                    umma_bf16(acc, duh + off, dlh + off, idesc, ks > 0);
                    umma_bf16(acc, duh + off, dll + off, idesc, 1);
                    umma_bf16(acc, dul + off, dlh + off, idesc, 1);
                }
                umma_commit(empty + s);
                umma_commit(tfull + a);
            }
            umma_commit(done);
            if (!mbar_wait(done, 0))
                s_fail = 1;
        }
    }
    else
    {
        // ---- epilogue warps 0-7: lane i of warp w is column (w & 1) * 32 + i of block
        // ((w & 3) < 2 ? ja : jb) and covers rows 32 (w >> 2) .. + 31 of the tile. Every
        // epilogue warp runs all of the CTA's tiles -- after a failed wait without waiting or
        // computing -- so the named barrier below always sees all eight warps.
        const int q = warp & 3, h = warp >> 2;
        const int cb_idx = q >> 1;
        const int col = (q & 1) * 32 + lane;
        bool failed = false; // warp-uniform
        int64_t i = 0;
        for (int64_t t = t0; t < t1; ++t, ++i)
        {
            const int a = (int)(i & 1);
            const int cs = (int)(i % kTcCSlots);
            if (!failed && !__all_sync(0xffffffffu, mbar_wait(tfull + a, (uint32_t)((i >> 1) & 1)) &&
                                                        mbar_wait(cfull + cs, (uint32_t)((i / kTcCSlots) & 1))))
            {
                s_fail = 1;
                failed = true;
            }
            if (!failed)
            {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                uint32_t v[32];
                tmem_load32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * 64 + h * 32), v);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0)
                    mbar_arrive(tempty + a);
                if (cb_idx == 0 || coff[2 * cs + 1] >= 0)
                {
                    float *c =
                        reinterpret_cast<float *>(cbuf + cs * kTcCBytes + cb_idx * 16384) + h * 32 * 64 + col;
#pragma unroll
                    for (int r = 0; r < 32; ++r)
                        c[r * 64] -= __uint_as_float(v[r]);
                }
            }
            // the bulk store reads what the generic stores wrote
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
            if (tid == 0 && !failed) // warp 0 saw this slot's C land, so its offsets are valid
            {
                const unsigned char *cb = cbuf + cs * kTcCBytes;
                bulk_s2g(slab + coff[2 * cs], cb, 16384);
                if (coff[2 * cs + 1] >= 0)
                    bulk_s2g(slab + coff[2 * cs + 1], cb + 16384, 16384);
                asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                mbar_arrive(cempty + cs);
            }
        }
        if (tid == 0)
            asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); // stores complete before exit
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0 && s_fail)
        atomicOr(status + ST_TIMEOUT, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
}

// ----------------------------------------------------------------------------------
// Two pivots per pass (a pair of consecutive single-pivot levels, Symbolic::PairShape):
// C(t,c) -= L(t,a) U(a,c) + L(t,b) U(b,c) over b's targets, with a's product only where a
// reaches the target. The tile is that of k_update64_tc (one target row t x two upper
// columns, M = 128, N = 64) with K = 128: a's three BF16 products, then b's, accumulate
// into one FP32 tensor-memory accumulator, and the target is read and written once for
// both pivots -- half the target traffic of two single-pivot passes.
//
// Shared memory holds both pivots' U pairs (64 KB; a column a does not reach is a zero
// block) and a four-entry ring of L blocks (one source each); the targets do not pass
// through shared memory: each epilogue thread loads its 32 values of the next tile into
// registers while the current tile's products run, and the producer lane prefetches the
// targets of tiles further ahead into L2. At ~130 KB of shared memory and <= 128 registers
// per thread the CTA leaves room on its SM for the next pivots' LU / row-solve CTAs.
constexpr int kTc2Threads = 320;
constexpr int kTc2LStages = 4;  // L(t, .) ring entries
constexpr int kTc2Prefetch = 2; // tiles ahead of the producer whose targets go to L2
constexpr int kTc2Smem = 4 * kSplitBytes + kTc2LStages * kSplitBytes + 256 + 1024;

struct Tc2Tile
{
    int32_t row; // index in b's lower column
    int32_t ja;  // index in b's upper row of the first column block
    int32_t jb;  // second column block, -1 if the tile has one
};

// Index x of a sequence with the positions s0 < s1 (-1: absent, present ones first) removed.
__host__ __device__ __forceinline__ int32_t skip_two(int32_t x, int32_t s0, int32_t s1)
{
    if (s0 >= 0 && x >= s0)
        ++x;
    if (s1 >= 0 && x >= s1)
        ++x;
    return x;
}

// Tile t of a pair pass. mode 0: every target, column pair major; mode 1: the priority rows
// pr.x, pr.y x every column pair, then the priority columns (pr.z, pr.w) of every other
// row in one tile; mode 2: the other rows x pairs of the other columns, column pair major.
__host__ __device__ __forceinline__ Tc2Tile tc2_tile(int32_t n_lc, int32_t n_up, int mode, int4 pr, int64_t t)
{
    Tc2Tile x;
    if (mode == 0)
    {
        const int32_t cp = (int32_t)(t / n_lc);
        x.row = (int32_t)(t - (int64_t)cp * n_lc);
        x.ja = 2 * cp;
        x.jb = x.ja + 1 < n_up ? x.ja + 1 : -1;
        return x;
    }
    const int32_t nri = (pr.x >= 0) + (pr.y >= 0), ncj = (pr.z >= 0) + (pr.w >= 0);
    if (mode == 1)
    {
        const int32_t ncp = (n_up + 1) / 2;
        const int64_t np = (int64_t)nri * ncp;
        if (t < np)
        {
            const int32_t r = (int32_t)(t / ncp), cp = (int32_t)(t - (int64_t)r * ncp);
            x.row = r == 0 ? pr.x : pr.y;
            x.ja = 2 * cp;
            x.jb = x.ja + 1 < n_up ? x.ja + 1 : -1;
        }
        else
        {
            x.row = skip_two((int32_t)(t - np), pr.x, pr.y);
            x.ja = pr.z;
            x.jb = pr.w;
        }
        return x;
    }
    const int32_t nr = n_lc - nri, nc = n_up - ncj;
    const int32_t cp = (int32_t)(t / nr);
    x.row = skip_two((int32_t)(t - (int64_t)cp * nr), pr.x, pr.y);
    const int32_t a = 2 * cp, b = a + 1;
    x.ja = skip_two(a, pr.z, pr.w);
    x.jb = b < nc ? skip_two(b, pr.z, pr.w) : -1;
    return x;
}

__device__ __forceinline__ void tmem_load16(uint32_t addr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                 "[%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                   "=r"(v[15])
                 : "r"(addr));
}

__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// ops_a / ops_b: the BF16 splits of the levels of a (slot pa) and b (slot pb), each its
// lower-column blocks then its upper-row blocks; tgt: b's target-offset table (k_split64);
// zero_split: one all-zero split block. Every wait is bounded; on expiry the CTA sets
// ST_TIMEOUT, lets its copies and MMAs finish and returns.
__global__ void __launch_bounds__(kTc2Threads, 1)
    k_update64_tc2(DevSym S, float *__restrict__ slab, const unsigned char *__restrict__ ops_a,
                   const unsigned char *__restrict__ ops_b, const int64_t *__restrict__ tgt,
                   const unsigned char *__restrict__ zero_split, int64_t pa, int64_t pb, int mode, int4 pr,
                   int64_t n_tiles, int *status, int reverse)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char *ua = base;                   // U(a, [ja jb]): hi (ja, jb) then lo (ja, jb)
    unsigned char *ub = base + 2 * kSplitBytes; // U(b, [ja jb])
    unsigned char *ring = base + 4 * kSplitBytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kTc2LStages * kSplitBytes);
    uint64_t *full = bars;                 // [kTc2LStages] L block landed
    uint64_t *empty = full + kTc2LStages;  // [kTc2LStages] L block consumed by the MMAs
    uint64_t *ufull = empty + kTc2LStages; // U pairs landed
    uint64_t *uempty = ufull + 1;          // MMAs on the previous U pairs done
    uint64_t *tfull = ufull + 2;           // [2] accumulator ready
    uint64_t *tempty = ufull + 4;          // [2] accumulator drained (one arrival per epilogue warp)
    uint64_t *done = ufull + 6;            // all MMAs of the CTA done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(ufull + 7);
    __shared__ int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t ka = S.piv[pa], kb = S.piv[pb];
    const int32_t n_lc_a = (int32_t)(S.lcol_ptr[ka + 1] - S.lcol_ptr[ka]);
    const int32_t n_lc = (int32_t)(S.lcol_ptr[kb + 1] - S.lcol_ptr[kb]);
    const int32_t n_up = (int32_t)(S.row_ptr[kb + 1] - S.diag_pos[kb] - 1);
    const int32_t *rmap = S.pair_map + S.split_pref[pb]; // b's lower row i -> a's, or -1
    const int32_t *cmap = rmap + n_lc;                    // b's upper column j -> a's, or -1
    const int64_t t0 = n_tiles * blockIdx.x / gridDim.x, t1 = n_tiles * (blockIdx.x + 1) / gridDim.x;
    auto tix = [&](int64_t t) { return reverse ? t0 + t1 - 1 - t : t; };
    auto tile = [&](int64_t t) { return tc2_tile(n_lc, n_up, mode, pr, tix(t)); };
    // whether a reaches any column of a tile's pair, and a given row
    auto a_cols = [&](const Tc2Tile &x) { return cmap[x.ja] >= 0 || (x.jb >= 0 && cmap[x.jb] >= 0); };
    if (tid == 0)
    {
        for (int i = 0; i < kTc2LStages; ++i)
        {
            mbar_init(full + i, 1);
            mbar_init(empty + i, 1);
        }
        mbar_init(ufull, 1);
        mbar_init(uempty, 1);
        mbar_init(tfull, 1);
        mbar_init(tfull + 1, 1);
        mbar_init(tempty, kTcEpiWarps);
        mbar_init(tempty + 1, kTcEpiWarps);
        mbar_init(done, 1);
        s_fail = schedule_aborted(status);
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(128));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const bool run = s_fail == 0; // read by every thread before any role can change it
    __syncthreads();

    if (!run)
    {
    }
    else if (warp == kTcEpiWarps)
    {
        // ---- producer: both U pairs on change, one L block per source and tile, and the
        // targets of a tile kTc2Prefetch ahead into L2
        if (lane == 0)
        {
            int32_t cur_a = -2, cur_b = -2;
            bool cols_a = false;
            uint32_t uloads = 0;
            int64_t e = 0;
            bool ok = true;
            for (int64_t t = t0; t < t1 && ok; ++t)
            {
                const Tc2Tile x = tile(t);
                if (x.ja != cur_a || x.jb != cur_b)
                {
                    if (uloads > 0 && !mbar_wait(uempty, (uloads - 1) & 1))
                    {
                        ok = false;
                        break;
                    }
                    cols_a = a_cols(x);
                    const int halves = x.jb >= 0 ? 2 : 1;
                    mbar_expect_tx(ufull, (uint32_t)(halves * (cols_a ? 2 : 1) * kSplitBytes));
                    for (int hsel = 0; hsel < halves; ++hsel)
                    {
                        const int32_t j = hsel ? x.jb : x.ja;
                        const unsigned char *sb = ops_b + (int64_t)(n_lc + j) * kSplitBytes;
                        bulk_g2s(ub + hsel * kSplitHalf, sb, kSplitHalf, ufull);
                        bulk_g2s(ub + kSplitBytes + hsel * kSplitHalf, sb + kSplitHalf, kSplitHalf, ufull);
                        if (cols_a)
                        {
                            const int32_t ja = cmap[j];
                            const unsigned char *sa =
                                ja >= 0 ? ops_a + (int64_t)(n_lc_a + ja) * kSplitBytes : zero_split;
                            bulk_g2s(ua + hsel * kSplitHalf, sa, kSplitHalf, ufull);
                            bulk_g2s(ua + kSplitBytes + hsel * kSplitHalf, sa + kSplitHalf, kSplitHalf, ufull);
                        }
                    }
                    ++uloads;
                    cur_a = x.ja;
                    cur_b = x.jb;
                }
                const int32_t ra = cols_a ? rmap[x.row] : -1;
                for (int src = ra >= 0 ? 0 : 1; src < 2; ++src)
                {
                    const int s = (int)(e % kTc2LStages);
                    if (e >= kTc2LStages && !mbar_wait(empty + s, (uint32_t)((e / kTc2LStages - 1) & 1)))
                    {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(full + s, kSplitBytes);
                    const unsigned char *sl =
                        src == 0 ? ops_a + (int64_t)ra * kSplitBytes : ops_b + (int64_t)x.row * kSplitBytes;
                    bulk_g2s(ring + s * kSplitBytes, sl, kSplitBytes, full + s);
                    ++e;
                }
                if (ok && t + kTc2Prefetch < t1)
                {
                    const Tc2Tile y = tile(t + kTc2Prefetch);
                    const int64_t *row_tgt = tgt + (int64_t)y.row * n_up;
                    prefetch_l2(slab + row_tgt[y.ja], 16384);
                    if (y.jb >= 0)
                        prefetch_l2(slab + row_tgt[y.jb], 16384);
                }
            }
            if (!ok)
                s_fail = 1;
            // drain: every copy issued lands before the CTA can leave
            for (int64_t j = e > kTc2LStages ? e - kTc2LStages : 0; j < e; ++j)
                if (!mbar_wait(full + (j % kTc2LStages), (uint32_t)((j / kTc2LStages) & 1)))
                    s_fail = 1;
            if (uloads > 0 && !mbar_wait(ufull, (uloads - 1) & 1))
                s_fail = 1;
        }
    }
    else if (warp == kTcEpiWarps + 1)
    {
        // ---- MMA issuer: per tile a's products (where a reaches it), then b's
        if (lane == 0)
        {
            constexpr uint32_t idesc = umma_idesc_bf16(128, 64);
            int32_t cur_a = -2, cur_b = -2;
            bool cols_a = false;
            uint32_t uloads = 0;
            int64_t e = 0, i = 0;
            bool ok = true;
            for (int64_t t = t0; t < t1 && ok; ++t, ++i)
            {
                const Tc2Tile x = tile(t);
                if (x.ja != cur_a || x.jb != cur_b)
                {
                    if (uloads > 0)
                        umma_commit(uempty);
                    if (!mbar_wait(ufull, uloads & 1))
                    {
                        ok = false;
                        break;
                    }
                    ++uloads;
                    cols_a = a_cols(x);
                    cur_a = x.ja;
                    cur_b = x.jb;
                }
                const int acc_i = (int)(i & 1);
                if (i >= 2 && !mbar_wait(tempty + acc_i, (uint32_t)(((i >> 1) - 1) & 1)))
                {
                    ok = false;
                    break;
                }
                const uint32_t acc = tmem + (uint32_t)(acc_i * 64);
                const bool use_a = cols_a && rmap[x.row] >= 0;
                for (int src = use_a ? 0 : 1; src < 2; ++src)
                {
                    const int s = (int)(e % kTc2LStages);
                    if (!mbar_wait(full + s, (uint32_t)((e / kTc2LStages) & 1)))
                    {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t uh = smem_u32(src == 0 ? ua : ub);
                    const uint64_t duh = umma_smem_desc(uh), dul = umma_smem_desc(uh + kSplitBytes);
                    const uint32_t lh = smem_u32(ring + s * kSplitBytes);
                    const uint64_t dlh = umma_smem_desc(lh), dll = umma_smem_desc(lh + kSplitHalf);
                    const bool first = src == (use_a ? 0 : 1);
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks)
                    {
                        const uint64_t off = (uint64_t)((ks * 32) >> 4); // 16 BF16 = 32 bytes along K
                        umma_bf16(acc, duh + off, dlh + off, idesc, (first && ks == 0) ? 0u : 1u);
                        umma_bf16(acc, duh + off, dll + off, idesc, 1);
                        umma_bf16(acc, dul + off, dlh + off, idesc, 1);
                    }
                    umma_commit(empty + s);
                    ++e;
                }
                if (ok)
                    umma_commit(tfull + acc_i);
            }
            if (!ok)
                s_fail = 1;
            umma_commit(done);
            if (!mbar_wait(done, 0))
                s_fail = 1;
        }
    }
    else
    {
        // ---- epilogue warps 0-7: lane i of warp w is column (w & 1) * 32 + i of block
        // ((w & 3) < 2 ? ja : jb), rows 32 (w >> 2) .. + 31 of the tile. The target values of
        // the next tile are loaded into registers before this tile's accumulator is awaited.
        const int q = warp & 3, h = warp >> 2;
        const int cb_idx = q >> 1;
        const int col = (q & 1) * 32 + lane;
        const int64_t rowoff = (int64_t)(h * 32) * 64 + col;
        auto target = [&](int64_t t) -> int64_t {
            const Tc2Tile x = tile(t);
            const int32_t j = cb_idx ? x.jb : x.ja;
            return j < 0 ? -1 : tgt[(int64_t)x.row * n_up + j];
        };
        float cn[32];
        int64_t on = t0 < t1 ? target(t0) : -1;
        if (on >= 0)
        {
            const float *src = slab + on + rowoff;
#pragma unroll
            for (int r = 0; r < 32; ++r)
                cn[r] = src[r * 64];
        }
        bool failed = false; // warp-uniform
        int64_t i = 0;
        for (int64_t t = t0; t < t1; ++t, ++i)
        {
            float cc[32];
#pragma unroll
            for (int r = 0; r < 32; ++r)
                cc[r] = cn[r];
            const int64_t oc = on;
            on = -1;
            if (!failed && t + 1 < t1)
            {
                on = target(t + 1);
                if (on >= 0)
                {
                    const float *src = slab + on + rowoff;
#pragma unroll
                    for (int r = 0; r < 32; ++r)
                        cn[r] = src[r * 64];
                }
            }
            const int acc_i = (int)(i & 1);
            if (!failed && !__all_sync(0xffffffffu, mbar_wait(tfull + acc_i, (uint32_t)((i >> 1) & 1))))
            {
                s_fail = 1;
                failed = true;
            }
            if (failed)
                continue;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // the accumulator in two halves of 16 rows, so only 16 of its values are live
            const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc_i * 64 + h * 32);
            float *dst = slab + oc + rowoff;
            uint32_t v[16];
            tmem_load16(ta, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (oc >= 0)
            {
#pragma unroll
                for (int r = 0; r < 16; ++r)
                    dst[r * 64] = cc[r] - __uint_as_float(v[r]);
            }
            tmem_load16(ta + 16, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                mbar_arrive(tempty + acc_i);
            if (oc >= 0)
            {
#pragma unroll
                for (int r = 0; r < 16; ++r)
                    dst[(r + 16) * 64] = cc[r + 16] - __uint_as_float(v[r]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0 && s_fail)
        atomicOr(status + ST_TIMEOUT, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
}

} // namespace hyb
