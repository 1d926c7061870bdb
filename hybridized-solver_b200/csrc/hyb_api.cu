// hyb_api.cu - the C ABI (include/hybsol_b200.h): handle lifecycle, device memory,
// the level schedule (captured into CUDA graphs), plain FP64 and mixed FP32+refinement
// solves.
#include "hyb_internal.h"
#include "hyb_kernels.cuh"
#include "hyb_krylov.cuh"
#include "hyb_pivot.cuh"
#include "hyb_umma.cuh"

#include "hybsol_b200.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

using hyb::DevSym;
using hyb::Symbolic;

namespace
{
thread_local std::string g_cuda_error;

int cuda_fail(cudaError_t e, const char *what)
{
    g_cuda_error = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation)
        return HYB_FAILED_ALLOC;
    return HYB_CUDA_ERROR;
}

#define HYB_CUDA(call)                                                                                                 \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess)                                                                                         \
            return cuda_fail(e_, #call);                                                                               \
    } while (0)

// Largest dynamic shared memory a CTA may request on this device (set once per kernel).
int g_smem_optin = 0;

int smem_optin()
{
    if (g_smem_optin == 0)
    {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        g_smem_optin = v > 0 ? v : 48 * 1024;
    }
    return g_smem_optin;
}

// Dynamic shared memory the forward solve stage may take (its static arrays aside).
int solve_smem_cap()
{
    return smem_optin() - 8192;
}

// Streaming multiprocessors of the current device.
int g_sm_count = 0;

int sm_count()
{
    if (g_sm_count == 0)
    {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        g_sm_count = v > 0 ? v : 1;
    }
    return g_sm_count;
}

// Lets `kernel` use up to `bytes` of dynamic shared memory; a failure is reported by the
// return code and cleared, so a later launch check does not pick it up.
template <typename K> cudaError_t allow_smem(K kernel, int bytes)
{
    // dynamic + static shared memory may not exceed the opt-in limit
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 std::min<int>(bytes, smem_optin() - (int)fa.sharedSizeBytes));
    // The SM's L1/shared split is fixed while a CTA is resident: with every kernel of the
    // factorization preferring the largest shared carveout, the next pivot's CTAs fit
    // beside a running update CTA instead of waiting for it to finish.
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    cudaGetLastError();
    return e;
}

__global__ void k_status_init(int *st)
{
    if (threadIdx.x == 0)
    {
        st[hyb::ST_ZERO_PIVOTS] = 0;
        st[hyb::ST_NON_FINITE] = 0;
        st[hyb::ST_FIRST_BAD] = INT_MAX;
        st[3] = 0;
        st[hyb::ST_GROWTH_FP64] = 0;
        st[hyb::ST_GROWTH_KEPT] = 0;
    }
}

// Size buckets of the update tuner: the pivot size and the largest target dimension of a
// level, each rounded up to one of 8, 16, 32, 64, 128, 256 or more.
constexpr int kSizeClasses = 7;
constexpr int hyb_tuning_buckets()
{
    return kSizeClasses * kSizeClasses;
}

int size_class(int x)
{
    int c = 0;
    for (int lim = 8; c < kSizeClasses - 1 && x > lim; lim *= 2)
        ++c;
    return c;
}

// Generic-size Schur-update kernels the tuner chooses among.
enum UpdateKernel
{
    UPD_TILE32 = 0, // k_update32: 64-thread CTAs of one 32x32 output tile (targets up to 256 wide)
    UPD_TILE64 = 1, // k_update: one 256-thread CTA per target, its 64x64 tiles in turn
    UPD_DMMA = 2,   // k_update_dmma: FP64 tensor pipe, one CTA per 64x64 tile (pivots up to 128 rows)
    UPD_KINDS = 3
};

struct GraphExec
{
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;
    ~GraphExec()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
    }
};

} // namespace

struct hyb_system
{
    Symbolic S;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr; // lookahead pivots (joined into `stream` inside graphs)
    cudaStream_t stream3 = nullptr; // operand splits beside a pivot launch (forked and joined per level)
    cudaEvent_t ev_prio = nullptr, ev_piv = nullptr, ev_join = nullptr, ev_fork3 = nullptr, ev_join3 = nullptr;
    bool lookahead = true;
    bool umma = true; // mixed-form updates of 64-blocks on the tcgen05 tensor cores
    bool flow = true; // dataflow substitution (enqueue_solve_flow) in hyb_solve
    uint64_t wait_ns = hyb::kWaitLimitNs; // limit of each wait of the dataflow solve
    int64_t withhold_slot = -1;           // fault injection: pivot slot whose early partials are never released
    int refinement = 0;                   // HYB_OPTION_REFINEMENT: 0 auto, 1 refinement only, 2 FGMRES
    bool fp64_refine = false;             // HYB_OPTION_FP64_REFINEMENT
    int krylov_restart = 30;              // HYB_OPTION_KRYLOV_RESTART
    float growth_limit = 1024.0f;         // HYB_OPTION_GROWTH_LIMIT (mixed form)
    bool block_scaling = true;            // HYB_OPTION_BLOCK_SCALING (mixed form)
    bool alternate_walk = true;           // HYB_OPTION_ALTERNATE_WALK
    int pair_passes = 1;                  // HYB_OPTION_PAIR_PASSES (mixed form; 2: inner update launched apart)
    int row_pivots = -1;                  // HYB_OPTION_ROW_PIVOTS: -1 per precision (mixed 2, FP64 0)
    int update_sm_reserve = 4;            // HYB_OPTION_UPDATE_SM_RESERVE
    // generic-size Schur updates: HYB_OPTION_UPDATE_KERNEL (-1: tuned per size bucket), and
    // the tuned choice per precision and bucket (-1: not tuned yet)
    int update_kernel = -1;
    int tuned[2][hyb_tuning_buckets()];
    hyb_system()
    {
        for (auto &row : tuned)
            for (int &v : row)
                v = -1;
    }
    bool factors_scaled = false;          // the current mixed factors are those of S A S
    double *d_bscale = nullptr;           // s_k per block row
    double *d_dscale = nullptr;           // s_k per unknown
    // mixed form, pivots of at most hyb::kGrowthSmallRows rows: FP64 LU of a high-growth
    // pivot (offsets per block row, -1 for larger ones) and the flags k_trsm reads
    int *d_hg = nullptr;
    double *d_piv64 = nullptr;
    int64_t *d_g64_off = nullptr;
    // FP64 LUs of high-growth 64-row pivots between k_lu64_once and k_trsm64_strips: two
    // level-parity halves of fused_half slots of 64 x 64 doubles
    double *d_piv64f = nullptr;
    int64_t fused_half = 0;
    int lu_once = -1; // HYB_OPTION_PIVOT_LU_ONCE: -1 per precision (FP64 once, mixed fused)
    int fp64_shape = 1; // HYB_OPTION_FP64_MMA_SHAPE (m16n8k8: 0.6% faster than m8n8k4 at 128x128 p=8)
    // independent systems stacked in one handle (hyb_system_set_segments): unknown offsets,
    // their device copy, norms per segment and column, and the last solve's results
    std::vector<int64_t> seg_off;
    int64_t *d_seg_off = nullptr;
    double *d_seg_norm = nullptr;
    int64_t seg_norm_cap = 0;
    std::vector<uint32_t> seg_first;
    std::vector<double> seg_relres;
    void *arena = nullptr;
    DevSym ds{};
    double *d_a = nullptr; // original values (FP64, CSR order)
    int *d_status = nullptr;
    int *d_tickets = nullptr; // per pivot: partial products of the solve stage already published
    // dataflow solve: per block row the tag of the last solve direction that finished it,
    // the solve's status words, and the partial products of every pivot (flow_nrhs columns)
    int *d_flags = nullptr;
    int *d_pflags = nullptr; // per pivot: tag of the solve direction whose early partials are summed
    int *d_lu_tickets = nullptr; // per pivot: CTAs of k_lu_trsm64 that have read the diagonal block
    int *d_solve_status = nullptr;
    uint32_t solve_epoch = 0;
    double *d_flow64 = nullptr;
    float *d_flow32 = nullptr;
    int64_t flow64_nrhs = 0, flow32_nrhs = 0;
    int factored = -1; // -1, HYB_PRECISION_FP64 or HYB_PRECISION_MIXED
    double *d_f64 = nullptr;
    float *d_f32 = nullptr;
    float *d_dinv = nullptr; // FP32 inverses of the 64-row diagonal blocks (mixed form), n_inv x 4096
    // BF16 operand splits of tensor-core levels, a ring of level slots of split_half bytes
    // each, then one all-zero split block
    unsigned char *d_ops = nullptr;
    size_t split_half = 0;
    // target-block offsets of tensor-core levels, a ring of level slots of tgt_half entries
    int64_t *d_tgt = nullptr;
    size_t tgt_half = 0;
    // solve buffers, sized for buf_nrhs right-hand sides
    int64_t buf_nrhs = 0;
    double *d_b = nullptr, *d_x = nullptr, *d_r = nullptr, *d_scr64 = nullptr, *d_part = nullptr, *d_norm = nullptr;
    float *d_yf = nullptr, *d_scr32 = nullptr;
    int n_norm_parts = 0;
    // refinement: correction and best iterate (FP64); FGMRES: kry_m + 1 basis vectors V,
    // kry_m preconditioned vectors Z, the product w, the Hessenberg column and the
    // combination coefficients (all sized for buf_nrhs right-hand sides)
    double *d_z = nullptr, *d_xb = nullptr, *d_w = nullptr, *d_V = nullptr, *d_Zk = nullptr, *d_h = nullptr,
           *d_coef = nullptr;
    int64_t kry_m = 0;
    // column view of the factors and of A (transposed solve, ||A||_1), built at first use
    void *t_arena = nullptr;
    hyb::DevTrans dt{};
    int64_t t_max_rows = 0;
    double *d_tscr = nullptr;
    int64_t tscr_nrhs = 0;
    double *d_colsum = nullptr;
    std::vector<int64_t> t_fu_pref, t_bu_pref; // host copies of dt's unit prefixes (grid sizes)
    std::map<int, std::unique_ptr<GraphExec>> g_solveT; // by nrhs
    std::unique_ptr<GraphExec> g_factor[2];
    std::map<std::pair<int, int>, std::unique_ptr<GraphExec>> g_solve; // (precision, nrhs)
    uint64_t launches = 0;
    uint64_t last_launches = 0;
    // profiling: one event pair around the Schur-update kernels of every profile-th level
    // that has an update (0: off)
    int profile = 0;
    std::vector<cudaEvent_t> prof_ev;
    std::vector<int64_t> prof_levels; // first level of the unit of each event pair
    std::vector<uint8_t> prof_pair;   // whether that unit is a two-pivot pass
    int64_t prof_update_levels = 0;   // update passes in the captured schedule (a pair counts once)
    int64_t prof_update_pivots = 0;   // levels with an update in the captured schedule
    // the same for the pivot work of every profile-th unit (on whichever stream runs it)
    std::vector<cudaEvent_t> prof_piv_ev;
    std::vector<uint8_t> prof_piv_levels; // levels of each timed unit
    int64_t prof_piv_units = 0;
    int prof_precision = -1;

    ~hyb_system()
    {
        free_profile_events();
        g_factor[0].reset();
        g_factor[1].reset();
        g_solve.clear();
        cudaFree(arena);
        cudaFree(d_a);
        cudaFree(d_status);
        cudaFree(d_tickets);
        cudaFree(d_flags);
        cudaFree(d_pflags);
        cudaFree(d_lu_tickets);
        cudaFree(d_solve_status);
        cudaFree(d_flow64);
        cudaFree(d_flow32);
        cudaFree(d_f64);
        cudaFree(d_f32);
        cudaFree(d_dinv);
        cudaFree(d_ops);
        cudaFree(d_tgt);
        g_solveT.clear();
        cudaFree(d_seg_off);
        cudaFree(d_seg_norm);
        cudaFree(d_hg);
        cudaFree(d_piv64f);
        cudaFree(d_bscale);
        cudaFree(d_dscale);
        cudaFree(d_piv64);
        cudaFree(d_g64_off);
        cudaFree(t_arena);
        cudaFree(d_tscr);
        cudaFree(d_colsum);
        free_solve_buffers();
        for (cudaEvent_t e : {ev_prio, ev_piv, ev_join, ev_fork3, ev_join3})
            if (e)
                cudaEventDestroy(e);
        if (stream3)
            cudaStreamDestroy(stream3);
        if (stream2)
            cudaStreamDestroy(stream2);
        if (stream)
            cudaStreamDestroy(stream);
    }

    void free_profile_events()
    {
        for (cudaEvent_t e : prof_ev)
            cudaEventDestroy(e);
        prof_ev.clear();
        prof_levels.clear();
        prof_pair.clear();
        prof_update_levels = 0;
        prof_update_pivots = 0;
        for (cudaEvent_t e : prof_piv_ev)
            cudaEventDestroy(e);
        prof_piv_ev.clear();
        prof_piv_levels.clear();
        prof_piv_units = 0;
    }

    void free_krylov()
    {
        for (void *p : {(void *)d_w, (void *)d_V, (void *)d_Zk, (void *)d_h, (void *)d_coef})
            cudaFree(p);
        d_w = d_V = d_Zk = d_h = d_coef = nullptr;
        kry_m = 0;
    }

    void free_solve_buffers()
    {
        for (void *p : {(void *)d_b, (void *)d_x, (void *)d_r, (void *)d_scr64, (void *)d_part, (void *)d_norm,
                        (void *)d_yf, (void *)d_scr32, (void *)d_z, (void *)d_xb})
            cudaFree(p);
        d_b = d_x = d_r = d_scr64 = d_part = d_norm = d_z = d_xb = nullptr;
        d_yf = d_scr32 = nullptr;
        free_krylov();
        buf_nrhs = 0;
        g_solve.clear();
        g_solveT.clear();
    }
};

namespace
{

// The lookahead stream gets the highest priority, so the block scheduler places the next
// pivot's CTAs ahead of the remaining update CTAs as soon as an SM has room; captured
// kernels keep their stream's priority as a node attribute (see run_graph).
cudaError_t create_streams(hyb_system *h)
{
    int lo = 0, hi = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, lo);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithPriority(&h->stream2, cudaStreamNonBlocking, hi);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithPriority(&h->stream3, cudaStreamNonBlocking, hi);
    for (cudaEvent_t *ev : {&h->ev_prio, &h->ev_piv, &h->ev_join, &h->ev_fork3, &h->ev_join3})
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    return e;
}

// Copies the symbolic arrays into one device allocation and fills the DevSym view.
int upload_symbolic(hyb_system *h)
{
    const Symbolic &S = h->S;
    struct Item
    {
        const void *src;
        size_t bytes;
        const void **dst;
    };
    DevSym &d = h->ds;
    d.n = S.n;
    std::vector<Item> items = {
        {S.size.data(), S.size.size() * 4, (const void **)&d.size},
        {S.dof_off.data(), S.dof_off.size() * 8, (const void **)&d.dof_off},
        {S.row_ptr.data(), S.row_ptr.size() * 8, (const void **)&d.row_ptr},
        {S.cols.data(), S.cols.size() * 4, (const void **)&d.cols},
        {S.diag_pos.data(), S.diag_pos.size() * 8, (const void **)&d.diag_pos},
        {S.blk_off.data(), S.blk_off.size() * 8, (const void **)&d.blk_off},
        {S.lcol_ptr.data(), S.lcol_ptr.size() * 8, (const void **)&d.lcol_ptr},
        {S.lcol_row.data(), S.lcol_row.size() * 4, (const void **)&d.lcol_row},
        {S.lcol_blk.data(), S.lcol_blk.size() * 4, (const void **)&d.lcol_blk},
        {S.piv.data(), S.piv.size() * 4, (const void **)&d.piv},
        {S.trsm_pref.data(), S.trsm_pref.size() * 8, (const void **)&d.trsm_pref},
        {S.lu_pref.data(), S.lu_pref.size() * 8, (const void **)&d.lu_pref},
        {S.upd_pref.data(), S.upd_pref.size() * 8, (const void **)&d.upd_pref},
        {S.upd2_pref.data(), S.upd2_pref.size() * 8, (const void **)&d.upd2_pref},
        {S.split_pref.data(), S.split_pref.size() * 8, (const void **)&d.split_pref},
        {S.tc_pref.data(), S.tc_pref.size() * 8, (const void **)&d.tc_pref},
        {S.fwd_pref.data(), S.fwd_pref.size() * 8, (const void **)&d.fwd_pref},
        {S.fwdu_pref.data(), S.fwdu_pref.size() * 8, (const void **)&d.fwdu_pref},
        {S.fwd_item_p.data(), S.fwd_item_p.size() * 4, (const void **)&d.fwd_item_p},
        {S.bwd_item_p.data(), S.bwd_item_p.size() * 4, (const void **)&d.bwd_item_p},
        {S.bwd_first.data(), S.bwd_first.size() * 8, (const void **)&d.bwd_first},
        {S.fwd_rows.data(), S.fwd_rows.size() * 8, (const void **)&d.fwd_rows},
        {S.bwd_rows.data(), S.bwd_rows.size() * 8, (const void **)&d.bwd_rows},
        {S.inv_idx.data(), S.inv_idx.size() * 4, (const void **)&d.inv_idx},
        {S.inv_row.data(), S.inv_row.size() * 4, (const void **)&d.inv_row},
        {S.mt_tgt.data(), S.mt_tgt.size() * 4, (const void **)&d.mt_tgt},
        {S.mt_row.data(), S.mt_row.size() * 4, (const void **)&d.mt_row},
        {S.mt_col.data(), S.mt_col.size() * 4, (const void **)&d.mt_col},
        {S.mt_src_ptr.data(), S.mt_src_ptr.size() * 8, (const void **)&d.mt_src_ptr},
        {S.mt_src_k.data(), S.mt_src_k.size() * 4, (const void **)&d.mt_src_k},
        {S.mt_src_l.data(), S.mt_src_l.size() * 4, (const void **)&d.mt_src_l},
        {S.mt_src_u.data(), S.mt_src_u.size() * 4, (const void **)&d.mt_src_u},
        {S.a_row_ptr.data(), S.a_row_ptr.size() * 8, (const void **)&d.a_row_ptr},
        {S.a_cols.data(), S.a_cols.size() * 4, (const void **)&d.a_cols},
        {S.a_val_off.data(), S.a_val_off.size() * 8, (const void **)&d.a_val_off},
        {S.a_to_f.data(), S.a_to_f.size() * 4, (const void **)&d.a_to_f},
        {S.pair_map.data(), S.pair_map.size() * 4, (const void **)&d.pair_map},
    };
    size_t total = 0;
    for (const Item &it : items)
        total += (it.bytes + 255) / 256 * 256 + 256;
    HYB_CUDA(cudaMalloc(&h->arena, total));
    std::vector<char> host(total, 0);
    size_t off = 0;
    for (const Item &it : items)
    {
        if (it.bytes)
            std::memcpy(host.data() + off, it.src, it.bytes);
        *it.dst = (const char *)h->arena + off;
        off += (it.bytes + 255) / 256 * 256 + 256;
    }
    HYB_CUDA(cudaMemcpy(h->arena, host.data(), total, cudaMemcpyHostToDevice));
    return HYB_SUCCESS;
}

template <typename T> int lu_smem_bytes(int m)
{
    return m * m * (int)sizeof(T);
}

template <typename T> int trsm_smem_bytes(int m)
{
    return (m * (m | 1) + m * (hyb::kTile | 1)) * (int)sizeof(T); // odd row strides (k_trsm)
}

// LU of the diagonal blocks of level l and the solves of their rows' upper blocks.
// Launch errors are caught at the launch that caused them, naming the kernel and level.
#define HYB_LAUNCHED(what, level)                                                                                      \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t e_ = cudaGetLastError();                                                                           \
        if (e_ != cudaSuccess)                                                                                         \
            return cuda_fail(e_, (std::string(what) + " launch at level " + std::to_string(level)).c_str());          \
    } while (0)

// Whether level l's Schur update runs on the tensor cores (mixed form, 64-blocks).
template <typename T> bool tc_level(const hyb_system *h, int64_t l)
{
    return std::is_same_v<T, float> && h->umma && h->d_ops && h->d_tgt && !h->S.lvl_listed[l] &&
           h->S.shape[l].uniform64;
}

// Operand splits and target tables live in a ring of kOpsSlots level slots: a two-pivot pass
// reads the slots of its two levels while the next pair's pivots write the next two.
constexpr int kOpsSlots = 4;

unsigned char *level_ops(hyb_system *h, int64_t l)
{
    return h->d_ops + (size_t)(l % kOpsSlots) * h->split_half;
}

int64_t *level_tgt(hyb_system *h, int64_t l)
{
    return h->d_tgt + (size_t)(l % kOpsSlots) * h->tgt_half;
}

// One all-zero BF16 split block after the ring (a column a pair's first pivot does not reach).
const unsigned char *zero_split(const hyb_system *h)
{
    return h->d_ops + (size_t)kOpsSlots * h->split_half;
}

// One FP32 64x64 block after it: a pair's U(c,d), for the updates of the second pivot's column.
float *pair_ucd(hyb_system *h)
{
    return reinterpret_cast<float *>(h->d_ops + (size_t)kOpsSlots * h->split_half + hyb::kSplitBytes);
}

// BF16 split of a tensor-core level's operands, once its pivots are factored.
template <typename T> int enqueue_split(hyb_system *h, T *slab, int64_t l, cudaStream_t st, uint64_t &launches)
{
    if constexpr (std::is_same_v<T, float>)
    {
        const Symbolic &S = h->S;
        if (!tc_level<T>(h, l))
            return HYB_SUCCESS;
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        const int64_t blocks = S.split_pref[p1] - S.split_pref[p0];
        if (blocks > 0)
        {
            hyb::k_split64<<<(unsigned)blocks, hyb::kSplitThreads, 0, st>>>(h->ds, slab, level_ops(h, l),
                                                                           level_tgt(h, l), p0, p1, 0);
            ++launches;
            HYB_LAUNCHED("k_split64", l);
        }
    }
    return HYB_SUCCESS;
}

// Whether a level's pivots take the 64-row kernels (33-64 rows, upper blocks up to 128 wide).
bool fused_pivots(const Symbolic::LevelShape &sh)
{
    return sh.max_piv > 32 && sh.max_piv <= 64 && sh.max_up <= 128;
}

// Whether level l's 64-row pivots take the inverse-and-products path (HYB_OPTION_ROW_PIVOTS 2,
// by default in the mixed form).
template <typename T> bool inverse_pivots(const hyb_system *h, int64_t l)
{
    const Symbolic::LevelShape &sh = h->S.shape[l];
    const int mode64 = h->row_pivots < 0 ? (std::is_same_v<T, float> ? 2 : 0) : h->row_pivots;
    return std::is_same_v<T, float> && fused_pivots(sh) && sh.piv64 && mode64 == 2 && tc_level<T>(h, l) && h->d_dinv;
}

// With pair_first (level l's pivot is the first of a pair on the inverse-and-products path),
// the first pivot's update of the second one's row and column is applied by the products
// kernel too; the caller then issues no separate update for it.
// With second_done (level l's pivot is the second of such a pair), its LU and inverse were
// formed by the first pivot's products launch: only its products (and splits) remain.
template <typename T>
int enqueue_pivots(hyb_system *h, T *slab, int64_t l, cudaStream_t st, uint64_t &launches, bool pair_first = false,
                   bool second_done = false)
{
    const Symbolic &S = h->S;
    const DevSym &ds = h->ds;
    const int optin = smem_optin();
    const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
    const Symbolic::LevelShape &sh = S.shape[l];
    // growth check and FP64 fallback of the mixed form (0: off, and always for FP64 factors)
    const float glim = std::is_same_v<T, float> && h->d_hg ? h->growth_limit : 0.0f;
    // 64-row pivots (HYB_OPTION_ROW_PIVOTS): the mixed form by default factors each pivot
    // once and takes its upper blocks as products with the inverse (2); 1 is the blocked
    // substitution kernel (bit-identical to the 256-thread kernels); the FP64 form keeps the
    // 256-thread kernels by default, since the blocked kernel's 115 KB of FP64 shared
    // memory displaces update CTAs (measured at 96x96 p=8: 2,229 against 2,138 ms)
    const int mode64 = h->row_pivots < 0 ? (std::is_same_v<T, float> ? 2 : 0) : h->row_pivots;
    if constexpr (std::is_same_v<T, float>)
    {
        if (inverse_pivots<T>(h, l))
        {
            const int64_t n_split = S.split_pref[p1] - S.split_pref[p0];
            const int64_t n_trsm = S.trsm_pref[p1] - S.trsm_pref[p0];
            double *inv64 = h->d_piv64f + (l & 1) * h->fused_half * 4096;
            HYB_CUDA(cudaEventRecord(h->ev_fork3, st));
            HYB_CUDA(cudaStreamWaitEvent(h->stream3, h->ev_fork3, 0));
            if (n_split > 0) // the lower blocks' splits beside the pivot work
            {
                hyb::k_split64<<<(unsigned)n_split, hyb::kSplitThreads, 0, h->stream3>>>(
                    ds, slab, level_ops(h, l), level_tgt(h, l), p0, p1, 1);
                ++launches;
                HYB_LAUNCHED("k_split64", l);
            }
            HYB_CUDA(cudaEventRecord(h->ev_join3, h->stream3));
            // a pair's first pivot: the second pivot's positions in its lower column and upper row
            const int32_t i0 = pair_first ? sh.la_i0 : -1, j0 = pair_first ? sh.la_j0 : -1;
            const int64_t n_col = pair_first ? S.lcol_ptr[S.piv[p0] + 1] - S.lcol_ptr[S.piv[p0]] - 1 : 0;
            // the second pivot's LU and inverse run in the first one's products launch
            const int64_t pd = pair_first ? S.lvl_ptr[l + 1] : -1;
            double *x64_d = h->d_piv64f + ((l + 1) & 1) * h->fused_half * 4096;
            if (!second_done)
            {
                hyb::k_piv64_inv<<<(unsigned)(p1 - p0), hyb::kPivThreads, hyb::kInvSmem, st>>>(
                    ds, slab, p0, h->d_status, glim, h->d_dinv, inv64, h->d_hg, j0, pair_ucd(h));
                ++launches;
                HYB_LAUNCHED("k_piv64_inv", l);
            }
            if (n_trsm + n_col > 0)
            {
                hyb::k_strips64_inv<<<(unsigned)(n_trsm + n_col), hyb::kPivThreads, pd >= 0 ? hyb::kInvSmem : 0,
                                      st>>>(ds, slab, p0, p1, h->d_dinv, inv64, h->d_hg, level_ops(h, l), i0, j0,
                                            pair_ucd(h), pd, x64_d, glim, h->d_status);
                ++launches;
                HYB_LAUNCHED("k_strips64_inv", l);
            }
            HYB_CUDA(cudaStreamWaitEvent(st, h->ev_join3, 0));
            return HYB_SUCCESS;
        }
    }
    if (fused_pivots(sh) && sh.piv64 && mode64 >= 1)
    {
        // blocked LU and row solves per upper block; on a tensor-core level the lower-column
        // splits run beside it on a third stream and the upper blocks' splits are written by
        // the row solves
        const int64_t n_lu = S.lu_pref[p1] - S.lu_pref[p0];
        if (tc_level<T>(h, l))
        {
            if constexpr (std::is_same_v<T, float>)
            {
                const int64_t n_split = S.split_pref[p1] - S.split_pref[p0];
                HYB_CUDA(cudaEventRecord(h->ev_fork3, st));
                HYB_CUDA(cudaStreamWaitEvent(h->stream3, h->ev_fork3, 0));
                if (n_split > 0) // the last pivots have no lower or upper blocks
                {
                    hyb::k_split64<<<(unsigned)n_split, hyb::kSplitThreads, 0, h->stream3>>>(
                        ds, slab, level_ops(h, l), level_tgt(h, l), p0, p1, 1);
                    ++launches;
                    HYB_LAUNCHED("k_split64", l);
                }
                HYB_CUDA(cudaEventRecord(h->ev_join3, h->stream3));
                hyb::k_piv64<float, true><<<(unsigned)n_lu, hyb::kPivThreads, hyb::piv64_smem<float>(), st>>>(
                    ds, slab, p0, p1, h->d_lu_tickets, h->d_status, glim, level_ops(h, l));
                ++launches;
                HYB_LAUNCHED("k_piv64", l);
                HYB_CUDA(cudaStreamWaitEvent(st, h->ev_join3, 0));
                return HYB_SUCCESS;
            }
        }
        hyb::k_piv64<T, false><<<(unsigned)n_lu, hyb::kPivThreads, hyb::piv64_smem<T>(), st>>>(
            ds, slab, p0, p1, h->d_lu_tickets, h->d_status, glim, nullptr);
        ++launches;
        HYB_LAUNCHED("k_piv64", l);
        return HYB_SUCCESS;
    }
    if (fused_pivots(sh))
    {
        // fused: diagonal LU (padded to 64x64) and the solves of the pivot rows' upper blocks;
        // pivots of up to 32 rows stay on the generic kernels, whose serial steps are short
        // measured at 128x128 p=8: FP64 6,369 ms once against 6,770 fused (the redundant FP64
        // LUs take SM time from the DMMA update); mixed 1,794 against 1,766 (its FP32 LU is
        // cheap, and the extra launch lands on the pivot chain)
        if (h->lu_once < 0 ? std::is_same_v<T, double> : h->lu_once != 0)
        {
            // each pivot factored once, then the strips from the stored factors
            int *hg = glim > 0 ? h->d_hg : nullptr;
            double *f64 = glim > 0 ? h->d_piv64f + (l & 1) * h->fused_half * 4096 : nullptr;
            if (sh.piv64)
                hyb::k_lu64_once<T, false><<<(unsigned)(p1 - p0), hyb::kThreads, hyb::lu64_once_smem<T>(), st>>>(
                    ds, slab, p0, h->d_status, glim, hg, f64);
            else
                hyb::k_lu64_once<T, true><<<(unsigned)(p1 - p0), hyb::kThreads, hyb::lu64_once_smem<T>(), st>>>(
                    ds, slab, p0, h->d_status, glim, hg, f64);
            ++launches;
            HYB_LAUNCHED("k_lu64_once", l);
            const int64_t n_trsm = S.trsm_pref[p1] - S.trsm_pref[p0];
            if (n_trsm > 0)
            {
                const dim3 grid((unsigned)n_trsm, sh.max_up > 64 ? 2u : 1u);
                if (sh.piv64)
                    hyb::k_trsm64_strips<T, false><<<grid, hyb::kThreads, hyb::lu_trsm64_smem<T>(), st>>>(
                        ds, slab, p0, p1, hg, f64);
                else
                    hyb::k_trsm64_strips<T, true><<<grid, hyb::kThreads, hyb::lu_trsm64_smem<T>(), st>>>(
                        ds, slab, p0, p1, hg, f64);
                ++launches;
                HYB_LAUNCHED("k_trsm64_strips", l);
            }
            return enqueue_split<T>(h, slab, l, st, launches);
        }
        const int64_t units = S.lu_pref[p1] - S.lu_pref[p0];
        const dim3 grid((unsigned)units, sh.max_up > 64 ? 2u : 1u);
        if (sh.piv64) // every pivot and upper block exactly 64: no padding
            hyb::k_lu_trsm64<T, false><<<grid, hyb::kThreads, hyb::lu_trsm64_smem<T>(), st>>>(
                ds, slab, p0, p1, ds.lu_pref, h->d_lu_tickets, h->d_status, glim);
        else
            hyb::k_lu_trsm64<T, true><<<grid, hyb::kThreads, hyb::lu_trsm64_smem<T>(), st>>>(
                ds, slab, p0, p1, ds.lu_pref, h->d_lu_tickets, h->d_status, glim);
        ++launches;
        HYB_LAUNCHED("k_lu_trsm64", l);
        return enqueue_split<T>(h, slab, l, st, launches);
    }
    const int lu_bytes = lu_smem_bytes<T>(sh.max_piv);
    int *hg = glim > 0 ? h->d_hg : nullptr;
    if (lu_bytes <= optin)
        hyb::k_lu<T, true><<<(unsigned)(p1 - p0), hyb::kThreads, lu_bytes, st>>>(ds, slab, p0, h->d_status, glim, hg,
                                                                                 h->d_piv64, h->d_g64_off);
    else
        hyb::k_lu<T, false><<<(unsigned)(p1 - p0), hyb::kThreads, 0, st>>>(ds, slab, p0, h->d_status, glim, hg,
                                                                          h->d_piv64, h->d_g64_off);
    ++launches;
    HYB_LAUNCHED("k_lu", l);
    const int64_t n_trsm = S.trsm_pref[p1] - S.trsm_pref[p0];
    if (n_trsm > 0)
    {
        dim3 grid((unsigned)n_trsm, (unsigned)((sh.max_up + hyb::kTile - 1) / hyb::kTile));
        int bytes = trsm_smem_bytes<T>(sh.max_piv);
        if (hg && sh.max_piv <= hyb::kGrowthSmallRows) // room for an FP64 strip of a refactored pivot
            bytes = std::max(bytes, sh.max_piv * (hyb::kTile | 1) * (int)sizeof(double));
        if (bytes <= optin)
            hyb::k_trsm<T, true><<<grid, hyb::kThreads, bytes, st>>>(ds, slab, p0, p1, hg, h->d_piv64, h->d_g64_off);
        else
            hyb::k_trsm<T, false><<<grid, hyb::kThreads, 0, st>>>(ds, slab, p0, p1, hg, h->d_piv64, h->d_g64_off);
        ++launches;
        HYB_LAUNCHED("k_trsm", l);
    }
    return enqueue_split<T>(h, slab, l, st, launches);
}

// Whether the pivot work of every level with 64-row pivots already wrote their FP32
// inverses (the mixed form's inverse-and-products path, HYB_OPTION_ROW_PIVOTS 2).
template <typename T> bool inverses_by_pivots(const hyb_system *h)
{
    const Symbolic &S = h->S;
    const int mode64 = h->row_pivots < 0 ? (std::is_same_v<T, float> ? 2 : 0) : h->row_pivots;
    if (!std::is_same_v<T, float> || mode64 != 2)
        return false;
    for (int64_t l = 0; l < S.n_levels; ++l)
    {
        bool has64 = false;
        for (int64_t p = S.lvl_ptr[l]; p < S.lvl_ptr[l + 1] && !has64; ++p)
            has64 = S.size[S.piv[p]] == 64;
        if (has64 && !(fused_pivots(S.shape[l]) && S.shape[l].piv64 && tc_level<T>(h, l)))
            return false;
    }
    return true;
}

// FP32 inverses of every 64-row diagonal block (mixed form), in one launch after the last
// level. Only the solves read them; launched beside the stages instead, they slowed the
// update CTAs that shared their SMs, and each level waits for its slowest update CTA.
template <typename T> int enqueue_inverses(hyb_system *h, T *slab, uint64_t &launches)
{
    if constexpr (std::is_same_v<T, float>)
    {
        if (!h->d_dinv || h->S.n_inv == 0 || inverses_by_pivots<T>(h))
            return HYB_SUCCESS;
        hyb::k_diag_inv64<float>
            <<<(unsigned)h->S.n_inv, hyb::kInvThreads, 0, h->stream>>>(h->ds, slab, h->d_dinv);
        ++launches;
        HYB_LAUNCHED("k_diag_inv64", h->S.n_levels - 1);
    }
    return HYB_SUCCESS;
}

// Whether a generic update kernel can run a level's shapes.
bool generic_kernel_fits(const Symbolic::LevelShape &sh, int kind)
{
    if (kind == UPD_TILE32)
        return std::max(sh.max_row, sh.max_col) <= 8 * hyb::kSmallTile;
    if (kind == UPD_DMMA)
        return sh.max_piv <= hyb::kDmmaMaxK;
    return true;
}

int level_bucket(const Symbolic::LevelShape &sh)
{
    return size_class(sh.max_piv) * kSizeClasses + size_class(std::max(sh.max_row, sh.max_col));
}

// The generic update kernel of level l: the forced one (HYB_OPTION_UPDATE_KERNEL) where it
// fits, else the tuned choice of the level's size bucket, else the fixed rule (32x32 tiles
// for targets up to 256 wide, 64x64 tiles beyond).
template <typename T> int generic_kernel(const hyb_system *h, int64_t l)
{
    const Symbolic::LevelShape &sh = h->S.shape[l];
    if (h->update_kernel >= 0 && generic_kernel_fits(sh, h->update_kernel))
        return h->update_kernel;
    const int tuned = h->tuned[std::is_same_v<T, float> ? 1 : 0][level_bucket(sh)];
    if (tuned >= 0 && generic_kernel_fits(sh, tuned))
        return tuned;
    return generic_kernel_fits(sh, UPD_TILE32) ? UPD_TILE32 : UPD_TILE64;
}

template <typename T>
int enqueue_generic_update(hyb_system *h, T *slab, int64_t l, cudaStream_t st, int mode, int64_t nu, int kind,
                           uint64_t &launches)
{
    const Symbolic &S = h->S;
    const DevSym &ds = h->ds;
    const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
    const Symbolic::LevelShape &sh = S.shape[l];
    if (kind == UPD_TILE32)
    {
        // 64-thread CTAs of one 32x32 tile each (grid.y: the tiles of the largest target)
        const unsigned t32 = (unsigned)(((sh.max_row + hyb::kSmallTile - 1) / hyb::kSmallTile) *
                                        ((sh.max_col + hyb::kSmallTile - 1) / hyb::kSmallTile));
        hyb::k_update32<T><<<dim3((unsigned)nu, t32), hyb::kSmallThreads, 0, st>>>(ds, slab, p0, p1, mode, sh.la_i0,
                                                                                  sh.la_j0);
        ++launches;
        HYB_LAUNCHED("k_update32", l);
        return HYB_SUCCESS;
    }
    if (kind == UPD_DMMA)
    {
        const unsigned t64 = (unsigned)(((sh.max_row + 63) / 64) * ((sh.max_col + 63) / 64));
        hyb::k_update_dmma<T><<<dim3((unsigned)nu, t64), hyb::kDmmaThreads, hyb::dmma_smem_bytes(sh.max_piv), st>>>(
            ds, slab, p0, p1, mode, sh.la_i0, sh.la_j0);
        ++launches;
        HYB_LAUNCHED("k_update_dmma", l);
        return HYB_SUCCESS;
    }
    // one CTA per target block, looping over its 64x64 tiles
    hyb::k_update<T><<<(unsigned)nu, hyb::kThreads, 0, st>>>(ds, slab, p0, p1, mode, sh.la_i0, sh.la_j0);
    ++launches;
    HYB_LAUNCHED("k_update", l);
    return HYB_SUCCESS;
}

// Tunes the generic update kernel of every size bucket the factorization meets (T's
// precision): on the bucket's level with the most update units, each kernel that fits is
// run once to warm up and then three times under CUDA events; the fastest is kept. It runs
// on the zeroed slab before the values are scattered (products of zeros: nothing changes).
template <typename T> int tune_updates(hyb_system *h, T *slab)
{
    const Symbolic &S = h->S;
    const int prec = std::is_same_v<T, float> ? 1 : 0;
    std::vector<int64_t> rep(hyb_tuning_buckets(), -1);
    for (int64_t l = 0; l < S.n_levels; ++l)
    {
        const Symbolic::LevelShape &sh = S.shape[l];
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        const int64_t nu = S.upd_pref[p1] - S.upd_pref[p0];
        if (S.lvl_listed[l] || nu == 0 || (std::is_same_v<T, double> && sh.uniform64) || tc_level<T>(h, l))
            continue;
        const int b = level_bucket(sh);
        if (h->tuned[prec][b] >= 0)
            continue;
        if (rep[b] < 0 || nu > S.upd_pref[S.lvl_ptr[rep[b] + 1]] - S.upd_pref[S.lvl_ptr[rep[b]]])
            rep[b] = l;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    HYB_CUDA(cudaEventCreate(&e0));
    HYB_CUDA(cudaEventCreate(&e1));
    int rc = HYB_SUCCESS;
    for (int b = 0; b < hyb_tuning_buckets() && rc == HYB_SUCCESS; ++b)
    {
        const int64_t l = rep[b];
        if (l < 0)
            continue;
        const Symbolic::LevelShape &sh = S.shape[l];
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        const int64_t nu = S.upd_pref[p1] - S.upd_pref[p0];
        float best = INFINITY;
        int best_kind = -1;
        for (int kind = 0; kind < UPD_KINDS && rc == HYB_SUCCESS; ++kind)
        {
            if (!generic_kernel_fits(sh, kind))
                continue;
            uint64_t dummy = 0;
            if ((rc = enqueue_generic_update<T>(h, slab, l, h->stream, 0, nu, kind, dummy)) != HYB_SUCCESS)
                break;
            cudaEventRecord(e0, h->stream);
            for (int r = 0; r < 3 && rc == HYB_SUCCESS; ++r)
                rc = enqueue_generic_update<T>(h, slab, l, h->stream, 0, nu, kind, dummy);
            cudaEventRecord(e1, h->stream);
            const cudaError_t e = cudaEventSynchronize(e1);
            float ms = 0;
            if (e == cudaSuccess)
                cudaEventElapsedTime(&ms, e0, e1);
            else
                rc = cuda_fail(e, "tuning the update kernels");
            if (rc == HYB_SUCCESS && ms < best)
            {
                best = ms;
                best_kind = kind;
            }
        }
        h->tuned[prec][b] = best_kind;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// Whether some level of the factorization in T's precision uses a generic update kernel
// whose size bucket has not been tuned yet.
template <typename T> bool needs_tuning(const hyb_system *h)
{
    const Symbolic &S = h->S;
    const int prec = std::is_same_v<T, float> ? 1 : 0;
    for (int64_t l = 0; l < S.n_levels; ++l)
    {
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        if (S.lvl_listed[l] || S.upd_pref[p1] == S.upd_pref[p0] || (std::is_same_v<T, double> && S.shape[l].uniform64) ||
            tc_level<T>(h, l))
            continue;
        if (h->tuned[prec][level_bucket(S.shape[l])] < 0)
            return true;
    }
    return false;
}

// Schur-complement updates of level l: mode 0 all of them, 1 / 2 the lookahead split.
template <typename T> int enqueue_update(hyb_system *h, T *slab, int64_t l, cudaStream_t st, int mode,
                                         uint64_t &launches)
{
    const Symbolic &S = h->S;
    const DevSym &ds = h->ds;
    const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
    const Symbolic::LevelShape &sh = S.shape[l];
    const unsigned tiles =
        (unsigned)(((sh.max_row + hyb::kTile - 1) / hyb::kTile) * ((sh.max_col + hyb::kTile - 1) / hyb::kTile));
    // alternate levels walk their targets backwards (the priority launch keeps its order)
    const int reverse = h->alternate_walk && mode != 1 && (l & 1) ? 1 : 0;
    if (S.lvl_listed[l])
    {
        const int64_t q0 = S.mt_lvl_ptr[l], nq = S.mt_lvl_ptr[l + 1] - q0;
        if (nq > 0)
        {
            hyb::k_update_listed<T><<<dim3((unsigned)nq, tiles), hyb::kThreads, 0, st>>>(ds, slab, q0);
            ++launches;
            HYB_LAUNCHED("k_update_listed", l);
        }
        return HYB_SUCCESS;
    }
    const int64_t nu =
        mode == 0 ? S.upd_pref[p1] - S.upd_pref[p0] : (mode == 1 ? sh.la_prio_units : sh.la_rest_units);
    if (nu <= 0)
        return HYB_SUCCESS;
    if constexpr (std::is_same_v<T, double>)
    {
        if (sh.uniform64)
        {
            // FP64 MMA instruction shape (HYB_OPTION_FP64_MMA_SHAPE); every shape applies the
            // same products, only the grouping of the K sums inside an instruction differs
            if (h->fp64_shape == 2)
                hyb::k_update64_f64<2><<<(unsigned)nu, hyb::kUpd64Threads, hyb::kUpd64Smem, st>>>(
                    ds, slab, p0, p1, mode, sh.la_i0, sh.la_j0, h->d_status, reverse);
            else if (h->fp64_shape == 1)
                hyb::k_update64_f64<1><<<(unsigned)nu, hyb::kUpd64Threads, hyb::kUpd64Smem, st>>>(
                    ds, slab, p0, p1, mode, sh.la_i0, sh.la_j0, h->d_status, reverse);
            else
                hyb::k_update64_f64<0><<<(unsigned)nu, hyb::kUpd64Threads, hyb::kUpd64Smem, st>>>(
                    ds, slab, p0, p1, mode, sh.la_i0, sh.la_j0, h->d_status, reverse);
            ++launches;
            HYB_LAUNCHED("k_update64_f64", l);
            return HYB_SUCCESS;
        }
    }
    else
    {
        // mixed form: split-BF16 products on the tensor cores, one persistent CTA per SM
        if (tc_level<T>(h, l))
        {
            const int64_t tiles = mode == 0   ? S.tc_pref[p1] - S.tc_pref[p0]
                                  : mode == 1 ? sh.la_prio_tiles
                                              : sh.la_rest_tiles;
            if (tiles > 0)
            {
                const unsigned grid = (unsigned)std::min<int64_t>(tiles, (int64_t)sm_count());
                hyb::k_update64_tc<<<grid, hyb::kTcThreads, hyb::kTcSmem, st>>>(
                    ds, slab, level_ops(h, l), level_tgt(h, l), p0, p1, mode, sh.la_i0, sh.la_j0, tiles,
                    h->d_status, reverse);
                ++launches;
                HYB_LAUNCHED("k_update64_tc", l);
            }
            return HYB_SUCCESS;
        }
    }
    return enqueue_generic_update<T>(h, slab, l, st, mode, nu, generic_kernel<T>(h, l), launches);
}

// Whether level l starts a two-pivot pass in T's factorization: the mixed form on the
// tensor cores, a pair of the symbolic phase (Symbolic::PairShape), option on.
template <typename T> bool pair_unit(const hyb_system *h, int64_t l)
{
    return std::is_same_v<T, float> && h->pair_passes != 0 && l + 1 < h->S.n_levels && h->S.pair_first[l] &&
           tc_level<T>(h, l) && tc_level<T>(h, l + 1);
}

// The pivot work of the unit that starts at level l. A single level: its LU, row solves and
// split. A pair (a, b): a's, then a's update of b's row and column -- a few hundred target
// blocks in FP32 on the CUDA cores, in CTAs small enough to run beside a tensor-core pass --
// then b's.
template <typename T> int enqueue_unit_pivots(hyb_system *h, T *slab, int64_t l, cudaStream_t st, uint64_t &launches)
{
    const bool pair = pair_unit<T>(h, l);
    const bool fold = pair && h->pair_passes == 1 && inverse_pivots<T>(h, l) && inverse_pivots<T>(h, l + 1) &&
                      h->S.shape[l].la_i0 >= 0 && h->S.shape[l].la_j0 >= 0;
    int rc = enqueue_pivots<T>(h, slab, l, st, launches, fold);
    if (rc != HYB_SUCCESS || !pair)
        return rc;
    const Symbolic::LevelShape &sh = h->S.shape[l];
    if (!fold && (rc = enqueue_generic_update<T>(h, slab, l, st, 1, sh.la_prio_units, UPD_TILE32, launches)) !=
                     HYB_SUCCESS)
        return rc;
    return enqueue_pivots<T>(h, slab, l + 1, st, launches, false, fold);
}

// The two-pivot pass of the pair that starts at level l: mode 0 every target of b, 1 / 2 the
// lookahead split (the next unit's rows and columns first).
template <typename T> int enqueue_pair_update(hyb_system *h, T *slab, int64_t l, cudaStream_t st, int mode,
                                              uint64_t &launches)
{
    if constexpr (std::is_same_v<T, float>)
    {
        const Symbolic &S = h->S;
        const Symbolic::PairShape &ps = S.pair[l];
        const int64_t tiles = mode == 0 ? ps.all_tiles : (mode == 1 ? ps.prio_tiles : ps.rest_tiles);
        if (tiles <= 0)
            return HYB_SUCCESS;
        const int4 pr = make_int4(ps.i0, ps.i1, ps.j0, ps.j1);
        // alternate passes walk their targets backwards (the priority launch keeps its order)
        const int reverse = h->alternate_walk && mode != 1 && ((l >> 1) & 1) ? 1 : 0;
        // the main launch may leave SMs free for the next unit's pivot work
        const int64_t sms = mode == 1 ? sm_count() : std::max(1, sm_count() - h->update_sm_reserve);
        const unsigned grid = (unsigned)std::min<int64_t>(tiles, sms);
        hyb::k_update64_tc2<<<grid, hyb::kTc2Threads, hyb::kTc2Smem, st>>>(
            h->ds, slab, level_ops(h, l), level_ops(h, l + 1), level_tgt(h, l + 1), zero_split(h), S.lvl_ptr[l],
            S.lvl_ptr[l + 1], mode, pr, tiles, h->d_status, reverse);
        ++launches;
        HYB_LAUNCHED("k_update64_tc2", l);
    }
    return HYB_SUCCESS;
}

// Issues the whole factorization (used under graph capture). Units -- one level, or a pair
// of levels applied in one two-pivot pass -- run in order on the handle's stream; where a
// unit and the next are single pivots (or pairs of them), the next unit's pivot work runs
// on the second stream as soon as the update of its rows and columns is done, overlapping
// the rest of this unit's update (lookahead).
template <typename T> int enqueue_factor(hyb_system *h, T *slab, uint64_t &launches)
{
    const Symbolic &S = h->S;
    cudaStream_t st = h->stream, st2 = h->stream2;
    HYB_CUDA(cudaGetLastError()); // nothing earlier may be blamed on this schedule
    k_status_init<<<1, 32, 0, st>>>(h->d_status);
    ++launches;
    HYB_CUDA(cudaMemsetAsync(h->d_lu_tickets, 0, S.n * sizeof(int), st)); // an aborted run may leave tickets
    if (std::is_same_v<T, float> && h->d_hg)
        HYB_CUDA(cudaMemsetAsync(h->d_hg, 0, S.n * sizeof(int), st));
    int rc = HYB_SUCCESS;
    bool next_pivots_issued = false, forked = false;
    int64_t nl = 1;
    // the pivot work of the unit at level lu on stream s, bracketed by events on every
    // profile-th unit
    auto unit_pivots = [&](int64_t lu, cudaStream_t s) -> int {
        const bool tp = h->profile > 0 && h->prof_piv_units++ % h->profile == 0;
        if (tp)
        {
            cudaEvent_t e0, e1;
            HYB_CUDA(cudaEventCreate(&e0));
            HYB_CUDA(cudaEventCreate(&e1));
            h->prof_piv_ev.push_back(e0);
            h->prof_piv_ev.push_back(e1);
            h->prof_piv_levels.push_back(pair_unit<T>(h, lu) ? 2 : 1);
            HYB_CUDA(cudaEventRecordWithFlags(e0, s, cudaEventRecordExternal));
        }
        const int r = enqueue_unit_pivots<T>(h, slab, lu, s, launches);
        if (r == HYB_SUCCESS && tp)
            HYB_CUDA(cudaEventRecordWithFlags(h->prof_piv_ev.back(), s, cudaEventRecordExternal));
        return r;
    };
    for (int64_t l = 0; l < S.n_levels; l += nl)
    {
        const bool pair = pair_unit<T>(h, l);
        nl = pair ? 2 : 1;
        const int64_t next = l + nl; // first level of the next unit
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        const Symbolic::LevelShape &sh = S.shape[l];
        if (next_pivots_issued)
            HYB_CUDA(cudaStreamWaitEvent(st, h->ev_piv, 0));
        else if ((rc = unit_pivots(l, st)) != HYB_SUCCESS)
            return rc;
        next_pivots_issued = false;
        const bool has_update =
            pair || (S.lvl_listed[l] ? S.mt_lvl_ptr[l + 1] > S.mt_lvl_ptr[l] : S.upd_pref[p1] > S.upd_pref[p0]);
        const bool timed = h->profile > 0 && has_update && h->prof_update_levels % h->profile == 0;
        h->prof_update_levels += has_update ? 1 : 0;
        h->prof_update_pivots += has_update ? nl : 0;
        if (timed)
        {
            cudaEvent_t e0, e1;
            HYB_CUDA(cudaEventCreate(&e0));
            HYB_CUDA(cudaEventCreate(&e1));
            h->prof_ev.push_back(e0);
            h->prof_ev.push_back(e1);
            h->prof_levels.push_back(l);
            h->prof_pair.push_back(pair ? 1 : 0);
            // external records become event nodes of the captured graph (a plain record
            // under capture is only a dependency marker and never fires)
            HYB_CUDA(cudaEventRecordWithFlags(e0, st, cudaEventRecordExternal));
        }
        // A single level's lookahead clears only the next pivot's row and column, so it is
        // not taken when the next unit is a pair (whose pivot work spans two of each).
        const bool lookahead =
            h->lookahead && (pair ? S.pair[l].lookahead : sh.lookahead && !pair_unit<T>(h, next));
        auto update = [&](int mode) {
            return pair ? enqueue_pair_update<T>(h, slab, l, st, mode, launches)
                        : enqueue_update<T>(h, slab, l, st, mode, launches);
        };
        if (lookahead)
        {
            if ((rc = update(1)) != HYB_SUCCESS)
                return rc;
            HYB_CUDA(cudaEventRecord(h->ev_prio, st));
            HYB_CUDA(cudaStreamWaitEvent(st2, h->ev_prio, 0));
            if ((rc = unit_pivots(next, st2)) != HYB_SUCCESS)
                return rc;
            HYB_CUDA(cudaEventRecord(h->ev_piv, st2));
            if ((rc = update(2)) != HYB_SUCCESS)
                return rc;
            next_pivots_issued = true;
            forked = true;
        }
        else if ((rc = update(0)) != HYB_SUCCESS)
        {
            return rc;
        }
        if (timed)
            HYB_CUDA(cudaEventRecordWithFlags(h->prof_ev.back(), st, cudaEventRecordExternal));
    }
    if (forked)
    {
        HYB_CUDA(cudaEventRecord(h->ev_join, st2));
        HYB_CUDA(cudaStreamWaitEvent(st, h->ev_join, 0));
    }
    if ((rc = enqueue_inverses<T>(h, slab, launches)) != HYB_SUCCESS)
        return rc;
    HYB_CUDA(cudaGetLastError());
    return HYB_SUCCESS;
}

// The FP32 diagonal inverses a solve with factors of type T uses (mixed form only).
template <typename T> const T *solve_dinv(const hyb_system *h)
{
    if constexpr (std::is_same_v<T, float>)
        return h->d_dinv;
    else
        return nullptr;
}

// Forward + backward substitution of y (type V, dof x nrhs) with the factors in `slab`.
template <typename T, typename V> int enqueue_solve(hyb_system *h, const T *slab, V *y, V *scratch, int nrhs,
                                                    uint64_t &launches)
{
    const Symbolic &S = h->S;
    const T *dinv = solve_dinv<T>(h);
    const DevSym &ds = h->ds;
    cudaStream_t st = h->stream;
    // tickets return to zero after every stage; clearing them guards against an aborted solve
    HYB_CUDA(cudaMemsetAsync(h->d_tickets, 0, S.n * sizeof(int), st));
    for (int64_t l = 0; l < S.n_levels; ++l)
    {
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        const int64_t units = S.fwdu_pref[p1] - S.fwdu_pref[p0];
        const int mp = S.shape[l].max_piv;
        const int acc_bytes = (mp * nrhs * (int)sizeof(V) + 15) / 16 * 16;
        const int diag_bytes = mp * (mp | 1) * (int)sizeof(T);
        const int stage = acc_bytes + diag_bytes <= solve_smem_cap() ? 1 : 0;
        hyb::k_fwd_stage<T, V><<<(unsigned)units, hyb::kThreads, acc_bytes + (stage ? diag_bytes : 0), st>>>(
            ds, slab, y, scratch, h->d_tickets, p0, p1, nrhs, stage, dinv);
        ++launches;
    }
    for (int64_t l = S.n_levels - 1; l >= 0; --l)
    {
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        const int64_t units = S.trsm_pref[p1] - S.trsm_pref[p0];
        if (units == 0)
            continue;
        hyb::k_bwd_stage<T, V><<<(unsigned)units, hyb::kThreads, 0, st>>>(ds, slab, y, scratch, h->d_tickets, p0,
                                                                         p1, nrhs);
        ++launches;
    }
    HYB_CUDA(cudaGetLastError());
    return HYB_SUCCESS;
}

// Largest diagonal block of the system.
int max_pivot(const Symbolic &S)
{
    int m = 0;
    for (const Symbolic::LevelShape &sh : S.shape)
        m = std::max(m, sh.max_piv);
    return m;
}

template <typename V> V *&flow_scratch(hyb_system *h);
template <> double *&flow_scratch<double>(hyb_system *h)
{
    return h->d_flow64;
}
template <> float *&flow_scratch<float>(hyb_system *h)
{
    return h->d_flow32;
}

// Dataflow substitution of y (dof x nrhs) with the factors in `slab`: one cooperative
// launch per direction. Returns HYB_TOO_LARGE (before anything is enqueued) when the
// device cannot keep a useful grid resident, in which case the caller uses the staged solve.
template <typename T, typename V> int enqueue_solve_flow(hyb_system *h, const T *slab, V *y, int nrhs, uint64_t &launches)
{
    const Symbolic &S = h->S;
    const int mp = max_pivot(S);
    const int acc_bytes = (mp * nrhs * (int)sizeof(V) + 15) / 16 * 16;
    const int diag_bytes = mp * (mp | 1) * (int)sizeof(T);
    int stage = acc_bytes + diag_bytes <= solve_smem_cap() ? 1 : 0;
    const int fwd_smem = acc_bytes + (stage ? diag_bytes : 0);
    int per_sm_f = 0, per_sm_b = 0, coop = 0, dev = 0;
    HYB_CUDA(cudaGetDevice(&dev));
    HYB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    HYB_CUDA(cudaFuncSetAttribute(hyb::k_fwd_flow<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, fwd_smem));
    HYB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, hyb::k_fwd_flow<T, V>, hyb::kThreads, fwd_smem));
    HYB_CUDA(cudaFuncSetAttribute(hyb::k_bwd_flow<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, acc_bytes));
    HYB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_b, hyb::k_bwd_flow<T, V>, hyb::kThreads, acc_bytes));
    if (!coop || per_sm_f < 1 || per_sm_b < 1)
        return HYB_TOO_LARGE;
    V *&scr = flow_scratch<V>(h);
    int64_t &have = std::is_same_v<V, double> ? h->flow64_nrhs : h->flow32_nrhs;
    if (have < nrhs)
    {
        cudaFree(scr);
        scr = nullptr;
        have = 0;
        const int64_t rows = std::max<int64_t>(1, std::max(S.fwd_rows[S.n], S.bwd_rows[S.n]));
        HYB_CUDA(cudaMalloc(&scr, rows * nrhs * sizeof(V)));
        have = nrhs;
    }
    cudaStream_t st = h->stream;
    HYB_CUDA(cudaMemsetAsync(h->d_tickets, 0, S.n * sizeof(int), st));
    if (h->withhold_slot >= 0)
    {
        // the pivot's early-partial ticket starts far past its count, so no CTA ever takes
        // the last one: the pre-sum is never released and the finisher's wait runs out
        static const int kPoison = 1 << 30;
        HYB_CUDA(cudaMemcpyAsync(h->d_tickets + h->withhold_slot, &kPoison, sizeof(int), cudaMemcpyHostToDevice, st));
    }
    h->solve_epoch = (h->solve_epoch + 1) & 0x3fffffffu;
    int tag_f = (int)(2 * h->solve_epoch + 1), tag_b = tag_f + 1;
    DevSym ds = h->ds;
    V *scratch = scr;
    int *tickets = h->d_tickets, *flags = h->d_flags, *pflags = h->d_pflags, *status = h->d_solve_status;
    const T *dinv = solve_dinv<T>(h);
    uint64_t wait_ns = h->wait_ns;
    int64_t nf = (int64_t)S.fwd_item_p.size(), nb = (int64_t)S.bwd_item_p.size();
    const int sms = sm_count();
    {
        const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nf, (int64_t)per_sm_f * sms));
        void *args[] = {&ds,    (void *)&slab, &y,    &scratch, &tickets, &flags,  &pflags,
                        &tag_f, &nf,           &nrhs, &stage,   &dinv,    &status, &wait_ns};
        HYB_CUDA(cudaLaunchCooperativeKernel((const void *)hyb::k_fwd_flow<T, V>, dim3(grid), dim3(hyb::kThreads),
                                             args, fwd_smem, st));
    }
    {
        const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nb, (int64_t)per_sm_b * sms));
        void *args[] = {&ds, (void *)&slab, &y, &scratch, &tickets, &flags, &pflags, &tag_b, &nb, &nrhs, &status, &wait_ns};
        HYB_CUDA(cudaLaunchCooperativeKernel((const void *)hyb::k_bwd_flow<T, V>, dim3(grid), dim3(hyb::kThreads),
                                             args, acc_bytes, st));
    }
    launches += 2;
    return HYB_SUCCESS;
}

// Runs `body` (which enqueues work and counts launches) through a cached CUDA graph.
template <typename F> int run_graph(hyb_system *h, std::unique_ptr<GraphExec> &slot, F body)
{
    if (!slot)
    {
        auto g = std::make_unique<GraphExec>();
        HYB_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        uint64_t count = 0;
        const int rc = body(count);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
        if (rc != HYB_SUCCESS)
        {
            if (graph)
                cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaStreamEndCapture");
        const cudaError_t ie = cudaGraphInstantiate(&g->exec, graph, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess)
            return cuda_fail(ie, "cudaGraphInstantiate");
        g->launches = count;
        slot = std::move(g);
    }
    HYB_CUDA(cudaGraphLaunch(slot->exec, h->stream));
    h->last_launches += slot->launches;
    return HYB_SUCCESS;
}

// One substitution of y with the factors in `slab`: the dataflow form when it is enabled
// and the device can run it, else the staged form through the cached graph `slot`.
template <typename T, typename V>
int substitute(hyb_system *h, const T *slab, V *y, V *scratch, int nrhs, std::unique_ptr<GraphExec> &slot)
{
    if (h->flow)
    {
        uint64_t count = 0;
        const int rc = enqueue_solve_flow<T, V>(h, slab, y, nrhs, count);
        h->last_launches += count;
        if (rc != HYB_TOO_LARGE)
            return rc;
    }
    return run_graph(h, slot, [&](uint64_t &count) { return enqueue_solve<T, V>(h, slab, y, scratch, nrhs, count); });
}

int ensure_solve_buffers(hyb_system *h, int64_t nrhs)
{
    if (h->buf_nrhs >= nrhs)
        return HYB_SUCCESS;
    h->free_solve_buffers();
    const Symbolic &S = h->S;
    const int64_t dof = S.dof_off[S.n];
    const int64_t scr = std::max(S.max_fwd_scratch_rows, S.max_bwd_scratch_rows) * nrhs + 1;
    h->n_norm_parts = 296;
    HYB_CUDA(cudaMalloc(&h->d_b, dof * nrhs * sizeof(double)));
    HYB_CUDA(cudaMalloc(&h->d_x, dof * nrhs * sizeof(double)));
    HYB_CUDA(cudaMalloc(&h->d_r, dof * nrhs * sizeof(double)));
    HYB_CUDA(cudaMalloc(&h->d_scr64, scr * sizeof(double)));
    HYB_CUDA(cudaMalloc(&h->d_yf, dof * nrhs * sizeof(float)));
    HYB_CUDA(cudaMalloc(&h->d_scr32, scr * sizeof(float)));
    HYB_CUDA(cudaMalloc(&h->d_part, (size_t)h->n_norm_parts * nrhs * sizeof(double)));
    HYB_CUDA(cudaMalloc(&h->d_norm, 2 * nrhs * sizeof(double)));
    HYB_CUDA(cudaMalloc(&h->d_z, dof * nrhs * sizeof(double)));
    HYB_CUDA(cudaMalloc(&h->d_xb, dof * nrhs * sizeof(double)));
    h->buf_nrhs = nrhs;
    return HYB_SUCCESS;
}

void enqueue_sumsq(hyb_system *h, const double *v, int64_t rows, int nrhs, double *out, uint64_t &launches)
{
    hyb::k_sumsq_partial<<<h->n_norm_parts, hyb::kThreads, 0, h->stream>>>(v, rows, nrhs, h->d_part);
    hyb::k_sumsq_final<<<1, 32, 0, h->stream>>>(h->d_part, h->n_norm_parts, nrhs, out);
    launches += 2;
}

void enqueue_residual(hyb_system *h, const double *b, const double *x, double *r, int nrhs, uint64_t &launches)
{
    const int64_t dof = h->S.dof_off[h->S.n];
    const int64_t warps = hyb::kThreads / 32;
    hyb::k_residual<<<(unsigned)((dof + warps - 1) / warps), hyb::kThreads, 0, h->stream>>>(h->ds, h->d_a, b, x, r,
                                                                                            dof, nrhs);
    ++launches;
}

unsigned elementwise_grid(int64_t n)
{
    return (unsigned)std::min<int64_t>((n + hyb::kThreads - 1) / hyb::kThreads, 148 * 32);
}

int check_handle(const hyb_system *h)
{
    return h ? HYB_SUCCESS : HYB_INVALID_ARGUMENT;
}


// Device workspace of the dense block entry points, one per device: grown to the largest
// request and kept until the process exits, so repeated calls allocate nothing. Callers hold
// g_ws_mutex while they use it.
constexpr int kWsDevices = 64;
std::mutex g_ws_mutex;
char *g_ws[kWsDevices] = {};
size_t g_ws_bytes[kWsDevices] = {};

int workspace(size_t bytes, char **out)
{
    int dev = 0;
    HYB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kWsDevices)
        return HYB_INVALID_ARGUMENT;
    if (g_ws_bytes[dev] < bytes)
    {
        if (g_ws[dev])
        {
            HYB_CUDA(cudaDeviceSynchronize()); // earlier users of the old buffer are done
            cudaFree(g_ws[dev]);
            g_ws[dev] = nullptr;
            g_ws_bytes[dev] = 0;
        }
        const size_t grow = std::max<size_t>(bytes, 1 << 20);
        HYB_CUDA(cudaMalloc(&g_ws[dev], grow));
        g_ws_bytes[dev] = grow;
    }
    *out = g_ws[dev];
    return HYB_SUCCESS;
}

// A device allocation released when it goes out of scope, so early returns do not leak.
struct DevBuf
{
    void *p = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf()
    {
        if (p)
            cudaFree(p);
    }
};

// ------------------------------------------------------------------------------------
// Refinement of the mixed form (and of the plain form with HYB_OPTION_FP64_REFINEMENT).

// Squared 2-norms of the columns of v (dof x nr) into dev_out (on the device) and `out`
// (host) -- for a segmented system, of every segment of every column (nseg x nr) -- with
// the solve's status words read in the same synchronization.
int column_sumsq(hyb_system *h, const double *v, int nr, double *dev_out, std::vector<double> &out, bool &timed_out,
                 uint64_t &cnt)
{
    const int64_t dof = h->S.dof_off[h->S.n];
    enqueue_sumsq(h, v, dof, nr, dev_out, cnt);
    int sst[hyb::ST_WORDS];
    const int64_t nseg = h->seg_off.empty() ? 0 : (int64_t)h->seg_off.size() - 1;
    const double *src = dev_out;
    if (nseg > 0)
    {
        if (h->seg_norm_cap < nseg * nr)
        {
            cudaFree(h->d_seg_norm);
            h->d_seg_norm = nullptr;
            h->seg_norm_cap = 0;
            HYB_CUDA(cudaMalloc(&h->d_seg_norm, nseg * nr * sizeof(double)));
            h->seg_norm_cap = nseg * nr;
        }
        hyb::k_sumsq_segments<<<(unsigned)nseg, hyb::kThreads, 0, h->stream>>>(v, h->d_seg_off, nr, h->d_seg_norm);
        ++cnt;
        src = h->d_seg_norm;
    }
    out.resize(nseg > 0 ? nseg * nr : nr);
    HYB_CUDA(cudaMemcpyAsync(out.data(), src, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    HYB_CUDA(cudaMemcpyAsync(sst, h->d_solve_status, sizeof(sst), cudaMemcpyDeviceToHost, h->stream));
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    timed_out = sst[hyb::ST_TIMEOUT] != 0;
    return HYB_SUCCESS;
}

// Per segment and column, the steps after which its relative residual was first measured
// at or below tol, and the latest relative residual (segmented systems).
void record_segments(hyb_system *h, const std::vector<double> &rn2, const std::vector<double> &bn2, double tol,
                     uint32_t iters)
{
    if (h->seg_off.empty())
        return;
    for (size_t i = 0; i < rn2.size(); ++i)
    {
        const double rel = bn2[i] > 0 ? std::sqrt(rn2[i] / bn2[i]) : std::sqrt(rn2[i]);
        h->seg_relres[i] = rel;
        if (rel <= tol && h->seg_first[i] == UINT32_MAX)
            h->seg_first[i] = iters;
    }
}

// Largest relative residual over the columns (segments and columns when segmented).
double max_relative(const std::vector<double> &rn2, const std::vector<double> &bn2)
{
    double m = 0;
    for (size_t r = 0; r < rn2.size(); ++r)
    {
        const double v = bn2[r] > 0 ? std::sqrt(rn2[r] / bn2[r]) : std::sqrt(rn2[r]);
        m = std::isnan(v) ? v : std::max(m, v);
        if (std::isnan(m))
            break;
    }
    return m;
}

// z = M^{-1} v, one substitution with the handle's factors: in the mixed form v is rounded
// to FP32, substituted with the FP32 factors and widened back; otherwise FP64 throughout.
int apply_factors(hyb_system *h, const double *v, double *z, int nr, uint64_t &cnt)
{
    const int64_t len = h->S.dof_off[h->S.n] * nr;
    if (h->factored == HYB_PRECISION_MIXED)
    {
        const int64_t dof = h->S.dof_off[h->S.n];
        const unsigned eg = elementwise_grid(len);
        // with scaled factors (of S A S): A^{-1} v ~ S (LU)^{-1} (S v)
        if (h->factors_scaled)
            hyb::k_convert_scaled<double, float><<<eg, hyb::kThreads, 0, h->stream>>>(v, h->d_yf, h->d_dscale, dof, nr);
        else
            hyb::k_convert<double, float><<<eg, hyb::kThreads, 0, h->stream>>>(v, h->d_yf, len);
        auto &slot = h->g_solve[{HYB_PRECISION_MIXED, nr}];
        const int rc = substitute<float, float>(h, h->d_f32, h->d_yf, h->d_scr32, nr, slot);
        if (rc != HYB_SUCCESS)
            return rc;
        if (h->factors_scaled)
            hyb::k_convert_scaled<float, double><<<eg, hyb::kThreads, 0, h->stream>>>(h->d_yf, z, h->d_dscale, dof, nr);
        else
            hyb::k_convert<float, double><<<eg, hyb::kThreads, 0, h->stream>>>(h->d_yf, z, len);
        cnt += 2;
        return HYB_SUCCESS;
    }
    if (z != v)
        HYB_CUDA(cudaMemcpyAsync(z, v, len * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    auto &slot = h->g_solve[{HYB_PRECISION_FP64, nr}];
    return substitute<double, double>(h, h->d_f64, z, h->d_scr64, nr, slot);
}

struct RefineResult
{
    uint32_t iters = 0;  // corrections applied (refinement steps + FGMRES iterations)
    uint32_t krylov = 0; // of them, FGMRES iterations
    double relres = -1;
    int status = HYB_SUCCESS;
};

// A refinement step must shrink the FP64 residual by at least this factor, or the
// automatic mode continues with FGMRES.
constexpr double kIrContraction = 0.1;

// Restarted FGMRES(m) in FP64 on A x = b from the current x (d_x), right-preconditioned
// by the factors: Z_j = M^{-1} V_j, w = A Z_j, modified Gram-Schmidt against V, Givens
// rotations on the host, x += Z y. Each column of a multi-RHS solve is its own Krylov
// process (the columns share the launches). The true FP64 residual is recomputed at every
// restart and decides convergence.
int fgmres(hyb_system *h, int nr, double tol, uint32_t max_iter, const std::vector<double> &bn2, RefineResult &o,
           uint64_t &cnt)
{
    const Symbolic &S = h->S;
    const int m = h->krylov_restart;
    const int64_t dof = S.dof_off[S.n], len = dof * nr;
    const unsigned eg = elementwise_grid(len);
    if (h->kry_m != m)
    {
        h->free_krylov();
        HYB_CUDA(cudaMalloc(&h->d_w, len * sizeof(double)));
        HYB_CUDA(cudaMalloc(&h->d_V, (size_t)(m + 1) * len * sizeof(double)));
        HYB_CUDA(cudaMalloc(&h->d_Zk, (size_t)m * len * sizeof(double)));
        HYB_CUDA(cudaMalloc(&h->d_h, (size_t)(m + 2) * nr * sizeof(double)));
        HYB_CUDA(cudaMalloc(&h->d_coef, (size_t)m * nr * sizeof(double)));
        h->kry_m = m;
    }
    // per column r: H (m+1 x m, row i column j at (r * (m + 1) + i) * m + j), rotations, g
    std::vector<double> H((size_t)nr * (m + 1) * m), cs((size_t)nr * m), sn((size_t)nr * m), g((size_t)nr * (m + 1));
    std::vector<double> hcol((size_t)(m + 2) * nr), coef((size_t)m * nr), rn2;
    // The Arnoldi estimate is the norm of a whole column; a column's residual is small
    // enough for every segment once it is below tol times the smallest segment norm of b.
    std::vector<double> col_scale(nr, INFINITY);
    for (size_t i = 0; i < bn2.size(); ++i)
    {
        const double v = std::sqrt(bn2[i]);
        col_scale[i % nr] = std::min(col_scale[i % nr], v > 0 ? v : 1.0);
    }
    bool to = false;
    int rc;
    for (;;)
    {
        enqueue_residual(h, h->d_b, h->d_x, h->d_r, nr, cnt);
        if ((rc = column_sumsq(h, h->d_r, nr, h->d_norm, rn2, to, cnt)) != HYB_SUCCESS)
            return rc;
        if (to)
        {
            o.status = HYB_DEVICE_TIMEOUT;
            return HYB_SUCCESS;
        }
        o.relres = max_relative(rn2, bn2);
        record_segments(h, rn2, bn2, tol, o.iters);
        if (o.relres <= tol)
            return HYB_SUCCESS;
        if (o.iters >= max_iter || !std::isfinite(o.relres))
        {
            o.status = HYB_NOT_CONVERGED;
            return HYB_SUCCESS;
        }
        hyb::k_normalize<<<eg, hyb::kThreads, 0, h->stream>>>(h->d_V, h->d_r, h->d_norm, dof, nr);
        ++cnt;
        std::fill(g.begin(), g.end(), 0.0);
        std::vector<double> beta2(nr, 0.0); // column norms of r (the segments' sums when segmented)
        for (size_t i = 0; i < rn2.size(); ++i)
            beta2[i % nr] += rn2[i];
        for (int r = 0; r < nr; ++r)
            g[(size_t)r * (m + 1)] = std::sqrt(std::max(beta2[r], 0.0));
        int j = 0;
        bool done = false;
        while (j < m && o.iters < max_iter && !done)
        {
            double *vj = h->d_V + (size_t)j * len, *zj = h->d_Zk + (size_t)j * len;
            if ((rc = apply_factors(h, vj, zj, nr, cnt)) != HYB_SUCCESS)
                return rc;
            enqueue_residual(h, nullptr, zj, h->d_w, nr, cnt); // w = A z_j
            for (int i = 0; i <= j; ++i)
            {
                const double *vi = h->d_V + (size_t)i * len;
                hyb::k_dot_partial<<<h->n_norm_parts, hyb::kThreads, 0, h->stream>>>(vi, h->d_w, dof, nr, h->d_part);
                hyb::k_sumsq_final<<<1, 32, 0, h->stream>>>(h->d_part, h->n_norm_parts, nr, h->d_h + (size_t)i * nr);
                hyb::k_sub_scaled<<<eg, hyb::kThreads, 0, h->stream>>>(h->d_w, vi, h->d_h + (size_t)i * nr, dof, nr);
                cnt += 3;
            }
            enqueue_sumsq(h, h->d_w, dof, nr, h->d_h + (size_t)(j + 1) * nr, cnt);
            hyb::k_normalize<<<eg, hyb::kThreads, 0, h->stream>>>(h->d_V + (size_t)(j + 1) * len, h->d_w,
                                                                   h->d_h + (size_t)(j + 1) * nr, dof, nr);
            ++cnt;
            int sst[hyb::ST_WORDS];
            HYB_CUDA(cudaMemcpyAsync(hcol.data(), h->d_h, (size_t)(j + 2) * nr * sizeof(double),
                                     cudaMemcpyDeviceToHost, h->stream));
            HYB_CUDA(cudaMemcpyAsync(sst, h->d_solve_status, sizeof(sst), cudaMemcpyDeviceToHost, h->stream));
            HYB_CUDA(cudaStreamSynchronize(h->stream));
            if (sst[hyb::ST_TIMEOUT])
            {
                o.status = HYB_DEVICE_TIMEOUT;
                return HYB_SUCCESS;
            }
            ++o.iters;
            ++o.krylov;
            double est = 0;
            for (int r = 0; r < nr; ++r)
            {
                auto Hc = [&](int i) -> double & { return H[((size_t)r * (m + 1) + i) * m + j]; };
                for (int i = 0; i <= j; ++i)
                    Hc(i) = hcol[(size_t)i * nr + r];
                Hc(j + 1) = std::sqrt(std::max(hcol[(size_t)(j + 1) * nr + r], 0.0));
                double *c = &cs[(size_t)r * m], *sv = &sn[(size_t)r * m], *gr = &g[(size_t)r * (m + 1)];
                for (int i = 0; i < j; ++i)
                {
                    const double t = c[i] * Hc(i) + sv[i] * Hc(i + 1);
                    Hc(i + 1) = -sv[i] * Hc(i) + c[i] * Hc(i + 1);
                    Hc(i) = t;
                }
                const double a = Hc(j), bb = Hc(j + 1), d = std::hypot(a, bb);
                c[j] = d > 0 ? a / d : 1.0;
                sv[j] = d > 0 ? bb / d : 0.0;
                Hc(j) = d;
                Hc(j + 1) = 0;
                gr[j + 1] = -sv[j] * gr[j];
                gr[j] = c[j] * gr[j];
                const double e = std::fabs(gr[j + 1]) / col_scale[r];
                est = std::isnan(e) ? e : std::max(est, e);
            }
            ++j;
            // the estimate is that of exact arithmetic: stop the cycle a little below the
            // tolerance and let the recomputed residual decide
            done = est <= 0.5 * tol;
        }
        // y = R^{-1} g on the j x j triangle, then x += Z y
        for (int r = 0; r < nr; ++r)
        {
            const double *gr = &g[(size_t)r * (m + 1)];
            std::vector<double> y(j);
            for (int i = j - 1; i >= 0; --i)
            {
                double sum = gr[i];
                for (int q = i + 1; q < j; ++q)
                    sum -= H[((size_t)r * (m + 1) + i) * m + q] * y[q];
                const double dii = H[((size_t)r * (m + 1) + i) * m + i];
                y[i] = dii != 0 ? sum / dii : 0.0;
            }
            for (int i = 0; i < j; ++i)
                coef[(size_t)i * nr + r] = y[i];
        }
        HYB_CUDA(cudaMemcpyAsync(h->d_coef, coef.data(), (size_t)j * nr * sizeof(double), cudaMemcpyHostToDevice,
                                 h->stream));
        hyb::k_add_combination<<<eg, hyb::kThreads, 0, h->stream>>>(h->d_x, h->d_Zk, len, h->d_coef, j, dof, nr);
        ++cnt;
    }
}

// x = M^{-1} b, then refinement: plain steps x += M^{-1} (b - A x) with the FP64 residual
// (HYB_OPTION_REFINEMENT 0 and 1), continued by FGMRES (0, when a step shrinks the
// residual less than kIrContraction, from the better of the last two iterates) or FGMRES
// from the start (2).
int refine(hyb_system *h, int nr, double tol, uint32_t max_iter, RefineResult &o, uint64_t &cnt)
{
    const Symbolic &S = h->S;
    const int64_t len = S.dof_off[S.n] * nr;
    const size_t bytes = len * sizeof(double);
    int rc = apply_factors(h, h->d_b, h->d_x, nr, cnt);
    if (rc != HYB_SUCCESS)
        return rc;
    std::vector<double> bn2, rn2;
    bool to = false;
    if ((rc = column_sumsq(h, h->d_b, nr, h->d_norm + nr, bn2, to, cnt)) != HYB_SUCCESS)
        return rc;
    if (!h->seg_off.empty())
    {
        h->seg_first.assign(bn2.size(), UINT32_MAX);
        h->seg_relres.assign(bn2.size(), -1.0);
    }
    double prev = INFINITY;
    bool krylov = h->refinement == 2;
    while (!krylov)
    {
        enqueue_residual(h, h->d_b, h->d_x, h->d_r, nr, cnt);
        if ((rc = column_sumsq(h, h->d_r, nr, h->d_norm, rn2, to, cnt)) != HYB_SUCCESS)
            return rc;
        if (to)
        {
            o.status = HYB_DEVICE_TIMEOUT;
            return HYB_SUCCESS;
        }
        o.relres = max_relative(rn2, bn2);
        record_segments(h, rn2, bn2, tol, o.iters);
        if (o.relres <= tol)
            return HYB_SUCCESS;
        if (h->refinement == 0 && o.iters > 0 && !(o.relres <= kIrContraction * prev))
        {
            if (!(o.relres <= prev)) // the last step made it worse: back to the iterate before it
            {
                HYB_CUDA(cudaMemcpyAsync(h->d_x, h->d_xb, bytes, cudaMemcpyDeviceToDevice, h->stream));
                o.relres = prev;
            }
            krylov = true;
            break;
        }
        if (o.iters >= max_iter || !std::isfinite(o.relres))
        {
            o.status = HYB_NOT_CONVERGED;
            return HYB_SUCCESS;
        }
        if (h->refinement == 0)
            HYB_CUDA(cudaMemcpyAsync(h->d_xb, h->d_x, bytes, cudaMemcpyDeviceToDevice, h->stream));
        if ((rc = apply_factors(h, h->d_r, h->d_z, nr, cnt)) != HYB_SUCCESS)
            return rc;
        hyb::k_add_correction<double><<<elementwise_grid(len), hyb::kThreads, 0, h->stream>>>(h->d_x, h->d_z, len);
        ++cnt;
        ++o.iters;
        prev = o.relres;
    }
    return fgmres(h, nr, tol, max_iter, bn2, o, cnt);
}

// ------------------------------------------------------------------------------------
// Solves with A^T and the condition estimate.

// Column view of the factors and of A (hyb::DevTrans), built and uploaded once per handle.
int ensure_trans(hyb_system *h)
{
    if (h->t_arena)
        return HYB_SUCCESS;
    const Symbolic &S = h->S;
    const int64_t n = S.n;
    std::vector<int64_t> ucol_ptr(n + 1, 0), fu_pref(n + 1, 0), fu_rows(n + 1, 0), bu_pref(n + 1, 0),
        bu_rows(n + 1, 0), acol_ptr(n + 1, 0);
    for (int64_t k = 0; k < n; ++k)
        for (int64_t j = S.diag_pos[k] + 1; j < S.row_ptr[k + 1]; ++j)
            ++ucol_ptr[S.cols[j] + 1];
    for (int64_t c = 0; c < n; ++c)
        ucol_ptr[c + 1] += ucol_ptr[c];
    std::vector<int32_t> ucol_row(ucol_ptr[n]), ucol_blk(ucol_ptr[n]);
    {
        std::vector<int64_t> next(ucol_ptr.begin(), ucol_ptr.end() - 1);
        for (int64_t k = 0; k < n; ++k) // ascending rows within every column
            for (int64_t j = S.diag_pos[k] + 1; j < S.row_ptr[k + 1]; ++j)
            {
                const int64_t e = next[S.cols[j]]++;
                ucol_row[e] = (int32_t)k;
                ucol_blk[e] = (int32_t)j;
            }
    }
    for (int64_t p = 0; p < n; ++p)
    {
        const int64_t k = S.piv[p], m = S.size[k];
        const int64_t nu = ucol_ptr[k + 1] - ucol_ptr[k], nl = S.lcol_ptr[k + 1] - S.lcol_ptr[k];
        fu_pref[p + 1] = fu_pref[p] + std::max<int64_t>(1, nu);
        fu_rows[p + 1] = fu_rows[p] + (nu * m + 3) / 4 * 4;
        bu_pref[p + 1] = bu_pref[p] + std::max<int64_t>(1, nl);
        bu_rows[p + 1] = bu_rows[p] + (nl * m + 3) / 4 * 4;
    }
    int64_t max_rows = 0;
    for (int64_t l = 0; l < S.n_levels; ++l)
    {
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        max_rows = std::max({max_rows, fu_rows[p1] - fu_rows[p0], bu_rows[p1] - bu_rows[p0]});
    }
    const int64_t nnz_a = S.nnz_a();
    for (int64_t j = 0; j < nnz_a; ++j)
        ++acol_ptr[S.a_cols[j] + 1];
    for (int64_t c = 0; c < n; ++c)
        acol_ptr[c + 1] += acol_ptr[c];
    std::vector<int32_t> acol_row(std::max<int64_t>(1, nnz_a)), acol_blk(std::max<int64_t>(1, nnz_a));
    {
        std::vector<int64_t> next(acol_ptr.begin(), acol_ptr.end() - 1);
        for (int64_t r = 0; r < n; ++r)
            for (int64_t j = S.a_row_ptr[r]; j < S.a_row_ptr[r + 1]; ++j)
            {
                const int64_t e = next[S.a_cols[j]]++;
                acol_row[e] = (int32_t)r;
                acol_blk[e] = (int32_t)j;
            }
    }
    struct Item
    {
        const void *src;
        size_t bytes;
        const void **dst;
    };
    hyb::DevTrans &d = h->dt;
    const std::vector<Item> items = {
        {ucol_ptr.data(), ucol_ptr.size() * 8, (const void **)&d.ucol_ptr},
        {ucol_row.data(), ucol_row.size() * 4, (const void **)&d.ucol_row},
        {ucol_blk.data(), ucol_blk.size() * 4, (const void **)&d.ucol_blk},
        {fu_pref.data(), fu_pref.size() * 8, (const void **)&d.fu_pref},
        {fu_rows.data(), fu_rows.size() * 8, (const void **)&d.fu_rows},
        {bu_pref.data(), bu_pref.size() * 8, (const void **)&d.bu_pref},
        {bu_rows.data(), bu_rows.size() * 8, (const void **)&d.bu_rows},
        {acol_ptr.data(), acol_ptr.size() * 8, (const void **)&d.acol_ptr},
        {acol_row.data(), acol_row.size() * 4, (const void **)&d.acol_row},
        {acol_blk.data(), acol_blk.size() * 4, (const void **)&d.acol_blk},
    };
    size_t total = 0;
    for (const Item &it : items)
        total += (it.bytes + 255) / 256 * 256 + 256;
    std::vector<char> host(total, 0);
    void *arena = nullptr;
    HYB_CUDA(cudaMalloc(&arena, total));
    size_t off = 0;
    for (const Item &it : items)
    {
        if (it.bytes)
            std::memcpy(host.data() + off, it.src, it.bytes);
        *it.dst = (const char *)arena + off;
        off += (it.bytes + 255) / 256 * 256 + 256;
    }
    const cudaError_t e = cudaMemcpy(arena, host.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
    {
        cudaFree(arena);
        return cuda_fail(e, "cudaMemcpy(transpose view)");
    }
    h->t_arena = arena;
    h->t_max_rows = max_rows;
    h->t_fu_pref = std::move(fu_pref);
    h->t_bu_pref = std::move(bu_pref);
    return HYB_SUCCESS;
}

// A^T y = z in place on y with the FP64 factors: the U^T pass by levels ascending, then
// the L^T pass by levels descending.
int enqueue_solve_transpose(hyb_system *h, double *y, double *scratch, int nrhs, uint64_t &launches)
{
    const Symbolic &S = h->S;
    cudaStream_t st = h->stream;
    HYB_CUDA(cudaMemsetAsync(h->d_tickets, 0, S.n * sizeof(int), st));
    for (int64_t l = 0; l < S.n_levels; ++l)
    {
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        const int64_t units = h->t_fu_pref[p1] - h->t_fu_pref[p0];
        hyb::k_fwdT_stage<double, double>
            <<<(unsigned)units, hyb::kThreads, 0, st>>>(h->ds, h->dt, h->d_f64, y, scratch, h->d_tickets, p0, p1, nrhs);
        ++launches;
    }
    for (int64_t l = S.n_levels - 1; l >= 0; --l)
    {
        const int64_t p0 = S.lvl_ptr[l], p1 = S.lvl_ptr[l + 1];
        const int64_t units = h->t_bu_pref[p1] - h->t_bu_pref[p0];
        const int smem = S.shape[l].max_piv * nrhs * (int)sizeof(double);
        hyb::k_bwdT_stage<double, double><<<(unsigned)units, hyb::kThreads, smem, st>>>(
            h->ds, h->dt, h->d_f64, y, scratch, h->d_tickets, p0, p1, nrhs);
        ++launches;
    }
    HYB_CUDA(cudaGetLastError());
    return HYB_SUCCESS;
}

// One solve of a host vector with A (plain FP64 substitution) or A^T, for the estimate.
int solve_host_once(hyb_system *h, const double *in, double *out, bool transpose)
{
    const int64_t dof = h->S.dof_off[h->S.n];
    HYB_CUDA(cudaMemcpyAsync(h->d_x, in, dof * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    int rc;
    if (transpose)
        rc = run_graph(h, h->g_solveT[1],
                       [&](uint64_t &c) { return enqueue_solve_transpose(h, h->d_x, h->d_tscr, 1, c); });
    else
        rc = substitute<double, double>(h, h->d_f64, h->d_x, h->d_scr64, 1, h->g_solve[{HYB_PRECISION_FP64, 1}]);
    if (rc != HYB_SUCCESS)
        return rc;
    int sst[hyb::ST_WORDS];
    HYB_CUDA(cudaMemcpyAsync(out, h->d_x, dof * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    HYB_CUDA(cudaMemcpyAsync(sst, h->d_solve_status, sizeof(sst), cudaMemcpyDeviceToHost, h->stream));
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    if (sst[hyb::ST_TIMEOUT])
    {
        g_cuda_error = "a wait of the dataflow solve ran out of its time limit";
        return HYB_DEVICE_TIMEOUT;
    }
    return HYB_SUCCESS;
}

// Scratch of the transposed solve's partial products for nrhs right-hand sides.
int ensure_trans_scratch(hyb_system *h, int64_t nrhs)
{
    if (h->tscr_nrhs >= nrhs)
        return HYB_SUCCESS;
    cudaFree(h->d_tscr);
    h->d_tscr = nullptr;
    h->tscr_nrhs = 0;
    h->g_solveT.clear();
    HYB_CUDA(cudaMalloc(&h->d_tscr, (h->t_max_rows * nrhs + 1) * sizeof(double)));
    h->tscr_nrhs = nrhs;
    return HYB_SUCCESS;
}

} // namespace

// =====================================================================================
extern "C" {

HYB_API const char *hyb_status_string(int status)
{
    switch (status)
    {
    case HYB_SUCCESS:
        return "success";
    case HYB_BLOCK_NOT_IN_SYSTEM:
        return "block not in system";
    case HYB_FAILED_ALLOC:
        return "memory allocation failed";
    case HYB_MAX_COLORS:
        return "maximum number of colors exceeded";
    case HYB_INVALID_ARGUMENT:
        return "invalid argument";
    case HYB_MISSING_DIAGONAL:
        return "a row has no diagonal block";
    case HYB_NOT_DECOMPOSED:
        return "the system has not been decomposed yet";
    case HYB_CUDA_ERROR:
        return "CUDA error";
    case HYB_NO_DEVICE:
        return "no sm_100 CUDA device";
    case HYB_ZERO_PIVOT:
        return "zero pivot";
    case HYB_NON_FINITE:
        return "non-finite pivot";
    case HYB_NOT_CONVERGED:
        return "iterative refinement did not converge";
    case HYB_TOO_LARGE:
        return "size beyond the supported limit";
    case HYB_DEVICE_TIMEOUT:
        return "a bounded device-side wait ran out";
    default:
        return "unknown status";
    }
}

HYB_API const char *hyb_last_cuda_error(void)
{
    return g_cuda_error.c_str();
}

HYB_API int hyb_version(void)
{
    return 100;
}

HYB_API int hyb_device_available(void)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return 0;
    }
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    return major == 10;
}

HYB_API int hyb_compute_ordering(uint64_t n, const uint64_t *row_ptr, const uint64_t *cols, int strategy,
                                 uint64_t max_colors, uint64_t *ordering)
{
    if (n && (!row_ptr || !ordering || (!cols && row_ptr[n])))
        return HYB_INVALID_ARGUMENT;
    try
    {
        return hyb::compute_ordering(n, row_ptr, cols, strategy, max_colors, ordering);
    }
    catch (const std::bad_alloc &)
    {
        return HYB_FAILED_ALLOC;
    }
}

HYB_API int hyb_analyze(uint64_t n, const uint64_t *block_sizes, const uint64_t *row_ptr, const uint64_t *cols,
                        hyb_analysis *out, uint64_t *filled_row_ptr, uint64_t *filled_cols, int64_t *ops)
{
    if (!out || !block_sizes || !row_ptr || (!cols && n && row_ptr[n]))
        return HYB_INVALID_ARGUMENT;
    try
    {
        Symbolic S;
        std::string err;
        const int rc = hyb::symbolic_build((int64_t)n, block_sizes, row_ptr, cols, S, err);
        if (rc != HYB_SUCCESS)
        {
            g_cuda_error = err;
            return rc;
        }
        out->filled_blocks = (uint64_t)S.nnz_f();
        out->factor_values = (uint64_t)S.factor_values;
        out->n_levels = (uint64_t)S.n_levels;
        out->nops = (uint64_t)(S.lcol_ptr[S.n] + S.n);
        out->slab_bytes_fp64 = (uint64_t)S.slab_elems() * sizeof(double);
        out->factor_flops = S.factor_flops;
        out->pair_levels = (uint64_t)S.n_pairs;
        if (filled_row_ptr)
            for (int64_t i = 0; i <= S.n; ++i)
                filled_row_ptr[i] = (uint64_t)S.row_ptr[i];
        if (filled_cols)
            for (int64_t j = 0; j < S.nnz_f(); ++j)
                filled_cols[j] = (uint64_t)S.cols[j];
        if (ops)
        {
            std::vector<int64_t> v;
            hyb::symbolic_operations(S, v);
            std::memcpy(ops, v.data(), v.size() * sizeof(int64_t));
        }
    }
    catch (const std::bad_alloc &)
    {
        return HYB_FAILED_ALLOC;
    }
    return HYB_SUCCESS;
}

HYB_API int hyb_system_create(uint64_t n, const uint64_t *block_sizes, const uint64_t *row_ptr, const uint64_t *cols,
                              hyb_system **out)
{
    if (!out || !block_sizes || !row_ptr || (!cols && n && row_ptr[n]))
        return HYB_INVALID_ARGUMENT;
    *out = nullptr;
    if (!hyb_device_available())
        return HYB_NO_DEVICE;
    std::unique_ptr<hyb_system> h;
    try
    {
        h = std::make_unique<hyb_system>();
        std::string err;
        const int rc = hyb::symbolic_build((int64_t)n, block_sizes, row_ptr, cols, h->S, err);
        if (rc != HYB_SUCCESS)
        {
            g_cuda_error = err;
            return rc;
        }
    }
    catch (const std::bad_alloc &)
    {
        return HYB_FAILED_ALLOC;
    }
    HYB_CUDA(cudaGetDevice(&h->device));
    HYB_CUDA(create_streams(h.get()));
    int rc = upload_symbolic(h.get());
    if (rc != HYB_SUCCESS)
        return rc;
    HYB_CUDA(cudaMalloc(&h->d_a, std::max<int64_t>(1, h->S.a_val_off.back()) * sizeof(double)));
    HYB_CUDA(cudaMemsetAsync(h->d_a, 0, std::max<int64_t>(1, h->S.a_val_off.back()) * sizeof(double), h->stream));
    HYB_CUDA(cudaMalloc(&h->d_status, hyb::ST_WORDS * sizeof(int)));
    HYB_CUDA(cudaMalloc(&h->d_tickets, h->S.n * sizeof(int)));
    HYB_CUDA(cudaMalloc(&h->d_flags, h->S.n * sizeof(int)));
    HYB_CUDA(cudaMemsetAsync(h->d_flags, 0, h->S.n * sizeof(int), h->stream));
    HYB_CUDA(cudaMalloc(&h->d_pflags, h->S.n * sizeof(int)));
    HYB_CUDA(cudaMemsetAsync(h->d_pflags, 0, h->S.n * sizeof(int), h->stream));
    HYB_CUDA(cudaMalloc(&h->d_lu_tickets, h->S.n * sizeof(int)));
    HYB_CUDA(cudaMemsetAsync(h->d_lu_tickets, 0, h->S.n * sizeof(int), h->stream));
    HYB_CUDA(cudaMalloc(&h->d_solve_status, hyb::ST_WORDS * sizeof(int)));
    HYB_CUDA(cudaMemsetAsync(h->d_tickets, 0, h->S.n * sizeof(int), h->stream));
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    *out = h.release();
    return HYB_SUCCESS;
}

HYB_API int hyb_system_destroy(hyb_system *h)
{
    if (!h)
        return HYB_SUCCESS;
    cudaStreamSynchronize(h->stream);
    delete h;
    return HYB_SUCCESS;
}

HYB_API int hyb_system_copy(const hyb_system *src, hyb_system **out)
{
    if (!src || !out)
        return HYB_INVALID_ARGUMENT;
    *out = nullptr;
    std::unique_ptr<hyb_system> h;
    try
    {
        h = std::make_unique<hyb_system>();
        h->S = src->S;
    }
    catch (const std::bad_alloc &)
    {
        return HYB_FAILED_ALLOC;
    }
    h->device = src->device;
    h->lookahead = src->lookahead;
    h->umma = src->umma;
    h->flow = src->flow;
    h->wait_ns = src->wait_ns;
    h->refinement = src->refinement;
    h->fp64_refine = src->fp64_refine;
    h->krylov_restart = src->krylov_restart;
    h->growth_limit = src->growth_limit;
    h->block_scaling = src->block_scaling;
    h->alternate_walk = src->alternate_walk;
    h->pair_passes = src->pair_passes;
    h->row_pivots = src->row_pivots;
    h->update_sm_reserve = src->update_sm_reserve;
    h->update_kernel = src->update_kernel;
    h->lu_once = src->lu_once;
    h->fp64_shape = src->fp64_shape;
    std::memcpy(h->tuned, src->tuned, sizeof(h->tuned));
    HYB_CUDA(create_streams(h.get()));
    int rc = upload_symbolic(h.get());
    if (rc != HYB_SUCCESS)
        return rc;
    const size_t a_bytes = std::max<int64_t>(1, h->S.a_val_off.back()) * sizeof(double);
    HYB_CUDA(cudaMalloc(&h->d_a, a_bytes));
    HYB_CUDA(cudaMalloc(&h->d_status, hyb::ST_WORDS * sizeof(int)));
    HYB_CUDA(cudaMalloc(&h->d_tickets, h->S.n * sizeof(int)));
    HYB_CUDA(cudaMalloc(&h->d_flags, h->S.n * sizeof(int)));
    HYB_CUDA(cudaMemsetAsync(h->d_flags, 0, h->S.n * sizeof(int), h->stream));
    HYB_CUDA(cudaMalloc(&h->d_pflags, h->S.n * sizeof(int)));
    HYB_CUDA(cudaMemsetAsync(h->d_pflags, 0, h->S.n * sizeof(int), h->stream));
    HYB_CUDA(cudaMalloc(&h->d_lu_tickets, h->S.n * sizeof(int)));
    HYB_CUDA(cudaMemsetAsync(h->d_lu_tickets, 0, h->S.n * sizeof(int), h->stream));
    HYB_CUDA(cudaMalloc(&h->d_solve_status, hyb::ST_WORDS * sizeof(int)));
    HYB_CUDA(cudaMemsetAsync(h->d_tickets, 0, h->S.n * sizeof(int), h->stream));
    HYB_CUDA(cudaStreamSynchronize(src->stream));
    HYB_CUDA(cudaMemcpyAsync(h->d_a, src->d_a, a_bytes, cudaMemcpyDeviceToDevice, h->stream));
    const size_t slab = std::max<int64_t>(1, h->S.slab_elems());
    if (src->d_f64)
    {
        HYB_CUDA(cudaMalloc(&h->d_f64, slab * sizeof(double)));
        HYB_CUDA(cudaMemcpyAsync(h->d_f64, src->d_f64, slab * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    }
    if (src->d_f32)
    {
        HYB_CUDA(cudaMalloc(&h->d_f32, slab * sizeof(float)));
        HYB_CUDA(cudaMemcpyAsync(h->d_f32, src->d_f32, slab * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    }
    if (src->d_dinv)
    {
        const size_t bytes = (size_t)h->S.n_inv * 4096 * sizeof(float);
        HYB_CUDA(cudaMalloc(&h->d_dinv, bytes));
        HYB_CUDA(cudaMemcpyAsync(h->d_dinv, src->d_dinv, bytes, cudaMemcpyDeviceToDevice, h->stream));
    }
    h->factored = src->factored;
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    *out = h.release();
    return HYB_SUCCESS;
}

HYB_API uint64_t hyb_system_value_count(const hyb_system *h)
{
    return h ? (uint64_t)h->S.a_val_off.back() : 0;
}

HYB_API uint64_t hyb_system_dof(const hyb_system *h)
{
    return h ? (uint64_t)h->S.dof_off[h->S.n] : 0;
}

HYB_API void *hyb_system_stream(const hyb_system *h)
{
    return h ? (void *)h->stream : nullptr;
}

HYB_API int hyb_system_set_option(hyb_system *h, int option, int64_t value)
{
    if (check_handle(h))
        return HYB_INVALID_ARGUMENT;
    switch (option)
    {
    case HYB_OPTION_LOOKAHEAD:
        if (h->lookahead != (value != 0))
        {
            h->lookahead = value != 0;
            h->g_factor[0].reset();
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_TENSOR_CORE_MIXED:
        if (h->umma != (value != 0))
        {
            h->umma = value != 0;
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_DATAFLOW_SOLVE:
        h->flow = value != 0;
        return HYB_SUCCESS;
    case HYB_OPTION_WAIT_LIMIT_NS:
        if (value <= 0)
            return HYB_INVALID_ARGUMENT;
        h->wait_ns = (uint64_t)std::max<int64_t>(value, 100000);
        return HYB_SUCCESS;
    case HYB_OPTION_REFINEMENT:
        if (value < 0 || value > 2)
            return HYB_INVALID_ARGUMENT;
        h->refinement = (int)value;
        return HYB_SUCCESS;
    case HYB_OPTION_FP64_REFINEMENT:
        h->fp64_refine = value != 0;
        return HYB_SUCCESS;
    case HYB_OPTION_KRYLOV_RESTART:
        if (value < 1 || value > 200)
            return HYB_INVALID_ARGUMENT;
        if (value != h->krylov_restart)
            h->free_krylov();
        h->krylov_restart = (int)value;
        return HYB_SUCCESS;
    case HYB_OPTION_FP64_MMA_SHAPE:
        if (value < 0 || value > 2)
            return HYB_INVALID_ARGUMENT;
        if (h->fp64_shape != (int)value)
        {
            h->fp64_shape = (int)value;
            h->g_factor[0].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_PIVOT_LU_ONCE:
        if (value < -1 || value > 1)
            return HYB_INVALID_ARGUMENT;
        if (h->lu_once != (int)value)
        {
            h->lu_once = (int)value;
            h->g_factor[0].reset();
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_UPDATE_KERNEL:
        if (value < -1 || value >= UPD_KINDS)
            return HYB_INVALID_ARGUMENT;
        if (value != h->update_kernel)
        {
            h->update_kernel = (int)value;
            h->g_factor[0].reset();
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_ALTERNATE_WALK:
        if (h->alternate_walk != (value != 0))
        {
            h->alternate_walk = value != 0;
            h->g_factor[0].reset();
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_UPDATE_SM_RESERVE:
        if (value < 0 || value > 64)
            return HYB_INVALID_ARGUMENT;
        if (h->update_sm_reserve != (int)value)
        {
            h->update_sm_reserve = (int)value;
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_ROW_PIVOTS:
        if (value < -1 || value > 2)
            return HYB_INVALID_ARGUMENT;
        if (h->row_pivots != (int)value)
        {
            h->row_pivots = (int)value;
            h->g_factor[0].reset();
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_PAIR_PASSES:
        if (value < 0 || value > 2)
            return HYB_INVALID_ARGUMENT;
        if (h->pair_passes != (int)value)
        {
            h->pair_passes = (int)value;
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_BLOCK_SCALING:
        h->block_scaling = value != 0;
        return HYB_SUCCESS;
    case HYB_OPTION_GROWTH_LIMIT:
        if (value < 0)
            return HYB_INVALID_ARGUMENT;
        if ((float)value != h->growth_limit)
        {
            h->growth_limit = (float)value;
            h->g_factor[1].reset();
        }
        return HYB_SUCCESS;
    case HYB_OPTION_WITHHOLD_ROW:
    {
        if (value < 0)
        {
            h->withhold_slot = -1;
            return HYB_SUCCESS;
        }
        const Symbolic &S = h->S;
        if (value >= S.n || S.diag_pos[value] - S.row_ptr[value] < 2)
            return HYB_INVALID_ARGUMENT;
        for (int64_t p = 0; p < S.n; ++p)
            if (S.piv[p] == value)
                h->withhold_slot = p;
        return HYB_SUCCESS;
    }
    default:
        return HYB_INVALID_ARGUMENT;
    }
}

HYB_API int hyb_system_set_segments(hyb_system *h, uint64_t nseg, const uint64_t *offsets)
{
    if (check_handle(h) || (nseg > 0 && !offsets))
        return HYB_INVALID_ARGUMENT;
    const int64_t dof = h->S.dof_off[h->S.n];
    if (nseg > 0 && (offsets[0] != 0 || offsets[nseg] != (uint64_t)dof || nseg > (uint64_t)dof))
        return HYB_INVALID_ARGUMENT;
    for (uint64_t s = 0; s < nseg; ++s)
        if (offsets[s + 1] <= offsets[s])
            return HYB_INVALID_ARGUMENT;
    cudaFree(h->d_seg_off);
    h->d_seg_off = nullptr;
    h->seg_off.clear();
    h->seg_first.clear();
    h->seg_relres.clear();
    if (nseg == 0)
        return HYB_SUCCESS;
    std::vector<int64_t> off(offsets, offsets + nseg + 1);
    HYB_CUDA(cudaMalloc(&h->d_seg_off, off.size() * sizeof(int64_t)));
    HYB_CUDA(cudaMemcpy(h->d_seg_off, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
    h->seg_off = std::move(off);
    return HYB_SUCCESS;
}

HYB_API int hyb_tuned_kernels(const hyb_system *h, int precision, int32_t kinds[49])
{
    if (check_handle(h) || !kinds || (precision != HYB_PRECISION_FP64 && precision != HYB_PRECISION_MIXED))
        return HYB_INVALID_ARGUMENT;
    static_assert(hyb_tuning_buckets() == 49, "the header declares 49 buckets");
    for (int b = 0; b < hyb_tuning_buckets(); ++b)
        kinds[b] = h->tuned[precision][b];
    return HYB_SUCCESS;
}

HYB_API int hyb_segment_results(const hyb_system *h, uint32_t *iterations, double *relative_residual)
{
    if (check_handle(h) || h->seg_off.empty())
        return HYB_INVALID_ARGUMENT;
    if (h->seg_first.empty())
        return HYB_NOT_DECOMPOSED; // no refined solve yet
    if (iterations)
        std::memcpy(iterations, h->seg_first.data(), h->seg_first.size() * sizeof(uint32_t));
    if (relative_residual)
        std::memcpy(relative_residual, h->seg_relres.data(), h->seg_relres.size() * sizeof(double));
    return HYB_SUCCESS;
}

HYB_API int hyb_system_set_values(hyb_system *h, const double *values, int memory)
{
    if (check_handle(h) || (!values && h->S.a_val_off.back() > 0))
        return HYB_INVALID_ARGUMENT;
    const size_t bytes = h->S.a_val_off.back() * sizeof(double);
    if (bytes)
        HYB_CUDA(cudaMemcpyAsync(h->d_a, values, bytes,
                                 memory == HYB_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 h->stream));
    h->factored = -1;
    if (memory != HYB_MEMORY_DEVICE)
        HYB_CUDA(cudaStreamSynchronize(h->stream)); // the caller may reuse a pageable buffer
    return HYB_SUCCESS;
}

HYB_API int hyb_decompose(hyb_system *h, int precision, hyb_decompose_info *info)
{
    if (check_handle(h) || (precision != HYB_PRECISION_FP64 && precision != HYB_PRECISION_MIXED))
        return HYB_INVALID_ARGUMENT;
    const Symbolic &S = h->S;
    const size_t slab = std::max<int64_t>(1, S.slab_elems());
    static bool attrs_set = false;
    if (!attrs_set)
    {
        const int optin = smem_optin();
        const cudaError_t errs[] = {
            allow_smem(hyb::k_lu<double, true>, optin),
            allow_smem(hyb::k_lu<float, true>, optin),
            allow_smem(hyb::k_trsm<double, true>, optin),
            allow_smem(hyb::k_trsm<float, true>, optin),
            allow_smem(hyb::k_fwd_stage<double, double>, optin),
            allow_smem(hyb::k_fwd_stage<float, float>, optin),
            allow_smem(hyb::k_update64_f64<0>, hyb::kUpd64Smem),
            allow_smem(hyb::k_update64_f64<1>, hyb::kUpd64Smem),
            allow_smem(hyb::k_update64_f64<2>, hyb::kUpd64Smem),
            allow_smem(hyb::k_lu_trsm64<double, false>, hyb::lu_trsm64_smem<double>()),
            allow_smem(hyb::k_lu_trsm64<float, false>, hyb::lu_trsm64_smem<float>()),
            allow_smem(hyb::k_lu_trsm64<double, true>, hyb::lu_trsm64_smem<double>()),
            allow_smem(hyb::k_lu_trsm64<float, true>, hyb::lu_trsm64_smem<float>()),
            allow_smem(hyb::k_update64_tc, hyb::kTcSmem),
            allow_smem(hyb::k_update64_tc2, hyb::kTc2Smem),
            allow_smem(hyb::k_piv64<double, false>, hyb::piv64_smem<double>()),
            allow_smem(hyb::k_piv64<float, false>, hyb::piv64_smem<float>()),
            allow_smem(hyb::k_piv64<float, true>, hyb::piv64_smem<float>()),
            allow_smem(hyb::k_piv64_inv, hyb::kInvSmem),
            allow_smem(hyb::k_strips64_inv, hyb::kInvSmem),
            allow_smem(hyb::k_split64, 0),
            allow_smem(hyb::k_update<double>, 0),
            allow_smem(hyb::k_update<float>, 0),
            allow_smem(hyb::k_update32<double>, 0),
            allow_smem(hyb::k_update32<float>, 0),
            allow_smem(hyb::k_update_dmma<double>, hyb::dmma_smem_bytes(hyb::kDmmaMaxK)),
            allow_smem(hyb::k_lu64_once<double, false>, hyb::lu64_once_smem<double>()),
            allow_smem(hyb::k_lu64_once<double, true>, hyb::lu64_once_smem<double>()),
            allow_smem(hyb::k_lu64_once<float, false>, hyb::lu64_once_smem<float>()),
            allow_smem(hyb::k_lu64_once<float, true>, hyb::lu64_once_smem<float>()),
            allow_smem(hyb::k_trsm64_strips<double, false>, hyb::lu_trsm64_smem<double>()),
            allow_smem(hyb::k_trsm64_strips<double, true>, hyb::lu_trsm64_smem<double>()),
            allow_smem(hyb::k_trsm64_strips<float, false>, hyb::lu_trsm64_smem<float>()),
            allow_smem(hyb::k_trsm64_strips<float, true>, hyb::lu_trsm64_smem<float>()),
            allow_smem(hyb::k_update_dmma<float>, hyb::dmma_smem_bytes(hyb::kDmmaMaxK)),
        };
        for (cudaError_t e : errs)
            if (e != cudaSuccess)
                return cuda_fail(e, "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)");
        attrs_set = true;
    }
    h->last_launches = 0;
    h->factored = -1;
    h->g_solveT.clear(); // captured with the FP64 slab's address, which may change below
    const unsigned sgrid = (unsigned)std::min<int64_t>(std::max<int64_t>(1, S.nnz_a()), 148 * 16);
    if (precision == HYB_PRECISION_FP64)
    {
        if (h->d_f32)
        {
            cudaFree(h->d_f32);
            cudaFree(h->d_dinv);
            h->d_f32 = nullptr;
            h->d_dinv = nullptr;
            h->g_factor[1].reset();
            h->g_solve.clear();
        }
        if (!h->d_f64)
        {
            HYB_CUDA(cudaMalloc(&h->d_f64, slab * sizeof(double)));
            h->g_factor[0].reset();
            h->g_solve.clear();
        }
        HYB_CUDA(cudaMemsetAsync(h->d_f64, 0, slab * sizeof(double), h->stream));
        if (h->update_kernel < 0 && needs_tuning<double>(h))
        {
            const int rc = tune_updates<double>(h, h->d_f64);
            if (rc != HYB_SUCCESS)
                return rc;
            h->g_factor[0].reset(); // recaptured with the chosen kernels
            HYB_CUDA(cudaMemsetAsync(h->d_f64, 0, slab * sizeof(double), h->stream));
        }
        hyb::k_scatter<double><<<sgrid, hyb::kThreads, 0, h->stream>>>(h->ds, h->d_a, h->d_f64, S.nnz_a(), nullptr);
        h->last_launches += 1;
        const int rc = run_graph(h, h->g_factor[0], [&](uint64_t &count) {
            h->free_profile_events();
            h->prof_precision = HYB_PRECISION_FP64;
            return enqueue_factor<double>(h, h->d_f64, count);
        });
        if (rc != HYB_SUCCESS)
            return rc;
    }
    else
    {
        if (h->d_f64)
        {
            cudaFree(h->d_f64);
            h->d_f64 = nullptr;
            h->g_factor[0].reset();
            h->g_solve.clear();
        }
        if (!h->d_f32)
        {
            HYB_CUDA(cudaMalloc(&h->d_f32, slab * sizeof(float)));
            if (S.n_inv > 0)
                HYB_CUDA(cudaMalloc(&h->d_dinv, (size_t)S.n_inv * 4096 * sizeof(float)));
            h->g_factor[1].reset();
            h->g_solve.clear();
        }
        if (!h->d_hg)
        {
            // FP64 LU slots for the high-growth fallback of pivots of at most kGrowthSmallRows rows
            std::vector<int64_t> off(S.n, -1);
            int64_t total = 0;
            for (int64_t k = 0; k < S.n; ++k)
                if (S.size[k] <= hyb::kGrowthSmallRows)
                {
                    off[k] = total;
                    total += (int64_t)S.size[k] * S.size[k];
                }
            HYB_CUDA(cudaMalloc(&h->d_hg, S.n * sizeof(int)));
            HYB_CUDA(cudaMalloc(&h->d_piv64, std::max<int64_t>(1, total) * sizeof(double)));
            HYB_CUDA(cudaMalloc(&h->d_g64_off, S.n * sizeof(int64_t)));
            HYB_CUDA(cudaMemcpy(h->d_g64_off, off.data(), S.n * sizeof(int64_t), cudaMemcpyHostToDevice));
            // slots for the FP64 LUs of high-growth pivots of the fused 33-64-row levels
            int64_t most = 0;
            for (int64_t l = 0; l < S.n_levels; ++l)
            {
                const Symbolic::LevelShape &sh = S.shape[l];
                if (fused_pivots(sh))
                    most = std::max(most, S.lvl_ptr[l + 1] - S.lvl_ptr[l]);
            }
            h->fused_half = std::max<int64_t>(1, most);
            HYB_CUDA(cudaMalloc(&h->d_piv64f, 2 * h->fused_half * 4096 * sizeof(double)));
            h->g_factor[1].reset();
        }
        if (h->umma && !h->d_ops && S.max_split_blocks > 0)
        {
            h->split_half = (size_t)S.max_split_blocks * hyb::kSplitBytes;
            h->tgt_half = (size_t)std::max<int64_t>(1, S.max_tc_targets);
            HYB_CUDA(cudaMalloc(&h->d_ops, kOpsSlots * h->split_half + 2 * hyb::kSplitBytes));
            HYB_CUDA(cudaMemset(h->d_ops + kOpsSlots * h->split_half, 0, hyb::kSplitBytes));
            HYB_CUDA(cudaMalloc(&h->d_tgt, kOpsSlots * h->tgt_half * sizeof(int64_t)));
            h->g_factor[1].reset();
        }
        HYB_CUDA(cudaMemsetAsync(h->d_f32, 0, slab * sizeof(float), h->stream));
        if (h->update_kernel < 0 && needs_tuning<float>(h))
        {
            const int rc = tune_updates<float>(h, h->d_f32);
            if (rc != HYB_SUCCESS)
                return rc;
            h->g_factor[1].reset();
            HYB_CUDA(cudaMemsetAsync(h->d_f32, 0, slab * sizeof(float), h->stream));
        }
        h->factors_scaled = false;
        if (h->block_scaling)
        {
            if (!h->d_bscale)
            {
                HYB_CUDA(cudaMalloc(&h->d_bscale, S.n * sizeof(double)));
                HYB_CUDA(cudaMalloc(&h->d_dscale, std::max<int64_t>(1, S.dof_off[S.n]) * sizeof(double)));
            }
            hyb::k_block_scales<<<(unsigned)S.n, 128, 0, h->stream>>>(h->ds, h->d_a, h->d_bscale, h->d_dscale);
            h->last_launches += 1;
            h->factors_scaled = true;
        }
        hyb::k_scatter<float><<<sgrid, hyb::kThreads, 0, h->stream>>>(h->ds, h->d_a, h->d_f32, S.nnz_a(),
                                                                       h->factors_scaled ? h->d_bscale : nullptr);
        h->last_launches += 1;
        const int rc = run_graph(h, h->g_factor[1], [&](uint64_t &count) {
            h->free_profile_events();
            h->prof_precision = HYB_PRECISION_MIXED;
            return enqueue_factor<float>(h, h->d_f32, count);
        });
        if (rc != HYB_SUCCESS)
            return rc;
    }
    int st[hyb::ST_WORDS];
    HYB_CUDA(cudaMemcpyAsync(st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    if (st[hyb::ST_TIMEOUT])
    {
        g_cuda_error = "a device-side wait of the factorization ran out of its time limit";
        return HYB_DEVICE_TIMEOUT;
    }
    h->factored = precision;
    h->launches += h->last_launches;
    if (info)
    {
        info->n_levels = (uint64_t)S.n_levels;
        info->filled_blocks = (uint64_t)S.nnz_f();
        info->factor_values = (uint64_t)S.factor_values;
        info->factor_flops = S.factor_flops;
        info->zero_pivots = (uint64_t)st[hyb::ST_ZERO_PIVOTS];
        info->non_finite = (uint64_t)st[hyb::ST_NON_FINITE];
        info->first_bad_pivot = st[hyb::ST_FIRST_BAD] == INT_MAX ? -1 : st[hyb::ST_FIRST_BAD];
        info->growth_fp64 = (uint64_t)st[hyb::ST_GROWTH_FP64];
        info->growth_kept = (uint64_t)st[hyb::ST_GROWTH_KEPT];
    }
    return HYB_SUCCESS;
}

HYB_API int hyb_residual(hyb_system *h, const double *b, const double *x, double *r, uint64_t nrhs, int memory)
{
    if (check_handle(h) || !b || !x || !r || nrhs == 0 || nrhs > 1024)
        return HYB_INVALID_ARGUMENT;
    int rc = ensure_solve_buffers(h, (int64_t)nrhs);
    if (rc != HYB_SUCCESS)
        return rc;
    const int64_t dof = h->S.dof_off[h->S.n];
    const size_t bytes = dof * nrhs * sizeof(double);
    const cudaMemcpyKind in = memory == HYB_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind outk = memory == HYB_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    HYB_CUDA(cudaMemcpyAsync(h->d_b, b, bytes, in, h->stream));
    HYB_CUDA(cudaMemcpyAsync(h->d_x, x, bytes, in, h->stream));
    uint64_t launches = 0;
    enqueue_residual(h, h->d_b, h->d_x, h->d_r, (int)nrhs, launches);
    HYB_CUDA(cudaMemcpyAsync(r, h->d_r, bytes, outk, h->stream));
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    return HYB_SUCCESS;
}

HYB_API int hyb_solve(hyb_system *h, const double *b, double *x, uint64_t nrhs, int memory, double tol,
                      uint32_t max_iter, hyb_solve_info *info)
{
    if (check_handle(h) || !b || !x || nrhs == 0 || nrhs > 1024)
        return HYB_INVALID_ARGUMENT;
    if (h->factored < 0)
        return HYB_NOT_DECOMPOSED;
    const Symbolic &S = h->S;
    for (int64_t l = 0; l < S.n_levels; ++l)
        if ((int64_t)S.shape[l].max_piv * (int64_t)nrhs * 8 > solve_smem_cap())
            return HYB_TOO_LARGE;
    int rc = ensure_solve_buffers(h, (int64_t)nrhs);
    if (rc != HYB_SUCCESS)
        return rc;
    h->last_launches = 0;
    const int nr = (int)nrhs;
    const int64_t dof = S.dof_off[S.n];
    const int64_t len = dof * nr;
    const size_t bytes = len * sizeof(double);
    const cudaMemcpyKind in = memory == HYB_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind outk = memory == HYB_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const bool want_residual = info != nullptr && tol > 0;
    if (tol <= 0)
        tol = 1e-12;
    HYB_CUDA(cudaMemcpyAsync(h->d_b, b, bytes, in, h->stream));
    HYB_CUDA(cudaMemsetAsync(h->d_solve_status, 0, hyb::ST_WORDS * sizeof(int), h->stream));
    RefineResult res;
    if (h->factored == HYB_PRECISION_FP64 && !h->fp64_refine)
    {
        // the plain drop-in solve: one substitution with the FP64 factors
        HYB_CUDA(cudaMemcpyAsync(h->d_x, h->d_b, bytes, cudaMemcpyDeviceToDevice, h->stream));
        auto &slot = h->g_solve[{HYB_PRECISION_FP64, nr}];
        rc = substitute<double, double>(h, h->d_f64, h->d_x, h->d_scr64, nr, slot);
        if (rc != HYB_SUCCESS)
            return rc;
        if (want_residual)
        {
            uint64_t cnt = 0;
            std::vector<double> bn2, rn2;
            bool to = false;
            enqueue_residual(h, h->d_b, h->d_x, h->d_r, nr, cnt);
            if ((rc = column_sumsq(h, h->d_r, nr, h->d_norm, rn2, to, cnt)) != HYB_SUCCESS ||
                (rc = column_sumsq(h, h->d_b, nr, h->d_norm + nr, bn2, to, cnt)) != HYB_SUCCESS)
                return rc;
            res.relres = max_relative(rn2, bn2);
            if (!h->seg_off.empty())
            {
                h->seg_first.assign(bn2.size(), UINT32_MAX);
                h->seg_relres.assign(bn2.size(), -1.0);
                record_segments(h, rn2, bn2, tol, 0);
            }
            h->last_launches += cnt;
        }
    }
    else
    {
        uint64_t cnt = 0;
        rc = refine(h, nr, tol, max_iter, res, cnt);
        h->last_launches += cnt;
        if (rc != HYB_SUCCESS)
            return rc;
    }
    HYB_CUDA(cudaGetLastError());
    HYB_CUDA(cudaMemcpyAsync(x, h->d_x, bytes, outk, h->stream));
    int sst[hyb::ST_WORDS];
    HYB_CUDA(cudaMemcpyAsync(sst, h->d_solve_status, sizeof(sst), cudaMemcpyDeviceToHost, h->stream));
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    if (sst[hyb::ST_TIMEOUT])
    {
        g_cuda_error = "a wait of the dataflow solve ran out of its time limit";
        return HYB_DEVICE_TIMEOUT;
    }
    h->launches += h->last_launches;
    if (info)
    {
        info->iterations = res.iters;
        info->relative_residual = res.relres;
        info->krylov_iterations = res.krylov;
    }
    return res.status;
}

HYB_API int hyb_solve_transpose(hyb_system *h, const double *b, double *x, uint64_t nrhs, int memory)
{
    if (check_handle(h) || !b || !x || nrhs == 0 || nrhs > 1024)
        return HYB_INVALID_ARGUMENT;
    if (h->factored != HYB_PRECISION_FP64 || !h->d_f64)
        return HYB_NOT_DECOMPOSED;
    const Symbolic &S = h->S;
    for (int64_t l = 0; l < S.n_levels; ++l)
        if ((int64_t)S.shape[l].max_piv * (int64_t)nrhs * 8 > solve_smem_cap())
            return HYB_TOO_LARGE;
    int rc;
    if ((rc = ensure_trans(h)) != HYB_SUCCESS || (rc = ensure_solve_buffers(h, (int64_t)nrhs)) != HYB_SUCCESS ||
        (rc = ensure_trans_scratch(h, (int64_t)nrhs)) != HYB_SUCCESS)
        return rc;
    HYB_CUDA(allow_smem(hyb::k_bwdT_stage<double, double>, smem_optin()));
    const size_t bytes = S.dof_off[S.n] * nrhs * sizeof(double);
    const cudaMemcpyKind in = memory == HYB_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind outk = memory == HYB_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    HYB_CUDA(cudaMemcpyAsync(h->d_x, b, bytes, in, h->stream));
    h->last_launches = 0;
    const int nr = (int)nrhs;
    rc = run_graph(h, h->g_solveT[nr], [&](uint64_t &c) { return enqueue_solve_transpose(h, h->d_x, h->d_tscr, nr, c); });
    if (rc != HYB_SUCCESS)
        return rc;
    HYB_CUDA(cudaMemcpyAsync(x, h->d_x, bytes, outk, h->stream));
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    h->launches += h->last_launches;
    return HYB_SUCCESS;
}

HYB_API int hyb_condition_estimate(hyb_system *h, hyb_condition *out)
{
    if (check_handle(h) || !out)
        return HYB_INVALID_ARGUMENT;
    if (h->factored != HYB_PRECISION_FP64 || !h->d_f64)
        return HYB_NOT_DECOMPOSED;
    const Symbolic &S = h->S;
    int rc;
    if ((rc = ensure_trans(h)) != HYB_SUCCESS || (rc = ensure_solve_buffers(h, 1)) != HYB_SUCCESS ||
        (rc = ensure_trans_scratch(h, 1)) != HYB_SUCCESS)
        return rc;
    HYB_CUDA(allow_smem(hyb::k_bwdT_stage<double, double>, smem_optin()));
    const int64_t n = S.dof_off[S.n];
    HYB_CUDA(cudaMemsetAsync(h->d_solve_status, 0, hyb::ST_WORDS * sizeof(int), h->stream));
    if (!h->d_colsum)
        HYB_CUDA(cudaMalloc(&h->d_colsum, std::max<int64_t>(1, n) * sizeof(double)));
    hyb::k_col_abs_sums<<<(unsigned)S.n, hyb::kThreads, 0, h->stream>>>(h->ds, h->dt, h->d_a, h->d_colsum);
    HYB_CUDA(cudaGetLastError());
    std::vector<double> v(n), y(n), z(n);
    std::vector<int> sgn(n);
    HYB_CUDA(cudaMemcpyAsync(v.data(), h->d_colsum, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    double norm1 = 0;
    for (double c : v)
        norm1 = std::max(norm1, c);
    // ||A^{-1}||_1 by Hager's method with Higham's refinements (Higham, ACM TOMS 14 (1988),
    // Algorithm 4.1): the 1-norm of A^{-1} is the maximum of ||A^{-1} x||_1 over the unit
    // vectors e_j; the gradient step z = A^{-T} sign(A^{-1} x) points at the next e_j to
    // try, and a final alternating test vector guards against unlucky cases.
    uint32_t solves = 0;
    auto with_a = [&](const std::vector<double> &in, std::vector<double> &o) {
        ++solves;
        return solve_host_once(h, in.data(), o.data(), false);
    };
    auto with_at = [&](const std::vector<double> &in, std::vector<double> &o) {
        ++solves;
        return solve_host_once(h, in.data(), o.data(), true);
    };
    auto norm_1 = [](const std::vector<double> &a) {
        double t = 0;
        for (double e : a)
            t += std::fabs(e);
        return t;
    };
    auto argmax_abs = [](const std::vector<double> &a) {
        size_t j = 0;
        for (size_t i = 1; i < a.size(); ++i)
            if (std::fabs(a[i]) > std::fabs(a[j]))
                j = i;
        return j;
    };
    std::fill(v.begin(), v.end(), 1.0 / (double)n);
    if ((rc = with_a(v, y)) != HYB_SUCCESS)
        return rc;
    double est = norm_1(y);
    if (n > 1)
    {
        for (int64_t i = 0; i < n; ++i)
        {
            sgn[i] = y[i] >= 0 ? 1 : -1;
            v[i] = sgn[i];
        }
        if ((rc = with_at(v, z)) != HYB_SUCCESS)
            return rc;
        size_t j = argmax_abs(z);
        for (int iter = 2;; ++iter)
        {
            std::fill(v.begin(), v.end(), 0.0);
            v[j] = 1.0;
            if ((rc = with_a(v, y)) != HYB_SUCCESS)
                return rc;
            const double old = est;
            est = norm_1(y);
            bool repeated = true;
            for (int64_t i = 0; i < n && repeated; ++i)
                repeated = (y[i] >= 0 ? 1 : -1) == sgn[i];
            if (repeated || est <= old) // converged, or no longer increasing
            {
                est = std::max(est, old);
                break;
            }
            for (int64_t i = 0; i < n; ++i)
            {
                sgn[i] = y[i] >= 0 ? 1 : -1;
                v[i] = sgn[i];
            }
            if ((rc = with_at(v, z)) != HYB_SUCCESS)
                return rc;
            const size_t jlast = j;
            j = argmax_abs(z);
            if (z[jlast] == std::fabs(z[j]) || iter >= 5)
                break;
        }
        // alternating test vector x_i = (-1)^i (1 + i / (n - 1))
        for (int64_t i = 0; i < n; ++i)
            v[i] = (i % 2 ? -1.0 : 1.0) * (1.0 + (double)i / (double)(n - 1));
        if ((rc = with_a(v, y)) != HYB_SUCCESS)
            return rc;
        est = std::max(est, 2.0 * norm_1(y) / (3.0 * (double)n));
    }
    out->norm1 = norm1;
    out->inv_norm1 = est;
    out->kappa1 = norm1 * est;
    out->solves = solves;
    return HYB_SUCCESS;
}

HYB_API int hyb_row_count(const hyb_system *h, uint64_t row, uint64_t *count)
{
    if (check_handle(h) || row >= (uint64_t)h->S.n || !count)
        return HYB_INVALID_ARGUMENT;
    if (h->factored >= 0)
        *count = (uint64_t)(h->S.row_ptr[row + 1] - h->S.row_ptr[row]);
    else
        *count = (uint64_t)(h->S.a_row_ptr[row + 1] - h->S.a_row_ptr[row]);
    return HYB_SUCCESS;
}

HYB_API int hyb_row_cols(const hyb_system *h, uint64_t row, uint64_t *cols)
{
    if (check_handle(h) || row >= (uint64_t)h->S.n || !cols)
        return HYB_INVALID_ARGUMENT;
    const bool f = h->factored >= 0;
    const int64_t b = f ? h->S.row_ptr[row] : h->S.a_row_ptr[row];
    const int64_t e = f ? h->S.row_ptr[row + 1] : h->S.a_row_ptr[row + 1];
    const int32_t *src = f ? h->S.cols.data() : h->S.a_cols.data();
    for (int64_t j = b; j < e; ++j)
        cols[j - b] = (uint64_t)src[j];
    return HYB_SUCCESS;
}

HYB_API int hyb_get_block(const hyb_system *h, uint64_t row, uint64_t col, double *out)
{
    if (check_handle(h) || row >= (uint64_t)h->S.n || col >= (uint64_t)h->S.n || !out)
        return HYB_INVALID_ARGUMENT;
    const Symbolic &S = h->S;
    const int64_t cnt = (int64_t)S.size[row] * S.size[col];
    if (h->factored < 0)
    {
        const int32_t *b = S.a_cols.data() + S.a_row_ptr[row];
        const int32_t *e = S.a_cols.data() + S.a_row_ptr[row + 1];
        const int32_t *p = std::lower_bound(b, e, (int32_t)col);
        if (p == e || *p != (int32_t)col)
            return HYB_BLOCK_NOT_IN_SYSTEM;
        const int64_t j = p - S.a_cols.data();
        HYB_CUDA(cudaMemcpyAsync(out, h->d_a + S.a_val_off[j], cnt * sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
        HYB_CUDA(cudaStreamSynchronize(h->stream));
        return HYB_SUCCESS;
    }
    const int64_t j = hyb::find_block(S, (int64_t)row, (int64_t)col);
    if (j < 0)
        return HYB_BLOCK_NOT_IN_SYSTEM;
    if (h->factored == HYB_PRECISION_FP64)
    {
        HYB_CUDA(cudaMemcpyAsync(out, h->d_f64 + S.blk_off[j], cnt * sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
        HYB_CUDA(cudaStreamSynchronize(h->stream));
    }
    else
    {
        std::vector<float> tmp(cnt);
        HYB_CUDA(cudaMemcpyAsync(tmp.data(), h->d_f32 + S.blk_off[j], cnt * sizeof(float), cudaMemcpyDeviceToHost,
                                 h->stream));
        HYB_CUDA(cudaStreamSynchronize(h->stream));
        for (int64_t i = 0; i < cnt; ++i)
            out[i] = tmp[i];
    }
    return HYB_SUCCESS;
}

HYB_API int hyb_operations(const hyb_system *h, uint64_t *nops, int64_t *ops)
{
    if (check_handle(h) || !nops)
        return HYB_INVALID_ARGUMENT;
    if (h->factored < 0)
        return HYB_NOT_DECOMPOSED;
    try
    {
        std::vector<int64_t> v;
        hyb::symbolic_operations(h->S, v);
        *nops = v.size() / 2;
        if (ops)
            std::memcpy(ops, v.data(), v.size() * sizeof(int64_t));
    }
    catch (const std::bad_alloc &)
    {
        return HYB_FAILED_ALLOC;
    }
    return HYB_SUCCESS;
}

HYB_API uint64_t hyb_last_launch_count(const hyb_system *h)
{
    return h ? h->last_launches : 0;
}

HYB_API int hyb_profile_enable(hyb_system *h, int stride)
{
    if (check_handle(h) || stride < 0)
        return HYB_INVALID_ARGUMENT;
    if (h->profile != stride)
    {
        h->profile = stride;
        // the factorization graphs are recaptured with (or without) the event nodes
        h->g_factor[0].reset();
        h->g_factor[1].reset();
        h->free_profile_events();
    }
    return HYB_SUCCESS;
}

HYB_API int hyb_profile_read(const hyb_system *h, hyb_kernel_profile *out)
{
    if (check_handle(h) || !out)
        return HYB_INVALID_ARGUMENT;
    *out = hyb_kernel_profile{};
    if (!h->profile || h->factored < 0 || h->factored != h->prof_precision)
        return HYB_NOT_DECOMPOSED;
    for (size_t i = 0; i < h->prof_levels.size(); ++i)
    {
        float ms = 0;
        const cudaError_t e = cudaEventElapsedTime(&ms, h->prof_ev[2 * i], h->prof_ev[2 * i + 1]);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            return cuda_fail(e, "cudaEventElapsedTime");
        }
        out->launches += 1;
        out->total_ms += ms;
        if (h->prof_pair[i])
        {
            const auto &ps = h->S.pair[h->prof_levels[i]];
            out->flops += ps.flops;
            out->c_elems += ps.c_elems;
            out->ab_elems += ps.ab_elems;
            out->pivots_timed += 2;
        }
        else
        {
            const auto &sh = h->S.shape[h->prof_levels[i]];
            out->flops += sh.upd_flops;
            out->c_elems += sh.upd_c_elems;
            out->ab_elems += sh.upd_ab_elems;
            out->pivots_timed += 1;
        }
    }
    out->levels = (uint64_t)h->prof_update_pivots;
    out->passes = (uint64_t)h->prof_update_levels;
    for (size_t i = 0; i < h->prof_piv_levels.size(); ++i)
    {
        float ms = 0;
        const cudaError_t e = cudaEventElapsedTime(&ms, h->prof_piv_ev[2 * i], h->prof_piv_ev[2 * i + 1]);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            return cuda_fail(e, "cudaEventElapsedTime");
        }
        out->pivot_ms += ms;
        out->pivot_units += 1;
        out->pivot_levels += h->prof_piv_levels[i];
    }
    return HYB_SUCCESS;
}

HYB_API int hyb_block_lu(uint64_t m, double *a, int memory)
{
    if (!a || m == 0 || m > 4096)
        return HYB_INVALID_ARGUMENT;
    if (!hyb_device_available())
        return HYB_NO_DEVICE;
    const size_t bytes = m * m * sizeof(double);
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    char *ws = nullptr;
    int rc = workspace(bytes + 256, &ws);
    if (rc != HYB_SUCCESS)
        return rc;
    int *st = reinterpret_cast<int *>(ws);
    double *d = a;
    if (memory != HYB_MEMORY_DEVICE)
    {
        d = reinterpret_cast<double *>(ws + 256);
        HYB_CUDA(cudaMemcpy(d, a, bytes, cudaMemcpyHostToDevice));
    }
    k_status_init<<<1, 32>>>(st);
    HYB_CUDA(allow_smem(hyb::k_dense_lu, smem_optin()));
    if ((int)bytes <= smem_optin())
        hyb::k_dense_lu<<<1, hyb::kThreads, bytes>>>(d, (int)m, st);
    else
        hyb::k_dense_lu_global<<<1, hyb::kThreads>>>(d, (int)m, st);
    HYB_CUDA(cudaGetLastError());
    if (memory != HYB_MEMORY_DEVICE)
        HYB_CUDA(cudaMemcpy(a, d, bytes, cudaMemcpyDeviceToHost));
    HYB_CUDA(cudaDeviceSynchronize());
    return HYB_SUCCESS;
}

HYB_API int hyb_block_lu_solve(uint64_t m, const double *lu, uint64_t ncols, const double *b, double *out,
                               int memory)
{
    if (!lu || !b || !out || m == 0 || ncols == 0 || m > 4096)
        return HYB_INVALID_ARGUMENT;
    if (memory == HYB_MEMORY_DEVICE && b != out)
        HYB_CUDA(cudaMemcpy(out, b, m * ncols * sizeof(double), cudaMemcpyDeviceToDevice));
    if (memory != HYB_MEMORY_DEVICE && b != out)
        std::memcpy(out, b, m * ncols * sizeof(double));
    double *const bs[1] = {out};
    return hyb_block_lu_solve_batched(m, lu, 1, &ncols, bs, memory);
}

HYB_API int hyb_block_lu_solve_batched(uint64_t m, const double *lu, uint64_t count, const uint64_t *n,
                                       double *const *b, int memory)
{
    if (!lu || m == 0 || m > 4096 || (count && (!n || !b)))
        return HYB_INVALID_ARGUMENT;
    for (uint64_t i = 0; i < count; ++i)
        if (!b[i] || n[i] == 0 || n[i] > (1u << 20))
            return HYB_INVALID_ARGUMENT;
    if (!hyb_device_available())
        return HYB_NO_DEVICE;
    if (count == 0)
        return HYB_SUCCESS;
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    const size_t lu_bytes = m * m * sizeof(double);
    std::vector<size_t> off(count + 1, 0);
    for (uint64_t i = 0; i < count; ++i)
        off[i + 1] = off[i] + (m * n[i] * sizeof(double) + 255) / 256 * 256;
    const double *dlu = lu;
    char *ws = nullptr;
    if (memory != HYB_MEMORY_DEVICE)
    {
        int rc = workspace((lu_bytes + 255) / 256 * 256 + off[count], &ws);
        if (rc != HYB_SUCCESS)
            return rc;
        // one staging buffer on the host, one copy in and one out
        std::vector<char> host((lu_bytes + 255) / 256 * 256 + off[count]);
        std::memcpy(host.data(), lu, lu_bytes);
        char *hb = host.data() + (lu_bytes + 255) / 256 * 256;
        for (uint64_t i = 0; i < count; ++i)
            std::memcpy(hb + off[i], b[i], m * n[i] * sizeof(double));
        HYB_CUDA(cudaMemcpy(ws, host.data(), host.size(), cudaMemcpyHostToDevice));
        dlu = reinterpret_cast<const double *>(ws);
        char *db = ws + (lu_bytes + 255) / 256 * 256;
        for (uint64_t i = 0; i < count; ++i)
            hyb::k_dense_lu_solve<<<(unsigned)((n[i] + hyb::kTile - 1) / hyb::kTile), hyb::kThreads>>>(
                dlu, (int)m, reinterpret_cast<double *>(db + off[i]), (int)n[i]);
        HYB_CUDA(cudaGetLastError());
        HYB_CUDA(cudaMemcpy(hb, db, off[count], cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < count; ++i)
            std::memcpy(b[i], hb + off[i], m * n[i] * sizeof(double));
        return HYB_SUCCESS;
    }
    for (uint64_t i = 0; i < count; ++i)
        hyb::k_dense_lu_solve<<<(unsigned)((n[i] + hyb::kTile - 1) / hyb::kTile), hyb::kThreads>>>(dlu, (int)m, b[i],
                                                                                                 (int)n[i]);
    HYB_CUDA(cudaGetLastError());
    HYB_CUDA(cudaDeviceSynchronize());
    return HYB_SUCCESS;
}

HYB_API int hyb_block_gemm(uint64_t m, uint64_t k, uint64_t n, const double *a, const double *b, double *c,
                           int subtract, int memory)
{
    if (!b || !c)
        return HYB_INVALID_ARGUMENT;
    const double *const bs[1] = {b};
    double *const cs[1] = {c};
    return hyb_block_gemm_batched(1, m, k, &n, a, bs, cs, subtract, memory);
}

HYB_API int hyb_block_gemm_batched(uint64_t count, uint64_t m, uint64_t k, const uint64_t *n, const double *a,
                                   const double *const *b, double *const *c, int subtract, int memory)
{
    if (!a || m == 0 || m > (1u << 20) || k > (1u << 20) || (count && (!n || !b || !c)))
        return HYB_INVALID_ARGUMENT;
    for (uint64_t i = 0; i < count; ++i)
        if (!b[i] || !c[i] || n[i] == 0 || n[i] > (1u << 20))
            return HYB_INVALID_ARGUMENT;
    if (!hyb_device_available())
        return HYB_NO_DEVICE;
    if (count == 0)
        return HYB_SUCCESS;
    auto launch = [&](const double *da, const double *db, double *dc, uint64_t ni) {
        const dim3 grid((unsigned)((ni + hyb::kTile - 1) / hyb::kTile), (unsigned)((m + hyb::kTile - 1) / hyb::kTile));
        hyb::k_dense_gemm<<<grid, hyb::kThreads>>>(da, db, dc, (int)m, (int)k, (int)ni, subtract);
    };
    if (memory == HYB_MEMORY_DEVICE)
    {
        for (uint64_t i = 0; i < count; ++i)
            launch(a, b[i], c[i], n[i]);
        HYB_CUDA(cudaGetLastError());
        HYB_CUDA(cudaDeviceSynchronize());
        return HYB_SUCCESS;
    }
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    auto pad = [](size_t x) { return (x + 255) / 256 * 256; };
    // workspace: a, then every b, then every c (each 256-byte aligned, 8 bytes of slack for
    // the tile loader's vector reads past a row's end)
    const size_t a_bytes = pad(m * k * sizeof(double) + 8);
    std::vector<size_t> boff(count + 1, 0), coff(count + 1, 0);
    for (uint64_t i = 0; i < count; ++i)
    {
        boff[i + 1] = boff[i] + pad(k * n[i] * sizeof(double) + 8);
        coff[i + 1] = coff[i] + pad(m * n[i] * sizeof(double));
    }
    const size_t in_bytes = a_bytes + boff[count] + (subtract ? coff[count] : 0);
    char *ws = nullptr;
    int rc = workspace(a_bytes + boff[count] + coff[count], &ws);
    if (rc != HYB_SUCCESS)
        return rc;
    std::vector<char> host(a_bytes + boff[count] + coff[count], 0);
    std::memcpy(host.data(), a, m * k * sizeof(double));
    for (uint64_t i = 0; i < count; ++i)
    {
        std::memcpy(host.data() + a_bytes + boff[i], b[i], k * n[i] * sizeof(double));
        if (subtract)
            std::memcpy(host.data() + a_bytes + boff[count] + coff[i], c[i], m * n[i] * sizeof(double));
    }
    HYB_CUDA(cudaMemcpy(ws, host.data(), in_bytes, cudaMemcpyHostToDevice));
    char *dc = ws + a_bytes + boff[count];
    for (uint64_t i = 0; i < count; ++i)
        launch(reinterpret_cast<const double *>(ws), reinterpret_cast<const double *>(ws + a_bytes + boff[i]),
               reinterpret_cast<double *>(dc + coff[i]), n[i]);
    HYB_CUDA(cudaGetLastError());
    HYB_CUDA(cudaMemcpy(host.data(), dc, coff[count], cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < count; ++i)
        std::memcpy(c[i], host.data() + coff[i], m * n[i] * sizeof(double));
    return HYB_SUCCESS;
}

HYB_API int hyb_system_add_blocks(hyb_system *h, uint64_t count, const uint64_t *rows, const uint64_t *cols,
                                  const double *values, int memory)
{
    if (check_handle(h) || (count && (!rows || !cols || !values)))
        return HYB_INVALID_ARGUMENT;
    if (count == 0)
        return HYB_SUCCESS;
    const Symbolic &S = h->S;
    // every input block's original-pattern index, checked before anything is added
    std::vector<int64_t> tgt_of(count), in_off(count + 1, 0);
    for (uint64_t i = 0; i < count; ++i)
    {
        if (rows[i] >= (uint64_t)S.n || cols[i] >= (uint64_t)S.n)
            return HYB_INVALID_ARGUMENT;
        const int32_t *b = S.a_cols.data() + S.a_row_ptr[rows[i]];
        const int32_t *e = S.a_cols.data() + S.a_row_ptr[rows[i] + 1];
        const int32_t *q = std::lower_bound(b, e, (int32_t)cols[i]);
        if (q == e || *q != (int32_t)cols[i])
            return HYB_BLOCK_NOT_IN_SYSTEM;
        tgt_of[i] = q - S.a_cols.data();
        in_off[i + 1] = in_off[i] + (int64_t)S.size[rows[i]] * S.size[cols[i]];
    }
    // input blocks grouped by target, each group in input order
    std::vector<int64_t> order(count);
    for (uint64_t i = 0; i < count; ++i)
        order[i] = (int64_t)i;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return tgt_of[x] < tgt_of[y]; });
    std::vector<int64_t> tgt, grp{0};
    for (uint64_t q = 0; q < count; ++q)
        if (q + 1 == count || tgt_of[order[q + 1]] != tgt_of[order[q]])
        {
            tgt.push_back(tgt_of[order[q]]);
            grp.push_back((int64_t)q + 1);
        }
    const size_t idx_bytes = (in_off.size() + order.size() + tgt.size() + grp.size()) * sizeof(int64_t);
    const size_t val_bytes = memory == HYB_MEMORY_DEVICE ? 0 : (size_t)in_off[count] * sizeof(double);
    DevBuf buf;
    HYB_CUDA(cudaMalloc(&buf.p, idx_bytes + val_bytes));
    int64_t *d_in = static_cast<int64_t *>(buf.p), *d_order = d_in + in_off.size(), *d_tgt = d_order + order.size(),
            *d_grp = d_tgt + tgt.size();
    std::vector<int64_t> packed;
    packed.reserve(idx_bytes / sizeof(int64_t));
    for (const auto *v : {&in_off, &order, &tgt, &grp})
        packed.insert(packed.end(), v->begin(), v->end());
    HYB_CUDA(cudaMemcpyAsync(d_in, packed.data(), idx_bytes, cudaMemcpyHostToDevice, h->stream));
    const double *vin = values;
    if (memory != HYB_MEMORY_DEVICE)
    {
        double *dv = reinterpret_cast<double *>(reinterpret_cast<char *>(buf.p) + idx_bytes);
        HYB_CUDA(cudaMemcpyAsync(dv, values, val_bytes, cudaMemcpyHostToDevice, h->stream));
        vin = dv;
    }
    hyb::k_add_blocks<<<(unsigned)tgt.size(), hyb::kThreads, 0, h->stream>>>(h->ds, h->d_a, vin, d_in, d_order, d_tgt,
                                                                             d_grp);
    HYB_CUDA(cudaGetLastError());
    HYB_CUDA(cudaStreamSynchronize(h->stream)); // the staging buffer is freed on return
    h->factored = -1;
    return HYB_SUCCESS;
}

} // extern "C"

// ------------------------------------------------------------------------------------
// Allocation-free FP64 solve (hyb_solve_fp64_noalloc).
//
// The per-stage partial block products of the substitution go to this fixed array
// instead of buffers the handle allocates. In host code `g_noalloc_scratch` only names
// the symbol; its device address is looked up once per device with cudaGetSymbolAddress.
// The partials are written before they are read in every stage, so the contents a previous
// call left need no clearing.
static __device__ __align__(256) double g_noalloc_scratch[HYB_NOALLOC_SCRATCH_DOUBLES];

namespace
{
constexpr int kMaxDevices = 64;
std::once_flag g_noalloc_once[kMaxDevices];
double *g_noalloc_ptr[kMaxDevices] = {};
cudaError_t g_noalloc_err[kMaxDevices] = {};

// Device address of the scratch array on `device`, which must be current: looked up once
// per device (concurrent first calls wait for the one lookup).
int noalloc_scratch(int device, double **out)
{
    if (device < 0 || device >= kMaxDevices)
        return HYB_INVALID_ARGUMENT;
    std::call_once(g_noalloc_once[device], [device]() {
        void *p = nullptr;
        g_noalloc_err[device] = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        g_noalloc_ptr[device] = static_cast<double *>(p);
    });
    if (g_noalloc_err[device] != cudaSuccess)
        return cuda_fail(g_noalloc_err[device], "cudaGetSymbolAddress(g_noalloc_scratch)");
    *out = g_noalloc_ptr[device];
    return HYB_SUCCESS;
}
} // namespace

extern "C" HYB_API int hyb_solve_fp64_noalloc(hyb_system *h, const double *b, double *x, uint64_t nrhs)
{
    if (check_handle(h) || !b || !x || nrhs == 0 || nrhs > 1024)
        return HYB_INVALID_ARGUMENT;
    if (h->factored != HYB_PRECISION_FP64 || !h->d_f64)
        return HYB_NOT_DECOMPOSED;
    const Symbolic &S = h->S;
    const int64_t need = std::max(S.max_fwd_scratch_rows, S.max_bwd_scratch_rows) * (int64_t)nrhs;
    if (need > (int64_t)HYB_NOALLOC_SCRATCH_DOUBLES)
    {
        g_cuda_error = "solve scratch of " + std::to_string(need) + " doubles exceeds the fixed array of " +
                       std::to_string(HYB_NOALLOC_SCRATCH_DOUBLES);
        return HYB_TOO_LARGE;
    }
    for (int64_t l = 0; l < S.n_levels; ++l)
        if ((int64_t)S.shape[l].max_piv * (int64_t)nrhs * 8 > solve_smem_cap())
            return HYB_TOO_LARGE;
    int dev = 0;
    HYB_CUDA(cudaGetDevice(&dev));
    if (dev != h->device)
        return HYB_INVALID_ARGUMENT;
    double *scratch = nullptr;
    int rc = noalloc_scratch(dev, &scratch);
    if (rc != HYB_SUCCESS)
        return rc;
    const int64_t dof = S.dof_off[S.n];
    const uintptr_t xb = reinterpret_cast<uintptr_t>(x), bb = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = (uintptr_t)dof * nrhs * sizeof(double);
    if (x != b && xb < bb + len && bb < xb + len)
        return HYB_INVALID_ARGUMENT; // overlapping but not identical: the copy below would be undefined
    if (x != b)
        HYB_CUDA(cudaMemcpyAsync(x, b, len, cudaMemcpyDeviceToDevice, h->stream));
    uint64_t launches = 0;
    rc = enqueue_solve<double, double>(h, h->d_f64, x, scratch, (int)nrhs, launches);
    if (rc != HYB_SUCCESS)
        return rc;
    HYB_CUDA(cudaStreamSynchronize(h->stream));
    h->last_launches = launches;
    return HYB_SUCCESS;
}
