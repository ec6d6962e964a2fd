// qs_tile_tmem.cu - tiled fused passes with the tile held in tensor memory
// (complex64).  Layout and rationale: qs_tile_tmem.cuh.
//
// One CTA per SM with four lane groups of 128 threads (4 warps); each group
// owns a 32 KB staging buffer, an mbarrier, a named barrier and 128 TMEM
// columns (two 64-column regions that alternate between a block's A operand
// - BF16 hi in 32 columns, lo in 32 - and its FP32 accumulator).  A group
// walks tiles  blockIdx.x * 4 + group  in steps of  gridDim.x * 4;  per tile:
//   1. wait for the tile's copies (issued one tile earlier) and gather each
//      thread's block-0 row from the swizzled staging buffer;
//   2. split the row into BF16 hi/lo and write it to the group's TMEM lanes
//      (tcgen05.st); barrier; one thread issues the block's 12 MMAs
//      (kind::f16, A from TMEM, B = the block matrix in shared memory,
//      D = x_hi R_hi + x_hi R_lo + x_lo R_hi in the other region) and commits
//      to the group's mbarrier (a one-block pass issues the next tile's
//      copies now);
//   3. per block: wait, load the row's 64 results (tcgen05.ld); before the
//      next block write them through the staging buffer (free since the
//      gather) and read the thread's row of the next block, split, write it as
//      the next A and issue the next MMAs - after the last exchange every
//      thread issues its copies of the next tile; after the last block store
//      the row to HBM (in place, or at the positions of a remapping pass's
//      StoreMap).
// The four groups' chains overlap each other on the SM.
//
// The previous pass's norm correction (a scalar) is folded into block 0's
// matrix when the CTA loads it; the input norm is summed on the plan's first
// pass only; every wait on an mbarrier is bounded (qs_tile::mbar_wait), and an
// expired wait is reported through the plan's error word.
#include <algorithm>
#include <cstring>

#include "qs_fused.h"
#include "qs_tile_core.cuh"
#include "qs_tile_tmem.cuh"
#include "qs_tile_tmem_dev.cuh"

using qs_tmem::TLayout;

// ------------------------------------------------------------------ host layout
int qs_tmem_layout_build(int n, const qs_tiled_desc *d, TLayout *L)
{
    memset(L, 0, sizeof(*L));
    const int nsub = d->nsub;
    if (nsub < 1 || nsub > qs_tmem::kMaxSub) return qs_fail(QS_ERR_ARG, "tiled pass: %d blocks", nsub);
    int local[64];
    for (int i = 0; i < 64; ++i) local[i] = -1;
    for (int t = 0; t < 12; ++t) {
        const int q = d->T[t];
        if (q < 0 || q >= n || (t && q <= d->T[t - 1]))
            return qs_fail(QS_ERR_ARG, "tiled pass: tile qubits must be ascending and in range");
        local[q] = t;
        L->tmask |= 1ull << q;
        L->tpos[t] = (int8_t)q;
    }
    if (d->T[0] != 0) return QS_ERR_UNSUPPORTED;       // 16-byte copies need tile bit 0 at position 0
    uint32_t qm[qs_tmem::kMaxSub] = {0, 0, 0};
    int mbit[qs_tmem::kMaxSub][12];
    for (int b = 0; b < nsub; ++b) {
        for (int t = 0; t < 12; ++t) mbit[b][t] = -1;
        for (int m = 0; m < 5; ++m) {
            const int q = d->qpos[b][m];
            const int t = (q >= 0 && q < n) ? local[q] : -1;
            if (t < 0 || ((qm[b] >> t) & 1))
                return qs_fail(QS_ERR_ARG, "tiled pass: block qubits must be distinct tile qubits");
            qm[b] |= 1u << t;
            mbit[b][t] = m;
        }
    }
    int WT[12];
    uint64_t wseen = 0;
    for (int t = 0; t < 12; ++t) {
        WT[t] = d->has_write ? d->wtile[t] : d->T[t];
        if (WT[t] < 0 || WT[t] >= n || ((wseen >> WT[t]) & 1))
            return qs_fail(QS_ERR_ARG, "tiled pass: write positions must be distinct and in range");
        wseen |= 1ull << WT[t];
    }
    const int last = nsub - 1;
    int z = -1;                                  // tile bit written at position 0
    for (int t = 0; t < 12; ++t)
        if (WT[t] == 0) z = t;

    // Each block's tile bits: 5 columns (register bits), 5 lanes, 2 warps.
    // Warps take the two non-column bits that matter least: for the last
    // block the highest write positions (its lanes then cover the lowest ones
    // and its stores coalesce), otherwise the highest tile bits; tile bit 0
    // stays a lane when it is not a column (an 8-byte gather's bank bit 0).
    // Lanes: tile bit 0 first, then ascending.  Registers: the bit written at
    // position 0 first in the last block (16-byte stores), tile bit 0 first in
    // block 0 (16-byte gathers), then ascending.
    int regs[qs_tmem::kMaxSub][5], lanes[qs_tmem::kMaxSub][5], warps[qs_tmem::kMaxSub][2];
    for (int b = 0; b < nsub; ++b) {
        int nonq[7], nn = 0;
        for (int t = 0; t < 12; ++t)
            if (!((qm[b] >> t) & 1)) nonq[nn++] = t;
        auto rank = [&](int t) { return (t == 0 ? -1000 : 0) + (b == last ? WT[t] : t); };
        std::stable_sort(nonq, nonq + 7, [&](int x, int y) { return rank(x) < rank(y); });
        warps[b][0] = nonq[5];
        warps[b][1] = nonq[6];
        std::sort(nonq, nonq + 5);                   // ascending, so tile bit 0 (if a lane) comes first
        for (int i = 0; i < 5; ++i) lanes[b][i] = nonq[i];
        int cols[5], nc = 0;
        for (int t = 0; t < 12; ++t)
            if ((qm[b] >> t) & 1) cols[nc++] = t;
        int head = -1;
        if (b == last && z >= 0 && ((qm[b] >> z) & 1)) head = z;
        else if (b == 0 && (qm[b] & 1u)) head = 0;
        int k = 0;
        if (head >= 0) regs[b][k++] = head;
        for (int c = 0; c < 5; ++c)
            if (cols[c] != head) regs[b][k++] = cols[c];
    }
    L->nsub = nsub;
    L->pair_in = regs[0][0] == 0;
    L->vec_out = WT[regs[last][0]] == 0;
    for (int b = 0; b < nsub; ++b)
        for (int p = 0; p < 5; ++p) L->mperm[b][p] = (int8_t)mbit[b][regs[b][p]];

    // staging swizzle: the lanes of one shared-memory phase of the gather
    // (lane bits 0..2 for 16-byte gathers, 0..3 for 8-byte ones) must read
    // distinct bank slots (stage-slot bits 1..3, and bit 0 for 8-byte reads);
    // tile bits >= 4 get the free ones through f
    uint16_t fbit[12] = {0};
    {
        const int phase = L->pair_in ? 3 : 4;
        uint32_t used = 0;
        for (int i = 0; i < phase; ++i)
            if (lanes[0][i] <= 3) used |= 1u << lanes[0][i];
        for (int i = 0; i < phase; ++i) {
            const int t = lanes[0][i];
            if (t <= 3) continue;
            for (int sb = 1; sb <= 3; ++sb)
                if (!((used >> sb) & 1)) { used |= 1u << sb; fbit[t] = (uint16_t)(1u << sb); break; }
        }
    }
    auto slot = [&](int t) { return (uint16_t)((1u << t) ^ fbit[t]); };
    for (int i = 0; i < 5; ++i) L->s_lane[i] = slot(lanes[0][i]);
    for (int v = 0; v < 2; ++v) L->s_warp[v] = slot(warps[0][v]);
    for (int j = 0; j < 32; ++j) {
        uint16_t sv = 0;
        for (int p = 0; p < 5; ++p)
            if ((j >> p) & 1) sv ^= slot(regs[0][p]);
        L->s_col[j] = sv;
    }

    // exchange swizzles: slot = index ^ g(index), g linear from tile bits >= 4
    // into slot bits 0..3, chosen so that the 16 lanes of a half warp hit 16
    // distinct 8-byte bank slots both when block b writes and when block b + 1
    // reads (their lane bits 0..3 must have independent bank vectors)
    for (int b = 0; b + 1 < nsub; ++b) {
        uint16_t g[12] = {0};
        const int *wl = lanes[b], *rl = lanes[b + 1];
        auto bank = [&](int t, const uint16_t *gg) { return (uint32_t)(t < 4 ? (1u << t) : gg[t]); };
        auto independent = [&](const int *ls, const uint16_t *gg) {
            for (uint32_t m = 1; m < 16; ++m) {
                uint32_t x = 0;
                for (int i = 0; i < 4; ++i)
                    if ((m >> i) & 1) x ^= bank(ls[i], gg);
                if (!x) return false;
            }
            return true;
        };
        int high[8], nh = 0;
        for (int i = 0; i < 4; ++i) {
            if (wl[i] >= 4 && std::find(high, high + nh, wl[i]) == high + nh) high[nh++] = wl[i];
            if (rl[i] >= 4 && std::find(high, high + nh, rl[i]) == high + nh) high[nh++] = rl[i];
        }
        uint32_t seed = 0x9e3779b9u;
        bool ok = false;
        for (int attempt = 0; attempt < 4096 && !ok; ++attempt) {
            for (int h = 0; h < nh; ++h) {
                seed = seed * 1664525u + 1013904223u;
                g[high[h]] = (uint16_t)(attempt == 0 ? (1u << (h & 3)) : 1u + (seed >> 28) % 15u);
            }
            ok = independent(wl, g) && independent(rl, g);
        }
        auto xs = [&](int t) { return (uint16_t)((1u << t) ^ g[t]); };
        for (int i = 0; i < 5; ++i) {
            L->xw_lane[b][i] = xs(lanes[b][i]);
            L->xr_lane[b][i] = xs(lanes[b + 1][i]);
        }
        for (int v = 0; v < 2; ++v) {
            L->xw_warp[b][v] = xs(warps[b][v]);
            L->xr_warp[b][v] = xs(warps[b + 1][v]);
        }
        for (int j = 0; j < 32; ++j) {
            uint16_t w = 0, rr = 0;
            for (int p = 0; p < 5; ++p)
                if ((j >> p) & 1) { w ^= xs(regs[b][p]); rr ^= xs(regs[b + 1][p]); }
            L->xw_col[b][j] = w;
            L->xr_col[b][j] = rr;
        }
    }
    for (int b = 0; b < 7; ++b) {
        L->g_bit[b] = 1ull << d->T[b + 1];
        L->cf_bit[b] = (uint16_t)(fbit[b + 1] >> 1);
    }
    for (int k = 0; k < 16; ++k) {
        uint64_t g = 0;
        uint16_t c = 0;
        for (int i = 0; i < 4; ++i)
            if ((k >> i) & 1) { g |= 1ull << d->T[8 + i]; c ^= (uint16_t)(fbit[8 + i] >> 1); }
        L->gk[k] = g;
        L->cf_k[k] = c;
    }
    for (int i = 0; i < 5; ++i) L->o_lane[i] = 1ull << WT[lanes[last][i]];
    for (int v = 0; v < 2; ++v) L->o_warp[v] = 1ull << WT[warps[last][v]];
    for (int j = 0; j < 32; ++j) {
        uint64_t o = 0;
        for (int p = 0; p < 5; ++p)
            if ((j >> p) & 1) o |= 1ull << WT[regs[last][p]];
        L->o_col[j] = o;
    }
    return QS_OK;
}

// ------------------------------------------------------------------ device
namespace {

using namespace qs_tile;
using namespace qs_tmem_dev;

constexpr int kGroups = 4;                       // lane groups (tiles in flight) per CTA
// TPR threads per tile row: 128 * TPR threads per group, each with 32 / TPR of
// its row's 32 columns (TPR = 2: two warps on each quarter of the TMEM lanes).
template <int TPR>
struct TShape {
    static constexpr int kGroupThreads = 128 * TPR;
    static constexpr int kCtaThreads = kGroups * kGroupThreads;
    static constexpr int kRegs = 32 / TPR;       // complex columns per thread
};
constexpr uint32_t kOffB = 0;                    // 3 blocks x (hi, lo) x 8 KB
constexpr uint32_t kOffStage = qs_tmem::kMaxSub * 2 * kB;
constexpr uint32_t kOffMisc = kOffStage + kGroups * kStage;
constexpr uint32_t kSmemUsed = kOffMisc + 64;
// Ask for more than half of the SM's shared memory, so that no other CTA that
// allocates tensor memory can share the SM (this one takes all 512 columns).
constexpr uint32_t kSmemBytes = kSmemUsed > 200 * 1024 ? kSmemUsed : 200 * 1024;
constexpr uint32_t kCols = 512;
static_assert(kSmemBytes + 1024 <= 228 * 1024, "one CTA per SM");
static_assert((kOffStage & 1023) == 0, "operands 1024-byte aligned");
static_assert(kGroups * 128 <= kCols, "TMEM columns per group");

struct TParams {
    TLayout L;
    StoreMap W;
    uint64_t tiles;
    const uint16_t *mat;         // nsub x [2][64][64] BF16 bits (hi, lo), the plan's column order
    int *err;
    int nparts;                  // norm partials per pass (>= gridDim.x; the tail is written as zeros)
    const double *norm0;
    const double *prev_out;
    double *in_parts;
    double *out_parts;
};

template <int TPR>
__global__ void __launch_bounds__(TShape<TPR>::kCtaThreads, 1) k_tile_tmem(const float *amp, float *out, TParams P)
{
    using S = TShape<TPR>;
    constexpr int kV = 64 / TPR;                     // floats per thread per row
    extern __shared__ __align__(1024) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = tid / S::kGroupThreads, ltid = tid % S::kGroupThreads, wq = (ltid >> 5) & 3;
    const int half = TPR == 2 ? ltid >> 7 : 0;       // which 16 of a row's 32 columns (TPR = 2)
    const int c0 = 16 * half;
    if (smem_u32(smem) & 1023u) {
        if (tid == 0) atomicExch(P.err, 2);
        return;
    }
    const TLayout &L = P.L;
    const uint32_t stage = smem_u32(smem + kOffStage + grp * kStage);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kOffMisc) + grp;
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + kOffMisc + 32);
    float *s_scale = reinterpret_cast<float *>(smem + kOffMisc + 36);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_holder)), "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (ltid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (warp == 1) {
        double n0 = 0, np = 0;
        if (P.norm0 && P.prev_out)
            for (int i = lane; i < P.nparts; i += 32) { n0 += P.norm0[i]; np += P.prev_out[i]; }
        for (int o = 16; o > 0; o >>= 1) {
            n0 += __shfl_xor_sync(0xffffffffu, n0, o);
            np += __shfl_xor_sync(0xffffffffu, np, o);
        }
        if (lane == 0) *s_scale = (P.norm0 && P.prev_out && np > 0) ? (float)sqrt(n0 / np) : 1.0f;
    }
    __syncthreads();
    load_b_perm(smem + kOffB, P.mat, L, *s_scale);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem_base = *tmem_holder;
    const uint32_t tgrp = tmem_base + (uint32_t)(grp * 128);          // the group's 128 columns
    const uint32_t tlane = tgrp + ((uint32_t)(wq * 32) << 16);        // this warp's 32 lanes
    const uint32_t mb = smem_u32(mbar);
    const int bar_id = 1 + grp;

    // per-thread parts of the gather, copy and store addresses
    uint32_t xrow = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i)
        if ((lane >> i) & 1) xrow ^= L.s_lane[i];
#pragma unroll
    for (int v = 0; v < 2; ++v)
        if ((wq >> v) & 1) xrow ^= L.s_warp[v];
    uint64_t orow = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i)
        if ((lane >> i) & 1) orow |= L.o_lane[i];
#pragma unroll
    for (int v = 0; v < 2; ++v)
        if ((wq >> v) & 1) orow |= L.o_warp[v];
    uint32_t xw0 = 0, xr0 = 0, xw1 = 0, xr1 = 0;       // the thread's exchange slots, transitions 0 and 1
#pragma unroll
    for (int i = 0; i < 5; ++i)
        if ((lane >> i) & 1) {
            xw0 ^= L.xw_lane[0][i]; xr0 ^= L.xr_lane[0][i];
            xw1 ^= L.xw_lane[1][i]; xr1 ^= L.xr_lane[1][i];
        }
#pragma unroll
    for (int v = 0; v < 2; ++v)
        if ((wq >> v) & 1) {
            xw0 ^= L.xw_warp[0][v]; xr0 ^= L.xr_warp[0][v];
            xw1 ^= L.xw_warp[1][v]; xr1 ^= L.xr_warp[1][v];
        }
    if (TPR == 2 && half) {                          // the thread's columns 16.. (every table is linear)
        xrow ^= L.s_col[16];
        orow |= L.o_col[16];
        xw0 ^= L.xw_col[0][16]; xr0 ^= L.xr_col[0][16];
        xw1 ^= L.xw_col[1][16]; xr1 ^= L.xr_col[1][16];
    }
    uint64_t g_t = 0;
    uint32_t cs_t = (uint32_t)ltid;                  // TPR = 2: bit 7 of ltid is bit 0 of k
#pragma unroll
    for (int b = 0; b < 7; ++b)
        if ((ltid >> b) & 1) { g_t |= L.g_bit[b]; cs_t ^= L.cf_bit[b]; }
    if (TPR == 2 && (ltid >> 7)) { g_t |= L.gk[1]; cs_t ^= L.cf_k[1]; }

    const bool want_in = P.in_parts != nullptr;
    uint32_t phase = 0;
    bool failed = false;
    double acc_in = 0, acc_out = 0;
    const uint64_t stride = (uint64_t)gridDim.x * kGroups;
    uint64_t tile = (uint64_t)blockIdx.x * kGroups + grp;
    const uint64_t step = tbase_of(stride, L);
    uint64_t tbase = tbase_of(tile, L);
    if (tile < P.tiles) copy_tile<TPR>(amp, tbase, L, stage, g_t, cs_t);
    for (; tile < P.tiles; tile += stride) {
        const uint64_t tnext = tile_base_advance(tbase, step, L.tmask);
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        group_bar<S::kGroupThreads>(bar_id);
        float y[kV];
        {
            // gather the thread's part of its block-0 row
            if (L.pair_in) {
#pragma unroll
                for (int j = 0; j < 16 / TPR; ++j) {
                    const uint32_t a = stage + ((xrow ^ L.s_col[2 * j]) << 3);
                    asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                                 : "=f"(y[4 * j]), "=f"(y[4 * j + 1]), "=f"(y[4 * j + 2]), "=f"(y[4 * j + 3])
                                 : "r"(a));
                }
            } else {
#pragma unroll
                for (int j = 0; j < 32 / TPR; ++j) {
                    const uint32_t a = stage + ((xrow ^ L.s_col[j]) << 3);
                    asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];" : "=f"(y[2 * j]), "=f"(y[2 * j + 1]) : "r"(a));
                }
            }
            if (want_in) acc_in += (double)sum_squares(y);
            split_store<TPR>(tlane, y, c0);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        group_bar<S::kGroupThreads>(bar_id);
        if (ltid == 0) issue_ts(tgrp + 64, tgrp, smem_u32(smem + kOffB), smem_u32(smem + kOffB + kB), mb);
        // a one-block pass needs the staging buffer no more: the next tile's copies
        if (L.nsub == 1 && tile + stride < P.tiles) copy_tile<TPR>(amp, tnext, L, stage, g_t, cs_t);

        for (int b = 0; b < L.nsub; ++b) {
            // every thread waits on the mbarrier itself (measured 2 % faster than
            // one poller per warp handing it on through the group barrier)
            const bool ok = mbar_wait(mb, phase);
            phase ^= 1;
            if (group_bar_or<S::kGroupThreads>(bar_id, !ok)) { failed = true; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t dreg = (b & 1) ? 0u : 64u;                    // this block's accumulator
#pragma unroll
            for (int q = 0; q < 2 / TPR; ++q) tmem_ld32(tlane + dreg + 2 * c0 + 32 * q, y + 32 * q);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (b + 1 < L.nsub) {
                exchange_through<TPR, S::kGroupThreads>(y, stage, b ? xw1 : xw0, b ? xr1 : xr0, L.xw_col[b], L.xr_col[b], bar_id);
                split_store<TPR>(tlane + dreg, y, c0);                   // the next block's A
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                group_bar<S::kGroupThreads>(bar_id);                                  // also: every exchange read is done
                if (ltid == 0)
                    issue_ts(tgrp + (dreg ^ 64u), tgrp + dreg, smem_u32(smem + kOffB + (2 * (b + 1)) * kB),
                             smem_u32(smem + kOffB + (2 * (b + 1) + 1) * kB), mb);
                // after the last exchange the staging buffer is free: the next tile's copies
                if (b + 2 == L.nsub && tile + stride < P.tiles) copy_tile<TPR>(amp, tnext, L, stage, g_t, cs_t);
            } else {
                const uint64_t obase = store_base(tile, tbase, P.W) | orow;
                if (L.vec_out) {
#pragma unroll
                    for (int j = 0; j < 16 / TPR; ++j)
                        *reinterpret_cast<float4 *>(out + 2 * (obase | L.o_col[2 * j])) =
                            make_float4(y[4 * j], y[4 * j + 1], y[4 * j + 2], y[4 * j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 32 / TPR; ++j)
                        *reinterpret_cast<float2 *>(out + 2 * (obase | L.o_col[j])) = make_float2(y[2 * j], y[2 * j + 1]);
                }
                acc_out += (double)sum_squares(y);                      // after the stores are issued
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        }
        if (failed) break;
        tbase = tnext;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    {
        double ai = acc_in, ao = acc_out;
        for (int o = 16; o > 0; o >>= 1) {
            ai += __shfl_xor_sync(0xffffffffu, ai, o);
            ao += __shfl_xor_sync(0xffffffffu, ao, o);
        }
        constexpr int kWarps = S::kCtaThreads / 32;
        double *red = reinterpret_cast<double *>(smem + kOffStage);      // group 0's staging buffer
        __syncthreads();                     // every copy of every group has landed
        if (lane == 0) { red[warp] = ai; red[kWarps + warp] = ao; }
        __syncthreads();
        if (tid == 0) {
            double a = 0, b = 0;
            for (int w = 0; w < kWarps; ++w) { a += red[w]; b += red[kWarps + w]; }
            if (P.in_parts) P.in_parts[blockIdx.x] = a;
            if (P.out_parts) P.out_parts[blockIdx.x] = b;
        }
        if (blockIdx.x == 0)                 // partials past this grid read as zero
            for (int i = (int)gridDim.x + tid; i < P.nparts; i += S::kCtaThreads) {
                if (P.in_parts) P.in_parts[i] = 0.0;
                if (P.out_parts) P.out_parts[i] = 0.0;
            }
    }
    if (failed) {
        if (ltid == 0) atomicExch(P.err, 1);
        mbar_wait(mb, phase ^ 1);            // bounded: the MMAs in flight, if any
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem_base), "r"(kCols));
    }
}

}  // namespace

int qs_tmem_grid(const qs_state *s)
{
    const uint64_t tiles = s->N >> 12, need = (tiles + kGroups - 1) / kGroups;
    return (int)(need < QS_SM_COUNT ? need : QS_SM_COUNT);
}

// Launch one tiled pass on k_tile_tmem.  QS_ERR_UNSUPPORTED (nothing
// launched, no error recorded) when the pass does not fit this kernel.
int qs_launch_tiled_tmem(qs_state *s, const qs_tiled_desc *d, int *err_dev)
{
    if (s->dtype != QS_C64 || s->n < 12) return QS_ERR_UNSUPPORTED;
    TParams P;
    memset(&P, 0, sizeof(P));
    int r = qs_tmem_layout_build(s->n, d, &P.L);
    if (r) return r;
    P.W.mode = d->has_write ? d->wmode : 0;
    P.W.ntb = s->n - 12;
    if (d->has_write && P.W.mode != 1 && P.W.mode != 2)
        return qs_fail(QS_ERR_ARG, "tiled pass: write mode %d", P.W.mode);
    if (P.W.mode == 2) {
        uint64_t seen = 0;
        for (int l = 0; l < 12; ++l) seen |= 1ull << d->wtile[l];
        for (int i = 0; i < P.W.ntb; ++i) {
            const int w = d->wpos[i];
            if (w < 0 || w >= s->n || ((seen >> w) & 1))
                return qs_fail(QS_ERR_ARG, "tiled pass: write positions must form a permutation");
            seen |= 1ull << w;
            P.W.wpos[i] = (int8_t)w;
        }
    } else if (P.W.mode == 1) {
        for (int l = 0; l < 12; ++l)
            if (d->wtile[l] >= 12) return qs_fail(QS_ERR_ARG, "tiled pass: contiguous writes need tile bits at 0..11");
    }
    P.tiles = s->N >> 12;
    P.mat = static_cast<const uint16_t *>(d->mat_dev);
    P.err = err_dev;
    P.nparts = qs_tiled_grid(s);
    P.norm0 = d->norm0;
    P.prev_out = d->prev_out;
    P.in_parts = d->in_parts;
    P.out_parts = d->out_parts;
    const float *in = static_cast<const float *>(d->amp_in ? d->amp_in : s->amp);
    float *out = static_cast<float *>(d->amp_out ? d->amp_out : s->amp);
    if ((d->amp_in != nullptr) != (d->amp_out != nullptr) || (d->amp_in && (const void *)in == (const void *)out))
        return qs_fail(QS_ERR_ARG, "tiled pass: set both buffers, and distinct, or neither");
    if (d->has_write && !d->amp_out)
        return qs_fail(QS_ERR_ARG, "tiled pass: remapped results need a separate output buffer");
    const unsigned grid = (unsigned)qs_tmem_grid(s);
    if (d->threads_per_row == 2) {
        QS_CUDA_TRY(cudaFuncSetAttribute(k_tile_tmem<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
        k_tile_tmem<2><<<grid, TShape<2>::kCtaThreads, kSmemBytes, s->stream>>>(in, out, P);
    } else {
        QS_CUDA_TRY(cudaFuncSetAttribute(k_tile_tmem<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
        k_tile_tmem<1><<<grid, TShape<1>::kCtaThreads, kSmemBytes, s->stream>>>(in, out, P);
    }
    QS_LAUNCH_CHECK("k_tile_tmem");
    return QS_OK;
}
