// qs_fused2.cu - tiled fused passes: up to three 5-qubit blocks per read and
// write of the state, on the tensor cores (complex64).
//
// A pass owns 12 tile qubits T (ascending; the lowest ones always included so
// that rows are runs of contiguous amplitudes).  The state splits into 2^(n-12)
// tiles of 4096 amplitudes that differ only in the T bits.  Each block b of
// the pass acts on 5 qubits Q_b within T; for it the tile is viewed as 128
// rows x 32 amplitudes: the row index is the 7 tile bits outside Q_b, the
// column index the 5 bits of Q_b.  One M=128, N=64, K=64 contraction per tile
// and block (split-BF16 x3, FP32 accumulation in TMEM, as in qs_fused.cu).
//
// Per tile, thread i of 128 owns row i and TMEM lane i (qs_tile_core.cuh):
//   1. its row of block 0 arrives by cp.async in a staging row of its own; it
//      reads it to registers and writes the BF16 hi/lo split into the
//      swizzled K-major A buffer (16-byte chunks);
//   2. for each block: one thread issues the 12 MMAs and commits to an
//      mbarrier; every thread waits, loads its 64 FP32 results from TMEM, and
//      either scatters them as BF16 hi/lo into the next block's A layout (one
//      XOR per result gives its offset there), or - after the last block -
//      stores them to HBM in place.
// A CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...; the global base
// of the next tile is one masked add away from the current one.
//
// Two shapes, chosen per pass by its number of blocks:
//   * up to 2 blocks: 64 KB of shared memory, three CTAs per SM.  The staging
//     rows live in the A region: the next tile's copies are issued as soon as
//     the last block's MMAs have finished reading A, and land while the
//     results go out to HBM;
//   * 3 blocks: 112 KB, two CTAs per SM, a separate staging area filled one
//     whole tile ahead.
// The extra resident CTA is what pays: each tile is a serial chain (copy,
// split, MMA, wait, scatter, MMA, wait, store) that one CTA cannot overlap.
// Norm tracking and bounded waits as in qs_fused.cu.
#include "qs_fused.h"
#include "qs_tile_core.cuh"

namespace {

using namespace qs_tile;

template <int SUB>
struct Shape {
    static constexpr bool kStageInA = SUB <= 2;
    static constexpr int kCtasPerSm = kStageInA ? 3 : 2;
    static constexpr uint32_t kOffA = 0;                          // A hi, A lo
    static constexpr uint32_t kOffB = 2 * kA;                     // B hi/lo per block
    static constexpr uint32_t kOffStage = kStageInA ? kOffA : kOffB + SUB * 2 * kB;
    static constexpr uint32_t kOffMisc = kOffB + SUB * 2 * kB + (kStageInA ? 0 : kStage);
    static constexpr uint32_t kSmemBytes = kOffMisc + 16;         // mbarrier (8), tmem address (4), scale (4)
    static_assert(kCtasPerSm * (kSmemBytes + 1024) <= 228 * 1024, "resident CTAs per SM");
    static_assert(!kStageInA || 2 * kA == kStage, "the A region holds one tile of staging rows");
};

struct TileParams {
    Layout L;
    uint64_t tiles;
    const uint16_t *mat;         // nsub x [2][64][64] BF16 bits (hi, lo) of R
    int *err;
    int nparts;                  // norm partials per pass (>= gridDim.x; the tail is written as zeros)
    const double *norm0;
    const double *prev_out;
    double *in_parts;
    double *out_parts;
};

template <int SUB>
__global__ void __launch_bounds__(kThreads, Shape<SUB>::kCtasPerSm) k_fused_tile(float *__restrict__ amp, TileParams P)
{
    using S = Shape<SUB>;
    extern __shared__ __align__(1024) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    if (smem_u32(smem) & 1023u) {             // swizzled operands need 1024-byte alignment
        if (tid == 0) atomicExch(P.err, 2);
        return;
    }
    const Layout &L = P.L;
    uint8_t *aHi = smem + S::kOffA, *aLo = smem + S::kOffA + kA;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + S::kOffMisc);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + S::kOffMisc + 8);
    float *s_scale = reinterpret_cast<float *>(smem + S::kOffMisc + 12);
    const uint32_t stage = smem_u32(smem + S::kOffStage);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_holder)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    load_b(smem + S::kOffB, P.mat, L.nsub);
    // scale undoing the previous pass's norm drift (fixed-order sums)
    if (warp == 1) {
        double n0 = 0, np = 0;
        if (P.norm0 && P.prev_out)
            for (int i = tid - 32; i < P.nparts; i += 32) { n0 += P.norm0[i]; np += P.prev_out[i]; }
        for (int o = 16; o > 0; o >>= 1) {
            n0 += __shfl_xor_sync(0xffffffffu, n0, o);
            np += __shfl_xor_sync(0xffffffffu, np, o);
        }
        if (tid == 32) *s_scale = (P.norm0 && P.prev_out && np > 0) ? (float)sqrt(n0 / np) : 1.0f;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_holder;
    const float scale = *s_scale;

    const int row = tid;
    uint64_t gC0 = 0, gCl = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b) {
        gC0 |= (uint64_t)((row >> b) & 1) << L.c0_glob[b];
        gCl |= (uint64_t)((row >> b) & 1) << L.cl_glob[b];
    }
    uint32_t scat_t[kMaxSub - 1] = {0, 0};
    for (int t = 0; t + 1 < L.nsub; ++t) scat_t[t] = scatter_thread_part(L, t, row);
    const uint32_t mb = smem_u32(mbar);
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t a_hi = smem_u32(aHi), a_lo = smem_u32(aLo);
    uint32_t phase = 0;
    bool failed = false;
    double acc_in = 0, acc_out = 0;

    uint64_t tile = blockIdx.x;
    const uint64_t step = tile_base(gridDim.x, L);
    uint64_t tbase = tile_base(tile, L);
    if (tile < P.tiles) prefetch_row(amp, tbase | gC0, L, stage, row);
    for (; tile < P.tiles; tile += gridDim.x) {
        const uint64_t tnext = tile_base_advance(tbase, step, L.tmask);
        const bool more = tile + gridDim.x < P.tiles;
        // ---- block 0 input: this thread's staging row -> registers -> A
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        float x[64];
        read_stage_row(stage, row, x);
        if constexpr (S::kStageInA)
            __syncthreads();                  // every staging row is read before A overwrites them
        else if (more)
            prefetch_row(amp, tnext | gC0, L, stage, row);
        {
            float t = 0.f;
#pragma unroll
            for (int e = 0; e < 64; ++e) { x[e] *= scale; t = fmaf(x[e], x[e], t); }
            acc_in += (double)t;
        }
        a_store_row(aHi, aLo, row, x);

        for (int b = 0; b < L.nsub; ++b) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0)
                issue_block_mma(tmem, a_hi, a_lo, smem_u32(smem + S::kOffB + (2 * b) * kB),
                                smem_u32(smem + S::kOffB + (2 * b + 1) * kB), mb);
            const bool ok = mbar_wait(mb, phase);
            phase ^= 1;
            if (__syncthreads_or(!ok)) { failed = true; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (S::kStageInA && b + 1 == L.nsub && more)
                prefetch_row(amp, tnext | gC0, L, stage, row);   // the MMAs are done with A
            uint32_t y[4][16];
#pragma unroll
            for (int q = 0; q < 4; ++q) tmem_ld16(taddr + 16 * q, y[q]);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (b + 1 < L.nsub) {
                // results become the next block's A operand
                const uint32_t tp = scat_t[b];
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        a_store_at(aHi, aLo, tp ^ L.scat[b][8 * q + e], __uint_as_float(y[q][2 * e]),
                                   __uint_as_float(y[q][2 * e + 1]));
            } else {
                float t = 0.f;
                const uint64_t obase = tbase | gCl;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) t = fmaf(__uint_as_float(y[q][e]), __uint_as_float(y[q][e]), t);
                    if (L.vecl) {
#pragma unroll
                        for (int e = 0; e < 8; e += 2) {
                            float4 v = make_float4(__uint_as_float(y[q][2 * e]), __uint_as_float(y[q][2 * e + 1]),
                                                   __uint_as_float(y[q][2 * e + 2]), __uint_as_float(y[q][2 * e + 3]));
                            *reinterpret_cast<float4 *>(amp + 2 * (obase | L.gl[8 * q + e])) = v;
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            float2 v = make_float2(__uint_as_float(y[q][2 * e]), __uint_as_float(y[q][2 * e + 1]));
                            *reinterpret_cast<float2 *>(amp + 2 * (obase | L.gl[8 * q + e])) = v;
                        }
                    }
                }
                acc_out += (double)t;
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
        double *red = reinterpret_cast<double *>(smem + S::kOffStage);   // staging is free now
        __syncthreads();
        if ((tid & 31) == 0) { red[warp] = ai; red[4 + warp] = ao; }
        __syncthreads();
        if (tid == 0) {
            double a = 0, b = 0;
            for (int w = 0; w < kThreads / 32; ++w) { a += red[w]; b += red[4 + w]; }
            if (P.in_parts) P.in_parts[blockIdx.x] = a;
            if (P.out_parts) P.out_parts[blockIdx.x] = b;
        }
        if (blockIdx.x == 0)                 // partials past this grid read as zero
            for (int i = (int)gridDim.x + tid; i < P.nparts; i += kThreads) {
                if (P.in_parts) P.in_parts[i] = 0.0;
                if (P.out_parts) P.out_parts[i] = 0.0;
            }
    }
    if (failed) {
        if (tid == 0) atomicExch(P.err, 1);
        mbar_wait(mb, phase ^ 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTmemCols));
    }
}

uint64_t grid_for(const qs_state *s, int ctas_per_sm)
{
    const uint64_t tiles = s->N >> 12, cap = (uint64_t)QS_SM_COUNT * ctas_per_sm;
    return tiles < cap ? tiles : cap;
}

template <int SUB>
int launch(qs_state *s, TileParams &P)
{
    using S = Shape<SUB>;
    QS_CUDA_TRY(cudaFuncSetAttribute(k_fused_tile<SUB>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kSmemBytes));
    const unsigned grid = (unsigned)grid_for(s, S::kCtasPerSm);
    k_fused_tile<SUB><<<grid, kThreads, S::kSmemBytes, s->stream>>>(static_cast<float *>(s->amp), P);
    QS_LAUNCH_CHECK("k_fused_tile");
    return QS_OK;
}

}  // namespace

int qs_tiled_grid(const qs_state *s)
{
    return (int)grid_for(s, Shape<2>::kCtasPerSm);    // the larger of the two grids
}

int qs_launch_tiled(qs_state *s, const qs_tiled_desc *d, int *err_dev)
{
    if (s->dtype != QS_C64) return qs_fail(QS_ERR_UNSUPPORTED, "tiled passes: complex64 states only");
    if (s->n < 12) return qs_fail(QS_ERR_UNSUPPORTED, "tiled passes: need at least 12 qubits");
    TileParams P;
    memset(&P, 0, sizeof(P));
    int r = qs_tile_layout_build(s->n, d->T, d->nsub, d->qpos, d->has_rows ? d->rows : nullptr, &P.L);
    if (r) return r;
    P.tiles = s->N >> 12;
    P.mat = static_cast<const uint16_t *>(d->mat_dev);
    P.err = err_dev;
    P.nparts = qs_tiled_grid(s);
    P.norm0 = d->norm0;
    P.prev_out = d->prev_out;
    P.in_parts = d->in_parts;
    P.out_parts = d->out_parts;
    return d->nsub <= 2 ? launch<2>(s, P) : launch<3>(s, P);
}
