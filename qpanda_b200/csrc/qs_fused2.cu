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
// Per tile, a lane of 128 threads (thread i owns row i and TMEM lane i,
// qs_tile_core.cuh) does:
//   1. the tile arrives by cp.async in tile order, each thread copying 16
//      chunks of 16 bytes (the 32 lanes of a warp fill 512 contiguous bytes of
//      shared memory per instruction); each thread then splits its own chunks
//      into BF16 hi/lo at their rows and columns of the swizzled K-major A
//      buffer and at once issues its copies of the lane's next tile into the
//      same slots, so that they land while this tile is computed;
//   2. for each block: one thread issues the 12 MMAs and commits to the
//      lane's mbarrier; every thread waits, loads its 64 FP32 results from
//      TMEM, and either scatters them as BF16 hi/lo into the next block's A
//      layout (one XOR per result gives its offset there), or - after the last
//      block - stores them to HBM: in place, or - for a remapping plan - into
//      the other buffer at the positions the pass's StoreMap gives.
// One CTA per SM holds three such lanes (two for passes of three blocks),
// each with its own A buffers, staging area, mbarrier, named barrier and 64
// TMEM columns; the blocks' B operands are loaded once per CTA and shared.
// Each lane's tile is a serial chain (copy, split, MMA, wait, scatter, MMA,
// wait, store); three independent lanes per SM overlap each other's chains,
// and every lane keeps its next tile's copies in flight throughout.
// A lane walks tiles  blockIdx.x * lanes + lane  in steps of gridDim.x * lanes;
// the global base of its next tile is one masked add away from the current one.
//
// The norm correction of the previous pass (a scalar) is folded into block
// 0's B operand when the CTA loads it, and the input norm is accumulated only
// on the plan's first pass (the only one whose input norm is used).
// Bounded waits as in qs_fused.cu.
#include "qs_fused.h"
#include "qs_tile_core.cuh"

namespace {

using namespace qs_tile;

template <int SUB, int TPR>
struct Shape {
    static constexpr int kLanes = SUB <= 2 ? 3 : 2;
    static constexpr int kLaneThreads = kThreads * TPR;       // 128 rows, TPR threads per row
    static constexpr int kCtaThreads = kLaneThreads * kLanes;
    static constexpr uint32_t kOffB = 0;                          // B hi/lo per block
    static constexpr uint32_t kLaneBytes = 2 * kA + kStage;       // A hi, A lo, staging rows
    static constexpr uint32_t kOffLane = kOffB + SUB * 2 * kB;
    static constexpr uint32_t kOffMisc = kOffLane + kLanes * kLaneBytes;
    // misc: one mbarrier per lane (8 B each, 32 reserved), tmem address (4), scale (4)
    static constexpr uint32_t kSmemBytes = kOffMisc + 48;
    static constexpr uint32_t kCols = kLanes <= 2 ? 128 : 256;    // TMEM columns (power of two >= 64 x lanes)
    static_assert(kSmemBytes + 1024 <= 228 * 1024, "one CTA per SM");
    static_assert(kLanes * kTmemCols <= kCols, "TMEM columns per lane");
    static_assert((kOffLane & 1023) == 0 && (kLaneBytes & 1023) == 0, "swizzled operands are 1024-byte aligned");
};

struct TileParams {
    Layout L;
    LoadMap M;
    StoreMap W;
    uint64_t tiles;
    const uint16_t *mat;         // nsub x [2][64][64] BF16 bits (hi, lo) of R
    int *err;
    int nparts;                  // norm partials per pass (>= gridDim.x; the tail is written as zeros)
    const double *norm0;
    const double *prev_out;
    double *in_parts;
    double *out_parts;
};

__device__ __forceinline__ void lane_bar(int id, int nthreads)
{
    asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(nthreads) : "memory");
}

// Named-barrier OR over the lane's threads.
__device__ __forceinline__ bool lane_bar_or(int id, int nthreads, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r) : "r"((uint32_t)v), "r"(id), "r"(nthreads) : "memory");
    return r != 0;
}

// B operands of a pass into the swizzled layout; block 0's matrix multiplied
// by `scale` (hi + lo recombined in FP32, scaled, split again).
__device__ __forceinline__ void load_b_scaled(uint8_t *dst, const uint16_t *mat, int nsub, float scale,
                                              int nthreads)
{
    const int first = scale != 1.0f ? 1 : 0;
    if (first) {
        for (int c = threadIdx.x; c < 64 * 8; c += nthreads) {
            const int row = c / 8, ch = c % 8;
            const uint4 h = *reinterpret_cast<const uint4 *>(mat + row * 64 + ch * 8);
            const uint4 l = *reinterpret_cast<const uint4 *>(mat + 64 * 64 + row * 64 + ch * 8);
            const uint32_t hw[4] = {h.x, h.y, h.z, h.w}, lw[4] = {l.x, l.y, l.z, l.w};
            uint32_t ho[4], lo[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float a = (__uint_as_float(hw[e] << 16) + __uint_as_float(lw[e] << 16)) * scale;
                const float b = (__uint_as_float(hw[e] & 0xffff0000u) + __uint_as_float(lw[e] & 0xffff0000u)) * scale;
                split_pair(a, b, ho[e], lo[e]);
            }
            const uint32_t off = row * 128 + ((ch ^ (row & 7)) << 4);
            *reinterpret_cast<uint4 *>(dst + off) = make_uint4(ho[0], ho[1], ho[2], ho[3]);
            *reinterpret_cast<uint4 *>(dst + kB + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        }
    }
    for (int c = threadIdx.x + first * 2 * 64 * 8; c < nsub * 2 * 64 * 8; c += nthreads) {
        const int mtx = c / (64 * 8), row = (c / 8) % 64, ch = c % 8;
        uint4 v = *reinterpret_cast<const uint4 *>(mat + (size_t)mtx * 64 * 64 + row * 64 + ch * 8);
        *reinterpret_cast<uint4 *>(dst + mtx * kB + row * 128 + ((ch ^ (row & 7)) << 4)) = v;
    }
}

template <int SUB, int TPR>
__global__ void __launch_bounds__(Shape<SUB, TPR>::kCtaThreads, 1) k_fused_tile(const float *amp, float *out,
                                                                              TileParams P)
{
    using S = Shape<SUB, TPR>;
    constexpr int kQ = 4 / TPR;                // 16-column TMEM loads per thread per block
    extern __shared__ __align__(1024) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int lane = tid / S::kLaneThreads, ltid = tid % S::kLaneThreads, lwarp = (ltid >> 5) & 3;
    const int half = TPR == 2 ? ltid >> 7 : 0;   // which 16 of a row's 32 columns (two threads per row)
    if (smem_u32(smem) & 1023u) {             // swizzled operands need 1024-byte alignment
        if (tid == 0) atomicExch(P.err, 2);
        return;
    }
    const Layout &L = P.L;
    uint8_t *lbase = smem + S::kOffLane + lane * S::kLaneBytes;
    uint8_t *aHi = lbase, *aLo = lbase + kA;
    const uint32_t stage = smem_u32(lbase + 2 * kA);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + S::kOffMisc) + lane;
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + S::kOffMisc + 32);
    float *s_scale = reinterpret_cast<float *>(smem + S::kOffMisc + 36);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_holder)), "r"(S::kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (ltid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
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
    __syncthreads();
    load_b_scaled(smem + S::kOffB, P.mat, L.nsub, *s_scale, S::kCtaThreads);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem_base = *tmem_holder;
    const uint32_t tmem = tmem_base + (uint32_t)(lane * kTmemCols);      // this lane's 64 columns

    const int row = ltid & (kThreads - 1);
    uint64_t gCl = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b) gCl |= (uint64_t)((row >> b) & 1) << L.cl_glob[b];
    uint32_t scat_t[kMaxSub - 1] = {0, 0};
    for (int t = 0; t + 1 < L.nsub; ++t) scat_t[t] = scatter_thread_part(L, t, row);
    const uint32_t mb = smem_u32(mbar);
    const uint32_t taddr = tmem + ((uint32_t)(lwarp * 32) << 16);
    const uint32_t a_hi = smem_u32(aHi), a_lo = smem_u32(aLo);
    const int bar_id = 1 + lane;
    const bool want_in = P.in_parts != nullptr;
    uint32_t phase = 0;
    bool failed = false;
    double acc_in = 0, acc_out = 0;

    const ChunkBase cb = chunk_base<TPR>(P.M, ltid);
    const uint64_t stride = (uint64_t)gridDim.x * S::kLanes;
    uint64_t tile = (uint64_t)blockIdx.x * S::kLanes + lane;
    const uint64_t step = tile_base(stride, L);
    uint64_t tbase = tile_base(tile, L);
    const int j0 = 16 * half;                 // this thread's columns: all 32, or 16 of them from j0
    if (tile < P.tiles) prefetch_tile_linear<TPR>(amp, tbase, P.M, stage, cb.g, ltid);
    for (; tile < P.tiles; tile += stride) {
        const uint64_t tnext = tile_base_advance(tbase, step, L.tmask);
        // ---- block 0 input: this thread's staged chunks -> A; then its
        // chunks of the lane's next tile (its own staging slots, just read)
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        {
            uint32_t hv[16 / TPR][2], lv[16 / TPR][2];
            const float ss = convert_load<TPR>(stage, ltid, hv, lv);
            if (want_in) acc_in += (double)ss;
            convert_store<TPR>(aHi, aLo, P.M, cb, hv, lv);
        }
        if (tile + stride < P.tiles) prefetch_tile_linear<TPR>(amp, tnext, P.M, stage, cb.g, ltid);

        for (int b = 0; b < L.nsub; ++b) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            lane_bar(bar_id, S::kLaneThreads);
            if (ltid == 0)
                issue_block_mma(tmem, a_hi, a_lo, smem_u32(smem + S::kOffB + (2 * b) * kB),
                                smem_u32(smem + S::kOffB + (2 * b + 1) * kB), mb);
            const bool ok = mbar_wait(mb, phase);
            phase ^= 1;
            if (lane_bar_or(bar_id, S::kLaneThreads, !ok)) { failed = true; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t y[kQ][16];
#pragma unroll
            for (int q = 0; q < kQ; ++q) tmem_ld16(taddr + 2 * j0 + 16 * q, y[q]);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (b + 1 < L.nsub) {
                // results become the next block's A operand
                const uint32_t tp = scat_t[b];
#pragma unroll
                for (int q = 0; q < kQ; ++q)
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        a_store_at(aHi, aLo, tp ^ L.scat[b][j0 + 8 * q + e], __uint_as_float(y[q][2 * e]),
                                   __uint_as_float(y[q][2 * e + 1]));
            } else {
                const uint64_t obase = store_base(tile, tbase, P.W) | gCl;
#pragma unroll
                for (int q = 0; q < kQ; ++q) {
                    if (L.vecl) {
#pragma unroll
                        for (int e = 0; e < 8; e += 2) {
                            float4 v = make_float4(__uint_as_float(y[q][2 * e]), __uint_as_float(y[q][2 * e + 1]),
                                                   __uint_as_float(y[q][2 * e + 2]), __uint_as_float(y[q][2 * e + 3]));
                            *reinterpret_cast<float4 *>(out + 2 * (obase | L.gl[j0 + 8 * q + e])) = v;
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            float2 v = make_float2(__uint_as_float(y[q][2 * e]), __uint_as_float(y[q][2 * e + 1]));
                            *reinterpret_cast<float2 *>(out + 2 * (obase | L.gl[j0 + 8 * q + e])) = v;
                        }
                    }
                }
                float t4[4] = {0.f, 0.f, 0.f, 0.f};               // after the stores are issued
#pragma unroll
                for (int q = 0; q < kQ; ++q)
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        t4[e & 3] = fmaf(__uint_as_float(y[q][e]), __uint_as_float(y[q][e]), t4[e & 3]);
                acc_out += (double)((t4[0] + t4[1]) + (t4[2] + t4[3]));
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
        double *red = reinterpret_cast<double *>(smem + S::kOffLane + 2 * kA);   // lane 0's staging rows
        __syncthreads();                     // every copy of every lane has landed
        if ((tid & 31) == 0) { red[warp] = ai; red[kWarps + warp] = ao; }
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
        mbar_wait(mb, phase ^ 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem_base), "r"(S::kCols));
    }
}

template <int SUB>
uint64_t grid_for(const qs_state *s)
{
    constexpr int lanes = Shape<SUB, 1>::kLanes;
    const uint64_t tiles = s->N >> 12, need = (tiles + lanes - 1) / lanes;
    return need < QS_SM_COUNT ? need : QS_SM_COUNT;
}

template <int SUB, int TPR>
int launch(qs_state *s, const float *in, float *out, TileParams &P)
{
    using S = Shape<SUB, TPR>;
    QS_CUDA_TRY(cudaFuncSetAttribute(k_fused_tile<SUB, TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     S::kSmemBytes));
    const unsigned grid = (unsigned)grid_for<SUB>(s);
    k_fused_tile<SUB, TPR><<<grid, S::kCtaThreads, S::kSmemBytes, s->stream>>>(in, out, P);
    QS_LAUNCH_CHECK("k_fused_tile");
    return QS_OK;
}

}  // namespace

int qs_tiled_grid(const qs_state *s)
{
    const uint64_t a = grid_for<2>(s), b = grid_for<3>(s);
    return (int)(a > b ? a : b);                      // the larger of the two grids
}

int qs_launch_tiled(qs_state *s, const qs_tiled_desc *d, int *err_dev)
{
    if (s->dtype != QS_C64) return qs_fail(QS_ERR_UNSUPPORTED, "tiled passes: complex64 states only");
    if (s->n < 12) return qs_fail(QS_ERR_UNSUPPORTED, "tiled passes: need at least 12 qubits");
    TileParams P;
    memset(&P, 0, sizeof(P));
    int r = qs_tile_layout_build(s->n, d->T, d->nsub, d->qpos, d->has_rows ? d->rows : nullptr, &P.L, &P.M,
                                 d->has_write ? d->wtile : nullptr);
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
    if (d->threads_per_row == 2)
        return d->nsub <= 2 ? launch<2, 2>(s, in, out, P) : launch<3, 2>(s, in, out, P);
    return d->nsub <= 2 ? launch<2, 1>(s, in, out, P) : launch<3, 1>(s, in, out, P);
}
