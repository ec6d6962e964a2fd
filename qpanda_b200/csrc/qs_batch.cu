// qs_batch.cu - many independent circuits in one persistent launch.
//
// The reference runs one program at a time (QPandaSDK::run, QPandaAPI.cpp:131-211);
// a parameter sweep is a loop of runs.  Here thousands of circuits of uneven
// width and depth share one launch: every circuit gets its own state buffer
// (at least 12 qubits: narrower ones are padded with idle qubits that stay in
// |0>), its own fused plan (tiled passes of up to three 5-qubit tensor-core
// blocks, qs_plan.cpp), and the kernel's CTAs take whole circuits from a
// queue, longest first.  A CTA runs all passes of its circuit over all of the
// circuit's tiles, so passes need no synchronisation between CTAs; states up
// to a few MB stay in L2 while their CTA works on them.  The first pass starts
// from |0...0> without reading memory; the last pass also accumulates the
// nearest-neighbour <Z_i Z_{i+1}> expectations of the circuit.
//
// Circuits with the same gate pattern (same operations on the same qubits)
// share one plan structure; only their block matrices are rebuilt.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "qs_fused.h"
#include "qs_plan_internal.h"
#include "qs_prim.h"
#include "qs_tile_core.cuh"
#include "qs_tile_tmem.cuh"
#include "qs_tile_tmem_dev.cuh"

int qs_tmem_layout_build(int n, const qs_tiled_desc *d, qs_tmem::TLayout *L);

namespace {

using namespace qs_tile;

constexpr int kMaxZZ = 23;                        // circuits of up to 24 qubits
constexpr uint32_t kLayoutBytes = (sizeof(Layout) + 15) & ~15u;
constexpr uint32_t kLoadBytes = (sizeof(LoadMap) + 15) & ~15u;

// Shared memory of the two shapes: with up to 2 blocks per pass the staging
// area is the A region and three CTAs fit per SM - the tile arrives in tile
// order (prefetch_tile_linear), each thread reads its own chunks to registers,
// and after a barrier writes them at their rows and columns of A; with 3
// blocks there is a separate staging area, each thread copies its own row
// (prefetch_row), and two CTAs fit per SM.
// Reductions (4 + 4 x kMaxZZ doubles) reuse the staging rows: they run only
// when no copy into staging is in flight and no MMA reads A.
template <int SUB>
struct BShape {
    static constexpr bool kStageInA = SUB <= 2;
    static constexpr int kCtasPerSm = kStageInA ? 3 : 2;
    static constexpr uint32_t kOffA = 0;
    static constexpr uint32_t kOffB = 2 * kA;
    static constexpr uint32_t kOffStage = kStageInA ? kOffA : kOffB + SUB * 2 * kB;
    static constexpr uint32_t kOffLayout = kOffB + SUB * 2 * kB + (kStageInA ? 0 : kStage);
    static constexpr uint32_t kOffLoad = kOffLayout + kLayoutBytes;            // tile-order shape only
    static constexpr uint32_t kOffMisc = kOffLoad + (kStageInA ? kLoadBytes : 0);   // mbarrier 8, tmem 4, circuit 4
    static constexpr uint32_t kSmemBytes = kOffMisc + 16;
    static constexpr uint32_t kOffRed = kOffStage;
    static_assert(kCtasPerSm * (kSmemBytes + 1024) <= 228 * 1024, "resident CTAs per SM");
    static_assert(!kStageInA || 2 * kA == kStage, "the A region holds one tile of staging rows");
    static_assert((4 + 4 * kMaxZZ) * 8 <= kStage, "reductions fit the staging rows");
};

struct BatchCirc {
    float *amp;                  // 2^nq_eff complex64
    const uint16_t *mats;        // the circuit's blocks, [2][64][64] BF16 each
    const Layout *layouts;       // its passes (Layout::pad = first block of the pass)
    const LoadMap *loads;        // their tile-order copy maps
    const qs_tmem::TLayout *tlayouts;   // its passes' tensor-memory layouts (k_batch_tmem), or null
    double *zz;                  // nq - 1 outputs
    int32_t npass, nq, nq_eff, pad;
};

struct BatchParams {
    const BatchCirc *circ;
    const int32_t *order;        // processing order (longest first)
    int32_t ncirc;
    int32_t *head;               // queue position, zeroed before the launch
    int *err;
};

template <int SUB>
__global__ void __launch_bounds__(kThreads, BShape<SUB>::kCtasPerSm) k_batch(BatchParams P)
{
    using S = BShape<SUB>;
    extern __shared__ __align__(1024) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (smem_u32(smem) & 1023u) {
        if (tid == 0) atomicExch(P.err, 2);
        return;
    }
    uint8_t *aHi = smem + S::kOffA, *aLo = smem + S::kOffA + kA;
    Layout &L = *reinterpret_cast<Layout *>(smem + S::kOffLayout);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + S::kOffMisc);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + S::kOffMisc + 8);
    int32_t *s_circ = reinterpret_cast<int32_t *>(smem + S::kOffMisc + 12);
    double *red = reinterpret_cast<double *>(smem + S::kOffRed);
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
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_holder;
    const uint32_t mb = smem_u32(mbar);
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t a_hi = smem_u32(aHi), a_lo = smem_u32(aLo);
    const int row = tid;
    uint32_t phase = 0;
    bool failed = false;

    while (!failed) {
        if (tid == 0) {
            const int c = atomicAdd(P.head, 1);
            *s_circ = c < P.ncirc ? P.order[c] : -1;
        }
        __syncthreads();
        const int ci = *s_circ;
        if (ci < 0) break;
        const BatchCirc C = P.circ[ci];
        const uint64_t tiles = 1ull << (C.nq_eff - 12);
        const int nzz = C.nq - 1;
        float scale = 1.0f;
        double zz[kMaxZZ];
#pragma unroll
        for (int i = 0; i < kMaxZZ; ++i) zz[i] = 0.0;
        double out_norm = 0.0;

        for (int p = 0; p < C.npass && !failed; ++p) {
            // the pass's layout and matrices into shared memory
            {
                const uint32_t *src = reinterpret_cast<const uint32_t *>(C.layouts + p);
                uint32_t *dst = reinterpret_cast<uint32_t *>(&L);
                for (int i = tid; i < (int)(sizeof(Layout) / 4); i += kThreads) dst[i] = src[i];
                if constexpr (S::kStageInA) {
                    const uint32_t *ls = reinterpret_cast<const uint32_t *>(C.loads + p);
                    uint32_t *ld = reinterpret_cast<uint32_t *>(smem + S::kOffLoad);
                    for (int i = tid; i < (int)(sizeof(LoadMap) / 4); i += kThreads) ld[i] = ls[i];
                }
            }
            __syncthreads();
            load_b(smem + S::kOffB, C.mats + (size_t)L.pad * 2 * 64 * 64, L.nsub);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            uint64_t gC0 = 0, gCl = 0;
#pragma unroll
            for (int b = 0; b < 7; ++b) {
                gC0 |= (uint64_t)((row >> b) & 1) << L.c0_glob[b];
                gCl |= (uint64_t)((row >> b) & 1) << L.cl_glob[b];
            }
            uint32_t baseR[kMaxSub - 1] = {0, 0}, baseJ[kMaxSub - 1] = {0, 0};
            for (int t = 0; t + 1 < L.nsub; ++t)
                for (int b = 0; b < 7; ++b) {
                    const uint32_t bit = (row >> b) & 1;
                    const int m = L.rowmap[t][b];
                    if (m >= 0) baseR[t] |= bit << m;
                    else baseJ[t] |= bit << (~m);
                }
            const bool last_pass = p + 1 == C.npass;
            double acc_out = 0;
            const uint64_t step = tile_base(1, L);
            uint64_t tbase = 0;                       // tile_base(0)
            const LoadMap &M = *reinterpret_cast<const LoadMap *>(smem + S::kOffLoad);
            ChunkBase cb{0, 0, 0};
            if constexpr (S::kStageInA) cb = chunk_base(M, tid);
            if (p > 0) {
                if constexpr (S::kStageInA) prefetch_tile_linear(C.amp, tbase, M, stage, cb.g, tid);
                else prefetch_row(C.amp, tbase | gC0, L, stage, row);
            }
            for (uint64_t tile = 0; tile < tiles; ++tile) {
                const uint64_t tnext = tile_base_advance(tbase, step, L.tmask);
                if (p == 0) {
                    // |0...0>: amplitude 0 is tile 0, the row with no row bits, column 0
                    float x[64];
#pragma unroll
                    for (int e = 0; e < 64; ++e) x[e] = 0.f;
                    if (tile == 0 && gC0 == 0) x[0] = 1.f;
#pragma unroll
                    for (int j = 0; j < 32; ++j) a_store_pair(aHi, aLo, row, j, x[2 * j], x[2 * j + 1]);
                } else if constexpr (S::kStageInA) {
                    // this thread's chunks of the tile (tile order, in the A
                    // region) to registers; once every thread has its chunks,
                    // their BF16 split at their rows and columns of A
                    asm volatile("cp.async.wait_group 0;" ::: "memory");
                    float4 v[16];
#pragma unroll
                    for (int k = 0; k < 16; ++k)
                        asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                                     : "=f"(v[k].x), "=f"(v[k].y), "=f"(v[k].z), "=f"(v[k].w)
                                     : "r"(stage + (uint32_t)(128 * k + tid) * 16u));
                    __syncthreads();
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const uint32_t r0 = cb.r ^ M.rk[k], j0 = cb.j ^ M.jk[k];
                        uint32_t h0, l0, h1, l1;
                        split_pair(v[k].x * scale, v[k].y * scale, h0, l0);
                        split_pair(v[k].z * scale, v[k].w * scale, h1, l1);
                        if (M.pair) {
                            const uint32_t off = a_offset(r0, j0);
                            *reinterpret_cast<uint2 *>(aHi + off) = make_uint2(h0, h1);
                            *reinterpret_cast<uint2 *>(aLo + off) = make_uint2(l0, l1);
                        } else {
                            const uint32_t o0 = a_offset(r0, j0), o1 = a_offset(r0 | M.dr, j0 | M.dj);
                            *reinterpret_cast<uint32_t *>(aHi + o0) = h0;
                            *reinterpret_cast<uint32_t *>(aLo + o0) = l0;
                            *reinterpret_cast<uint32_t *>(aHi + o1) = h1;
                            *reinterpret_cast<uint32_t *>(aLo + o1) = l1;
                        }
                    }
                } else {
                    asm volatile("cp.async.wait_group 0;" ::: "memory");
                    float x[64];
                    read_stage_row(stage, row, x);
                    if (tile + 1 < tiles) prefetch_row(C.amp, tnext | gC0, L, stage, row);
#pragma unroll
                    for (int e = 0; e < 64; ++e) x[e] *= scale;
#pragma unroll
                    for (int j = 0; j < 32; ++j) a_store_pair(aHi, aLo, row, j, x[2 * j], x[2 * j + 1]);
                }

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
                    if constexpr (S::kStageInA)
                        if (p > 0 && b + 1 == L.nsub && tile + 1 < tiles)
                            prefetch_tile_linear(C.amp, tnext, M, stage, cb.g, tid);   // the MMAs are done with A
                    uint32_t y[4][16];
#pragma unroll
                    for (int q = 0; q < 4; ++q) tmem_ld16(taddr + 16 * q, y[q]);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (b + 1 < L.nsub) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                const int j = 8 * q + e;
                                const int r2 = baseR[b] | L.tabR[b][j], j2 = baseJ[b] | L.tabJ[b][j];
                                a_store_pair(aHi, aLo, r2, j2, __uint_as_float(y[q][2 * e]),
                                             __uint_as_float(y[q][2 * e + 1]));
                            }
                    } else {
                        const uint64_t obase = tbase | gCl;
                        float t4[4] = {0.f, 0.f, 0.f, 0.f};                  // four chains, fixed order
                        float zt[kMaxZZ];
#pragma unroll
                        for (int i = 0; i < kMaxZZ; ++i) zt[i] = 0.f;
#pragma unroll
                        for (int q = 0; q < 4; ++q)
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                const float re = __uint_as_float(y[q][2 * e]), im = __uint_as_float(y[q][2 * e + 1]);
                                const uint64_t g = obase | L.gl[8 * q + e];
                                *reinterpret_cast<float2 *>(C.amp + 2 * g) = make_float2(re, im);
                                const float pr = fmaf(re, re, im * im);
                                t4[e & 3] += pr;
                                if (last_pass) {
                                    const uint32_t par = (uint32_t)(g ^ (g >> 1));   // bit i: x_i xor x_{i+1}
#pragma unroll
                                    for (int i = 0; i < kMaxZZ; ++i) zt[i] += ((par >> i) & 1u) ? -pr : pr;
                                }
                            }
                        acc_out += (double)((t4[0] + t4[1]) + (t4[2] + t4[3]));
                        if (last_pass)
#pragma unroll
                            for (int i = 0; i < kMaxZZ; ++i) zz[i] += (double)zt[i];
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                }
                if (failed) break;
                tbase = tnext;
            }
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            // the pass's output norm (fixed order), and the next pass's scale
            for (int o = 16; o > 0; o >>= 1) acc_out += __shfl_xor_sync(0xffffffffu, acc_out, o);
            __syncthreads();
            if (lane == 0) red[warp] = acc_out;
            __syncthreads();
            out_norm = red[0] + red[1] + red[2] + red[3];
            scale = out_norm > 0 ? (float)(1.0 / sqrt(out_norm)) : 1.0f;
            // this pass's stores must be visible to the next pass's loads
            __threadfence();
            __syncthreads();
        }
        if (failed) break;
        // <Z_i Z_{i+1}> of the normalised final state
#pragma unroll
        for (int i = 0; i < kMaxZZ; ++i)
            for (int o = 16; o > 0; o >>= 1) zz[i] += __shfl_xor_sync(0xffffffffu, zz[i], o);
        if (lane == 0)
#pragma unroll
            for (int i = 0; i < kMaxZZ; ++i) red[4 + warp * kMaxZZ + i] = zz[i];
        __syncthreads();
        for (int i = tid; i < nzz; i += kThreads)
            C.zz[i] = (red[4 + i] + red[4 + kMaxZZ + i] + red[4 + 2 * kMaxZZ + i] + red[4 + 3 * kMaxZZ + i]) /
                      out_norm;
        __syncthreads();
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

// The same sweep with the tile in tensor memory: k_tile_tmem's pass body
// (qs_tile_tmem.cu: staging copies in tile order, the row gather, the tile as
// the MMAs' A operand in TMEM, the exchange between blocks through the staging
// buffer, the stores of the last block) run by one 128-thread CTA per circuit,
// three CTAs per SM, passes of up to two blocks; what k_batch adds stays as it
// is: the queue, |0...0> on the first pass without reading memory, the
// previous pass's norm folded into the first block's matrix, and the
// <Z_i Z_{i+1}> of the last pass's output.
constexpr int kTmThreads = 128;
constexpr int kTmCtasPerSm = 3;
constexpr uint32_t kTmOffB = 0;                                      // 2 blocks x (hi, lo) x 8 KB
constexpr uint32_t kTmOffStage = 2 * 2 * kB;                         // 32 KB of staging
constexpr uint32_t kTmOffLayout = kTmOffStage + kStage;
constexpr uint32_t kTmLayoutBytes = (sizeof(qs_tmem::TLayout) + 15) & ~15u;
constexpr uint32_t kTmOffMisc = kTmOffLayout + kTmLayoutBytes;       // mbarrier 8, tmem 4, circuit 4
constexpr uint32_t kTmSmemBytes = kTmOffMisc + 16;
constexpr uint32_t kTmCols = 128;
static_assert(kTmCtasPerSm * (kTmSmemBytes + 1024) <= 228 * 1024, "resident CTAs per SM");
static_assert(kTmCtasPerSm * kTmCols <= 512, "TMEM columns per SM");
static_assert((4 + 4 * kMaxZZ) * 8 <= kStage, "reductions fit the staging buffer");

__global__ void __launch_bounds__(kTmThreads, kTmCtasPerSm) k_batch_tmem(BatchParams P)
{
    namespace D = qs_tmem_dev;
    extern __shared__ __align__(1024) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (smem_u32(smem) & 1023u) {
        if (tid == 0) atomicExch(P.err, 2);
        return;
    }
    qs_tmem::TLayout &L = *reinterpret_cast<qs_tmem::TLayout *>(smem + kTmOffLayout);
    const uint32_t stage = smem_u32(smem + kTmOffStage);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kTmOffMisc);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + kTmOffMisc + 8);
    int32_t *s_circ = reinterpret_cast<int32_t *>(smem + kTmOffMisc + 12);
    double *red = reinterpret_cast<double *>(smem + kTmOffStage);   // when no copy is in flight

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_holder)), "r"(kTmCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tgrp = *tmem_holder;
    const uint32_t tlane = tgrp + ((uint32_t)(warp * 32) << 16);
    const uint32_t mb = smem_u32(mbar);
    uint32_t phase = 0;
    bool failed = false;

    while (!failed) {
        if (tid == 0) {
            const int c = atomicAdd(P.head, 1);
            *s_circ = c < P.ncirc ? P.order[c] : -1;
        }
        __syncthreads();
        const int ci = *s_circ;
        if (ci < 0) break;
        const BatchCirc C = P.circ[ci];
        const uint64_t tiles = 1ull << (C.nq_eff - 12);
        const int nzz = C.nq - 1;
        float scale = 1.0f;
        double zz[kMaxZZ];
#pragma unroll
        for (int i = 0; i < kMaxZZ; ++i) zz[i] = 0.0;
        double out_norm = 0.0;

        for (int p = 0; p < C.npass && !failed; ++p) {
            {
                const uint32_t *src = reinterpret_cast<const uint32_t *>(C.tlayouts + p);
                uint32_t *dst = reinterpret_cast<uint32_t *>(&L);
                for (int i = tid; i < (int)(sizeof(qs_tmem::TLayout) / 4); i += kTmThreads) dst[i] = src[i];
            }
            __syncthreads();
            D::load_b_perm(smem + kTmOffB, C.mats + (size_t)C.layouts[p].pad * 2 * 64 * 64, L, scale);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // per-thread parts of the gather, exchange, copy and store addresses
            uint32_t xrow = 0, xw0 = 0, xr0 = 0;
            uint64_t orow = 0, g_t = 0;
            uint32_t cs_t = (uint32_t)tid;
#pragma unroll
            for (int i = 0; i < 5; ++i)
                if ((lane >> i) & 1) {
                    xrow ^= L.s_lane[i];
                    orow |= L.o_lane[i];
                    xw0 ^= L.xw_lane[0][i];
                    xr0 ^= L.xr_lane[0][i];
                }
#pragma unroll
            for (int v = 0; v < 2; ++v)
                if ((warp >> v) & 1) {
                    xrow ^= L.s_warp[v];
                    orow |= L.o_warp[v];
                    xw0 ^= L.xw_warp[0][v];
                    xr0 ^= L.xr_warp[0][v];
                }
#pragma unroll
            for (int b = 0; b < 7; ++b)
                if ((tid >> b) & 1) { g_t |= L.g_bit[b]; cs_t ^= L.cf_bit[b]; }
            const bool last_pass = p + 1 == C.npass;
            double acc_out = 0;
            const uint64_t step = D::tbase_of(1, L);
            uint64_t tbase = 0;
            if (p > 0) D::copy_tile<1>(C.amp, tbase, L, stage, g_t, cs_t);
            for (uint64_t tile = 0; tile < tiles; ++tile) {
                const uint64_t tnext = tile_base_advance(tbase, step, L.tmask);
                float y[64];
                if (p == 0) {
                    // |0...0>: amplitude 0 is tile 0, the row with no row bits, column 0
#pragma unroll
                    for (int e = 0; e < 64; ++e) y[e] = 0.f;
                    if (tile == 0 && tid == 0) y[0] = 1.f;
                } else {
                    asm volatile("cp.async.wait_group 0;" ::: "memory");
                    __syncthreads();
                    if (L.pair_in) {
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                                         : "=f"(y[4 * j]), "=f"(y[4 * j + 1]), "=f"(y[4 * j + 2]), "=f"(y[4 * j + 3])
                                         : "r"(stage + ((xrow ^ L.s_col[2 * j]) << 3)));
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];"
                                         : "=f"(y[2 * j]), "=f"(y[2 * j + 1]) : "r"(stage + ((xrow ^ L.s_col[j]) << 3)));
                    }
                }
                D::split_store<1>(tlane, y, 0u);
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncthreads();
                if (tid == 0) D::issue_ts(tgrp + 64, tgrp, smem_u32(smem + kTmOffB), smem_u32(smem + kTmOffB + kB), mb);
                if (p > 0 && L.nsub == 1 && tile + 1 < tiles) D::copy_tile<1>(C.amp, tnext, L, stage, g_t, cs_t);
                for (int b = 0; b < L.nsub; ++b) {
                    const bool ok = mbar_wait(mb, phase);
                    phase ^= 1;
                    if (__syncthreads_or(!ok)) { failed = true; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t dreg = (b & 1) ? 0u : 64u;                // this block's accumulator
                    D::tmem_ld32(tlane + dreg, y);
                    D::tmem_ld32(tlane + dreg + 32, y + 32);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (b + 1 < L.nsub) {
                        D::exchange_through<1, kTmThreads>(y, stage, xw0, xr0, L.xw_col[0], L.xr_col[0], 0);
                        D::split_store<1>(tlane + dreg, y, 0u);              // the next block's A
                        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                        __syncthreads();                                     // also: every exchange read is done
                        if (tid == 0)
                            D::issue_ts(tgrp + (dreg ^ 64u), tgrp + dreg, smem_u32(smem + kTmOffB + 2 * kB),
                                        smem_u32(smem + kTmOffB + 3 * kB), mb);
                        if (p > 0 && tile + 1 < tiles) D::copy_tile<1>(C.amp, tnext, L, stage, g_t, cs_t);
                    } else {
                        const uint64_t obase = tbase | orow;
                        if (L.vec_out) {
#pragma unroll
                            for (int j = 0; j < 16; ++j)
                                *reinterpret_cast<float4 *>(C.amp + 2 * (obase | L.o_col[2 * j])) =
                                    make_float4(y[4 * j], y[4 * j + 1], y[4 * j + 2], y[4 * j + 3]);
                        } else {
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                *reinterpret_cast<float2 *>(C.amp + 2 * (obase | L.o_col[j])) =
                                    make_float2(y[2 * j], y[2 * j + 1]);
                        }
                        acc_out += (double)D::sum_squares(y);
                        if (last_pass) {
                            float zt[kMaxZZ];
#pragma unroll
                            for (int i = 0; i < kMaxZZ; ++i) zt[i] = 0.f;
#pragma unroll
                            for (int j = 0; j < 32; ++j) {
                                const uint64_t g = obase | L.o_col[j];
                                const float pr = fmaf(y[2 * j], y[2 * j], y[2 * j + 1] * y[2 * j + 1]);
                                const uint32_t par = (uint32_t)(g ^ (g >> 1));       // bit i: x_i xor x_{i+1}
#pragma unroll
                                for (int i = 0; i < kMaxZZ; ++i) zt[i] += ((par >> i) & 1u) ? -pr : pr;
                            }
#pragma unroll
                            for (int i = 0; i < kMaxZZ; ++i) zz[i] += (double)zt[i];
                        }
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                }
                if (failed) break;
                tbase = tnext;
            }
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            // the pass's output norm (fixed order), and the next pass's scale
            for (int o = 16; o > 0; o >>= 1) acc_out += __shfl_xor_sync(0xffffffffu, acc_out, o);
            __syncthreads();
            if (lane == 0) red[warp] = acc_out;
            __syncthreads();
            out_norm = red[0] + red[1] + red[2] + red[3];
            scale = out_norm > 0 ? (float)(1.0 / sqrt(out_norm)) : 1.0f;
            // this pass's stores must be visible to the next pass's loads
            __threadfence();
            __syncthreads();
        }
        if (failed) break;
#pragma unroll
        for (int i = 0; i < kMaxZZ; ++i)
            for (int o = 16; o > 0; o >>= 1) zz[i] += __shfl_xor_sync(0xffffffffu, zz[i], o);
        if (lane == 0)
#pragma unroll
            for (int i = 0; i < kMaxZZ; ++i) red[4 + warp * kMaxZZ + i] = zz[i];
        __syncthreads();
        for (int i = tid; i < nzz; i += kTmThreads)
            C.zz[i] = (red[4 + i] + red[4 + kMaxZZ + i] + red[4 + 2 * kMaxZZ + i] + red[4 + 3 * kMaxZZ + i]) /
                      out_norm;
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) atomicExch(P.err, 1);
        mbar_wait(mb, phase ^ 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tgrp), "r"(kTmCols));
    }
}

}  // namespace

// ------------------------------------------------------------------ host
struct qs_batch {
    int n = 0;
    qs_batch_opts opts;
    std::vector<int> nq, nq_eff;
    std::vector<size_t> zz_off;          // output offsets (nq - 1 each)
    std::vector<size_t> amp_off;         // state offsets (bytes)
    std::vector<int32_t> order;
    int dev = -1;
    void *d_states = nullptr;            // all states
    void *d_mats = nullptr;              // all block matrices
    void *d_layouts = nullptr;           // layouts of the distinct plan structures
    void *d_loads = nullptr;             // their tile-order copy maps
    void *d_tlayouts = nullptr;          // their tensor-memory layouts (k_batch_tmem)
    bool use_tmem = false;
    void *d_circ = nullptr;              // BatchCirc[n]
    void *d_order = nullptr;
    double *d_zz = nullptr;
    int32_t *d_head = nullptr;           // queue head + error flag
    size_t zz_count = 0, state_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t graph_stream = nullptr;
};

namespace {

void batch_free(qs_batch *B)
{
    if (B->graph_exec) cudaGraphExecDestroy(B->graph_exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    for (void *p : {B->d_states, B->d_mats, B->d_layouts, B->d_loads, B->d_tlayouts, B->d_circ, B->d_order,
                    (void *)B->d_zz, (void *)B->d_head})
        if (p) cudaFree(p);
    delete B;
}

std::string signature(int nq, const qs_gate *g, size_t count)
{
    std::string s(reinterpret_cast<const char *>(&nq), sizeof(nq));
    for (size_t i = 0; i < count; ++i) {
        s.append(reinterpret_cast<const char *>(&g[i].op), sizeof(int32_t));
        s.append(reinterpret_cast<const char *>(g[i].q), sizeof(g[i].q));
        s.append(reinterpret_cast<const char *>(&g[i].nctrl), sizeof(int32_t));
        s.append(reinterpret_cast<const char *>(g[i].ctrl), sizeof(int32_t) * (size_t)std::max(0, g[i].nctrl));
    }
    return s;
}

}  // namespace

extern "C" int qs_batch_default_opts(qs_batch_opts *o)
{
    if (!o) return qs_fail(QS_ERR_ARG, "qs_batch_default_opts: null");
    o->max_sub = 2;              // three CTAs per SM (BShape)
    o->low_qubits = 3;
    o->order = QS_BATCH_LONGEST_FIRST;
    o->use_graph = 1;
    o->block_qubits = 5;
    o->tile_in_tmem = 1;
    return QS_OK;
}

extern "C" int qs_batch_create(int n_circ, const int *n_qubits, const qs_gate *gates, const size_t *offsets,
                               const qs_batch_opts *opts, qs_batch **out)
{
    if (!out) return qs_fail(QS_ERR_ARG, "qs_batch_create: null output");
    *out = nullptr;
    if (n_circ < 1 || !n_qubits || !offsets || (!gates && offsets[n_circ] > 0))
        return qs_fail(QS_ERR_ARG, "qs_batch_create: bad arguments");
    qs_batch_opts o;
    if (opts) o = *opts;
    else qs_batch_default_opts(&o);
    if (o.max_sub < 1 || o.max_sub > 3 || o.low_qubits < 1 || o.low_qubits > 5 || o.block_qubits < 4 ||
        o.block_qubits > 5)
        return qs_fail(QS_ERR_ARG, "qs_batch_create: max_sub 1..3, low_qubits 1..5, block_qubits 4..5");
    for (int c = 0; c < n_circ; ++c) {
        if (n_qubits[c] < 1 || n_qubits[c] > kMaxZZ + 1)
            return qs_fail(QS_ERR_UNSUPPORTED, "qs_batch_create: circuit %d has %d qubits (batched circuits: 1..%d)",
                           c, n_qubits[c], kMaxZZ + 1);
        if (offsets[c + 1] < offsets[c]) return qs_fail(QS_ERR_ARG, "qs_batch_create: offsets must not decrease");
    }
    qs_batch *B = new qs_batch();
    B->n = n_circ;
    B->opts = o;
    int r = QS_OK;
    cudaError_t e = cudaGetDevice(&B->dev);
    if (e != cudaSuccess) { delete B; return qs_cuda_fail(e, "qs_batch_create"); }

    // ---- plans: one structure per gate pattern, rebound per circuit
    qs_plan_opts po;
    qs_plan_default_opts(&po);
    po.max_sub = o.max_sub;
    po.low_qubits = o.low_qubits;
    po.block_qubits = o.block_qubits;
    std::map<std::string, int> proto_of;              // signature -> index in protos
    std::vector<qs_plan *> protos, plans(n_circ, nullptr);
    std::vector<int> proto_id(n_circ), proto_rep;     // proto_rep: a circuit of each structure
    B->nq.resize(n_circ);
    B->nq_eff.resize(n_circ);
    for (int c = 0; c < n_circ && !r; ++c) {
        B->nq[c] = n_qubits[c];
        B->nq_eff[c] = std::max(12, n_qubits[c]);
        const qs_gate *g = gates + offsets[c];
        const size_t cnt = offsets[c + 1] - offsets[c];
        for (size_t i = 0; i < cnt && !r; ++i)
            if (qs_gate_qubits(&g[i]) >> n_qubits[c])
                r = qs_fail(QS_ERR_ARG, "qs_batch_create: circuit %d gate %zu uses a qubit >= %d", c, i, n_qubits[c]);
        if (r) break;
        auto ins = proto_of.emplace(signature(B->nq_eff[c], g, cnt), (int)proto_rep.size());
        if (ins.second) proto_rep.push_back(c);
        proto_id[c] = ins.first->second;
    }
    // Host work in parallel: the plan of each structure with its pass layouts,
    // then every circuit's block matrices rebound onto its structure's plan.
    const int nt = std::max(1, (int)std::min(16u, std::thread::hardware_concurrency()));
    auto parallel = [nt](int count, const std::function<void(int)> &f) {
        std::vector<std::thread> th;
        for (int t = 0; t < std::min(nt, count); ++t)
            th.emplace_back([&, t]() {
                for (int i = t; i < count; i += nt) f(i);
            });
        for (auto &x : th) x.join();
    };
    const int input_mode = o.max_sub <= 2 ? 0 : 1;   // tile-order staging, or per-row copies
    const int np = (int)proto_rep.size();
    protos.assign(np, nullptr);
    std::vector<std::vector<Layout>> p_layouts(np);
    std::vector<std::vector<LoadMap>> p_loads(np);
    std::vector<std::vector<qs_tmem::TLayout>> p_tl(np);
    std::vector<char> tl_ok(np, 1);
    bool want_tmem = o.tile_in_tmem && o.max_sub <= 2;
    std::vector<int> prc(np, QS_OK);
    std::vector<std::string> perr(np);
    if (!r)
        parallel(np, [&](int pi) {
            const int c = proto_rep[pi];
            int rr = qs_plan_create_ex(B->nq_eff[c], gates + offsets[c], offsets[c + 1] - offsets[c], &po, &protos[pi]);
            const qs_plan *pp = protos[pi];
            for (size_t u = 0; !rr && u < pp->passes.size(); ++u) {
                const PlanPass &pass = pp->passes[u];
                Layout L;
                LoadMap M;
                int qpos[3][5];
                for (size_t b = 0; b < pass.count; ++b)
                    for (int j = 0; j < 5; ++j) qpos[b][j] = pp->blocks[pass.first + b].q[j];
                int rows[3][7];
                if ((rr = qs_tile_row_orders(pp->n, pass.T, (int)pass.count, qpos, rows, nullptr, input_mode))) break;
                if ((rr = qs_tile_layout_build(pp->n, pass.T, (int)pass.count, qpos, rows, &L, &M))) break;
                L.pad = (int32_t)pass.first;
                p_layouts[pi].push_back(L);
                p_loads[pi].push_back(M);
                if (want_tmem && tl_ok[pi]) {
                    // the same pass for k_batch_tmem: in place, natural layout
                    qs_tiled_desc d;
                    memset(&d, 0, sizeof(d));
                    for (int t = 0; t < 12; ++t) d.T[t] = pass.T[t];
                    d.nsub = (int)pass.count;
                    for (size_t b = 0; b < pass.count; ++b)
                        for (int j = 0; j < 5; ++j) d.qpos[b][j] = qpos[b][j];
                    qs_tmem::TLayout TL;
                    if (qs_tmem_layout_build(pp->n, &d, &TL) == QS_OK) p_tl[pi].push_back(TL);
                    else tl_ok[pi] = 0;                         // this structure stays on k_batch
                }
            }
            if (rr) perr[pi] = qs_last_error();
            prc[pi] = rr;
        });
    for (int pi = 0; pi < np && !r; ++pi)
        if (prc[pi]) r = qs_fail(prc[pi], "qs_batch_create: circuit %d: %s", proto_rep[pi], perr[pi].c_str());
    if (!r) {
        std::vector<int> rc(n_circ, QS_OK);
        parallel(n_circ, [&](int c) {
            rc[c] = qs_plan_rebind(protos[proto_id[c]], gates + offsets[c], offsets[c + 1] - offsets[c], &plans[c]);
        });
        for (int c = 0; c < n_circ && !r; ++c)
            if (rc[c]) r = qs_fail(QS_ERR_ARG, "qs_batch_create: rebinding circuit %d failed", c);
    }
    // ---- device memory
    std::vector<Layout> layouts;                      // per proto, concatenated
    std::vector<LoadMap> loads;                       // their tile-order copy maps
    std::vector<qs_tmem::TLayout> tlayouts;           // and tensor-memory layouts (same indices)
    std::vector<size_t> layout_first(np);
    for (int pi = 0; pi < np && want_tmem; ++pi) want_tmem = tl_ok[pi] != 0;   // one kernel for the batch
    B->use_tmem = want_tmem;
    for (int pi = 0; pi < np && !r; ++pi) {
        layout_first[pi] = layouts.size();
        layouts.insert(layouts.end(), p_layouts[pi].begin(), p_layouts[pi].end());
        loads.insert(loads.end(), p_loads[pi].begin(), p_loads[pi].end());
        if (want_tmem) tlayouts.insert(tlayouts.end(), p_tl[pi].begin(), p_tl[pi].end());
    }
    std::vector<size_t> mat_off(n_circ);
    size_t mat_total = 0;
    B->amp_off.resize(n_circ);
    B->zz_off.resize(n_circ);
    for (int c = 0; c < n_circ && !r; ++c) {
        mat_off[c] = mat_total;
        mat_total += plans[c]->blocks.size() * 2 * 64 * 64;
        B->amp_off[c] = B->state_bytes;
        B->state_bytes += ((8ull << B->nq_eff[c]) + 255) & ~255ull;
        B->zz_off[c] = B->zz_count;
        B->zz_count += (size_t)(B->nq[c] - 1);
    }
    std::vector<BatchCirc> hc(n_circ);
    if (!r) {
        e = cudaMalloc(&B->d_states, B->state_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&B->d_mats, std::max<size_t>(mat_total * 2, 16));
        if (e == cudaSuccess) e = cudaMalloc(&B->d_layouts, std::max<size_t>(layouts.size() * sizeof(Layout), 16));
        if (e == cudaSuccess) e = cudaMalloc(&B->d_loads, std::max<size_t>(loads.size() * sizeof(LoadMap), 16));
        if (e == cudaSuccess && want_tmem)
            e = cudaMalloc(&B->d_tlayouts, std::max<size_t>(tlayouts.size() * sizeof(qs_tmem::TLayout), 16));
        if (e == cudaSuccess) e = cudaMalloc(&B->d_circ, sizeof(BatchCirc) * n_circ);
        if (e == cudaSuccess) e = cudaMalloc(&B->d_order, sizeof(int32_t) * n_circ);
        if (e == cudaSuccess) e = cudaMalloc((void **)&B->d_zz, std::max<size_t>(B->zz_count, 1) * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc((void **)&B->d_head, 2 * sizeof(int32_t));
        // The block matrices as BF16: a run of consecutive circuits at a time
        // is converted on the host threads into one of two pinned buffers
        // while the other's copy to the device is in flight.
        constexpr size_t kPerBlock = 2 * 64 * 64;     // BF16 values of one block (hi, lo)
        size_t chunk = 32ull << 20;                    // bytes per pinned buffer, at least one circuit's
        for (int c = 0; c < n_circ; ++c) chunk = std::max(chunk, plans[c]->blocks.size() * kPerBlock * 2);
        uint16_t *pin[2] = {nullptr, nullptr};
        cudaEvent_t copied[2] = {nullptr, nullptr};
        cudaStream_t up = nullptr;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking);
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
            e = cudaHostAlloc((void **)&pin[k], chunk, cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&copied[k], cudaEventDisableTiming);
        }
        bool in_flight[2] = {false, false};
        for (int c0 = 0, k = 0; c0 < n_circ && e == cudaSuccess; k ^= 1) {
            int c1 = c0;
            while (c1 < n_circ && (mat_off[c1] + plans[c1]->blocks.size() * kPerBlock - mat_off[c0]) * 2 <= chunk) ++c1;
            if (in_flight[k] && (e = cudaEventSynchronize(copied[k])) != cudaSuccess) break;
            uint16_t *buf = pin[k];
            const size_t base = mat_off[c0];
            parallel(c1 - c0, [&](int i) {
                const int c = c0 + i;
                for (size_t b = 0; b < plans[c]->blocks.size(); ++b)
                    qs_plan_block_bf16(plans[c], b, buf + (mat_off[c] - base) + b * kPerBlock);
            });
            const size_t elems = (c1 < n_circ ? mat_off[c1] : mat_total) - base;
            if (elems) {
                e = cudaMemcpyAsync(static_cast<uint16_t *>(B->d_mats) + base, buf, elems * 2, cudaMemcpyHostToDevice, up);
                if (e == cudaSuccess) e = cudaEventRecord(copied[k], up);
                in_flight[k] = e == cudaSuccess;
            }
            c0 = c1;
        }
        if (up) {
            const cudaError_t e2 = cudaStreamSynchronize(up);
            if (e == cudaSuccess) e = e2;
        }
        for (int k = 0; k < 2; ++k) {
            if (copied[k]) cudaEventDestroy(copied[k]);
            if (pin[k]) cudaFreeHost(pin[k]);
        }
        if (up) cudaStreamDestroy(up);
        if (e == cudaSuccess && !layouts.empty())
            e = cudaMemcpy(B->d_layouts, layouts.data(), layouts.size() * sizeof(Layout), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !loads.empty())
            e = cudaMemcpy(B->d_loads, loads.data(), loads.size() * sizeof(LoadMap), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && want_tmem && !tlayouts.empty())
            e = cudaMemcpy(B->d_tlayouts, tlayouts.data(), tlayouts.size() * sizeof(qs_tmem::TLayout),
                           cudaMemcpyHostToDevice);
        if (e != cudaSuccess) r = qs_cuda_fail(e, "qs_batch_create: device memory");
    }
    if (!r) {
        for (int c = 0; c < n_circ; ++c) {
            const qs_plan *pp = protos[proto_id[c]];
            BatchCirc &bc = hc[c];
            bc.amp = reinterpret_cast<float *>(static_cast<char *>(B->d_states) + B->amp_off[c]);
            bc.mats = static_cast<const uint16_t *>(B->d_mats) + mat_off[c];
            bc.layouts = static_cast<const Layout *>(B->d_layouts) + layout_first[proto_id[c]];
            bc.loads = static_cast<const LoadMap *>(B->d_loads) + layout_first[proto_id[c]];
            bc.tlayouts = want_tmem ? static_cast<const qs_tmem::TLayout *>(B->d_tlayouts) + layout_first[proto_id[c]]
                                    : nullptr;
            bc.zz = B->d_zz + B->zz_off[c];
            bc.npass = (int32_t)pp->passes.size();
            bc.nq = B->nq[c];
            bc.nq_eff = B->nq_eff[c];
        }
        // processing order: longest first (tiles x passes), or as given
        B->order.resize(n_circ);
        for (int c = 0; c < n_circ; ++c) B->order[c] = c;
        if (o.order == QS_BATCH_LONGEST_FIRST)
            std::stable_sort(B->order.begin(), B->order.end(), [&](int32_t a, int32_t b) {
                return (double)hc[a].npass * (double)(1ull << hc[a].nq_eff) >
                       (double)hc[b].npass * (double)(1ull << hc[b].nq_eff);
            });
        e = cudaMemcpy(B->d_circ, hc.data(), sizeof(BatchCirc) * n_circ, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(B->d_order, B->order.data(), sizeof(int32_t) * n_circ, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) r = qs_cuda_fail(e, "qs_batch_create: tables");
    }
    for (qs_plan *p : plans) qs_plan_destroy(p);
    for (qs_plan *p : protos) qs_plan_destroy(p);
    if (r) { batch_free(B); return r; }
    *out = B;
    return QS_OK;
}

namespace {

int batch_launch(qs_batch *B, cudaStream_t st)
{
    QS_CUDA_TRY(cudaMemsetAsync(B->d_head, 0, 2 * sizeof(int32_t), st));
    BatchParams P;
    P.circ = static_cast<const BatchCirc *>(B->d_circ);
    P.order = static_cast<const int32_t *>(B->d_order);
    P.ncirc = B->n;
    P.head = B->d_head;
    P.err = B->d_head + 1;
    if (B->use_tmem) {
        const unsigned grid = (unsigned)std::min(B->n, QS_SM_COUNT * kTmCtasPerSm);
        k_batch_tmem<<<grid, kTmThreads, kTmSmemBytes, st>>>(P);
    } else if (B->opts.max_sub <= 2) {
        const unsigned grid = (unsigned)std::min(B->n, QS_SM_COUNT * BShape<2>::kCtasPerSm);
        k_batch<2><<<grid, kThreads, BShape<2>::kSmemBytes, st>>>(P);
    } else {
        const unsigned grid = (unsigned)std::min(B->n, QS_SM_COUNT * BShape<3>::kCtasPerSm);
        k_batch<3><<<grid, kThreads, BShape<3>::kSmemBytes, st>>>(P);
    }
    QS_LAUNCH_CHECK("k_batch");
    return QS_OK;
}

}  // namespace

extern "C" int qs_batch_run(qs_batch *B, void *stream)
{
    if (!B) return qs_fail(QS_ERR_ARG, "qs_batch_run: null batch");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    QS_CUDA_TRY(cudaFuncSetAttribute(k_batch<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, BShape<2>::kSmemBytes));
    QS_CUDA_TRY(cudaFuncSetAttribute(k_batch<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, BShape<3>::kSmemBytes));
    QS_CUDA_TRY(cudaFuncSetAttribute(k_batch_tmem, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmSmemBytes));
    if (!B->opts.use_graph) return batch_launch(B, st);
    if (!B->graph_exec) {
        // capture once on a private stream; replay on the caller's stream
        if (!B->graph_stream) QS_CUDA_TRY(cudaStreamCreateWithFlags(&B->graph_stream, cudaStreamNonBlocking));
        QS_CUDA_TRY(cudaStreamBeginCapture(B->graph_stream, cudaStreamCaptureModeThreadLocal));
        int r = batch_launch(B, B->graph_stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(B->graph_stream, &g);
        if (r) { if (g) cudaGraphDestroy(g); return r; }
        if (e != cudaSuccess) return qs_cuda_fail(e, "qs_batch_run: capture");
        B->graph = g;
        QS_CUDA_TRY(cudaGraphInstantiate(&B->graph_exec, B->graph, 0));
    }
    QS_CUDA_TRY(cudaGraphLaunch(B->graph_exec, st));
    return QS_OK;
}

extern "C" int qs_batch_zz(qs_batch *B, double *out, size_t *count)
{
    if (!B || !count) return qs_fail(QS_ERR_ARG, "qs_batch_zz: null argument");
    *count = B->zz_count;
    if (!out) return QS_OK;
    QS_CUDA_TRY(cudaDeviceSynchronize());
    int32_t flag[2] = {0, 0};
    QS_CUDA_TRY(cudaMemcpy(flag, B->d_head, sizeof(flag), cudaMemcpyDeviceToHost));
    if (flag[1] == 2) return qs_fail(QS_ERR_STATE, "qs_batch: dynamic shared memory not 1024-byte aligned");
    if (flag[1]) return qs_fail(QS_ERR_STATE, "qs_batch: a bounded wait in the batch kernel expired");
    QS_CUDA_TRY(cudaMemcpy(out, B->d_zz, B->zz_count * sizeof(double), cudaMemcpyDeviceToHost));
    return QS_OK;
}

extern "C" int qs_batch_zz_offsets(const qs_batch *B, size_t *offsets)
{
    if (!B || !offsets) return qs_fail(QS_ERR_ARG, "qs_batch_zz_offsets: null argument");
    for (int c = 0; c < B->n; ++c) offsets[c] = B->zz_off[c];
    offsets[B->n] = B->zz_count;
    return QS_OK;
}

extern "C" int qs_batch_state(qs_batch *B, int c, void *host_out, int host_dtype)
{
    if (!B || c < 0 || c >= B->n || !host_out) return qs_fail(QS_ERR_ARG, "qs_batch_state: bad arguments");
    if (host_dtype != QS_C64 && host_dtype != QS_C128) return qs_fail(QS_ERR_ARG, "qs_batch_state: bad dtype");
    QS_CUDA_TRY(cudaDeviceSynchronize());
    const size_t N = 1ull << B->nq[c];               // idle padding qubits are |0>: the first 2^nq amplitudes
    std::vector<float> tmp(2 * N);
    QS_CUDA_TRY(cudaMemcpy(tmp.data(), static_cast<char *>(B->d_states) + B->amp_off[c], 8 * N,
                           cudaMemcpyDeviceToHost));
    if (host_dtype == QS_C64) memcpy(host_out, tmp.data(), 8 * N);
    else
        for (size_t i = 0; i < 2 * N; ++i) static_cast<double *>(host_out)[i] = tmp[i];
    return QS_OK;
}

extern "C" int qs_batch_info(const qs_batch *B, size_t *state_bytes, size_t *passes_total)
{
    if (!B) return qs_fail(QS_ERR_ARG, "qs_batch_info: null batch");
    if (state_bytes) *state_bytes = B->state_bytes;
    if (passes_total) *passes_total = 0;
    return QS_OK;
}

extern "C" int qs_batch_destroy(qs_batch *B)
{
    if (!B) return QS_OK;
    cudaDeviceSynchronize();
    if (B->graph_stream) cudaStreamDestroy(B->graph_stream);
    batch_free(B);
    return QS_OK;
}

// Autotuner: time candidate options on a sample of the circuits (every
// `stride`-th one) and return the fastest.  Candidates: blocks per pass
// (1, 2, 3) x lowest tile qubits (3, 5) x queue order (longest first, as
// given).  Each candidate is built, run once untimed, then timed over two runs
// with CUDA events on a private stream.
extern "C" int qs_batch_autotune(int n_circ, const int *n_qubits, const qs_gate *gates, const size_t *offsets,
                                 int stride, qs_batch_opts *best, double *best_ms)
{
    if (!best || n_circ < 1 || stride < 1) return qs_fail(QS_ERR_ARG, "qs_batch_autotune: bad arguments");
    std::vector<int> nq;
    std::vector<qs_gate> g;
    std::vector<size_t> off(1, 0);
    for (int c = 0; c < n_circ; c += stride) {
        nq.push_back(n_qubits[c]);
        g.insert(g.end(), gates + offsets[c], gates + offsets[c + 1]);
        off.push_back(g.size());
    }
    cudaStream_t st;
    QS_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double bt = 1e300;
    int r = QS_OK;
    for (int bq : {5, 4})
    for (int ms : {1, 2, 3})
        for (int lq : {3, 5})
            for (int order : {QS_BATCH_LONGEST_FIRST, QS_BATCH_INPUT_ORDER}) {
                qs_batch_opts o;
                qs_batch_default_opts(&o);
                o.block_qubits = bq;
                o.max_sub = ms;
                o.low_qubits = lq;
                o.order = order;
                o.use_graph = 0;
                qs_batch *b = nullptr;
                if ((r = qs_batch_create((int)nq.size(), nq.data(), g.data(), off.data(), &o, &b))) goto done;
                if ((r = qs_batch_run(b, st))) { qs_batch_destroy(b); goto done; }
                cudaEventRecord(e0, st);
                for (int k = 0; k < 2 && !r; ++k) r = qs_batch_run(b, st);
                cudaEventRecord(e1, st);
                cudaStreamSynchronize(st);
                float t = 0;
                cudaEventElapsedTime(&t, e0, e1);
                size_t cnt = 0;
                if (!r) r = qs_batch_zz(b, nullptr, &cnt);
                qs_batch_destroy(b);
                if (r) goto done;
                if (t / 2 < bt) {
                    bt = t / 2;
                    *best = o;
                }
            }
done:
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (r) return r;
    best->use_graph = 1;
    if (best_ms) *best_ms = bt;
    return QS_OK;
}

// ---------------------------------------------------------------- tuning cache
namespace {

// FNV-1a over the device and the sampled circuits' gate pattern.
uint64_t tune_key(int n_circ, const int *n_qubits, const qs_gate *gates, const size_t *offsets, int stride,
                  int dev)
{
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; ++i) { h ^= c[i]; h *= 1099511628211ull; }
    };
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
        mix(prop.name, strlen(prop.name));
        mix(&prop.multiProcessorCount, sizeof(int));
    }
    mix(&stride, sizeof(int));
    for (int c = 0; c < n_circ; c += stride) {
        mix(&n_qubits[c], sizeof(int));
        for (size_t i = offsets[c]; i < offsets[c + 1]; ++i) {
            const qs_gate &g = gates[i];
            mix(&g.op, sizeof(int32_t));
            mix(&g.dagger, sizeof(int32_t));
            mix(g.q, sizeof(g.q));
            mix(&g.nctrl, sizeof(int32_t));
            mix(g.ctrl, sizeof(int32_t) * (size_t)std::max(0, std::min(g.nctrl, QS_MAX_CTRL)));
        }
    }
    return h;
}

}  // namespace

extern "C" int qs_batch_autotune_cached(int n_circ, const int *n_qubits, const qs_gate *gates,
                                        const size_t *offsets, int stride, const char *cache_path,
                                        qs_batch_opts *best, double *best_ms, int *from_cache)
{
    if (!best || !cache_path || n_circ < 1 || stride < 1 || !n_qubits || !offsets)
        return qs_fail(QS_ERR_ARG, "qs_batch_autotune_cached: bad arguments");
    int dev = 0;
    QS_CUDA_TRY(cudaGetDevice(&dev));
    const uint64_t key = tune_key(n_circ, n_qubits, gates, offsets, stride, dev);
    if (from_cache) *from_cache = 0;
    if (FILE *f = fopen(cache_path, "r")) {
        char line[256];
        while (fgets(line, sizeof(line), f)) {
            unsigned long long k = 0;
            int ms, lq, order, bq, tm;
            double t;
            if (sscanf(line, "%llx %d %d %d %d %d %lf", &k, &ms, &lq, &order, &bq, &tm, &t) == 7 && k == key) {
                qs_batch_default_opts(best);
                best->max_sub = ms;
                best->low_qubits = lq;
                best->order = order;
                best->block_qubits = bq;
                best->tile_in_tmem = tm;
                if (best_ms) *best_ms = t;
                if (from_cache) *from_cache = 1;
                fclose(f);
                return QS_OK;
            }
        }
        fclose(f);
    }
    double t = 0;
    int r = qs_batch_autotune(n_circ, n_qubits, gates, offsets, stride, best, &t);
    if (r) return r;
    if (best_ms) *best_ms = t;
    FILE *f = fopen(cache_path, "a");
    if (!f) return qs_fail(QS_ERR_IO, "qs_batch_autotune_cached: cannot write %s", cache_path);
    fprintf(f, "%016llx %d %d %d %d %d %.6f\n", (unsigned long long)key, best->max_sub, best->low_qubits,
            best->order, best->block_qubits, best->tile_in_tmem, t);
    fclose(f);
    return QS_OK;
}
