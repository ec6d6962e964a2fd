// qs_tile_core.cuh - device building blocks of the tiled tensor-core passes
// (qs_fused2.cu: one circuit, many CTAs; qs_batch.cu: many circuits, one CTA
// each).  A tile is 4096 complex64 amplitudes that differ in 12 tile qubits;
// for a 5-qubit block it is 128 rows (7 tile bits) x 32 columns (the block's
// 5 bits).  Thread i of 128 owns row i and TMEM lane i (with two threads per
// row, threads i and 128 + i share row i, 16 columns each).
#pragma once

#include <cuda_bf16.h>

#include "qs_common.cuh"

namespace qs_tile {

constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kA = 128 * 64 * 2;             // 16 KB: one BF16 A buffer (128 rows x 64)
constexpr uint32_t kB = 64 * 64 * 2;              //  8 KB: one BF16 B buffer
constexpr uint32_t kStage = 128 * 256;            // 32 KB: 128 rows x 32 complex64
constexpr int kMaxSub = 3;
// instruction descriptor: D f32 (bits 4-5 = 1), A and B bf16 (7-9, 10-12 = 1),
// both K-major, N = 64 (N>>3 at 17-22), M = 128 (M>>4 at 24-28)
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(64 >> 3) << 17) |
                            ((uint32_t)(128 >> 4) << 24);
constexpr unsigned long long kWaitNs = 2000000000ull;   // bound on every wait

// Layout of one pass over a tile: where block 0's rows come from, how each
// block's results feed the next block's rows and columns, where the last
// block's results go.  Built on the host (qs_tile_layout_build).
struct Layout {
    uint64_t tmask;              // the 12 tile positions as a bit mask
    uint64_t g0[32];             // global offset of column j, block 0
    uint64_t gl[32];             // global offset of column j, last block
    int32_t c0_glob[7];          // global position of row bit i, block 0
    int32_t cl_glob[7];          // global position of row bit i, last block
    int32_t nsub, vec0, vecl, pad;
    int8_t tpos[12];             // global position of tile bit i (= T[i], ascending)
    int8_t cl_loc[7];            // tile bit of row bit i, last block
    int8_t pad2;
    uint16_t lout[32];           // tile bits of column j, last block (a 12-bit tile index)
    int8_t rowmap[kMaxSub - 1][7];   // row bit i of block b -> row bit (>= 0) or ~column bit of block b+1
    // Byte offset, within block b+1's swizzled A buffer, of the result in
    // column j of block b is  thread_part ^ scat[b][j]: the row/column bits a
    // result gets in block b+1 come either from the thread's row or from j,
    // never both, so the swizzled offset splits into two XOR-able halves.
    uint16_t scat[kMaxSub - 1][32];
    uint8_t tabR[kMaxSub - 1][32];   // column j of block b -> row bits of block b+1
    uint8_t tabJ[kMaxSub - 1][32];   // column j of block b -> column bits of block b+1
};

// Warp-contiguous copies of block 0's input (prefetch_tile): chunk c of a
// tile holds tile indices 2c, 2c+1, with c = 128 k + thread.  Built on the
// host beside the Layout (qs_tile_layout_build).
struct LoadMap {
    uint64_t gk[16];             // tile index bits 8..11 = k: global offset
    uint8_t rk[16];              //   ... block-0 row bits
    uint8_t jk[16];              //   ... block-0 column bits
    int8_t tpos[12];             // global position of tile bit t
    int8_t tmap0[12];            // tile bit t in block 0: row bit (>= 0) or ~column bit
    // A chunk's second amplitude (tile bit 0 set) sits at (row ^ dr, column ^ dj)
    // of the first; pair = 1 when tile bit 0 is block 0's column bit 0 (dj = 1,
    // dr = 0: the two are adjacent columns of one row).
    uint8_t dr, dj, pair;
    int8_t pad[5];
};

// Thread part of the scatter offset (see Layout::scat).
__device__ __forceinline__ uint32_t scatter_thread_part(const Layout &L, int t, int row)
{
    uint32_t r2 = 0, j2 = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b) {
        const uint32_t bit = (row >> b) & 1;
        const int m = L.rowmap[t][b];
        if (m >= 0) r2 |= bit << m;
        else j2 |= bit << (~m);
    }
    return (r2 << 7) | ((((j2 >> 2) ^ (r2 & 7)) & 7) << 4) | ((j2 & 3) << 2);
}

// Global offset of amplitude 0 of tile `tile`: the tile index with zeros
// inserted at the 12 tile positions.  Called once per kernel; the loop is
// deliberately not unrolled fully (a fully unrolled copy inside the tile loop
// made the pass 1.85x slower).
__device__ __forceinline__ uint64_t tile_base(uint64_t tile, const Layout &L)
{
#pragma unroll 4
    for (int j = 0; j < 12; ++j) {
        const uint64_t low = (1ull << L.tpos[j]) - 1;
        tile = ((tile & ~low) << 1) | (tile & low);
    }
    return tile;
}

// tile_base(t + d) from base = tile_base(t) and step = tile_base(d): with the
// tile positions set to one, the carries of the add run across them.
__device__ __forceinline__ uint64_t tile_base_advance(uint64_t base, uint64_t step, uint64_t tmask)
{
    return ((base | tmask) + step) & ~tmask;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Stores to shared memory by 32-bit shared-window address (st.shared, never
// the generic path).
__device__ __forceinline__ void sts32(uint32_t addr, uint32_t v)
{
    asm volatile("st.shared.b32 [%0], %1;" :: "r"(addr), "r"(v));
}
__device__ __forceinline__ void sts64(uint32_t addr, uint32_t a, uint32_t b)
{
    asm volatile("st.shared.v2.b32 [%0], {%1, %2};" :: "r"(addr), "r"(a), "r"(b));
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, rows of 128 B in
// 8-row groups 1024 B apart, version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase: false after limit_ns (kWaitNs).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, unsigned long long limit_ns = kWaitNs)
{
    const unsigned long long t0 = globaltimer();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (globaltimer() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(acc));
}

// D = A_hi*B_hi + A_hi*B_lo + A_lo*B_hi (12 MMAs of K = 16), then commit.
__device__ __forceinline__ void issue_block_mma(uint32_t tmem, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi,
                                                uint32_t b_lo, uint32_t mbar)
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint64_t dAh = umma_desc(a_hi), dAl = umma_desc(a_lo), dBh = umma_desc(b_hi), dBl = umma_desc(b_lo);
#pragma unroll
    for (int k = 0; k < 4; ++k) mma_bf16(tmem, dAh + 2 * k, dBh + 2 * k, k > 0);
#pragma unroll
    for (int k = 0; k < 4; ++k) mma_bf16(tmem, dAh + 2 * k, dBl + 2 * k, 1);
#pragma unroll
    for (int k = 0; k < 4; ++k) mma_bf16(tmem, dAl + 2 * k, dBh + 2 * k, 1);
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(mbar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Staging row of thread `row`: 16 chunks of 16 B (2 amplitudes), chunk k at
// position k ^ (row & 15) so that a quarter warp's 8 rows hit distinct banks.
__device__ __forceinline__ uint32_t stage_addr(uint32_t stage, int row, int chunk)
{
    return stage + row * 256 + ((chunk ^ (row & 15)) << 4);
}

// Asynchronous copies of this thread's row of block 0 (tile base `base`)
// into its staging row.  L2-only copies (.cg) when columns come in 16-byte
// pairs; 8-byte copies otherwise.
__device__ __forceinline__ void prefetch_row(const float *amp, uint64_t base, const Layout &L, uint32_t stage,
                                             int row)
{
    if (L.vec0) {
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            const float *src = amp + 2 * (base | L.g0[j]);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(stage_addr(stage, row, j >> 1)),
                         "l"(src) : "memory");
        }
    } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const float *src = amp + 2 * (base | L.g0[j]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;"
                         :: "r"(stage_addr(stage, row, j >> 1) + ((j & 1) << 3)), "l"(src) : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Per-thread part of prefetch_tile's addresses: tile index bits 1..7 = the
// thread's index within its 128.
struct ChunkBase {
    uint64_t g;
    uint32_t r, j;
};

// t: the thread's index among the lane's nt = 128 x tpr threads, which copy
// chunks c = nt k + t: tile index bits 1 .. log2(nt) come from t.
template <int TPR = 1>
__device__ __forceinline__ ChunkBase chunk_base(const LoadMap &L, int t128)
{
    ChunkBase c{0, 0, 0};
    constexpr int kBits = TPR == 2 ? 9 : 8;
#pragma unroll
    for (int t = 1; t < kBits; ++t) {
        if (!((t128 >> (t - 1)) & 1)) continue;
        c.g |= 1ull << L.tpos[t];
        const int m = L.tmap0[t];
        if (m >= 0) c.r |= 1u << m;
        else c.j |= 1u << (~m);
    }
    return c;
}

// Tile-order staging (k_fused_tile): chunk c of the tile - tile indices 2c,
// 2c+1 - is copied to byte 16c, chunk c = 128 k + thread, so the 32 lanes of a
// warp fill 512 contiguous bytes of shared memory per copy instruction, however
// short the tile's contiguous runs in global memory are.  Each thread later
// reads back only its own chunks (convert_load): no barrier separates the
// copies from the reads, nor the reads from the next tile's copies.
// With tpr threads per row the lane's 128 tpr threads each copy 16 / tpr
// chunks, c = 128 tpr k + t; tile index bits above log2(128 tpr) come from k,
// so the LoadMap's tables (indexed by tile bits 8..11) are read at k tpr.
template <int TPR = 1>
__device__ __forceinline__ void prefetch_tile_linear(const float *amp, uint64_t base, const LoadMap &M,
                                                     uint32_t stage, uint64_t g_thread, int t128)
{
#pragma unroll
    for (int k = 0; k < 16 / TPR; ++k) {
        const float *src = amp + 2 * (base | g_thread | M.gk[k * TPR]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;"
                     :: "r"(stage + (uint32_t)(128 * TPR * k + t128) * 16u), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void read_stage_row(uint32_t stage, int row, float (&x)[64])
{
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        float4 v;
        asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                     : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(stage_addr(stage, row, k)));
        x[4 * k] = v.x; x[4 * k + 1] = v.y; x[4 * k + 2] = v.z; x[4 * k + 3] = v.w;
    }
}

// BF16 hi/lo split of a complex pair: hi = bf16(x), lo = bf16(x - hi).
__device__ __forceinline__ void split_pair(float re, float im, uint32_t &hv, uint32_t &lv)
{
    hv = pack_bf16x2(re, im);
    lv = pack_bf16x2(re - __uint_as_float(hv << 16), im - __uint_as_float(hv & 0xffff0000u));
}

// Byte offset of (row r, column j) in a swizzled K-major A buffer.
__device__ __forceinline__ uint32_t a_offset(uint32_t r, uint32_t j)
{
    return r * 128 + ((((j >> 2) ^ (r & 7)) & 7) << 4) + ((j & 3) << 2);
}

// Block 0's input in two steps, so that the wait for the tensor cores to
// release the A buffers can sit between them (k_fused_tile):
// convert_load reads the thread's own staged chunks (all reads issued before
// the first use) and splits them into BF16 hi/lo pairs in registers, returning
// their sum of squares; convert_store writes the pairs at their block-0 rows
// and columns of the swizzled A buffers.  Column pairs (tile bit 0 = block-0
// column bit 0) go out as one 8-byte store per buffer; otherwise the two
// amplitudes of a chunk sit at (r, j) and (r | dr, j | dj) and go out as
// 4-byte stores.
template <int TPR = 1>
__device__ __forceinline__ float convert_load(uint32_t stage, int t128, uint32_t (&hv)[16 / TPR][2],
                                              uint32_t (&lv)[16 / TPR][2])
{
    constexpr int kChunks = 16 / TPR;
    float4 vv[kChunks];
#pragma unroll
    for (int k = 0; k < kChunks; ++k)
        asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                     : "=f"(vv[k].x), "=f"(vv[k].y), "=f"(vv[k].z), "=f"(vv[k].w)
                     : "r"(stage + (uint32_t)(128 * TPR * k + t128) * 16u));
    float ss = 0.f;
#pragma unroll
    for (int k = 0; k < kChunks; ++k) {
        const float4 v = vv[k];
        ss = fmaf(v.x, v.x, fmaf(v.y, v.y, fmaf(v.z, v.z, fmaf(v.w, v.w, ss))));
        split_pair(v.x, v.y, hv[k][0], lv[k][0]);
        split_pair(v.z, v.w, hv[k][1], lv[k][1]);
    }
    return ss;
}

template <int TPR = 1>
__device__ __forceinline__ void convert_store(uint8_t *aHi, uint8_t *aLo, const LoadMap &M, const ChunkBase &cb,
                                              const uint32_t (&hv)[16 / TPR][2], const uint32_t (&lv)[16 / TPR][2])
{
    constexpr int kChunks = 16 / TPR;
    const uint32_t hi_s = smem_u32(aHi), lo_s = smem_u32(aLo);
#pragma unroll
    for (int k = 0; k < kChunks; ++k) {
        const uint32_t row = cb.r ^ M.rk[k * TPR], j = cb.j ^ M.jk[k * TPR];
        if (M.pair) {
            const uint32_t off = a_offset(row, j);            // j even: columns j, j+1 are adjacent
            sts64(hi_s + off, hv[k][0], hv[k][1]);
            sts64(lo_s + off, lv[k][0], lv[k][1]);
        } else {
            const uint32_t o0 = a_offset(row, j), o1 = a_offset(row | M.dr, j | M.dj);
            sts32(hi_s + o0, hv[k][0]);
            sts32(lo_s + o0, lv[k][0]);
            sts32(hi_s + o1, hv[k][1]);
            sts32(lo_s + o1, lv[k][1]);
        }
    }
}

// Where a pass writes a tile's results (k_fused_tile).  The 12 tile bits go
// to the positions in the Layout's gl / cl_glob; the tile index bits (the
// other n - 12 positions, ascending as read) go to
//   mode 0: the positions they were read from (the pass writes in place);
//   mode 1: positions 12, 13, ... (a tile's results are one contiguous run);
//   mode 2: wpos[i] for tile index bit i.
struct StoreMap {
    int32_t mode;
    int32_t ntb;                 // tile index bits (n - 12)
    int8_t wpos[52];
};

// Global offset of a tile's results (see StoreMap).
__device__ __forceinline__ uint64_t store_base(uint64_t tile, uint64_t read_base, const StoreMap &W)
{
    if (W.mode == 0) return read_base;
    if (W.mode == 1) return tile << 12;
    uint64_t b = 0;
    for (int i = 0; i < W.ntb; ++i) b |= ((tile >> i) & 1ull) << W.wpos[i];
    return b;
}

// One complex amplitude as BF16 hi/lo pairs at row r, column j of the
// swizzled K-major A buffers.
__device__ __forceinline__ void a_store_pair(uint8_t *aHi, uint8_t *aLo, int r, int j, float re, float im)
{
    uint32_t hv, lv;
    split_pair(re, im, hv, lv);
    const uint32_t off = r * 128 + ((((j >> 2) ^ (r & 7))) << 4) + ((j & 3) << 2);
    *reinterpret_cast<uint32_t *>(aHi + off) = hv;
    *reinterpret_cast<uint32_t *>(aLo + off) = lv;
}

// One complex amplitude as BF16 hi/lo pairs at byte offset `off` of the A buffers.
__device__ __forceinline__ void a_store_at(uint8_t *aHi, uint8_t *aLo, uint32_t off, float re, float im)
{
    uint32_t hv, lv;
    split_pair(re, im, hv, lv);
    sts32(smem_u32(aHi) + off, hv);
    sts32(smem_u32(aLo) + off, lv);
}

// B operands of a pass (nsub blocks, hi and lo each) into the swizzled layout.
__device__ __forceinline__ void load_b(uint8_t *dst, const uint16_t *mat, int nsub)
{
    for (int c = threadIdx.x; c < nsub * 2 * 64 * 8; c += kThreads) {
        const int mtx = c / (64 * 8), row = (c / 8) % 64, ch = c % 8;
        uint4 v = *reinterpret_cast<const uint4 *>(mat + (size_t)mtx * 64 * 64 + row * 64 + ch * 8);
        *reinterpret_cast<uint4 *>(dst + mtx * kB + row * 128 + ((ch ^ (row & 7)) << 4)) = v;
    }
}

}  // namespace qs_tile

// Host: the Layout of a pass with tile qubits T[12] (ascending, global) and
// nsub blocks on qpos[b][5] (ascending, within T).  QS_OK or QS_ERR_ARG.
// T: the 12 tile positions, ascending; qpos[b]: block b's 5 positions in
// column-bit order (distinct tile positions); rows[b]: its other 7 in row-bit
// order (NULL: ascending).  With M non-null, also the LoadMap of
// prefetch_tile.  With wtile non-null, results are written with tile bit l at
// position wtile[l] instead of T[l] (the last block's gl and cl_glob).
int qs_tile_layout_build(int n, const int *T, int nsub, const int (*qpos)[5], const int (*rows)[7],
                         qs_tile::Layout *L, qs_tile::LoadMap *M = nullptr, const int *wtile = nullptr);
