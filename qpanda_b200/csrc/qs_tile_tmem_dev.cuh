// qs_tile_tmem_dev.cuh - device helpers of the tiled passes that hold the
// tile in tensor memory: k_tile_tmem (qs_tile_tmem.cu, one pass over a state)
// and k_batch_tmem (qs_batch_tmem.cu, all passes of many circuits).  The
// layout tables they read are qs_tmem::TLayout (qs_tile_tmem.cuh).
#pragma once

#include "qs_tile_core.cuh"
#include "qs_tile_tmem.cuh"

namespace qs_tmem_dev {

using namespace qs_tile;
using qs_tmem::TLayout;

// Named barrier of the NT threads of one lane group.
template <int NT>
__device__ __forceinline__ void group_bar(int id)
{
    asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(NT) : "memory");
}

template <int NT>
__device__ __forceinline__ bool group_bar_or(int id, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r) : "r"((uint32_t)v), "r"(id), "r"(NT) : "memory");
    return r != 0;
}

// tile_base / tile_base_advance on the TLayout's positions
__device__ __forceinline__ uint64_t tbase_of(uint64_t tile, const TLayout &L)
{
#pragma unroll 4
    for (int j = 0; j < 12; ++j) {
        const uint64_t low = (1ull << L.tpos[j]) - 1;
        tile = ((tile & ~low) << 1) | (tile & low);
    }
    return tile;
}

// Block matrices into the swizzled B layout, each permuted to this kernel's
// column order (register bit p = matrix bit mperm[b][p], for rows and
// columns alike); block 0's scaled by `scale` (hi + lo recombined, scaled,
// split again).
__device__ inline void load_b_perm(uint8_t *dst, const uint16_t *mat, const TLayout &L, float scale)
{
    const int total = L.nsub * 64 * 32;
    for (int it = threadIdx.x; it < total; it += blockDim.x) {
        const int b = it >> 11, np = (it >> 5) & 63, cp = it & 31;
        const uint32_t n = 2 * qs_tmem::tmem_matrix_index((uint32_t)np >> 1, L.mperm[b]) + (np & 1);
        const uint32_t k = 2 * qs_tmem::tmem_matrix_index((uint32_t)cp, L.mperm[b]);
        const uint16_t *src = mat + (size_t)b * 2 * 4096;
        uint32_t hi = *reinterpret_cast<const uint32_t *>(src + n * 64 + k);
        uint32_t lo = *reinterpret_cast<const uint32_t *>(src + 4096 + n * 64 + k);
        if (b == 0 && scale != 1.0f) {
            const float a = (__uint_as_float(hi << 16) + __uint_as_float(lo << 16)) * scale;
            const float c = (__uint_as_float(hi & 0xffff0000u) + __uint_as_float(lo & 0xffff0000u)) * scale;
            split_pair(a, c, hi, lo);
        }
        const uint32_t off = qs_tmem::tmem_b_offset((uint32_t)np, 2u * cp);
        *reinterpret_cast<uint32_t *>(dst + (2 * b) * kB + off) = hi;
        *reinterpret_cast<uint32_t *>(dst + (2 * b + 1) * kB + off) = lo;
    }
}

// D (TMEM) = A_hi B_hi + A_hi B_lo + A_lo B_hi with A in TMEM (hi at a_tmem,
// lo 32 columns further), B in shared memory; 12 MMAs of K = 16, then commit.
__device__ __forceinline__ void issue_ts(uint32_t d_tmem, uint32_t a_tmem, uint32_t b_hi, uint32_t b_lo,
                                         uint32_t mbar)
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint64_t dBh = umma_desc(b_hi), dBl = umma_desc(b_lo);
#pragma unroll
    for (int pr = 0; pr < 3; ++pr) {
        const uint32_t a = a_tmem + (pr == 2 ? 32u : 0u);
        const uint64_t db = pr == 1 ? dBl : dBh;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t acc = (pr | k) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %3, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %4, p;\n\t}\n"
                :
                : "r"(d_tmem), "r"(a + 8u * k), "l"(db + 2ull * k), "r"(acc), "r"(kIdesc));
        }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(mbar) : "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
        :: "r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
           "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]),
           "r"(v[15])
        : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *y)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; ++i) y[i] = __uint_as_float(r[i]);
}

// The thread's row values (32 / TPR complex, y[2j] real, y[2j+1] imaginary:
// its columns c0 .. c0 + 32 / TPR - 1) as BF16 hi/lo pairs into its TMEM
// lane: hi at columns a + c0.., lo at a + 32 + c0.., 16 columns at a time.
template <int TPR>
__device__ __forceinline__ void split_store(uint32_t taddr, const float (&y)[64 / TPR], uint32_t c0)
{
#pragma unroll
    for (int h = 0; h < 2 / TPR; ++h) {
        uint32_t hv[16], lv[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) split_pair(y[32 * h + 2 * j], y[32 * h + 2 * j + 1], hv[j], lv[j]);
        tmem_st16(taddr + c0 + 16 * h, hv);
        tmem_st16(taddr + 32 + c0 + 16 * h, lv);
    }
}

// Sum of squares in four independent chains (fixed order).
template <int NV>
__device__ __forceinline__ float sum_squares(const float (&y)[NV])
{
    float t[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < NV; ++i) t[i & 3] = fmaf(y[i], y[i], t[i & 3]);
    return (t[0] + t[1]) + (t[2] + t[3]);
}

// Between two blocks: the thread's results (y[2j], y[2j+1] = its register j)
// to their slots of the staging buffer (xw ^ wcol[j]), a barrier of the group,
// then its part of the next block's row from slots xr ^ rcol[j].  8-byte
// accesses; the swizzle makes each half warp's 16 accesses hit distinct
// banks.  xw / xr include the thread's column base (the tables are linear).
template <int TPR, int NT>
__device__ __forceinline__ void exchange_through(float (&y)[64 / TPR], uint32_t stage, uint32_t xw, uint32_t xr,
                                                 const uint16_t *wcol, const uint16_t *rcol, int bar_id)
{
#pragma unroll
    for (int j = 0; j < 32 / TPR; ++j)
        asm volatile("st.shared.v2.f32 [%0], {%1, %2};"
                     :: "r"(stage + ((xw ^ wcol[j]) << 3)), "f"(y[2 * j]), "f"(y[2 * j + 1]) : "memory");
    group_bar<NT>(bar_id);
#pragma unroll
    for (int j = 0; j < 32 / TPR; ++j)
        asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];"
                     : "=f"(y[2 * j]), "=f"(y[2 * j + 1]) : "r"(stage + ((xr ^ rcol[j]) << 3)) : "memory");
}

// The group's copies of a tile: chunk c = 128 k + t (tile indices 2c, 2c+1,
// adjacent in memory) to stage chunk c ^ cf_t ^ cf_k[k]; with TPR = 2 the
// group's 256 threads take chunks 256 kk + t (k = 2 kk + bit 7 of t, that bit
// folded into g_t / cs_t by the caller: the tables are linear in k).
template <int TPR>
__device__ __forceinline__ void copy_tile(const float *amp, uint64_t base, const TLayout &L, uint32_t stage,
                                          uint64_t g_t, uint32_t cs_t)
{
#pragma unroll
    for (int kk = 0; kk < 16 / TPR; ++kk) {
        const int k = TPR * kk;
        const float *src = amp + 2 * (base | g_t | L.gk[k]);
        const uint32_t dst = stage + ((cs_t ^ ((uint32_t)k << 7) ^ L.cf_k[k]) << 4);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}


}  // namespace qs_tmem_dev
