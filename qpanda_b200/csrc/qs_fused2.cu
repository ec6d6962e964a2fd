// qs_fused2.cu - tiled fused passes: up to three 5-qubit blocks per read and
// write of the state, on the tensor cores (complex64).
//
// A pass owns 12 tile qubits T (ascending; the lowest ones always included so
// that rows are runs of contiguous amplitudes).  The state splits into 2^(n-12)
// tiles of 4096 amplitudes that differ only in the T bits.  Each block b of
// the pass acts on 5 qubits Q_b within T; for it the tile is viewed as 128
// rows x 32 amplitudes: the row index is the 7 tile bits C_b outside Q_b, the
// column index the 5 bits of Q_b.  One M=128, N=64, K=64 contraction per tile
// and block (split-BF16 x3, FP32 accumulation in TMEM, as in qs_fused.cu).
//
// Per tile, thread i of 128 owns row i and TMEM lane i:
//   1. its row of block 0 arrives by cp.async (issued one tile ahead) in a
//      staging row of its own; it reads it to registers, immediately issues
//      the copies of the next tile into the same staging row, and writes the
//      BF16 hi/lo split into the swizzled K-major A buffer;
//   2. for each block: one thread issues the 12 MMAs and commits to an
//      mbarrier; every thread waits, loads its 64 FP32 results from TMEM, and
//      either scatters them as BF16 hi/lo into the A layout of the next block
//      (a result's tile index gives its row and column there), or - after the
//      last block - stores them to HBM in place.
// Two CTAs per SM (112 KB of shared memory each); the staging copies keep a
// tile of loads in flight per CTA while the other steps run.
//
// Norm tracking and bounded waits as in qs_fused.cu.
#include <cuda_bf16.h>

#include "qs_common.cuh"
#include "qs_fused.h"

namespace {

constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kA = 128 * 64 * 2;             // 16 KB: one BF16 A buffer (128 rows x 64)
constexpr uint32_t kB = 64 * 64 * 2;              //  8 KB: one BF16 B buffer
constexpr uint32_t kStage = 128 * 256;            // 32 KB: 128 rows x 32 complex64
constexpr int kMaxSub = 3;
constexpr uint32_t kOffA = 0;                     // A hi, A lo
constexpr uint32_t kOffB = 2 * kA;                // B hi/lo per block
constexpr uint32_t kOffStage = kOffB + kMaxSub * 2 * kB;
constexpr uint32_t kOffMisc = kOffStage + kStage; // mbarrier (8), tmem address (4), scale (4)
constexpr uint32_t kSmemBytes = kOffMisc + 16;
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(64 >> 3) << 17) |
                            ((uint32_t)(128 >> 4) << 24);
constexpr unsigned long long kWaitNs = 2000000000ull;

struct TileParams {
    uint64_t tiles;
    Holes outer;                 // the 12 tile positions
    int nsub;
    int c0_glob[7];              // global position of row bit i, block 0
    uint64_t g0[32];             // global offset of column j, block 0
    int vec0;                    // block 0 contains qubit 0: columns (j, j+1) adjacent
    int8_t rowmap[kMaxSub - 1][7];   // row bit i of block b -> row bit (>= 0) or ~col bit of block b+1
    uint8_t tabR[kMaxSub - 1][32];   // column j of block b -> row bits of block b+1
    uint8_t tabJ[kMaxSub - 1][32];   // column j of block b -> column bits of block b+1
    int cl_glob[7];              // last block
    uint64_t gl[32];
    int vecl;
    const uint16_t *mat;         // nsub x [2][64][64] BF16 bits (hi, lo) of R
    int *err;
    const double *norm0;
    const double *prev_out;
    double *in_parts;
    double *out_parts;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

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

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
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
        if (globaltimer() - t0 > kWaitNs) return false;
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

// Staging row of thread `row`: 16 chunks of 16 B (2 amplitudes each), chunk k
// stored at position k ^ (row & 15) so that the 8 rows of a quarter warp hit
// distinct banks.
__device__ __forceinline__ uint32_t stage_addr(uint32_t stage, int row, int chunk)
{
    return stage + row * 256 + ((chunk ^ (row & 15)) << 4);
}

// Copies of this thread's row of block 0 of tile `base` into its staging row.
__device__ __forceinline__ void prefetch_row(const float *amp, uint64_t base, const TileParams &P, uint32_t srow,
                                             int row)
{
    if (P.vec0) {
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            const float *src = amp + 2 * (base | P.g0[j]);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(stage_addr(srow, row, j >> 1)), "l"(src)
                         : "memory");
        }
    } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const float *src = amp + 2 * (base | P.g0[j]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;"
                         :: "r"(stage_addr(srow, row, j >> 1) + ((j & 1) << 3)), "l"(src) : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void a_store_pair(uint8_t *aHi, uint8_t *aLo, int r, int j, float re, float im)
{
    const uint32_t hv = pack_bf16x2(re, im);
    const float hre = __uint_as_float(hv << 16), him = __uint_as_float(hv & 0xffff0000u);
    const uint32_t lv = pack_bf16x2(re - hre, im - him);
    const uint32_t off = r * 128 + ((((j >> 2) ^ (r & 7))) << 4) + ((j & 3) << 2);
    *reinterpret_cast<uint32_t *>(aHi + off) = hv;
    *reinterpret_cast<uint32_t *>(aLo + off) = lv;
}

__global__ void __launch_bounds__(kThreads, 2) k_fused_tile(float *__restrict__ amp, TileParams P)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    if (smem_u32(smem) & 1023u) {             // swizzled operands need 1024-byte alignment
        if (tid == 0) atomicExch(P.err, 2);
        return;
    }
    uint8_t *aHi = smem + kOffA, *aLo = smem + kOffA + kA;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kOffMisc);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + kOffMisc + 8);
    float *s_scale = reinterpret_cast<float *>(smem + kOffMisc + 12);
    const uint32_t stage = smem_u32(smem + kOffStage);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_holder)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    // the blocks' B operands, swizzled: row n at n*128, chunk c at c ^ (n & 7)
    for (int c = tid; c < P.nsub * 2 * 64 * 8; c += kThreads) {
        const int mtx = c / (64 * 8), row = (c / 8) % 64, ch = c % 8;   // mtx = 2*block + (lo ? 1 : 0)
        uint4 v = *reinterpret_cast<const uint4 *>(P.mat + (size_t)mtx * 64 * 64 + row * 64 + ch * 8);
        *reinterpret_cast<uint4 *>(smem + kOffB + mtx * kB + row * 128 + ((ch ^ (row & 7)) << 4)) = v;
    }
    // scale undoing the previous pass's norm drift (fixed-order sums)
    if (warp == 1) {
        double n0 = 0, np = 0;
        if (P.norm0 && P.prev_out)
            for (int i = tid - 32; i < (int)gridDim.x; i += 32) { n0 += P.norm0[i]; np += P.prev_out[i]; }
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
        gC0 |= (uint64_t)((row >> b) & 1) << P.c0_glob[b];
        gCl |= (uint64_t)((row >> b) & 1) << P.cl_glob[b];
    }
    uint32_t baseR[kMaxSub - 1] = {0, 0}, baseJ[kMaxSub - 1] = {0, 0};
    for (int t = 0; t + 1 < P.nsub; ++t)
        for (int b = 0; b < 7; ++b) {
            const uint32_t bit = (row >> b) & 1;
            const int m = P.rowmap[t][b];
            if (m >= 0) baseR[t] |= bit << m;
            else baseJ[t] |= bit << (~m);
        }
    const uint32_t mb = smem_u32(mbar);
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t a_hi = smem_u32(aHi), a_lo = smem_u32(aLo);
    uint32_t phase = 0;
    bool failed = false;
    double acc_in = 0, acc_out = 0;

    uint64_t tile = blockIdx.x;
    if (tile < P.tiles) prefetch_row(amp, insert_holes(tile, P.outer) | gC0, P, stage, row);
    for (; tile < P.tiles; tile += gridDim.x) {
        const uint64_t tbase = insert_holes(tile, P.outer);
        // ---- block 0 input: this thread's staging row -> registers
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        float x[64];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            float4 v;
            asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                         : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(stage_addr(stage, row, k)));
            x[4 * k] = v.x; x[4 * k + 1] = v.y; x[4 * k + 2] = v.z; x[4 * k + 3] = v.w;
        }
        if (tile + gridDim.x < P.tiles)
            prefetch_row(amp, insert_holes(tile + gridDim.x, P.outer) | gC0, P, stage, row);
        {
            float t = 0.f;
#pragma unroll
            for (int e = 0; e < 64; ++e) { x[e] *= scale; t = fmaf(x[e], x[e], t); }
            acc_in += (double)t;
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) a_store_pair(aHi, aLo, row, j, x[2 * j], x[2 * j + 1]);

        for (int b = 0; b < P.nsub; ++b) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t bh = smem_u32(smem + kOffB + (2 * b) * kB), bl = smem_u32(smem + kOffB + (2 * b + 1) * kB);
                const uint64_t dAh = umma_desc(a_hi), dAl = umma_desc(a_lo), dBh = umma_desc(bh), dBl = umma_desc(bl);
#pragma unroll
                for (int k = 0; k < 4; ++k) mma_bf16(tmem, dAh + 2 * k, dBh + 2 * k, k > 0);
#pragma unroll
                for (int k = 0; k < 4; ++k) mma_bf16(tmem, dAh + 2 * k, dBl + 2 * k, 1);
#pragma unroll
                for (int k = 0; k < 4; ++k) mma_bf16(tmem, dAl + 2 * k, dBh + 2 * k, 1);
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             :: "r"(mb) : "memory");
            }
            const bool ok = mbar_wait(mb, phase);
            phase ^= 1;
            if (__syncthreads_or(!ok)) { failed = true; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t y[4][16];
#pragma unroll
            for (int q = 0; q < 4; ++q) tmem_ld16(taddr + 16 * q, y[q]);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (b + 1 < P.nsub) {
                // results become the next block's A operand
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int j = 8 * q + e;
                        const int r2 = baseR[b] | P.tabR[b][j], j2 = baseJ[b] | P.tabJ[b][j];
                        a_store_pair(aHi, aLo, r2, j2, __uint_as_float(y[q][2 * e]), __uint_as_float(y[q][2 * e + 1]));
                    }
            } else {
                float t = 0.f;
                const uint64_t obase = tbase | gCl;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) t = fmaf(__uint_as_float(y[q][e]), __uint_as_float(y[q][e]), t);
                    if (P.vecl) {
#pragma unroll
                        for (int e = 0; e < 8; e += 2) {
                            float4 v = make_float4(__uint_as_float(y[q][2 * e]), __uint_as_float(y[q][2 * e + 1]),
                                                   __uint_as_float(y[q][2 * e + 2]), __uint_as_float(y[q][2 * e + 3]));
                            *reinterpret_cast<float4 *>(amp + 2 * (obase | P.gl[8 * q + e])) = v;
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            float2 v = make_float2(__uint_as_float(y[q][2 * e]), __uint_as_float(y[q][2 * e + 1]));
                            *reinterpret_cast<float2 *>(amp + 2 * (obase | P.gl[8 * q + e])) = v;
                        }
                    }
                }
                acc_out += (double)t;
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        }
        if (failed) break;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    {
        double ai = acc_in, ao = acc_out;
        for (int o = 16; o > 0; o >>= 1) {
            ai += __shfl_xor_sync(0xffffffffu, ai, o);
            ao += __shfl_xor_sync(0xffffffffu, ao, o);
        }
        double *red = reinterpret_cast<double *>(smem + kOffStage);     // staging is free now
        __syncthreads();
        if ((tid & 31) == 0) { red[warp] = ai; red[4 + warp] = ao; }
        __syncthreads();
        if (tid == 0) {
            double a = 0, b = 0;
            for (int w = 0; w < kThreads / 32; ++w) { a += red[w]; b += red[4 + w]; }
            if (P.in_parts) P.in_parts[blockIdx.x] = a;
            if (P.out_parts) P.out_parts[blockIdx.x] = b;
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

}  // namespace

int qs_tiled_grid(const qs_state *s)
{
    uint64_t tiles = s->N >> 12;
    return (int)(tiles < (uint64_t)QS_SM_COUNT * 2 ? tiles : (uint64_t)QS_SM_COUNT * 2);
}

int qs_launch_tiled(qs_state *s, const qs_tiled_desc *d, int *err_dev)
{
    if (s->dtype != QS_C64) return qs_fail(QS_ERR_UNSUPPORTED, "tiled passes: complex64 states only");
    if (s->n < 12) return qs_fail(QS_ERR_UNSUPPORTED, "tiled passes: need at least 12 qubits");
    if (d->nsub < 1 || d->nsub > kMaxSub) return qs_fail(QS_ERR_ARG, "tiled pass: %d blocks", d->nsub);
    TileParams P;
    memset(&P, 0, sizeof(P));
    uint64_t tmask = 0;
    int local[64];
    for (int i = 0; i < 64; ++i) local[i] = -1;
    for (int i = 0; i < 12; ++i) {
        const int q = d->T[i];
        if (q < 0 || q >= s->n || (i && q <= d->T[i - 1]))
            return qs_fail(QS_ERR_ARG, "tiled pass: tile qubits must be ascending and in range");
        tmask |= 1ull << q;
        local[q] = i;
    }
    // per block: Q (5 local positions) and C (7 local positions), ascending
    int Q[kMaxSub][5], Cp[kMaxSub][7];
    for (int b = 0; b < d->nsub; ++b) {
        uint32_t qm = 0;
        for (int i = 0; i < 5; ++i) {
            const int q = d->qpos[b][i];
            if (q < 0 || q >= s->n || local[q] < 0 || (i && q <= d->qpos[b][i - 1]))
                return qs_fail(QS_ERR_ARG, "tiled pass: block qubits must be ascending tile qubits");
            Q[b][i] = local[q];
            qm |= 1u << local[q];
        }
        for (int p = 0, c = 0; p < 12; ++p)
            if (!(qm & (1u << p))) Cp[b][c++] = p;
    }
    P.outer = holes_from_mask(tmask);
    P.nsub = d->nsub;
    const int L = d->nsub - 1;
    for (int i = 0; i < 7; ++i) {
        P.c0_glob[i] = d->T[Cp[0][i]];
        P.cl_glob[i] = d->T[Cp[L][i]];
    }
    for (int j = 0; j < 32; ++j) {
        uint64_t a = 0, b = 0;
        for (int i = 0; i < 5; ++i)
            if (j & (1 << i)) { a |= 1ull << d->T[Q[0][i]]; b |= 1ull << d->T[Q[L][i]]; }
        P.g0[j] = a;
        P.gl[j] = b;
    }
    P.vec0 = d->T[Q[0][0]] == 0;
    P.vecl = d->T[Q[L][0]] == 0;
    for (int t = 0; t + 1 < d->nsub; ++t) {
        // where local position p lands in block t+1's layout
        int rowbit[12], colbit[12];
        for (int p = 0; p < 12; ++p) rowbit[p] = colbit[p] = -1;
        for (int i = 0; i < 7; ++i) rowbit[Cp[t + 1][i]] = i;
        for (int i = 0; i < 5; ++i) colbit[Q[t + 1][i]] = i;
        for (int i = 0; i < 7; ++i) {
            const int p = Cp[t][i];
            P.rowmap[t][i] = (int8_t)(rowbit[p] >= 0 ? rowbit[p] : ~colbit[p]);
        }
        for (int j = 0; j < 32; ++j) {
            uint32_t rr = 0, jj = 0;
            for (int i = 0; i < 5; ++i) {
                if (!(j & (1 << i))) continue;
                const int p = Q[t][i];
                if (rowbit[p] >= 0) rr |= 1u << rowbit[p];
                else jj |= 1u << colbit[p];
            }
            P.tabR[t][j] = (uint8_t)rr;
            P.tabJ[t][j] = (uint8_t)jj;
        }
    }
    P.tiles = s->N >> 12;
    P.mat = static_cast<const uint16_t *>(d->mat_dev);
    P.err = err_dev;
    P.norm0 = d->norm0;
    P.prev_out = d->prev_out;
    P.in_parts = d->in_parts;
    P.out_parts = d->out_parts;
    QS_CUDA_TRY(cudaFuncSetAttribute(k_fused_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
    const unsigned grid = (unsigned)qs_tiled_grid(s);
    k_fused_tile<<<grid, kThreads, kSmemBytes, s->stream>>>(static_cast<float *>(s->amp), P);
    QS_LAUNCH_CHECK("k_fused_tile");
    return QS_OK;
}
