// qs_fused.cu - fused 5-qubit blocks applied on the 5th-generation tensor
// cores (tcgen05.mma, accumulator in TMEM), complex64 state.
//
// A fused block is a dense 32x32 complex unitary U on qubits Q = {q0<..<q4}.
// Written over reals with interleaved (re, im) it is a 64x64 real matrix R:
//   R[2r+a][2c+b] = [[Re U, -Im U], [Im U, Re U]][a][b]   at (r, c).
// The state is cut into tiles of 128 rows x 32 amplitudes: a row is the 32
// amplitudes that differ only in the Q bits; the 128 rows of a tile differ in
// C, the 7 lowest qubits not in Q; the tile index fills the remaining bits.
// Per tile, D[128 x 64] = A[128 x 64] * R^T is one M=128, N=64, K=64 MMA.
//
// Precision: FP32 state, BF16 tensor-core inputs, FP32 accumulation.  Both
// operands are split x = x_hi + x_lo with x_hi = bf16(x), x_lo =
// bf16(x - x_hi), which represents x to ~2^-17 relative; the product uses
// three passes x_hi*R_hi + x_hi*R_lo + x_lo*R_hi (the dropped x_lo*R_lo term
// is ~2^-18 relative), accumulated in the same TMEM tile.
//
// Data flow per tile (one CTA of 128 threads, thread i = row i = TMEM lane i):
//   HBM -> registers (each thread loads its row's 32 amplitudes; a warp's
//   addresses differ in the low C bits, so each access covers whole sectors)
//   -> bf16 hi/lo split -> shared memory in the 128-byte-swizzled K-major
//   layout -> 12 x tcgen05.mma (K=16 each) issued by one thread -> commit to an
//   mbarrier -> tcgen05.ld of the thread's 64 FP32 results -> HBM (same
//   addresses, in place).  Four CTAs per SM overlap one another's loads,
//   MMAs and stores.
//
// Norm: every pass accumulates sum |in|^2 and sum |out|^2 in FP64 (one
// partial per CTA).  The truncating FP32 accumulation of the tensor cores
// loses ~3e-7 of the norm per pass, always in the same direction; the next
// pass rescales its input by sqrt(N0 / N_prev), N0 being the input norm of the
// plan's first pass, so the drift does not build up over a circuit.  That
// leaves the last pass's own drift, which the split products' rounding makes
// coherent when a circuit undoes an earlier one (a plan and then its inverse
// lost 1.3e-5 of the norm at 32 qubits); k_norm_fix, launched after a plan's
// last pass, scales the state by sqrt(N0 / N_last) when the two differ by
// more than 2^-21 relative, deciding on the device.
#include <cuda_bf16.h>

#include "qs_common.cuh"
#include "qs_fused.h"

namespace {

constexpr int kRows = 128;                       // MMA M
constexpr int kReal = 64;                        // MMA K and N: 32 amplitudes x (re, im)
constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kSmemA = kRows * kReal * 2;   // 16 KB per bf16 buffer
constexpr uint32_t kSmemB = kReal * kReal * 2;   //  8 KB per bf16 buffer
constexpr uint32_t kSmemUsed = 2 * kSmemA + 2 * kSmemB + 64;
constexpr uint32_t kSmemBytes = kSmemUsed + 1024;          // + alignment slack
// instruction descriptor: D f32 (bits 4-5 = 1), A bf16 (7-9 = 1), B bf16
// (10-12 = 1), both K-major, N>>3 at bits 17-22, M>>4 at bits 24-28
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kReal >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);
constexpr unsigned long long kWaitNs = 2000000000ull;      // 2 s bound on any wait

struct FusedParams {
    uint64_t tiles;
    Holes outer;                 // the 12 positions of Q and C
    uint64_t offQ[32];           // amplitude offset of block index j
    int cpos[7];                 // C positions, ascending
    int vec;                     // 1: qubit 0 is in Q, amplitude pairs (j, j+1) are adjacent
    const uint16_t *mat;         // [2][64][64] bf16 bits of R: hi then lo, row-major (n, k)
    int *err;
    // Norm tracking (FP64, one partial per CTA, fixed grid): the pass scales
    // its input by sqrt(sum(norm0) / sum(prev_out)) when both are given, and
    // writes sum |input|^2 to in_parts (if given) and sum |output|^2 to out_parts.
    const double *norm0;
    const double *prev_out;
    double *in_parts;
    double *out_parts;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, rows of 128 B in
// 8-row groups 1024 B apart (SBO), version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

__device__ __forceinline__ float bf16_lo_as_float(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi_as_float(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase.  Returns false after kWaitNs.
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

__global__ void __launch_bounds__(kThreads, 4) k_fused_tc(float *__restrict__ amp, FusedParams P)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *sA_hi = smem;
    uint8_t *sA_lo = smem + kSmemA;
    uint8_t *sB_hi = smem + 2 * kSmemA;
    uint8_t *sB_lo = sB_hi + kSmemB;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sB_lo + kSmemB);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(mbar + 1);

    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_holder)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    // B = R (hi, lo) into the swizzled layout: row n at n*128, 16-byte chunk c
    // at position c ^ (n & 7).
    for (int c = tid; c < 2 * kReal * 8; c += kThreads) {
        const int buf = c / (kReal * 8), row = (c / 8) % kReal, ch = c % 8;
        uint4 v = *reinterpret_cast<const uint4 *>(P.mat + (size_t)buf * kReal * kReal + row * kReal + ch * 8);
        uint8_t *dst = (buf ? sB_lo : sB_hi) + row * 128 + ((ch ^ (row & 7)) * 16);
        *reinterpret_cast<uint4 *>(dst) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_holder;

    const int row = tid;
    uint64_t depC = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b) depC |= (uint64_t)((row >> b) & 1) << P.cpos[b];
    const uint32_t a_hi = smem_u32(sA_hi), a_lo = smem_u32(sA_lo);
    const uint32_t b_hi = smem_u32(sB_hi), b_lo = smem_u32(sB_lo);
    const uint32_t mb = smem_u32(mbar);
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    uint8_t *rowA_hi = sA_hi + row * 128, *rowA_lo = sA_lo + row * 128;
    uint32_t phase = 0;
    bool failed = false;

    // Scale that undoes the systematic norm drift of the previous pass (the
    // tensor cores' FP32 accumulation does not round to nearest).  Warp 1 sums
    // the partials in a fixed order; every CTA computes the same value.
    __shared__ float s_scale;
    if (warp == 1) {
        double n0 = 0, np = 0;
        if (P.norm0 && P.prev_out)
            for (int i = tid - 32; i < (int)gridDim.x; i += 32) { n0 += P.norm0[i]; np += P.prev_out[i]; }
        for (int o = 16; o > 0; o >>= 1) {
            n0 += __shfl_xor_sync(0xffffffffu, n0, o);
            np += __shfl_xor_sync(0xffffffffu, np, o);
        }
        if (tid == 32) s_scale = (P.norm0 && P.prev_out && np > 0) ? (float)sqrt(n0 / np) : 1.0f;
    }
    __syncthreads();
    const float scale = s_scale;
    double acc_in = 0, acc_out = 0;

    for (uint64_t tile = blockIdx.x; tile < P.tiles; tile += gridDim.x) {
        const uint64_t base = insert_holes(tile, P.outer) | depC;
        // ---- load this row's 32 amplitudes
        float x[64];
        if (P.vec) {
#pragma unroll
            for (int j = 0; j < 32; j += 2) {
                float4 v = *reinterpret_cast<const float4 *>(amp + 2 * (base | P.offQ[j]));
                x[2 * j] = v.x; x[2 * j + 1] = v.y; x[2 * j + 2] = v.z; x[2 * j + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                float2 v = *reinterpret_cast<const float2 *>(amp + 2 * (base | P.offQ[j]));
                x[2 * j] = v.x; x[2 * j + 1] = v.y;
            }
        }
        {
            float t = 0.f;
#pragma unroll
            for (int e = 0; e < 64; ++e) { x[e] *= scale; t = fmaf(x[e], x[e], t); }
            acc_in += (double)t;
        }
        // ---- split into bf16 hi/lo and store the row (chunk c = reals 8c..8c+7)
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            uint4 h, l;
            uint32_t *hp = reinterpret_cast<uint32_t *>(&h), *lp = reinterpret_cast<uint32_t *>(&l);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float f0 = x[8 * c + 2 * e], f1 = x[8 * c + 2 * e + 1];
                const uint32_t hv = pack_bf16x2(f0, f1);
                hp[e] = hv;
                lp[e] = pack_bf16x2(f0 - bf16_lo_as_float(hv), f1 - bf16_hi_as_float(hv));
            }
            const int pos = (c ^ (row & 7)) * 16;
            *reinterpret_cast<uint4 *>(rowA_hi + pos) = h;
            *reinterpret_cast<uint4 *>(rowA_lo + pos) = l;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // ---- 3 x 4 MMAs (K = 16 each) into TMEM, then commit to the mbarrier
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint64_t dAh = umma_desc(a_hi), dAl = umma_desc(a_lo);
            const uint64_t dBh = umma_desc(b_hi), dBl = umma_desc(b_lo);
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
        // ---- TMEM -> registers -> HBM (same addresses)
        uint32_t y[4][16];
#pragma unroll
        for (int q = 0; q < 4; ++q) tmem_ld16(taddr + 16 * q, y[q]);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        {
            float t = 0.f;
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int e = 0; e < 16; ++e) t = fmaf(__uint_as_float(y[q][e]), __uint_as_float(y[q][e]), t);
            acc_out += (double)t;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (P.vec) {
#pragma unroll
                for (int j = 0; j < 8; j += 2) {
                    float4 v = make_float4(__uint_as_float(y[q][2 * j]), __uint_as_float(y[q][2 * j + 1]),
                                           __uint_as_float(y[q][2 * j + 2]), __uint_as_float(y[q][2 * j + 3]));
                    *reinterpret_cast<float4 *>(amp + 2 * (base | P.offQ[8 * q + j])) = v;
                }
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float2 v = make_float2(__uint_as_float(y[q][2 * j]), __uint_as_float(y[q][2 * j + 1]));
                    *reinterpret_cast<float2 *>(amp + 2 * (base | P.offQ[8 * q + j])) = v;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    // per-CTA norm partials (fixed order: warp shuffles, then warp 0)
    {
        __shared__ double red[2][kThreads / 32];
        for (int o = 16; o > 0; o >>= 1) {
            acc_in += __shfl_xor_sync(0xffffffffu, acc_in, o);
            acc_out += __shfl_xor_sync(0xffffffffu, acc_out, o);
        }
        if ((tid & 31) == 0) { red[0][warp] = acc_in; red[1][warp] = acc_out; }
        __syncthreads();
        if (tid == 0) {
            double a = 0, b = 0;
            for (int w = 0; w < kThreads / 32; ++w) { a += red[0][w]; b += red[1][w]; }
            if (P.in_parts) P.in_parts[blockIdx.x] = a;
            if (P.out_parts) P.out_parts[blockIdx.x] = b;
        }
    }
    if (failed) {
        if (tid == 0) atomicExch(P.err, 1);
        // Let the MMA still in flight (the phase that timed out) finish
        // before TMEM is released; this wait is bounded too.
        mbar_wait(mb, phase ^ 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTmemCols));
    }
}

// Every CTA sums the two sets of partials in the same fixed order and gets
// the same factor; nothing is written when the norms agree within kNormTol.
constexpr double kNormTol = 1.0 / (1 << 21);
constexpr int kFixThreads = 256;

__global__ void __launch_bounds__(kFixThreads) k_norm_fix(float4 *amp, uint64_t n4, const double *n0p,
                                                          const double *nlp, int nparts)
{
    __shared__ float s_c;
    if (threadIdx.x < 32) {
        double a = 0.0, b = 0.0;
        for (int i = threadIdx.x; i < nparts; i += 32) { a += n0p[i]; b += nlp[i]; }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (threadIdx.x == 0) s_c = (a > 0.0 && b > 0.0 && fabs(b / a - 1.0) > kNormTol) ? (float)sqrt(a / b) : 0.f;
    }
    __syncthreads();
    const float c = s_c;
    if (c == 0.f) return;
    const uint64_t stride = (uint64_t)gridDim.x * kFixThreads;
    uint64_t i = (uint64_t)blockIdx.x * kFixThreads + threadIdx.x;
    for (; i + 3 * stride < n4; i += 4 * stride) {
        float4 v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = amp[i + k * stride];
#pragma unroll
        for (int k = 0; k < 4; ++k) amp[i + k * stride] = make_float4(v[k].x * c, v[k].y * c, v[k].z * c, v[k].w * c);
    }
    for (; i < n4; i += stride) {
        const float4 v = amp[i];
        amp[i] = make_float4(v.x * c, v.y * c, v.z * c, v.w * c);
    }
}

}  // namespace

int qs_launch_norm_fix(qs_state *s, const double *norm0, const double *last_out, int nparts)
{
    if (s->dtype != QS_C64) return QS_OK;
    k_norm_fix<<<QS_SM_COUNT * 4, kFixThreads, 0, s->stream>>>(static_cast<float4 *>(s->amp), s->N / 2, norm0,
                                                              last_out, nparts);
    QS_LAUNCH_CHECK("k_norm_fix");
    return QS_OK;
}

int qs_fused_grid(const qs_state *s)
{
    uint64_t tiles = s->N >> 12;
    return (int)(tiles < (uint64_t)QS_SM_COUNT * 4 ? tiles : (uint64_t)QS_SM_COUNT * 4);
}

int qs_launch_fused(qs_state *s, const qs_fused_desc *d, int *err_dev)
{
    if (s->dtype != QS_C64) return qs_fail(QS_ERR_UNSUPPORTED, "fused blocks: complex64 states only");
    if (s->n < 12) return qs_fail(QS_ERR_UNSUPPORTED, "fused blocks: need at least 12 qubits");
    FusedParams P;
    memset(&P, 0, sizeof(P));
    uint64_t qmask = 0;
    for (int b = 0; b < 5; ++b) {
        if (d->qpos[b] < 0 || d->qpos[b] >= s->n || (b && d->qpos[b] <= d->qpos[b - 1]))
            return qs_fail(QS_ERR_ARG, "fused block: qubits must be ascending and in range");
        qmask |= 1ull << d->qpos[b];
    }
    uint64_t cmask = 0;
    for (int q = 0, c = 0; q < s->n && c < 7; ++q)
        if (!(qmask & (1ull << q))) { P.cpos[c++] = q; cmask |= 1ull << q; }
    P.outer = holes_from_mask(qmask | cmask);
    for (int j = 0; j < 32; ++j) {
        uint64_t o = 0;
        for (int b = 0; b < 5; ++b)
            if (j & (1 << b)) o |= 1ull << d->qpos[b];
        P.offQ[j] = o;
    }
    P.vec = d->qpos[0] == 0;
    P.tiles = s->N >> 12;
    P.mat = static_cast<const uint16_t *>(d->mat_dev);
    P.err = err_dev;
    P.norm0 = d->norm0;
    P.prev_out = d->prev_out;
    P.in_parts = d->in_parts;
    P.out_parts = d->out_parts;
    QS_CUDA_TRY(cudaFuncSetAttribute(k_fused_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
    const unsigned grid = (unsigned)qs_fused_grid(s);
    k_fused_tc<<<grid, kThreads, kSmemBytes, s->stream>>>(static_cast<float *>(s->amp), P);
    QS_LAUNCH_CHECK("k_fused_tc");
    return QS_OK;
}
