// qs_measure.cu - probabilities, measurement collapse, marginals and shots.
//
// Reference behaviour (QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp):
//   qubitMeasure (:1071-1126): p0 = sum over bit q == 0 of |a|^2 (serial sum,
//     FP64), outcome = ((float)u > p0), kept half scaled by 1/sqrt(p), other
//     half zeroed.
//   pMeasure (:159-190): out[idx] += |a_i|^2 with idx bit j = bit qubits[j] of i.
//
// Here every sum is FP64 and deterministic: each CTA reduces a fixed slice
// (warp shuffles, then shared memory) into one partial, and a single CTA adds
// the partials in a fixed order.  The partials live in the state's scratch
// buffer; the outcome decision is taken on the device so that the collapse
// kernel needs no host round trip.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "qs_common.cuh"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block reduction; result valid in thread 0.
__device__ double block_sum(double v)
{
    __shared__ double red[kThreads / 32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double r = 0;
    if (wid == 0) {
        r = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

template <typename T>
__device__ __forceinline__ double p2(T re, T im)
{
    double r = (double)re, i = (double)im;
    return fma(r, r, i * i);
}

// sum |a_i|^2 over i with bit q == 0 (q < 0: over all i), read in chunks of
// two neighbouring amplitudes (one 16-byte load for complex64): chunk c holds
// amplitudes 2c, 2c + 1.  q < 0: every chunk, both halves; q == 0: every
// chunk, first half; q >= 1: the chunks with bit q - 1 of c clear (the pair
// index with a zero inserted), both halves.  A thread keeps four chunks in
// flight; the per-thread order, and so the partials, are fixed by the grid.
template <typename T>
struct Chunk2 {
    T r0, i0, r1, i1;
};

template <typename T>
__device__ __forceinline__ Chunk2<T> load_chunk(const T *a, uint64_t c, bool first_only)
{
    Chunk2<T> x;
    if constexpr (sizeof(T) == 4) {
        const float4 v = reinterpret_cast<const float4 *>(a)[c];
        x.r0 = v.x; x.i0 = v.y; x.r1 = v.z; x.i1 = v.w;
    } else {
        const double2 *p = reinterpret_cast<const double2 *>(a) + 2 * c;
        const double2 v0 = p[0];
        x.r0 = v0.x; x.i0 = v0.y;
        if (first_only) {
            x.r1 = 0; x.i1 = 0;
        } else {
            const double2 v1 = p[1];
            x.r1 = v1.x; x.i1 = v1.y;
        }
    }
    return x;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_half_sum(const T *__restrict__ a, uint64_t items, int q, double *partials)
{
    const bool first_only = q == 0;
    const int sh = q > 0 ? q - 1 : 63;
    const uint64_t lowm = q > 0 ? (1ull << sh) - 1 : ~0ull;
    auto chunk = [&](uint64_t w) -> uint64_t { return q > 0 ? (((w >> sh) << (sh + 1)) | (w & lowm)) : w; };
    auto val = [&](const Chunk2<T> &x) -> double {
        return first_only ? p2(x.r0, x.i0) : p2(x.r0, x.i0) + p2(x.r1, x.i1);
    };
    double acc = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; w + 3 * stride < items; w += 4 * stride) {
        Chunk2<T> x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = load_chunk(a, chunk(w + u * stride), first_only);
#pragma unroll
        for (int u = 0; u < 4; ++u) acc += val(x[u]);
    }
    for (; w < items; w += stride) acc += val(load_chunk(a, chunk(w), first_only));
    double s = block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

struct MeasureResult {
    double p0;
    double scale;
    int outcome;
    int status;          // 0 ok, 1 = the selected outcome has probability <= 0
};

// mode 0: res->p0 = sum; mode 1: measurement decision with uniform u.
__global__ void k_finalize(const double *partials, int count, MeasureResult *res, int mode, double u)
{
    double acc = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partials[i];
    double tot = block_sum(acc);
    if (threadIdx.x == 0) {
        res->p0 = tot;
        res->status = 0;
        res->outcome = 0;
        res->scale = 1.0;
        if (mode == 1) {
            float fi = (float)u;
            int out = ((double)fi > tot) ? 1 : 0;
            double psel = out ? 1.0 - tot : tot;
            res->outcome = out;
            if (!(psel > 0.0)) res->status = 1;
            else res->scale = 1.0 / sqrt(psel);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_collapse(T *__restrict__ a, uint64_t pairs, int q, const MeasureResult *res)
{
    if (res->status) return;
    typedef typename vec2<T>::type V;
    V *pa = reinterpret_cast<V *>(a);
    const int out = res->outcome;
    const T sc = (T)res->scale;
    const uint64_t st = 1ull << q;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < pairs; w += stride) {
        uint64_t lo = w & (st - 1);
        uint64_t i0 = ((w >> q) << (q + 1)) | lo;
        uint64_t ik = out ? i0 + st : i0, iz = out ? i0 : i0 + st;
        V x = pa[ik];
        pa[ik] = V{x.x * sc, x.y * sc};
        pa[iz] = V{(T)0, (T)0};
    }
}

// -------------------------------------------------------------- marginals
// Stage 1: CTA (o, g) handles the chunks (2^c contiguous amplitudes) whose
// measured high bits equal o and whose unmeasured high bits lie in slice g;
// it adds |a|^2 into 2^mlo bins (measured low bits) and writes the bins at
// their full output index in partial slice g.
struct MargParams {
    int c;                       // chunk bits (<= 12)
    int mlo, ulo;                // measured / unmeasured positions below c
    int mhi, uhi;                // measured / unmeasured positions at or above c
    int m;                       // total measured
    int mlo_pos[12], mlo_out[12];
    int ulo_pos[12];
    int mhi_pos[40], mhi_out[40];
    int uhi_pos[40];
    uint64_t G, R;               // slices of the unmeasured high space, chunks per CTA
};

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_marginal(const T *__restrict__ a, MargParams P, double *__restrict__ part)
{
    extern __shared__ double sm[];
    const int C = 1 << P.c;
    const int nb = 1 << P.mlo;           // bins
    const int tpb = 1 << P.ulo;          // terms per bin
    double *p = sm;                      // C
    double *acc = p + C;                 // nb
    double *red = acc + nb;              // kThreads
    uint32_t *tabM = reinterpret_cast<uint32_t *>(red + kThreads);   // nb
    uint32_t *tabU = tabM + nb;                                      // tpb
    const int t = threadIdx.x;
    for (int b = t; b < nb; b += kThreads) {
        uint32_t v = 0;
        for (int r = 0; r < P.mlo; ++r) v |= ((b >> r) & 1u) << P.mlo_pos[r];
        tabM[b] = v;
        acc[b] = 0;
    }
    for (int u = t; u < tpb; u += kThreads) {
        uint32_t v = 0;
        for (int r = 0; r < P.ulo; ++r) v |= ((u >> r) & 1u) << P.ulo_pos[r];
        tabU[u] = v;
    }
    const uint64_t o = blockIdx.x / P.G;         // compact measured-high value
    const uint64_t g = blockIdx.x % P.G;
    uint64_t hm = 0, out_hi = 0;
    for (int r = 0; r < P.mhi; ++r) {
        uint64_t bit = (o >> r) & 1ull;
        hm |= bit << P.mhi_pos[r];
        out_hi |= bit << P.mhi_out[r];
    }
    typedef typename vec2<T>::type V;
    const V *pa = reinterpret_cast<const V *>(a);
    // fewer bins than threads: thread t sums fixed positions of every chunk
    // (bin t / tpbt, terms u = t % tpbt + k tpbt) into a register, and the
    // threads of a bin combine once at the end
    const int tpbt = nb < kThreads ? kThreads / nb : 1;
    const int mb = t / tpbt, msub = t % tpbt;
    double mine = 0;
    __syncthreads();
    for (uint64_t r = 0; r < P.R; ++r) {
        uint64_t uidx = g * P.R + r, hu = 0;
        for (int j = 0; j < P.uhi; ++j) hu |= ((uidx >> j) & 1ull) << P.uhi_pos[j];
        const uint64_t base = (hm | hu) << P.c;
        // all of the thread's loads of the chunk (up to 4096 / kThreads) go
        // out before the first store, so that enough bytes are in flight to
        // stream the state at HBM speed
        constexpr int kPer = 4096 / kThreads;
        double v[kPer];
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int l = t + i * kThreads;
            if (l < C) {
                const V x = pa[base + l];
                v[i] = p2(x.x, x.y);
            }
        }
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int l = t + i * kThreads;
            if (l < C) p[l] = v[i];
        }
        __syncthreads();
        if (nb >= kThreads) {
            for (int b = t; b < nb; b += kThreads) {
                double s = 0;
                for (int u = 0; u < tpb; ++u) s += p[tabM[b] | tabU[u]];
                acc[b] += s;
            }
        } else {
            double s = 0;
            for (int u = msub; u < tpb; u += tpbt) s += p[tabM[mb] | tabU[u]];
            mine += s;
        }
        __syncthreads();
    }
    if (nb < kThreads) {
        red[t] = mine;
        __syncthreads();
        for (int w = tpbt >> 1; w > 0; w >>= 1) {
            if (msub < w) red[t] += red[t + w];
            __syncthreads();
        }
        if (msub == 0) acc[mb] = red[t];
        __syncthreads();
    }
    double *dst = part + g * (1ull << P.m);
    for (int b = t; b < nb; b += kThreads) {
        uint64_t oi = out_hi;
        for (int r = 0; r < P.mlo; ++r) oi |= (uint64_t)((b >> r) & 1) << P.mlo_out[r];
        dst[oi] = acc[b];
    }
}

// The same marginal on chunks of 4096 (states of 12 qubits and more): a
// thread owns fixed chunk positions and adds their |a|^2 in registers, chunk
// after chunk, with 16-byte loads (two complex64 or one complex128 amplitude
// each) and two chunks' loads in flight before their first use.  When every
// chunk bit is measured (P.ulo == 0) each position is a bin - the order
// k_marginal adds them in, so the bins are bit-identical - and no shared
// memory is used; otherwise the CTA folds its 4096 position sums into the
// 2^mlo bins once, at the end, in a fixed order.
template <typename T, bool FOLD>
__global__ void __launch_bounds__(kThreads)
k_marginal_direct(const T *__restrict__ a, MargParams P, double *__restrict__ part)
{
    constexpr int kApl = sizeof(T) == 4 ? 2 : 1;            // amplitudes per 16-byte load
    constexpr int kLoads = 4096 / (kThreads * kApl);          // per thread and chunk
    typedef typename std::conditional<sizeof(T) == 4, float4, double2>::type L16;
    const L16 *pa = reinterpret_cast<const L16 *>(a);
    const int t = threadIdx.x;
    const uint64_t o = blockIdx.x / P.G, g = blockIdx.x % P.G;
    uint64_t hm = 0, out_hi = 0;
    for (int r = 0; r < P.mhi; ++r) {
        const uint64_t bit = (o >> r) & 1ull;
        hm |= bit << P.mhi_pos[r];
        out_hi |= bit << P.mhi_out[r];
    }
    double acc[kLoads * kApl];
#pragma unroll
    for (int i = 0; i < kLoads * kApl; ++i) acc[i] = 0.0;
    auto chunk_base = [&](uint64_t r) {
        const uint64_t uidx = g * P.R + r;
        uint64_t hu = 0;
        for (int j = 0; j < P.uhi; ++j) hu |= ((uidx >> j) & 1ull) << P.uhi_pos[j];
        return ((hm | hu) << 12) / kApl;                       // in 16-byte units
    };
    auto add = [&](const L16 (&v)[kLoads]) {
#pragma unroll
        for (int i = 0; i < kLoads; ++i) {
            if constexpr (sizeof(T) == 4) {
                const float4 x = *reinterpret_cast<const float4 *>(&v[i]);
                acc[2 * i] += p2(x.x, x.y);
                acc[2 * i + 1] += p2(x.z, x.w);
            } else {
                const double2 x = *reinterpret_cast<const double2 *>(&v[i]);
                acc[i] += p2(x.x, x.y);
            }
        }
    };
    uint64_t r = 0;
    for (; r + 2 <= P.R; r += 2) {
        const uint64_t b0 = chunk_base(r), b1 = chunk_base(r + 1);
        L16 v0[kLoads], v1[kLoads];
#pragma unroll
        for (int i = 0; i < kLoads; ++i) v0[i] = __ldg(pa + b0 + t + i * kThreads);
#pragma unroll
        for (int i = 0; i < kLoads; ++i) v1[i] = __ldg(pa + b1 + t + i * kThreads);
        add(v0);
        add(v1);
    }
    if (r < P.R) {
        const uint64_t b0 = chunk_base(r);
        L16 v0[kLoads];
#pragma unroll
        for (int i = 0; i < kLoads; ++i) v0[i] = __ldg(pa + b0 + t + i * kThreads);
        add(v0);
    }
    double *dst = part + g * (1ull << P.m);
    if constexpr (!FOLD) {                                    // every chunk position is a bin
#pragma unroll
        for (int i = 0; i < kLoads * kApl; ++i) {
            const int l = (t + (i / kApl) * kThreads) * kApl + (i % kApl);   // chunk position
            uint64_t oi = out_hi;
            for (int b = 0; b < P.mlo; ++b) oi |= (uint64_t)((l >> P.mlo_pos[b]) & 1) << P.mlo_out[b];
            dst[oi] = acc[i];
        }
        return;
    }
    // some chunk bits unmeasured: fold the 4096 position sums into the 2^mlo
    // bins once per CTA, in a fixed order (shared memory: 4096 + kThreads doubles)
    extern __shared__ double fold[];
    double *red = fold + 4096;
#pragma unroll
    for (int i = 0; i < kLoads * kApl; ++i) fold[(t + (i / kApl) * kThreads) * kApl + (i % kApl)] = acc[i];
    __syncthreads();
    const int nb = 1 << P.mlo, tpb = 1 << P.ulo;
    auto position = [&](int b, int u) {
        uint32_t l = 0;
        for (int r = 0; r < P.mlo; ++r) l |= (uint32_t)((b >> r) & 1) << P.mlo_pos[r];
        for (int r = 0; r < P.ulo; ++r) l |= (uint32_t)((u >> r) & 1) << P.ulo_pos[r];
        return l;
    };
    auto out_index = [&](int b) {
        uint64_t oi = out_hi;
        for (int r = 0; r < P.mlo; ++r) oi |= (uint64_t)((b >> r) & 1) << P.mlo_out[r];
        return oi;
    };
    if (nb >= kThreads) {
        for (int b = t; b < nb; b += kThreads) {
            double sum = 0;
            for (int u = 0; u < tpb; ++u) sum += fold[position(b, u)];
            dst[out_index(b)] = sum;
        }
    } else {
        const int tpbt = kThreads / nb, b = t / tpbt, sub = t % tpbt;
        double sum = 0;
        for (int u = sub; u < tpb; u += tpbt) sum += fold[position(b, u)];
        red[t] = sum;
        __syncthreads();
        for (int w = tpbt >> 1; w > 0; w >>= 1) {
            if (sub < w) red[t] += red[t + w];
            __syncthreads();
        }
        if (sub == 0) dst[out_index(b)] = red[t];
    }
}

__global__ void k_marginal_combine(const double *__restrict__ part, uint64_t G, uint64_t nout,
                                   double *__restrict__ out)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nout; o += stride) {
        double s = 0;
        for (uint64_t g = 0; g < G; ++g) s += part[g * nout + o];
        out[o] = s;
    }
}

size_t marginal_smem(const MargParams &P)
{
    size_t C = 1ull << P.c, nb = 1ull << P.mlo, tpb = 1ull << P.ulo;
    return (C + nb + kThreads) * sizeof(double) + (nb + tpb) * sizeof(uint32_t);
}

// -------------------------------------------------------------- shots
// tree[2^k + x] = P(first k measured outcomes = x) for k <= K0.
__global__ void k_fold(double *tree, int k)
{
    const uint64_t n = 1ull << k;
    double *dst = tree + n;
    const double *src = tree + 2 * n;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += stride)
        dst[x] = src[x] + src[x + n];
}

// One warp per shot.  Levels k < K0 read the tree; deeper levels sum the
// amplitudes that match the outcomes so far (2^(n-k-1) of them).
template <typename T>
__global__ void k_shots(const T *__restrict__ a, const double *__restrict__ tree, int K0, int m,
                        const Holes *__restrict__ deep, const int *__restrict__ qubits,
                        const double *__restrict__ u, uint64_t shots, int n,
                        uint64_t *__restrict__ out)
{
    typedef typename vec2<T>::type V;
    const V *pa = reinterpret_cast<const V *>(a);
    const int lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t s = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < shots; s += warps) {
        uint64_t x = 0;          // outcomes so far, bit k = qubits[k]
        uint64_t F = 0;          // the same outcomes placed at their qubit positions
        double S = 1.0;          // normalisation the reference state carries
        for (int k = 0; k < m; ++k) {
            double L;
            if (k < K0) {
                L = tree[(2ull << k) + x];
            } else {
                const Holes &h = deep[k - K0];
                const uint64_t cnt = 1ull << (n - k - 1);
                double acc = 0;
                for (uint64_t w = lane; w < cnt; w += 32) {
                    V v = pa[insert_holes(w, h) | F];
                    acc += p2(v.x, v.y);
                }
                L = warp_sum(acc);
            }
            const double p0 = L * S;
            const float fi = (float)u[s * (uint64_t)m + k];
            const int b = ((double)fi > p0) ? 1 : 0;
            const double psel = b ? 1.0 - p0 : p0;
            const double sc = 1.0 / sqrt(psel);
            S *= sc * sc;
            x |= (uint64_t)b << k;
            F |= (uint64_t)b << qubits[k];
        }
        if (lane == 0) out[s] = x;
    }
}

// -------------------------------------------------------------- norm, inner
template <typename Ta, typename Tb>
__global__ void __launch_bounds__(kThreads)
k_inner(const Ta *__restrict__ a, const Tb *__restrict__ b, uint64_t N, double *partials)
{
    typedef typename vec2<Ta>::type VA;
    typedef typename vec2<Tb>::type VB;
    const VA *pa = reinterpret_cast<const VA *>(a);
    const VB *pb = reinterpret_cast<const VB *>(b);
    // four elements in flight per thread, two accumulator pairs (fixed order)
    double re[2] = {0, 0}, im[2] = {0, 0};
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < N; i += 4 * stride) {
        VA x[4];
        VB y[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) { x[u] = pa[i + u * stride]; y[u] = pb[i + u * stride]; }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double xr = x[u].x, xi = x[u].y, yr = y[u].x, yi = y[u].y;
            re[u & 1] += xr * yr + xi * yi;          // conj(x) * y
            im[u & 1] += xr * yi - xi * yr;
        }
    }
    for (; i < N; i += stride) {
        const VA x = pa[i];
        const VB y = pb[i];
        const double xr = x.x, xi = x.y, yr = y.x, yi = y.y;
        re[0] += xr * yr + xi * yi;
        im[0] += xr * yi - xi * yr;
    }
    double sre = block_sum(re[0] + re[1]);
    double sim = block_sum(im[0] + im[1]);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = sre;
        partials[2 * blockIdx.x + 1] = sim;
    }
}

template <typename Ta, typename Tb>
__global__ void __launch_bounds__(kThreads)
k_diff(const Ta *__restrict__ a, const Tb *__restrict__ b, uint64_t N, double *partials)
{
    typedef typename vec2<Ta>::type VA;
    typedef typename vec2<Tb>::type VB;
    const VA *pa = reinterpret_cast<const VA *>(a);
    const VB *pb = reinterpret_cast<const VB *>(b);
    double mx = 0, ss = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < N; i += 4 * stride) {            // four elements in flight
        VA x[4];
        VB y[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) { x[u] = pa[i + u * stride]; y[u] = pb[i + u * stride]; }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double dr = (double)x[u].x - (double)y[u].x, di = (double)x[u].y - (double)y[u].y;
            const double d2 = dr * dr + di * di;
            ss += d2;
            mx = fmax(mx, d2);
        }
    }
    for (; i < N; i += stride) {
        VA x = pa[i];
        VB y = pb[i];
        double dr = (double)x.x - (double)y.x, di = (double)x.y - (double)y.y;
        double d2 = dr * dr + di * di;
        ss += d2;
        mx = fmax(mx, d2);
    }
    // max via shuffles, sum via block_sum
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    __shared__ double wmax[kThreads / 32];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = mx;
    double s2 = block_sum(ss);
    if (threadIdx.x == 0) {
        double m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, wmax[w]);
        partials[2 * blockIdx.x] = m;
        partials[2 * blockIdx.x + 1] = s2;
    }
}

__global__ void k_finalize_diff(const double *partials, int count, double *res)
{
    if (threadIdx.x == 0) {
        double m = 0, s = 0;
        for (int i = 0; i < count; ++i) { m = fmax(m, partials[2 * i]); s += partials[2 * i + 1]; }
        res[0] = sqrt(m);
        res[1] = s;
    }
}

__global__ void k_finalize2(const double *partials, int count, double *res)
{
    double re = 0, im = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        re += partials[2 * i];
        im += partials[2 * i + 1];
    }
    double r = block_sum(re);
    double s = block_sum(im);
    if (threadIdx.x == 0) { res[0] = r; res[1] = s; }
}

template <typename T>
__global__ void k_convert(const void *__restrict__ src, int src_dtype, T *__restrict__ dst, uint64_t n)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 2 * n; i += stride)
        dst[i] = src_dtype == QS_C64 ? (T) static_cast<const float *>(src)[i]
                                     : (T) static_cast<const double *>(src)[i];
}

// Scratch layout: [0, 64 KB) partials; [64 KB, 64 KB + 64 B) results; the rest
// per-operation buffers.
constexpr size_t kPartOff = 0;
constexpr size_t kResOff = 64 * 1024;
constexpr size_t kBufOff = kResOff + 256;

template <typename T>
int half_sum(qs_state *s, int q, int *nblocks)
{
    // chunks of two amplitudes (k_half_sum); q < n, so q >= 1 implies N >= 4
    const uint64_t items = q > 0 ? s->N >> 2 : s->N >> 1;
    unsigned grid = grid_for(items, kThreads, 8);
    double *part = reinterpret_cast<double *>(static_cast<char *>(s->scratch) + kPartOff);
    k_half_sum<T><<<grid, kThreads, 0, s->stream>>>(static_cast<const T *>(s->amp), items, q, part);
    QS_LAUNCH_CHECK("k_half_sum");
    *nblocks = (int)grid;
    return QS_OK;
}

int read_result(qs_state *s, size_t off, size_t bytes)
{
    QS_CUDA_TRY(cudaMemcpyAsync(s->pinned, static_cast<char *>(s->scratch) + off, bytes,
                                cudaMemcpyDeviceToHost, s->stream));
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return QS_OK;
}

template <typename T>
int prob_zero_t(qs_state *s, int q, double *p0)
{
    int nb, r;
    if ((r = half_sum<T>(s, q, &nb))) return r;
    double *part = reinterpret_cast<double *>(static_cast<char *>(s->scratch) + kPartOff);
    MeasureResult *res = reinterpret_cast<MeasureResult *>(static_cast<char *>(s->scratch) + kResOff);
    k_finalize<<<1, kThreads, 0, s->stream>>>(part, nb, res, 0, 0.0);
    QS_LAUNCH_CHECK("k_finalize");
    if ((r = read_result(s, kResOff, sizeof(MeasureResult)))) return r;
    *p0 = static_cast<MeasureResult *>(s->pinned)->p0;
    return QS_OK;
}

template <typename T>
int measure_t(qs_state *s, int q, double u, int *outcome)
{
    int nb, r;
    if ((r = half_sum<T>(s, q, &nb))) return r;
    double *part = reinterpret_cast<double *>(static_cast<char *>(s->scratch) + kPartOff);
    MeasureResult *res = reinterpret_cast<MeasureResult *>(static_cast<char *>(s->scratch) + kResOff);
    k_finalize<<<1, kThreads, 0, s->stream>>>(part, nb, res, 1, u);
    QS_LAUNCH_CHECK("k_finalize");
    uint64_t pairs = s->N >> 1;
    k_collapse<T><<<grid_for(pairs, kThreads), kThreads, 0, s->stream>>>(static_cast<T *>(s->amp), pairs, q, res);
    QS_LAUNCH_CHECK("k_collapse");
    if ((r = read_result(s, kResOff, sizeof(MeasureResult)))) return r;
    const MeasureResult *h = static_cast<const MeasureResult *>(s->pinned);
    if (h->status)
        return qs_fail(QS_ERR_STATE, "qs_measure: outcome %d of qubit %d has probability %.3g",
                       h->outcome, q, h->outcome ? 1.0 - h->p0 : h->p0);
    *outcome = h->outcome;
    return QS_OK;
}

// Marginal over qubits[0..m): plan the launch.  *part_bytes receives the
// scratch the partial slices need (0 when one slice covers the space).
MargParams marginal_plan(const qs_state *s, const int *qubits, int m, size_t *part_bytes)
{
    MargParams P;
    memset(&P, 0, sizeof(P));
    const int n = s->n;
    P.c = n < 12 ? n : 12;
    P.m = m;
    uint64_t meas = 0;
    for (int j = 0; j < m; ++j) {
        int q = qubits[j];
        meas |= 1ull << q;
        if (q < P.c) { P.mlo_pos[P.mlo] = q; P.mlo_out[P.mlo] = j; P.mlo++; }
        else { P.mhi_pos[P.mhi] = q - P.c; P.mhi_out[P.mhi] = j; P.mhi++; }
    }
    for (int q = 0; q < n; ++q) {
        if (meas & (1ull << q)) continue;
        if (q < P.c) P.ulo_pos[P.ulo++] = q;
        else P.uhi_pos[P.uhi++] = q - P.c;
    }
    // Aim for ~4 CTAs per SM in total.
    uint64_t ohi = 1ull << P.mhi, uspace = 1ull << P.uhi;
    uint64_t G = 1;
    while (G < uspace && ohi * G < (uint64_t)QS_SM_COUNT * 4) G <<= 1;
    P.G = G;
    P.R = uspace / G;
    *part_bytes = G > 1 ? G * (8ull << m) : 0;
    return P;
}

// Launch a planned marginal into dev_out (2^m doubles, device).  part must
// hold part_bytes from marginal_plan (unused when that was 0).  Neither
// pointer may move during the call: this function does not touch scratch.
template <typename T>
int marginal_launch(qs_state *s, const MargParams &P, double *dev_out, double *part)
{
    const uint64_t ohi = 1ull << P.mhi, G = P.G;
    if (G == 1) part = dev_out;
    uint64_t ctas = ohi * G;
    if (ctas > 0x7fffffffull) return qs_fail(QS_ERR_UNSUPPORTED, "qs_probs: too many output bins");
    if (P.c == 12) {
        // chunk positions accumulated in registers; folded into bins at the end
        // when some chunk bits are unmeasured (4096 + kThreads doubles of shared memory)
        if (P.ulo == 0)
            k_marginal_direct<T, false><<<(unsigned)ctas, kThreads, 0, s->stream>>>(static_cast<const T *>(s->amp), P, part);
        else
            k_marginal_direct<T, true><<<(unsigned)ctas, kThreads, (4096 + kThreads) * sizeof(double), s->stream>>>(
                static_cast<const T *>(s->amp), P, part);
        QS_LAUNCH_CHECK("k_marginal_direct");
    } else {
        size_t smem = marginal_smem(P);
        QS_CUDA_TRY(cudaFuncSetAttribute(k_marginal<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
        k_marginal<T><<<(unsigned)ctas, kThreads, smem, s->stream>>>(static_cast<const T *>(s->amp), P, part);
        QS_LAUNCH_CHECK("k_marginal");
    }
    if (G > 1) {
        uint64_t nout = 1ull << P.m;
        k_marginal_combine<<<grid_for(nout, kThreads), kThreads, 0, s->stream>>>(part, G, nout, dev_out);
        QS_LAUNCH_CHECK("k_marginal_combine");
    }
    return QS_OK;
}

int check_qubit_list(const qs_state *s, const int *qubits, int m, const char *who)
{
    if (m < 0 || m > s->n) return qs_fail(QS_ERR_ARG, "%s: bad qubit count %d", who, m);
    uint64_t seen = 0;
    for (int j = 0; j < m; ++j) {
        if (qubits[j] < 0 || qubits[j] >= s->n)
            return qs_fail(QS_ERR_ARG, "%s: qubit %d out of range [0,%d)", who, qubits[j], s->n);
        if (seen & (1ull << qubits[j])) return qs_fail(QS_ERR_ARG, "%s: qubit %d listed twice", who, qubits[j]);
        seen |= 1ull << qubits[j];
    }
    return QS_OK;
}

template <typename T>
int probs_t(qs_state *s, const int *qubits, int m, double *out)
{
    size_t outb = 8ull << m, part_b = 0;
    MargParams P = marginal_plan(s, qubits, m, &part_b);
    const size_t o_part = kBufOff + ((outb + 255) & ~255ull);
    int r = qs_ensure_scratch(s, o_part + part_b);
    if (r) return r;
    char *sc = static_cast<char *>(s->scratch);
    double *dev = reinterpret_cast<double *>(sc + kBufOff);
    if ((r = marginal_launch<T>(s, P, dev, reinterpret_cast<double *>(sc + o_part)))) return r;
    QS_CUDA_TRY(cudaMemcpyAsync(out, dev, outb, cudaMemcpyDeviceToHost, s->stream));
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return QS_OK;
}

template <typename T>
int sample_t(qs_state *s, const int *qubits, int m, const double *u, size_t shots, uint64_t *out)
{
    const int K0 = m < 20 ? m : 20;
    const size_t tree_b = 16ull << K0;            // 2^(K0+1) doubles
    const size_t u_b = 8ull * shots * (size_t)m;
    const size_t out_b = 8ull * shots;
    const int ndeep = m - K0;
    const size_t deep_b = sizeof(Holes) * (size_t)(ndeep > 0 ? ndeep : 1);
    const size_t q_b = 4ull * (m > 0 ? m : 1);
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t o_tree = kBufOff, o_u = o_tree + al(tree_b), o_out = o_u + al(u_b),
           o_deep = o_out + al(out_b), o_q = o_deep + al(deep_b), o_part = o_q + al(q_b);
    size_t part_b = 0;
    MargParams P = marginal_plan(s, qubits, K0, &part_b);
    // Size scratch once, before any pointer into it is taken.
    int r = qs_ensure_scratch(s, o_part + part_b);
    if (r) return r;
    char *sc = static_cast<char *>(s->scratch);
    double *tree = reinterpret_cast<double *>(sc + o_tree);
    // Level K0 = marginal over the first K0 measured qubits, stored at tree + 2^K0.
    if ((r = marginal_launch<T>(s, P, tree + (1ull << K0), reinterpret_cast<double *>(sc + o_part)))) return r;
    for (int k = K0 - 1; k >= 0; --k) {
        k_fold<<<grid_for(1ull << k, kThreads), kThreads, 0, s->stream>>>(tree, k);
        QS_LAUNCH_CHECK("k_fold");
    }
    std::vector<Holes> deep((size_t)(ndeep > 0 ? ndeep : 0));
    for (int k = K0; k < m; ++k) {
        uint64_t mask = 0;
        for (int j = 0; j <= k; ++j) mask |= 1ull << qubits[j];
        deep[(size_t)(k - K0)] = holes_from_mask(mask);
    }
    QS_CUDA_TRY(cudaMemcpyAsync(sc + o_u, u, u_b, cudaMemcpyHostToDevice, s->stream));
    if (ndeep > 0)
        QS_CUDA_TRY(cudaMemcpyAsync(sc + o_deep, deep.data(), sizeof(Holes) * deep.size(),
                                    cudaMemcpyHostToDevice, s->stream));
    QS_CUDA_TRY(cudaMemcpyAsync(sc + o_q, qubits, 4ull * m, cudaMemcpyHostToDevice, s->stream));
    const int thr = 256;
    uint64_t warps_needed = shots;
    unsigned grid = (unsigned)std::min<uint64_t>((warps_needed * 32 + thr - 1) / thr, (uint64_t)QS_SM_COUNT * 8);
    if (grid < 1) grid = 1;
    k_shots<T><<<grid, thr, 0, s->stream>>>(static_cast<const T *>(s->amp), tree, K0, m,
                                            reinterpret_cast<const Holes *>(sc + o_deep),
                                            reinterpret_cast<const int *>(sc + o_q),
                                            reinterpret_cast<const double *>(sc + o_u), shots, s->n,
                                            reinterpret_cast<uint64_t *>(sc + o_out));
    QS_LAUNCH_CHECK("k_shots");
    QS_CUDA_TRY(cudaMemcpyAsync(out, sc + o_out, out_b, cudaMemcpyDeviceToHost, s->stream));
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return QS_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" int qs_prob_zero(qs_state *s, int q, double *p0)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (q < 0 || q >= s->n) return qs_fail(QS_ERR_ARG, "qs_prob_zero: qubit %d out of range", q);
    if (!p0) return qs_fail(QS_ERR_ARG, "qs_prob_zero: null output");
    return s->dtype == QS_C64 ? prob_zero_t<float>(s, q, p0) : prob_zero_t<double>(s, q, p0);
}

extern "C" int qs_measure(qs_state *s, int q, double u, int *outcome)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (q < 0 || q >= s->n) return qs_fail(QS_ERR_ARG, "qs_measure: qubit %d out of range", q);
    if (!outcome) return qs_fail(QS_ERR_ARG, "qs_measure: null output");
    return s->dtype == QS_C64 ? measure_t<float>(s, q, u, outcome) : measure_t<double>(s, q, u, outcome);
}

extern "C" int qs_probs(qs_state *s, const int *qubits, int m, double *out)
{
    int r = qs_check_state(s);
    if (r) return r;
    if ((r = check_qubit_list(s, qubits, m, "qs_probs"))) return r;
    if (!out) return qs_fail(QS_ERR_ARG, "qs_probs: null output");
    return s->dtype == QS_C64 ? probs_t<float>(s, qubits, m, out) : probs_t<double>(s, qubits, m, out);
}

// Marginal into a caller-provided device buffer (2^m doubles); asynchronous.
extern "C" int qs_probs_device(qs_state *s, const int *qubits, int m, double *dev_out)
{
    int r = qs_check_state(s);
    if (r) return r;
    if ((r = check_qubit_list(s, qubits, m, "qs_probs_device"))) return r;
    if (!dev_out) return qs_fail(QS_ERR_ARG, "qs_probs_device: null output");
    size_t part_b = 0;
    MargParams P = marginal_plan(s, qubits, m, &part_b);
    if ((r = qs_ensure_scratch(s, kBufOff + part_b))) return r;
    double *part = reinterpret_cast<double *>(static_cast<char *>(s->scratch) + kBufOff);
    return s->dtype == QS_C64 ? marginal_launch<float>(s, P, dev_out, part)
                              : marginal_launch<double>(s, P, dev_out, part);
}

extern "C" int qs_sample(qs_state *s, const int *qubits, int m, const double *u, size_t shots,
                         uint64_t *out)
{
    int r = qs_check_state(s);
    if (r) return r;
    if ((r = check_qubit_list(s, qubits, m, "qs_sample"))) return r;
    if (m < 1 || m > 64) return qs_fail(QS_ERR_ARG, "qs_sample: need 1..64 qubits");
    if (shots == 0) return QS_OK;
    if (!u || !out) return qs_fail(QS_ERR_ARG, "qs_sample: null buffer");
    return s->dtype == QS_C64 ? sample_t<float>(s, qubits, m, u, shots, out)
                              : sample_t<double>(s, qubits, m, u, shots, out);
}

extern "C" int qs_norm2(qs_state *s, double *norm2)
{
    int r = qs_check_state(s);
    if (r) return r;
    int nb;
    r = s->dtype == QS_C64 ? half_sum<float>(s, -1, &nb) : half_sum<double>(s, -1, &nb);
    if (r) return r;
    double *part = reinterpret_cast<double *>(static_cast<char *>(s->scratch) + kPartOff);
    MeasureResult *res = reinterpret_cast<MeasureResult *>(static_cast<char *>(s->scratch) + kResOff);
    k_finalize<<<1, kThreads, 0, s->stream>>>(part, nb, res, 0, 0.0);
    QS_LAUNCH_CHECK("k_finalize");
    if ((r = read_result(s, kResOff, sizeof(MeasureResult)))) return r;
    *norm2 = static_cast<MeasureResult *>(s->pinned)->p0;
    return QS_OK;
}

extern "C" int qs_inner(qs_state *a, qs_state *b, double *re, double *im)
{
    int r = qs_check_state(a);
    if (r) return r;
    if ((r = qs_check_state(b))) return r;
    if (a->n != b->n) return qs_fail(QS_ERR_ARG, "qs_inner: qubit counts differ (%d vs %d)", a->n, b->n);
    // Order b's pending work before a's reduction.
    QS_CUDA_TRY(cudaStreamSynchronize(b->stream));
    unsigned grid = grid_for(a->N, kThreads, 8);
    double *part = reinterpret_cast<double *>(static_cast<char *>(a->scratch) + kPartOff);
    if (a->dtype == QS_C64 && b->dtype == QS_C64)
        k_inner<float, float><<<grid, kThreads, 0, a->stream>>>((const float *)a->amp, (const float *)b->amp, a->N, part);
    else if (a->dtype == QS_C64)
        k_inner<float, double><<<grid, kThreads, 0, a->stream>>>((const float *)a->amp, (const double *)b->amp, a->N, part);
    else if (b->dtype == QS_C64)
        k_inner<double, float><<<grid, kThreads, 0, a->stream>>>((const double *)a->amp, (const float *)b->amp, a->N, part);
    else
        k_inner<double, double><<<grid, kThreads, 0, a->stream>>>((const double *)a->amp, (const double *)b->amp, a->N, part);
    QS_LAUNCH_CHECK("k_inner");
    double *res = reinterpret_cast<double *>(static_cast<char *>(a->scratch) + kResOff);
    k_finalize2<<<1, kThreads, 0, a->stream>>>(part, (int)grid, res);
    QS_LAUNCH_CHECK("k_finalize2");
    if ((r = read_result(a, kResOff, 16))) return r;
    *re = static_cast<double *>(a->pinned)[0];
    *im = static_cast<double *>(a->pinned)[1];
    return QS_OK;
}

extern "C" int qs_diff(qs_state *a, qs_state *b, double *max_abs, double *sum_sq)
{
    int r = qs_check_state(a);
    if (r) return r;
    if ((r = qs_check_state(b))) return r;
    if (a->n != b->n) return qs_fail(QS_ERR_ARG, "qs_diff: qubit counts differ (%d vs %d)", a->n, b->n);
    QS_CUDA_TRY(cudaStreamSynchronize(b->stream));
    unsigned grid = grid_for(a->N, kThreads, 8);
    double *part = reinterpret_cast<double *>(static_cast<char *>(a->scratch) + kPartOff);
    if (a->dtype == QS_C64 && b->dtype == QS_C64)
        k_diff<float, float><<<grid, kThreads, 0, a->stream>>>((const float *)a->amp, (const float *)b->amp, a->N, part);
    else if (a->dtype == QS_C64)
        k_diff<float, double><<<grid, kThreads, 0, a->stream>>>((const float *)a->amp, (const double *)b->amp, a->N, part);
    else if (b->dtype == QS_C64)
        k_diff<double, float><<<grid, kThreads, 0, a->stream>>>((const double *)a->amp, (const float *)b->amp, a->N, part);
    else
        k_diff<double, double><<<grid, kThreads, 0, a->stream>>>((const double *)a->amp, (const double *)b->amp, a->N, part);
    QS_LAUNCH_CHECK("k_diff");
    double *res = reinterpret_cast<double *>(static_cast<char *>(a->scratch) + kResOff);
    k_finalize_diff<<<1, 32, 0, a->stream>>>(part, (int)grid, res);
    QS_LAUNCH_CHECK("k_finalize_diff");
    if ((r = read_result(a, kResOff, 16))) return r;
    if (max_abs) *max_abs = static_cast<double *>(a->pinned)[0];
    if (sum_sq) *sum_sq = static_cast<double *>(a->pinned)[1];
    return QS_OK;
}

// Host <-> device copies with dtype conversion through a staging area in scratch.
int qs_copy_in(qs_state *s, const void *host, int host_dtype)
{
    if (host_dtype == s->dtype) {
        QS_CUDA_TRY(cudaMemcpyAsync(s->amp, host, s->amp_bytes(), cudaMemcpyHostToDevice, s->stream));
        QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
        return QS_OK;
    }
    const size_t hsz = host_dtype == QS_C64 ? 8 : 16;
    const uint64_t chunk = 1ull << 22;           // amplitudes per staging step
    int r = qs_ensure_scratch(s, kBufOff + chunk * 16);
    if (r) return r;
    char *stage = static_cast<char *>(s->scratch) + kBufOff;
    for (uint64_t i = 0; i < s->N; i += chunk) {
        uint64_t cnt = std::min<uint64_t>(chunk, s->N - i);
        QS_CUDA_TRY(cudaMemcpyAsync(stage, static_cast<const char *>(host) + i * hsz, cnt * hsz,
                                    cudaMemcpyHostToDevice, s->stream));
        if (s->dtype == QS_C64)
            k_convert<float><<<grid_for(2 * cnt, 256), 256, 0, s->stream>>>(stage, host_dtype, (float *)s->amp + 2 * i, cnt);
        else
            k_convert<double><<<grid_for(2 * cnt, 256), 256, 0, s->stream>>>(stage, host_dtype, (double *)s->amp + 2 * i, cnt);
        QS_LAUNCH_CHECK("k_convert");
        QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    return QS_OK;
}

int qs_copy_out(qs_state *s, void *host, int host_dtype)
{
    if (host_dtype == s->dtype) {
        QS_CUDA_TRY(cudaMemcpyAsync(host, s->amp, s->amp_bytes(), cudaMemcpyDeviceToHost, s->stream));
        QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
        return QS_OK;
    }
    const size_t hsz = host_dtype == QS_C64 ? 8 : 16;
    const uint64_t chunk = 1ull << 22;
    int r = qs_ensure_scratch(s, kBufOff + chunk * 16);
    if (r) return r;
    char *stage = static_cast<char *>(s->scratch) + kBufOff;
    for (uint64_t i = 0; i < s->N; i += chunk) {
        uint64_t cnt = std::min<uint64_t>(chunk, s->N - i);
        const char *src = static_cast<const char *>(s->amp) + i * (s->dtype == QS_C64 ? 8 : 16);
        if (host_dtype == QS_C64)
            k_convert<float><<<grid_for(2 * cnt, 256), 256, 0, s->stream>>>(src, s->dtype, (float *)stage, cnt);
        else
            k_convert<double><<<grid_for(2 * cnt, 256), 256, 0, s->stream>>>(src, s->dtype, (double *)stage, cnt);
        QS_LAUNCH_CHECK("k_convert");
        QS_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(host) + i * hsz, stage, cnt * hsz,
                                    cudaMemcpyDeviceToHost, s->stream));
        QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    return QS_OK;
}
