// qs_lowstage.cu - the per-gate path with the low-stride qubits staged in
// shared memory.
//
// A gate whose target bits (the pair it mixes, or none for a phase) lie below
// qubit K (= 10) mixes amplitudes inside aligned runs of 2^K.  A run of such
// gates - consecutive in the gate list; their controls and phase masks may
// include any qubits - is applied in one pass: each CTA loads a 2^K-amplitude
// tile (16-byte loads), applies every gate of the run to it in shared memory
// with a barrier between gates, and writes it back.  A gate whose controls or
// mask bits at or above K are not all set in the tile's base leaves the tile
// alone.  The per-amplitude arithmetic is k_pair's and k_phase's
// (qs_gates.cu), so the state after the run is the state after the gates one
// by one.  Gates on higher targets keep the streaming kernels, whose
// pair-index remapping handles any stride.
#include <cstring>
#include <vector>

#include "qs_common.cuh"
#include "qs_prim.h"

namespace {

constexpr int kLowBits = 10;
constexpr int kMaxRun = 24;
constexpr int kThreads = 256;

template <typename T>
struct LowPrim {
    uint64_t need;               // bits >= K that every touched amplitude has set
    uint32_t holes;              // bits < K with a zero inserted when enumerating
    uint32_t set;                // bits < K set in every touched amplitude
    uint32_t off0, off1;         // pair members (kind PAIR)
    uint32_t nholes;
    uint32_t kind;
    T m[8];                      // PAIR: 2x2 row-major complex; PHASE: m[0] + i m[1]
};

template <typename T>
struct LowRun {
    int count;
    LowPrim<T> p[kMaxRun];
};

template <typename T>
__device__ __forceinline__ void cmul_add2(T &xr, T &xi, T ar, T ai, T br, T bi, const T *r0, const T *r1)
{
    T re = r0[0] * ar - r0[1] * ai;
    T im = r0[0] * ai + r0[1] * ar;
    re = fma(r1[0], br, re); re = fma(-r1[1], bi, re);
    im = fma(r1[0], bi, im); im = fma(r1[1], br, im);
    xr = re; xi = im;
}

// insert a zero at every set bit of `holes` (ascending)
__device__ __forceinline__ uint32_t spread(uint32_t w, uint32_t holes)
{
    while (holes) {
        const uint32_t low = (holes & (0u - holes)) - 1;     // bits below the lowest hole
        w = ((w & ~low) << 1) | (w & low);
        holes &= holes - 1;
    }
    return w;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_lowstage(T *__restrict__ a, uint64_t tiles, int K, LowRun<T> R)
{
    typedef typename vec2<T>::type V;
    extern __shared__ __align__(16) unsigned char lsm[];
    V *tile = reinterpret_cast<V *>(lsm);
    const uint32_t TN = 1u << K;
    V *pa = reinterpret_cast<V *>(a);
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t base = t << K;
        // load: 16-byte vectors
        if constexpr (sizeof(T) == 4) {
            const float4 *src = reinterpret_cast<const float4 *>(pa + base);
            float4 *dst = reinterpret_cast<float4 *>(tile);
            for (uint32_t i = threadIdx.x; i < TN / 2; i += kThreads) dst[i] = src[i];
        } else {
            for (uint32_t i = threadIdx.x; i < TN; i += kThreads) tile[i] = pa[base + i];
        }
        __syncthreads();
        for (int g = 0; g < R.count; ++g) {
            const LowPrim<T> &p = R.p[g];
            if ((base & p.need) != p.need) continue;          // the same for the whole CTA
            const uint32_t items = TN >> p.nholes;
            if (p.kind == QS_PRIM_PAIR) {
                for (uint32_t w = threadIdx.x; w < items; w += kThreads) {
                    const uint32_t i = spread(w, p.holes) | p.set;
                    V x = tile[i | p.off0], y = tile[i | p.off1];
                    T xr, xi, yr, yi;
                    cmul_add2(xr, xi, x.x, x.y, y.x, y.y, &p.m[0], &p.m[2]);
                    cmul_add2(yr, yi, x.x, x.y, y.x, y.y, &p.m[4], &p.m[6]);
                    tile[i | p.off0] = V{xr, xi};
                    tile[i | p.off1] = V{yr, yi};
                }
            } else {
                const T pr = p.m[0], pi = p.m[1];
                for (uint32_t w = threadIdx.x; w < items; w += kThreads) {
                    const uint32_t i = spread(w, p.holes) | p.set;
                    const V x = tile[i];
                    tile[i] = V{x.x * pr - x.y * pi, x.x * pi + x.y * pr};
                }
            }
            __syncthreads();
        }
        if constexpr (sizeof(T) == 4) {
            float4 *dst = reinterpret_cast<float4 *>(pa + base);
            const float4 *src = reinterpret_cast<const float4 *>(tile);
            for (uint32_t i = threadIdx.x; i < TN / 2; i += kThreads) dst[i] = src[i];
        } else {
            for (uint32_t i = threadIdx.x; i < TN; i += kThreads) pa[base + i] = tile[i];
        }
        __syncthreads();
    }
}

template <typename T>
int launch_run(qs_state *s, const std::vector<qs_prim> &run, int K)
{
    LowRun<T> R;
    memset(&R, 0, sizeof(R));
    R.count = (int)run.size();
    const uint64_t low = (1ull << K) - 1;
    for (size_t g = 0; g < run.size(); ++g) {
        const qs_prim &q = run[g];
        LowPrim<T> &p = R.p[g];
        p.kind = (uint32_t)q.kind;
        if (q.kind == QS_PRIM_PAIR) {
            p.need = q.cmask & ~low;
            p.holes = (uint32_t)(q.holes & low);             // target/exchange bits and low controls
            p.set = (uint32_t)(q.cmask & low);
            p.off0 = (uint32_t)q.off0;
            p.off1 = (uint32_t)q.off1;
            for (int j = 0; j < 8; ++j) p.m[j] = (T)q.m[j];
        } else {
            p.need = q.holes & ~low;
            p.holes = (uint32_t)(q.holes & low);
            p.set = (uint32_t)(q.holes & low);
            p.m[0] = (T)q.m[0];
            p.m[1] = (T)q.m[1];
        }
        p.nholes = (uint32_t)__builtin_popcount(p.holes);
    }
    const uint64_t tiles = s->N >> K;
    const size_t smem = sizeof(typename vec2<T>::type) << K;
    const unsigned grid = grid_for(tiles, 1, 8);
    k_lowstage<T><<<grid, kThreads, smem, s->stream>>>(static_cast<T *>(s->amp), tiles, K, R);
    QS_LAUNCH_CHECK("k_lowstage");
    return QS_OK;
}

}  // namespace

// Width of the staged tiles for an n-qubit state.
int qs_lowstage_bits(int n) { return n < kLowBits ? n : kLowBits; }

// Whether primitive p can join a staged run on an n-qubit state: its target
// bits below the tile width (controls and phase masks may be anywhere).
bool qs_lowstage_fits(const qs_prim &p, int n)
{
    const uint64_t low = (1ull << qs_lowstage_bits(n)) - 1;
    if (p.kind == QS_PRIM_PHASE) return true;
    return ((p.holes & ~p.cmask) & ~low) == 0 && (p.off0 & ~low) == 0 && (p.off1 & ~low) == 0;
}

int qs_lowstage_max_run() { return kMaxRun; }

// HBM traffic of primitive p on the per-gate kernels, in full passes over the
// state: the amplitudes it touches, counted in whole 32-byte sectors (4
// complex64 or 2 complex128 amplitudes).  Each control or phase-mask bit at
// or above the sector halves it; so does an exchange whose higher bit is.
double qs_lowstage_traffic(const qs_prim &p, int dtype)
{
    const int sb = dtype == QS_C64 ? 2 : 1;
    const uint64_t above = ~((1ull << sb) - 1);
    int halvings;
    if (p.kind == QS_PRIM_PHASE) {
        halvings = __builtin_popcountll(p.holes & above);
    } else {
        halvings = __builtin_popcountll(p.cmask & above);
        const uint64_t ex = p.off0 | p.off1;
        if (p.off0 && (ex & above)) ++halvings;      // the exchange family touches a != b only
    }
    return 1.0 / (double)(1ull << halvings);
}

// Apply a run of primitives that all fit (qs_lowstage_fits) in one pass.
int qs_launch_lowstage(qs_state *s, const std::vector<qs_prim> &run)
{
    if (run.empty()) return QS_OK;
    if ((int)run.size() > kMaxRun) return qs_fail(QS_ERR_ARG, "staged run of %zu gates (at most %d)", run.size(), kMaxRun);
    const int K = qs_lowstage_bits(s->n);
    return s->dtype == QS_C64 ? launch_run<float>(s, run, K) : launch_run<double>(s, run, K);
}
