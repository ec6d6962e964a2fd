// qs_lowstage.cu - the per-gate path with runs of gates staged in shared
// memory and registers.
//
// A gate whose target bits (the pair it mixes, or none for a phase) lie in a
// set Q of K (= 10) qubits mixes amplitudes inside the tiles of Q: the 2^K
// amplitudes that agree on every other qubit.  A run of such gates -
// consecutive in the gate list, their targets together within K qubits
// (qubit 0, and 1 for complex64, always in Q; the rest of Q the lowest
// qubits left); their controls and phase masks may include any qubits - is
// applied in one pass: each CTA loads a tile (16-byte copies; qubits 0..2 in
// Q make them whole 32- or 64-byte runs of the state) into shared memory and
// each of its 2^(K-3) threads takes 8 of the tile's amplitudes into
// registers.  Which 3 tile bits index a
// thread's registers (its *layout*) is chosen on the host per stretch of the
// run so that every gate's target bits are register bits when it is applied:
// the gate then mixes register pairs of one thread, with no shared-memory
// traffic and no barrier.  Only when the next gate needs other register bits
// do the amplitudes go back through shared memory (8 stores, a barrier, 8
// loads per thread).  A gate whose controls or mask bits outside Q are not
// all set in the tile's base leaves the tile alone; controls and mask bits in
// Q are a per-amplitude predicate.  The per-amplitude arithmetic is k_pair's
// and k_phase's (qs_gates.cu), so the state after the run is the state after
// the gates one by one.  A run that would not save traffic (a lone gate, a
// pair of controlled phases) keeps the streaming kernels, whose pair-index
// remapping handles any stride.
//
// The layouts, the shared-memory swizzle (every access phase on distinct
// banks) and the planner are in qs_lowstage.cuh.
#include <cstring>
#include <vector>

#include "qs_common.cuh"
#include "qs_lowstage.cuh"
#include "qs_prim.h"

namespace {

using namespace qs_low;

template <typename T>
__device__ __forceinline__ void cmul_add2(T &xr, T &xi, T ar, T ai, T br, T bi, const T *r0, const T *r1)
{
    T re = r0[0] * ar - r0[1] * ai;
    T im = r0[0] * ai + r0[1] * ar;
    re = fma(r1[0], br, re); re = fma(-r1[1], bi, re);
    im = fma(r1[0], bi, im); im = fma(r1[1], br, im);
    xr = re; xi = im;
}

// the pairs (r | B0, r | B1) over r with no bit of HB: one thread's share of
// a pair gate whose target bits are register bits; PRED: low control bits
// (set) to check per pair
template <typename T, int HB, int B0, int B1, bool PRED>
__device__ __forceinline__ void apply_pairs(T (&vr)[8], T (&vi)[8], const T (&m)[8], uint32_t tb,
                                            const uint32_t (&rb)[kRegBits], uint32_t set)
{
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        if (r & HB) continue;
        if (PRED && ((tb | reg_off(r, rb)) & set) != set) continue;
        const T ar = vr[r | B0], ai = vi[r | B0], br = vr[r | B1], bi = vi[r | B1];
        cmul_add2(vr[r | B0], vi[r | B0], ar, ai, br, bi, &m[0], &m[2]);
        cmul_add2(vr[r | B1], vi[r | B1], ar, ai, br, bi, &m[4], &m[6]);
    }
}

// The pairs (r, r | B) of a 1-qubit gate with a diagonal matrix (FLIP =
// false: x' = m00 x, y' = m11 y) or an anti-diagonal one (FLIP: x' = m01 y,
// y' = m10 x): cmul_add2's arithmetic with the zero entries' products, exact
// zeros there, left out.
template <typename T, int B, bool FLIP, bool PRED>
__device__ __forceinline__ void apply_sparse(T (&vr)[8], T (&vi)[8], const T (&m)[8], uint32_t tb,
                                             const uint32_t (&rb)[kRegBits], uint32_t set)
{
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        if (r & B) continue;
        if (PRED && ((tb | reg_off(r, rb)) & set) != set) continue;
        const T ar = vr[r], ai = vi[r], br = vr[r | B], bi = vi[r | B];
        // each output in the form cmul_add2 gives it when its first operand
        // (r0) or its second (r1) is the zero entry
        if (FLIP) {
            vr[r] = fma(-m[3], bi, m[2] * br);
            vi[r] = fma(m[3], br, m[2] * bi);
            vr[r | B] = m[4] * ar - m[5] * ai;
            vi[r | B] = m[4] * ai + m[5] * ar;
        } else {
            vr[r] = m[0] * ar - m[1] * ai;
            vi[r] = m[0] * ai + m[1] * ar;
            vr[r | B] = fma(-m[7], bi, m[6] * br);
            vi[r | B] = fma(m[7], br, m[6] * bi);
        }
    }
}

template <typename T>
__device__ __forceinline__ void apply_phase(T (&vr)[8], T (&vi)[8], T pr, T pi, uint32_t tb,
                                            const uint32_t (&rb)[kRegBits], uint32_t set)
{
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        if (((tb | reg_off(r, rb)) & set) != set) continue;
        const T x = vr[r], y = vi[r];
        vr[r] = x * pr - y * pi;
        vi[r] = x * pi + y * pr;
    }
}

template <typename T>
__global__ void __launch_bounds__(kMaxThreads) k_lowstage(T *__restrict__ a, uint64_t tiles, int K, Run<T> R)
{
    typedef typename vec2<T>::type V;
    extern __shared__ __align__(16) unsigned char lsm[];
    V *tile = reinterpret_cast<V *>(lsm);
    const int tbits = K - kRegBits;
    const uint32_t t = threadIdx.x;
    // 16-byte chunks per thread: the tile's 2^K amplitudes over 2^(K-3) threads
    constexpr uint32_t kChunks = sizeof(T) == 4 ? 4 : 8;
    // per layout, this thread's tile offset and its slot: computed once per CTA
    uint2 *lt = reinterpret_cast<uint2 *>(lsm + (sizeof(V) << K));
    for (int l = 0; l < R.nlayouts; ++l) {
        const uint32_t o = thread_off(R.L[l], t, tbits);
        lt[l * blockDim.x + t] = make_uint2(o, phys<T>(o));
    }
    uint32_t tb = 0, pt = 0, rb[kRegBits], pr[kRegBits];
    auto set_layout = [&](int l) {
        const uint2 v = lt[l * blockDim.x + t];
        tb = v.x;
        pt = v.y;
#pragma unroll
        for (int j = 0; j < kRegBits; ++j) {
            rb[j] = R.L[l].rb[j];
            pr[j] = R.L[l].pr[j];
        }
    };
    T vr[8], vi[8];
    auto read_regs = [&]() {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const V x = tile[pt ^ reg_off(r, pr)];
            vr[r] = x.x;
            vi[r] = x.y;
        }
    };
    auto write_regs = [&]() {
#pragma unroll
        for (int r = 0; r < 8; ++r) tile[pt ^ reg_off(r, pr)] = V{vr[r], vi[r]};
    };
    // the thread's part of every copy offset (its chunks differ in the bits above)
    const uint64_t cto = copy_thread_off<T>(t, K, R.qoff);
    for (uint64_t tl = blockIdx.x; tl < tiles; tl += gridDim.x) {
        const uint64_t base = tile_base(tl, K, R.qpos);
        // HBM -> shared memory, 16-byte chunks: all of a thread's chunks
        // loaded before any is stored (their loads in flight together)
        if constexpr (sizeof(T) == 4) {
            const float4 *src = reinterpret_cast<const float4 *>(a);
            float4 *dst = reinterpret_cast<float4 *>(lsm);
            float4 v[kChunks];
#pragma unroll
            for (uint32_t k = 0; k < kChunks; ++k) v[k] = src[(base | cto | copy_chunk_off<T>(k, K, R.qoff)) >> 1];
#pragma unroll
            for (uint32_t k = 0; k < kChunks; ++k) {
                const uint32_t p = phys<T>(2 * (t + k * blockDim.x));
                dst[p >> 1] = (p & 1) ? make_float4(v[k].z, v[k].w, v[k].x, v[k].y) : v[k];
            }
        } else {
            const double2 *src = reinterpret_cast<const double2 *>(a);
            double2 v[kChunks];
#pragma unroll
            for (uint32_t k = 0; k < kChunks; ++k) v[k] = src[base | cto | copy_chunk_off<T>(k, K, R.qoff)];
#pragma unroll
            for (uint32_t k = 0; k < kChunks; ++k) tile[phys<T>(t + k * blockDim.x)] = v[k];
        }
        __syncthreads();
        set_layout(0);
        read_regs();
        for (int g = 0; g < R.count; ++g) {
            const Op<T> &op = R.op[g];
            if (op.layout >= 0) {                         // the same for the whole CTA
                write_regs();                             // own slots: no barrier needed before
                __syncthreads();
                set_layout(op.layout);
                read_regs();
            }
            if ((base & op.need) != op.need) continue;    // the same for the whole CTA
            T m[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) m[j] = op.m[j];
            const bool pred = op.set != 0;
            switch (op.kind + (pred ? OP_KINDS : 0)) {
            case OP_PHASE:
            case OP_PHASE + OP_KINDS: apply_phase(vr, vi, m[0], m[1], tb, rb, op.set); break;
#define QS_LOW_PAIR_CASES(P, OFF)                                                             \
            case OFF + OP_1Q + 0: apply_pairs<T, 1, 0, 1, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_1Q + 1: apply_pairs<T, 2, 0, 2, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_1Q + 2: apply_pairs<T, 4, 0, 4, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_EX + 0: apply_pairs<T, 3, 1, 2, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_EX + 1: apply_pairs<T, 5, 1, 4, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_EX + 2: apply_pairs<T, 6, 2, 4, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_EX + 3: apply_pairs<T, 3, 2, 1, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_EX + 4: apply_pairs<T, 5, 4, 1, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_EX + 5: apply_pairs<T, 6, 4, 2, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_DIAG + 0: apply_sparse<T, 1, false, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_DIAG + 1: apply_sparse<T, 2, false, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_DIAG + 2: apply_sparse<T, 4, false, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_FLIP + 0: apply_sparse<T, 1, true, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_FLIP + 1: apply_sparse<T, 2, true, P>(vr, vi, m, tb, rb, op.set); break; \
            case OFF + OP_FLIP + 2: apply_sparse<T, 4, true, P>(vr, vi, m, tb, rb, op.set); break;
            QS_LOW_PAIR_CASES(false, 0)
            QS_LOW_PAIR_CASES(true, OP_KINDS)
#undef QS_LOW_PAIR_CASES
            default: break;
            }
        }
        write_regs();
        __syncthreads();
        // shared memory -> HBM
        if constexpr (sizeof(T) == 4) {
            float4 *dst = reinterpret_cast<float4 *>(a);
            const float4 *src = reinterpret_cast<const float4 *>(lsm);
#pragma unroll
            for (uint32_t k = 0; k < kChunks; ++k) {
                const uint32_t p = phys<T>(2 * (t + k * blockDim.x));
                const float4 v = src[p >> 1];
                dst[(base | cto | copy_chunk_off<T>(k, K, R.qoff)) >> 1] = (p & 1) ? make_float4(v.z, v.w, v.x, v.y) : v;
            }
        } else {
            double2 *dst = reinterpret_cast<double2 *>(a);
#pragma unroll
            for (uint32_t k = 0; k < kChunks; ++k)
                dst[base | cto | copy_chunk_off<T>(k, K, R.qoff)] = tile[phys<T>(t + k * blockDim.x)];
        }
        __syncthreads();
    }
}

template <typename T>
int launch_run(qs_state *s, const std::vector<qs_prim> &run, const TileMap &M)
{
    const int K = M.K;
    Run<T> R;
    plan_run_on(run, M, s->n, &R);
    const uint64_t tiles = s->N >> K;
    // the tile, then per layout each thread's (tile offset, slot)
    const size_t smem = (sizeof(typename vec2<T>::type) << K) + sizeof(uint2) * R.nlayouts * (1u << (K - kRegBits));
    const unsigned grid = grid_for(tiles, 1, 16);
    k_lowstage<T><<<grid, 1u << (K - kRegBits), smem, s->stream>>>(static_cast<T *>(s->amp), tiles, K, R);
    QS_LAUNCH_CHECK("k_lowstage");
    return QS_OK;
}

}  // namespace

// Width of the staged tiles for an n-qubit state (0: no staging on states
// this small).
int qs_lowstage_bits(int n) { return n < kMinLowBits ? 0 : n < kLowBits ? n : kLowBits; }

// The qubits a primitive mixes (none for a phase): they must be tile qubits.
static uint64_t prim_targets(const qs_prim &p) { return p.kind == QS_PRIM_PHASE ? 0 : (p.off0 | p.off1); }

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

// The passes of a lowered gate list on an n-qubit state of dtype: runs of
// consecutive primitives whose targets, with the qubits of a 64-byte run of
// the state (0..2 for complex64, 0..1 for complex128), fit K =
// qs_lowstage_bits(n) qubits - at most kMaxRun each - staged in one
// pass on the tile of those qubits and the lowest others (K in all), when
// that moves fewer bytes than the gates one by one would, or when `stage_all`
// (the CPU emulation's coverage); otherwise each primitive on its own.
void qs_lowstage_passes(const std::vector<qs_prim> &prims, int n, int dtype, bool stage_all,
                        std::vector<Pass> &out)
{
    out.clear();
    const int K = qs_lowstage_bits(n);
    if (!K) {
        for (size_t i = 0; i < prims.size(); ++i) out.push_back({i, 1, 0});
        return;
    }
    const uint64_t all = n >= 64 ? ~0ull : (1ull << n) - 1;
    const uint64_t seed = (dtype == QS_C64 ? 7ull : 3ull) & all;
    size_t first = 0;
    uint64_t q = seed;
    auto close = [&](size_t end) {
        const size_t count = end - first;
        if (!count) return;
        double per_gate = 0;
        for (size_t i = first; i < end; ++i) per_gate += qs_lowstage_traffic(prims[i], dtype);
        if (stage_all || (count > 1 && per_gate > 1.0)) {
            uint64_t m = q;
            for (int b = 0; b < n && __builtin_popcountll(m) < K; ++b) m |= 1ull << b;
            out.push_back({first, count, m});
        } else {
            for (size_t i = first; i < end; ++i) out.push_back({i, 1, 0});
        }
        first = end;
        q = seed;
    };
    for (size_t i = 0; i < prims.size(); ++i) {
        const uint64_t t = prim_targets(prims[i]);
        if ((int)(i - first) == kMaxRun || __builtin_popcountll(q | t) > K) close(i);
        q |= t;
    }
    close(prims.size());
}

// Apply a run of primitives whose targets lie in the qubits of qmask (K =
// qs_lowstage_bits(n) of them, qubit 0 among them: a 16-byte copy then holds
// two tile neighbours) in one pass.
int qs_launch_lowstage(qs_state *s, const std::vector<qs_prim> &run, uint64_t qmask)
{
    if (run.empty()) return QS_OK;
    if ((int)run.size() > kMaxRun) return qs_fail(QS_ERR_ARG, "staged run of %zu gates (at most %d)", run.size(), kMaxRun);
    const int K = qs_lowstage_bits(s->n);
    if (!K) return qs_fail(QS_ERR_ARG, "staged run on a %d-qubit state (at least %d qubits)", s->n, kMinLowBits);
    if (__builtin_popcountll(qmask) != K || !(qmask & 1ull) || (s->n < 64 && (qmask >> s->n)))
        return qs_fail(QS_ERR_ARG, "staged run: tile qubits 0x%llx (%d of them, with qubit 0)",
                       (unsigned long long)qmask, K);
    for (const qs_prim &p : run)
        if (prim_targets(p) & ~qmask) return qs_fail(QS_ERR_ARG, "staged run: a gate's targets are not tile qubits");
    const TileMap M = {K, qmask};
    return s->dtype == QS_C64 ? launch_run<float>(s, run, M) : launch_run<double>(s, run, M);
}
