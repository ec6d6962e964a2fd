// qs_lowstage.cuh - the plan of a staged run (k_lowstage, qs_lowstage.cu):
// the tile's qubits, register layouts, the shared-memory swizzle and the op
// list.  Host code plus the index helpers the kernel shares; included by the
// kernel and by the CPU emulation of its index arithmetic.
//
// A tile is the 2^K amplitudes that agree on every qubit outside a set Q of K
// qubits (qubit 0 always among them, and qubit 1 for complex64, so that the
// copies move whole 32-byte sectors); tile bit k is the k-th qubit of Q in
// ascending order.  A run is planned on its gates with every mask carried by
// the tile map (the qubits of Q -> bits 0..K-1, the others -> K, K+1, ... in
// ascending order), so below K every mask speaks of tile bits; a gate's
// controls outside Q are a per-tile condition, in the state's own bits.
//
// A CTA owns a tile; each of its 2^(K-3) threads holds 8
// amplitudes in registers.  A layout names the tile bit behind each of the 3
// register index bits and each thread index bit: thread t's register r holds
// tile index  tb(t) | rb(r),  tb / rb the deposits of t / r's bits at those
// positions.  The planner gives every pair gate a layout in which its target
// bits are register bits.
//
// Shared memory is XOR-swizzled: tile index i lives in slot
//   phys(i) = i ^ f(i),  f(i) = ((i >> lb) & (2^lb - 1)) ^ (parity(i >> 2lb) ? 2^lb - 1 : 0)
// with 2^lb amplitudes per 128-byte bank row (lb = 4 for complex64, 3 for
// complex128).  phys is linear over GF(2) and moves only bits below lb, so it
// is a permutation of every aligned 2^K block (K >= lb) and a thread's 8
// slots are its base slot XOR'd with the slots of its register bits.  The
// banks of one access phase (16 lanes of 8-byte accesses, 8 lanes of 16-byte
// ones) are the images of its lane bits under phys; each layout orders its
// thread bits so that the first lb have linearly independent images, which
// puts every phase on distinct banks.  On a full 10-bit tile, for any 3
// register bits the 7 others always hold lb such bits: bits b and b + lb have
// image e_b, bits >= 2lb the all-ones vector.  (Narrower tiles - whole states
// below 10 qubits - may not, and then clash on some accesses.)  The 16-byte
// copies between HBM and shared memory move 8 consecutive chunks per quarter
// warp, on which f is constant.
#pragma once

#include <stdint.h>
#include <string.h>

#include <vector>

#include "qs_prim.h"

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace qs_low {

constexpr int kLowBits = 10;
constexpr int kMinLowBits = 5;
constexpr int kRegBits = 3;
constexpr int kMaxRun = 24;
constexpr int kMaxThreads = 1 << (kLowBits - kRegBits);

// op kinds: a phase; a pair on register bit k (1 + k); an exchange pair whose
// members have register bit ja and jb set, (ja, jb) = (0,1), (0,2), (1,2),
// (1,0), (2,0), (2,1) (4 .. 9) - both orders, so that the arithmetic is
// k_pair's operand for operand; a pair on register bit k whose matrix is
// diagonal (10 + k: RZ, a phase on the target) or anti-diagonal (13 + k: X,
// Y, the CNOT and Toffoli targets), which skip the products with its zero
// entries (k_pair adds them as exact zeros)
enum : uint8_t { OP_PHASE = 0, OP_1Q = 1, OP_EX = 4, OP_DIAG = 10, OP_FLIP = 13, OP_KINDS = 16 };

struct Layout {
    uint16_t rb[kRegBits];                   // tile offset (a power of two) of register index bit j
    uint16_t pr[kRegBits];                   // phys(rb[j]): its shared-memory slot offset
    uint16_t tb[kLowBits - kRegBits];        // tile offset of thread index bit k (K - 3 of them used)
};

template <typename T>
struct Op {
    uint64_t need;               // bits >= K that every touched amplitude has set
    uint32_t set;                // bits < K set in every touched amplitude
    int16_t layout;              // >= 0: move the registers to this layout first
    uint8_t kind;
    T m[8];                      // pair: 2x2 row-major complex; phase: m[0] + i m[1]
};

template <typename T>
struct Run {
    int count;
    int nlayouts;
    Layout L[kMaxRun + 1];
    Op<T> op[kMaxRun];
    uint64_t qoff[kLowBits];     // 2^q of the tile's qubit q behind tile bit k
    int8_t qpos[kLowBits];       // the tile's qubits, ascending
};

// The tile's qubits: the set bits of qmask (K of them), ascending.
struct TileMap {
    int K;
    uint64_t qmask;
};

// A mask in the state's bits -> tile-map order (see the top of this file).
inline uint64_t map_bits(uint64_t m, const TileMap &M, int n)
{
    uint64_t out = 0;
    int lo = 0, hi = M.K;
    for (int q = 0; q < n; ++q) {
        const int to = ((M.qmask >> q) & 1) ? lo++ : hi++;
        if ((m >> q) & 1) out |= 1ull << to;
    }
    return out;
}

// The inverse of map_bits.
inline uint64_t unmap_bits(uint64_t m, const TileMap &M, int n)
{
    uint64_t out = 0;
    int lo = 0, hi = M.K;
    for (int q = 0; q < n; ++q) {
        const int from = ((M.qmask >> q) & 1) ? lo++ : hi++;
        if ((m >> from) & 1) out |= 1ull << q;
    }
    return out;
}

// State offset of tile tl's first amplitude: tl's bits spread over the
// qubits outside the tile (zeros inserted at the tile's qubits).
__host__ __device__ __forceinline__ uint64_t tile_base(uint64_t tl, int K, const int8_t *qpos)
{
    for (int j = 0; j < K; ++j) {
        const uint64_t low = (1ull << qpos[j]) - 1;
        tl = ((tl & ~low) << 1) | (tl & low);
    }
    return tl;
}

// The copies between the state and shared memory: thread t's chunk k is the
// tile's chunk c = t + k 2^(K-3), a 16-byte vector (two complex64 amplitudes,
// tile indices 2c and 2c + 1; or one complex128, tile index c).  Its state
// offset from the tile base is copy_thread_off(t) | copy_chunk_off(k): the
// thread's bits land on tile bits 1.. (complex64) or 0.. (complex128), k's on
// the 2 (3) tile bits above them.
template <typename T>
__host__ __device__ __forceinline__ uint64_t copy_thread_off(uint32_t t, int K, const uint64_t *qoff)
{
    const int first = sizeof(T) == 4 ? 1 : 0;
    uint64_t o = 0;
    for (int j = 0; j < K - kRegBits; ++j)
        if ((t >> j) & 1u) o |= qoff[first + j];
    return o;
}

template <typename T>
__host__ __device__ __forceinline__ uint64_t copy_chunk_off(uint32_t k, int K, const uint64_t *qoff)
{
    const int kb = sizeof(T) == 4 ? 2 : 3;
    uint64_t o = 0;
    for (int j = 0; j < kb; ++j)
        if ((k >> j) & 1u) o |= qoff[K - kb + j];
    return o;
}

template <typename T>
__host__ __device__ constexpr int bank_row_bits() { return sizeof(T) == 4 ? 4 : 3; }

template <typename T>
__host__ __device__ __forceinline__ uint32_t phys(uint32_t i)
{
    constexpr int lb = bank_row_bits<T>();
    constexpr uint32_t m = (1u << lb) - 1;
#ifdef __CUDA_ARCH__
    const uint32_t par = __popc(i >> (2 * lb)) & 1;
#else
    const uint32_t par = __builtin_popcount(i >> (2 * lb)) & 1;
#endif
    return i ^ ((i >> lb) & m) ^ (par ? m : 0);
}

// offset of register r in a layout with register-bit offsets b[]
__host__ __device__ __forceinline__ uint32_t reg_off(int r, const uint32_t (&b)[kRegBits])
{
    return ((r & 1) ? b[0] : 0u) ^ ((r & 2) ? b[1] : 0u) ^ ((r & 4) ? b[2] : 0u);
}

// thread t's tile offset in layout L (tbits thread bits)
__host__ __device__ __forceinline__ uint32_t thread_off(const Layout &L, uint32_t t, int tbits)
{
    uint32_t tb = 0;
    for (int k = 0; k < tbits; ++k) tb |= ((t >> k) & 1u) * L.tb[k];
    return tb;
}

// Bank bits (within one 128-byte row) of tile bit b under phys.
template <typename T>
inline uint32_t bank_image(int b)
{
    constexpr int lb = bank_row_bits<T>();
    if (b < lb) return 1u << b;
    if (b < 2 * lb) return 1u << (b - lb);
    return (1u << lb) - 1;
}

// A layout whose register bits are `regs` (in order): the other tile bits are
// the thread bits, the first lb of them with independent bank images, the
// rest ascending.
template <typename T>
inline Layout make_layout(const std::vector<int> &regs, int K)
{
    Layout L;
    memset(&L, 0, sizeof(L));
    for (int j = 0; j < kRegBits; ++j) {
        L.rb[j] = (uint16_t)(1u << regs[j]);
        L.pr[j] = (uint16_t)phys<T>(L.rb[j]);
    }
    std::vector<int> rest, order;
    for (int b = 0; b < K; ++b)
        if (b != regs[0] && b != regs[1] && b != regs[2]) rest.push_back(b);
    uint32_t basis[8] = {0};                       // echelon basis, by leading bit
    std::vector<bool> used(rest.size(), false);
    for (size_t k = 0; k < rest.size() && (int)order.size() < bank_row_bits<T>(); ++k) {
        uint32_t v = bank_image<T>(rest[k]);
        for (int hb = 7; hb >= 0 && v; --hb)
            if (((v >> hb) & 1) && basis[hb]) v ^= basis[hb];
        if (!v) continue;
        basis[31 - __builtin_clz(v)] = v;
        order.push_back(rest[k]);
        used[k] = true;
    }
    for (size_t k = 0; k < rest.size(); ++k)
        if (!used[k]) order.push_back(rest[k]);
    for (size_t k = 0; k < order.size(); ++k) L.tb[k] = (uint16_t)(1u << order[k]);
    return L;
}

// The plan of a run of primitives that all fit a K-bit tile (1 <= size <=
// kMaxRun, K in [kMinLowBits, kLowBits]).  Layouts: the first pair gate's
// target bits, then those of the following pair gates while they fit, then
// the lowest free bits; a new layout only where a pair gate's targets are
// not all register bits.
template <typename T>
inline void plan_run(const std::vector<qs_prim> &run, int K, Run<T> *R)
{
    memset(R, 0, sizeof(*R));
    R->count = (int)run.size();
    const uint64_t low = (1ull << K) - 1;
    auto targets = [&](const qs_prim &q) -> uint32_t {
        return q.kind == QS_PRIM_PAIR ? (uint32_t)((q.off0 | q.off1) & low) : 0u;
    };
    auto plan_layout = [&](size_t from, std::vector<int> &regs) -> uint32_t {
        regs.clear();
        uint32_t have = 0;
        for (size_t g = from; g < run.size(); ++g) {
            const uint32_t tg = targets(run[g]);
            if (!tg) continue;
            if (__builtin_popcount(have | tg) > kRegBits) break;
            for (int b = 0; b < K; ++b)
                if (((tg >> b) & 1) && !((have >> b) & 1)) regs.push_back(b);
            have |= tg;
        }
        for (int b = 0; b < K && (int)regs.size() < kRegBits; ++b)
            if (!((have >> b) & 1)) {
                regs.push_back(b);
                have |= 1u << b;
            }
        return have;
    };
    std::vector<int> regs;
    uint32_t cur = plan_layout(0, regs);
    R->L[R->nlayouts++] = make_layout<T>(regs, K);
    for (size_t g = 0; g < run.size(); ++g) {
        const qs_prim &q = run[g];
        Op<T> &p = R->op[g];
        p.layout = -1;
        const uint32_t tg = targets(q);
        if (tg & ~cur) {
            cur = plan_layout(g, regs);
            p.layout = (int16_t)R->nlayouts;
            R->L[R->nlayouts++] = make_layout<T>(regs, K);
        }
        auto reg_of = [&](int bit) {
            for (int j = 0; j < kRegBits; ++j)
                if (regs[j] == bit) return j;
            return 0;                                   // not reached: targets are register bits
        };
        if (q.kind == QS_PRIM_PAIR) {
            p.need = q.cmask & ~low;
            p.set = (uint32_t)(q.cmask & low);
            if (q.off0 == 0) {
                const int rk = reg_of(__builtin_ctzll(q.off1));
                const bool diag = q.m[2] == 0 && q.m[3] == 0 && q.m[4] == 0 && q.m[5] == 0;
                const bool flip = q.m[0] == 0 && q.m[1] == 0 && q.m[6] == 0 && q.m[7] == 0;
                p.kind = (uint8_t)((diag ? OP_DIAG : flip ? OP_FLIP : OP_1Q) + rk);
            } else {
                static const int8_t ex_kind[3][3] = {{0, 0, 1}, {3, 0, 2}, {4, 5, 0}};
                p.kind = (uint8_t)(OP_EX + ex_kind[reg_of(__builtin_ctzll(q.off0))][reg_of(__builtin_ctzll(q.off1))]);
            }
            for (int j = 0; j < 8; ++j) p.m[j] = (T)q.m[j];
        } else {
            p.kind = OP_PHASE;
            p.need = q.holes & ~low;
            p.set = (uint32_t)(q.holes & low);
            p.m[0] = (T)q.m[0];
            p.m[1] = (T)q.m[1];
        }
    }
}

// The plan of a run on the tile of qubits M.qmask of an n-qubit state: the
// run's masks carried by the tile map, planned by plan_run, each op's
// per-tile condition carried back to the state's bits.
template <typename T>
inline void plan_run_on(const std::vector<qs_prim> &run, const TileMap &M, int n, Run<T> *R)
{
    std::vector<qs_prim> loc(run);
    for (qs_prim &p : loc) {
        p.holes = map_bits(p.holes, M, n);
        p.cmask = map_bits(p.cmask, M, n);
        p.off0 = map_bits(p.off0, M, n);
        p.off1 = map_bits(p.off1, M, n);
    }
    plan_run(loc, M.K, R);
    for (int g = 0; g < R->count; ++g) R->op[g].need = unmap_bits(R->op[g].need, M, n);
    int k = 0;
    for (int q = 0; q < n && k < M.K; ++q)
        if ((M.qmask >> q) & 1) {
            R->qpos[k] = (int8_t)q;
            R->qoff[k] = 1ull << q;
            ++k;
        }
}

// The passes of a lowered gate list (qs_lowstage_passes, qs_lowstage.cu):
// prims [first, first + count) as one staged pass on the tile of qubits
// qmask, or, with qmask 0, one per-gate launch each.
struct Pass {
    size_t first, count;
    uint64_t qmask;
};

}  // namespace qs_low
