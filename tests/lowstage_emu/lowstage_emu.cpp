// lowstage_emu.cpp - CPU emulation of the staged low-qubit runs, for tests.
//
// Applies a gate list to a complex128 host state the way qs_gates_apply does
// on the GPU: gates lowered by the library (qs_lower_gate), split into passes
// by the library (qs_lowstage_passes: runs of consecutive gates whose targets
// fit one tile's qubits), and each run moved exactly as k_lowstage
// (qpanda_b200/csrc/qs_lowstage.cu) moves it: the plan from the library's own
// planner (qs_low::plan_run_on), the tile bases and 16-byte copy offsets in
// the state (qs_low::tile_base, copy_thread_off, copy_chunk_off: every
// amplitude of the state copied in exactly once and out exactly once per
// run), the copies into the swizzled tile, each
// thread's 8 registers at  thread_off ^ reg_off  through phys, the register
// pairs of every op kind, the predicates on low controls and masks, the
// tile-uniform skip on high ones, and the round trips through shared memory
// at every layout switch.  The arithmetic is FP64 here whatever the dtype; the
// dtype picks the plan (lane order and swizzle for 8- or 16-byte amplitudes).
// Checks: every shared-memory slot written exactly once per copy and per
// register write-back, every slot read exactly once per register read, and
// the bank conflicts of every access phase (counted, not assumed: 16 lanes of
// 8-byte accesses, or 8 lanes of 16-byte ones, on the slots they touch).
// Runs are staged whatever their size (stage_all: the library stages only
// runs that save traffic).
//
// Built by tests/test_lowstage_emulation.py against the library (host code
// only runs; nvcc because the shared header holds device helpers):
//   nvcc -O2 -std=c++17 -x cu -shared -Xcompiler -fPIC lowstage_emu.cpp
//        -I<csrc> -I<include> -L<lib> -lqsb200
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "qs_lowstage.cuh"
#include "qs_prim.h"

int qs_lowstage_bits(int n);
void qs_lowstage_passes(const std::vector<qs_prim> &prims, int n, int dtype, bool stage_all,
                        std::vector<qs_low::Pass> &out);

namespace {

typedef std::complex<double> cd;
char g_err[256];

int fail(const char *msg, long long a = 0, long long b = 0)
{
    snprintf(g_err, sizeof(g_err), msg, a, b);
    return 1;
}

// a primitive on the whole state, as k_pair / k_phase define it
void apply_direct(std::vector<cd> &a, const qs_prim &p)
{
    const uint64_t N = a.size();
    if (p.kind == QS_PRIM_PHASE) {
        const cd ph(p.m[0], p.m[1]);
        for (uint64_t i = 0; i < N; ++i)
            if ((i & p.holes) == p.holes) a[i] *= ph;
        return;
    }
    const cd m00(p.m[0], p.m[1]), m01(p.m[2], p.m[3]), m10(p.m[4], p.m[5]), m11(p.m[6], p.m[7]);
    for (uint64_t i = 0; i < N; ++i) {
        if ((i & p.holes) != p.cmask) continue;         // base: holes clear except the controls
        const cd x = a[i | p.off0], y = a[i | p.off1];
        a[i | p.off0] = m00 * x + m01 * y;
        a[i | p.off1] = m10 * x + m11 * y;
    }
}

struct Stats {
    long long reg_conflicts;     // extra shared-memory wavefronts of register reads / writes
    long long copy_conflicts;    // extra wavefronts of the HBM <-> shared copies
    long long layout_switches;
    long long runs;
};

// extra wavefronts of one access instruction: lanes -> slots, phases of
// `per_phase` lanes, `units` slots per 128-byte row
long long conflicts(const std::vector<int64_t> &slot_of_lane, int per_phase, int units)
{
    long long extra = 0;
    for (size_t p0 = 0; p0 < slot_of_lane.size(); p0 += per_phase) {
        std::vector<std::vector<int64_t>> by(units);
        for (size_t l = p0; l < p0 + per_phase && l < slot_of_lane.size(); ++l) {
            const int64_t s = slot_of_lane[l];
            if (s < 0) continue;
            bool dup = false;
            for (int64_t o : by[s % units]) dup |= o == s;
            if (!dup) by[s % units].push_back(s);
        }
        size_t worst = 1;
        for (auto &v : by) worst = std::max(worst, v.size());
        extra += (long long)worst - 1;
    }
    return extra;
}

template <typename T>
int emulate_run(std::vector<cd> &a, int n, const std::vector<qs_prim> &run, uint64_t qmask, Stats &st)
{
    using namespace qs_low;
    const int K = qs_lowstage_bits(n);
    if (K < kMinLowBits || K > kLowBits) return fail("tile width %lld out of range", K);
    if (__builtin_popcountll(qmask) != K || !(qmask & 1) || (qmask >> n)) return fail("tile qubits 0x%llx", (long long)qmask);
    for (const qs_prim &p : run)
        if (p.kind == QS_PRIM_PAIR && ((p.off0 | p.off1) & ~qmask)) return fail("a gate's targets are not tile qubits");
    Run<T> R;
    const TileMap M = {K, qmask};
    plan_run_on(run, M, n, &R);
    if (R.count != (int)run.size() || R.nlayouts < 1 || R.nlayouts > kMaxRun + 1) return fail("bad plan");
    const uint32_t TN = 1u << K;
    const int tbits = K - kRegBits;
    const uint32_t threads = 1u << tbits;
    const int units = bank_row_bits<T>() == 4 ? 16 : 8;     // amplitude slots per 128-byte row
    const int phase = sizeof(T) == 4 ? 16 : 8;              // lanes per shared-memory phase
    // every layout must be a bijection of (thread, register) onto the tile
    for (int l = 0; l < R.nlayouts; ++l) {
        std::vector<int> seen(TN, 0);
        uint32_t rb[kRegBits];
        for (int j = 0; j < kRegBits; ++j) rb[j] = R.L[l].rb[j];
        for (uint32_t t = 0; t < threads; ++t)
            for (int r = 0; r < 8; ++r) {
                const uint32_t i = thread_off(R.L[l], t, tbits) | reg_off(r, rb);
                if (i >= TN || seen[i]++) return fail("layout %lld does not cover the tile (index %lld)", l, i);
            }
    }
    std::vector<cd> slot(TN);
    std::vector<int> wr(TN), rd(TN);
    std::vector<cd> vals(threads * 8);
    uint32_t tb[kMaxThreads], pt[kMaxThreads], rb[kRegBits], pr[kRegBits];
    auto set_layout = [&](const Layout &L) {
        for (uint32_t t = 0; t < threads; ++t) {
            tb[t] = thread_off(L, t, tbits);
            pt[t] = phys<T>(tb[t]);
        }
        for (int j = 0; j < kRegBits; ++j) {
            rb[j] = L.rb[j];
            pr[j] = L.pr[j];                          // the kernel's slot offsets, from the plan
        }
    };
    auto access = [&](bool write) -> int {
        std::fill(write ? wr.begin() : rd.begin(), write ? wr.end() : rd.end(), 0);
        for (int r = 0; r < 8; ++r) {
            std::vector<int64_t> lanes(threads);
            for (uint32_t t = 0; t < threads; ++t) {
                const uint32_t s = pt[t] ^ reg_off(r, pr);
                if (s >= TN) return fail("slot %lld out of the tile", s);
                lanes[t] = s;
                if (write) {
                    if (wr[s]++) return fail("slot %lld written twice", s);
                    slot[s] = vals[t * 8 + r];
                } else {
                    if (rd[s]++) return fail("slot %lld read twice", s);
                    vals[t * 8 + r] = slot[s];
                }
            }
            st.reg_conflicts += conflicts(lanes, phase, units);
        }
        return 0;
    };
    // state offset of tile index i (the copies' view): chunk c = t + k threads
    // of thread t holds tile indices 2c, 2c + 1 (complex64) or c (complex128)
    std::vector<uint64_t> off(TN);
    for (uint32_t t = 0; t < threads; ++t)
        for (uint32_t k = 0; k < (sizeof(T) == 4 ? 4u : 8u); ++k) {
            const uint64_t o = copy_thread_off<T>(t, K, R.qoff) | copy_chunk_off<T>(k, K, R.qoff);
            const uint32_t c = t + k * threads;
            if (sizeof(T) == 4) {
                if (o & 1) return fail("16-byte copy at an odd amplitude (thread %lld, chunk %lld)", t, k);
                off[2 * c] = o;
                off[2 * c + 1] = o | 1;
            } else {
                off[c] = o;
            }
        }
    std::vector<uint8_t> touched(a.size(), 0);
    const uint64_t tiles = a.size() >> K;
    for (uint64_t tl = 0; tl < tiles; ++tl) {
        const uint64_t base = tile_base(tl, K, R.qpos);
        for (uint32_t i = 0; i < TN; ++i) {
            const uint64_t at = base | off[i];
            if (at >= a.size() || touched[at]++) return fail("amplitude %lld copied twice or out of range", (long long)at);
        }
        // HBM -> shared memory
        std::fill(wr.begin(), wr.end(), 0);
        if (sizeof(T) == 4) {
            std::vector<int64_t> lanes;
            for (uint32_t c = 0; c < TN / 2; ++c) {
                const uint32_t p = phys<T>(2 * c);
                const uint32_t s0 = (p >> 1) * 2;              // the float4 slot pair
                slot[s0] = (p & 1) ? a[base | off[2 * c + 1]] : a[base | off[2 * c]];
                slot[s0 + 1] = (p & 1) ? a[base | off[2 * c]] : a[base | off[2 * c + 1]];
                if (wr[s0]++ || wr[s0 + 1]++) return fail("copy slot %lld written twice", s0);
                lanes.push_back(p >> 1);
            }
            st.copy_conflicts += conflicts(lanes, 8, 8);
        } else {
            std::vector<int64_t> lanes;
            for (uint32_t c = 0; c < TN; ++c) {
                const uint32_t s = phys<T>(c);
                if (s >= TN || wr[s]++) return fail("copy slot %lld written twice", s);
                slot[s] = a[base | off[c]];
                lanes.push_back(s);
            }
            st.copy_conflicts += conflicts(lanes, 8, 8);
        }
        set_layout(R.L[0]);
        if (access(false)) return 1;
        for (int g = 0; g < R.count; ++g) {
            const Op<T> &op = R.op[g];
            if (op.layout >= 0) {
                if (access(true)) return 1;
                set_layout(R.L[op.layout]);
                if (access(false)) return 1;
                if (base == 0) ++st.layout_switches;
            }
            if ((base & op.need) != op.need) continue;
            int HB, B0, B1;
            if (op.kind == OP_PHASE) {
                HB = B0 = B1 = 0;
            } else if (op.kind < OP_EX) {
                HB = B1 = 1 << (op.kind - OP_1Q);
                B0 = 0;
            } else if (op.kind >= OP_DIAG && op.kind < OP_FLIP + 3) {
                // the full 2x2 on the pair: its zero entries must be zeros
                const bool flip = op.kind >= OP_FLIP;
                HB = B1 = 1 << (op.kind - (flip ? OP_FLIP : OP_DIAG));
                B0 = 0;
                const int z0 = flip ? 0 : 2, z1 = flip ? 6 : 4;
                if (op.m[z0] != 0 || op.m[z0 + 1] != 0 || op.m[z1] != 0 || op.m[z1 + 1] != 0)
                    return fail("op %lld: nonzero entries off its sparse pattern", g);
            } else {
                static const int ex[6][2] = {{1, 2}, {1, 4}, {2, 4}, {2, 1}, {4, 1}, {4, 2}};
                if (op.kind - OP_EX >= 6) return fail("bad op kind %lld", op.kind);
                B0 = ex[op.kind - OP_EX][0];
                B1 = ex[op.kind - OP_EX][1];
                HB = B0 | B1;
            }
            const cd m00(op.m[0], op.m[1]), m01(op.m[2], op.m[3]), m10(op.m[4], op.m[5]), m11(op.m[6], op.m[7]);
            for (uint32_t t = 0; t < threads; ++t) {
                cd *v = &vals[t * 8];
                for (int r = 0; r < 8; ++r) {
                    if (((tb[t] | reg_off(r, rb)) & op.set) != op.set) continue;
                    if (op.kind == OP_PHASE) {
                        v[r] *= m00;
                        continue;
                    }
                    if (r & HB) continue;
                    const cd x = v[r | B0], y = v[r | B1];
                    v[r | B0] = m00 * x + m01 * y;
                    v[r | B1] = m10 * x + m11 * y;
                }
            }
        }
        if (access(true)) return 1;
        for (uint32_t i = 0; i < TN; ++i)
            if (wr[i] != 1) return fail("slot %lld not written back", i);
        // shared memory -> HBM
        for (uint32_t i = 0; i < TN; ++i) a[base | off[i]] = slot[phys<T>(i)];
    }
    for (uint64_t i = 0; i < a.size(); ++i)
        if (touched[i] != 1) return fail("amplitude %lld not in exactly one tile", (long long)i);
    ++st.runs;
    return 0;
}

}  // namespace

extern "C" const char *lowstage_emu_error(void) { return g_err; }

// amp: 2^n complex128, in place.  gates: qs_gate records.  dtype: QS_C64 or
// QS_C128 (the plan's).  stats[4]: register-access conflicts, copy
// conflicts, layout switches (first tile), runs.  Returns 0 or 1.
extern "C" int lowstage_emu_apply(double *amp, int n, const void *gates, int count, int dtype, long long *stats)
{
    g_err[0] = 0;
    std::vector<cd> a((size_t)1 << n);
    memcpy(a.data(), amp, sizeof(cd) * a.size());
    const qs_gate *g = static_cast<const qs_gate *>(gates);
    Stats st = {0, 0, 0, 0};
    std::vector<qs_prim> prims(count);
    for (int i = 0; i < count; ++i)
        if (qs_lower_gate(n, &g[i], &prims[i])) return fail("gate %lld does not lower", i);
    std::vector<qs_low::Pass> passes;
    qs_lowstage_passes(prims, n, dtype, true, passes);
    size_t next = 0;
    for (const qs_low::Pass &ps : passes) {
        if (ps.first != next || ps.count < 1 || (int)ps.count > qs_low::kMaxRun)
            return fail("passes do not cover the gate list in order (at %lld)", (long long)next);
        next = ps.first + ps.count;
        if (!ps.qmask) {
            apply_direct(a, prims[ps.first]);
            continue;
        }
        std::vector<qs_prim> run(prims.begin() + ps.first, prims.begin() + ps.first + ps.count);
        if (dtype == QS_C64 ? emulate_run<float>(a, n, run, ps.qmask, st)
                            : emulate_run<double>(a, n, run, ps.qmask, st))
            return 1;
    }
    if (next != (size_t)count) return fail("passes end at %lld", (long long)next);
    memcpy(amp, a.data(), sizeof(cd) * a.size());
    stats[0] = st.reg_conflicts;
    stats[1] = st.copy_conflicts;
    stats[2] = st.layout_switches;
    stats[3] = st.runs;
    return 0;
}

// The passes qs_gates_apply makes for a gate list: out[0] staged passes,
// out[1] per-gate launches, out[2] gates in staged passes.  Returns 0 or 1.
extern "C" int lowstage_emu_passes(int n, const void *gates, int count, int dtype, long long *out)
{
    g_err[0] = 0;
    const qs_gate *g = static_cast<const qs_gate *>(gates);
    std::vector<qs_prim> prims(count);
    for (int i = 0; i < count; ++i)
        if (qs_lower_gate(n, &g[i], &prims[i])) return fail("gate %lld does not lower", i);
    std::vector<qs_low::Pass> passes;
    qs_lowstage_passes(prims, n, dtype, false, passes);
    out[0] = out[1] = out[2] = 0;
    for (const qs_low::Pass &ps : passes) {
        if (ps.qmask) {
            ++out[0];
            out[2] += (long long)ps.count;
        } else {
            ++out[1];
        }
    }
    return 0;
}
