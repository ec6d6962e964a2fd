// qs_plan.cpp - gate fusion: runs of gates -> dense k-qubit blocks.
//
// A plan is built once on the host from a gate list and applied to any
// state of the same qubit count.  Blocks are formed greedily in list order:
// a gate joins the open block when every earlier gate on its qubits has
// already been placed (so moving it forward only passes gates on other
// qubits, with which it commutes) and the block's qubit set stays within k.
// Each block's 2^k x 2^k unitary is the product of its gates, computed in
// FP64 by applying the same primitive operations the per-gate path uses
// (qs_lower_gate) to the columns of the identity.  Blocks with fewer than 5
// qubits are widened with the lowest free qubits so that every pass uses the
// same 5-qubit tensor-core kernel (qs_fused.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <cstring>
#include <vector>

#include "qs_common.cuh"
#include "qs_fused.h"
#include "qs_prim.h"

typedef std::complex<double> cd;

#include "qs_plan_internal.h"

namespace {

uint64_t remap(uint64_t mask, const int *q, int k)
{
    uint64_t r = 0;
    for (int b = 0; b < k; ++b)
        if (mask & (1ull << q[b])) r |= 1ull << b;
    return r;
}

uint16_t bf16_bits(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    u += 0x7fffu + ((u >> 16) & 1u);      // round to nearest even
    return (uint16_t)(u >> 16);
}

float bf16_float(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// What a scan in list order has passed over without placing: a later gate
// may be placed ahead of those earlier gates only if it commutes with each of
// them - it shares no qubit with it, or both are diagonal in the computational
// basis (RZ and CR with any controls: phases, which commute with each other
// whatever their qubits).  Diagonality is decided by the gate's kind, never by
// its angle, so that plans rebound to other angles keep a valid order.
struct Blocker {
    uint64_t any = 0;                    // qubits of passed non-diagonal gates
    uint64_t diag = 0;                   // qubits of passed diagonal gates
    bool free(uint64_t m, bool d) const { return !(m & any) && (d || !(m & diag)); }
    void add(uint64_t m, bool d) { (d ? diag : any) |= m; }
};

// Greedy fusion of the gates idx[] (in list order) into groups of at most k
// qubits: a gate joins the open group when every earlier unplaced gate
// commutes with it (Blocker) and the group stays within k qubits.  Returns
// the groups' member lists and qubit masks.
std::vector<std::pair<uint64_t, std::vector<size_t>>> greedy_groups(const std::vector<size_t> &idx,
                                                                    const std::vector<uint64_t> &mask,
                                                                    const std::vector<char> &diag, int k,
                                                                    uint64_t seed_mask = 0, int max_groups = 0)
{
    std::vector<std::pair<uint64_t, std::vector<size_t>>> out;
    std::vector<char> done(idx.size(), 0);
    size_t left = idx.size(), first = 0;
    while (left) {
        uint64_t Q = seed_mask;
        std::vector<size_t> mem;
        bool changed = true;
        while (changed) {
            changed = false;
            Blocker bl;
            while (first < idx.size() && done[first]) ++first;
            for (size_t t = first; t < idx.size(); ++t) {
                if (done[t]) continue;
                const uint64_t m = mask[idx[t]];
                const bool d = diag[idx[t]];
                if (bl.free(m, d) && __builtin_popcountll(Q | m) <= k) {
                    done[t] = 1;
                    --left;
                    Q |= m;
                    mem.push_back(idx[t]);
                    changed = true;
                } else {
                    bl.add(m, d);
                }
            }
        }
        out.push_back(std::make_pair(Q, std::move(mem)));
        if (max_groups && (int)out.size() > max_groups) break;
    }
    return out;
}

typedef std::vector<std::pair<uint64_t, std::vector<size_t>>> Groups;

// Closure-first fusion of the gates idx[] (in list order) into groups of at
// most k qubits.  A group starts with the first unplaced gate, then takes
// every available gate whose qubits it already has (available: no earlier
// unplaced gate fails to commute with it - Blocker), and only when none is
// left grows by one available gate:
// the one after which the next closure would take the most gates (ratio =
// false), or the most gates per qubit added (ratio = true); then the one
// adding the fewest qubits, then the earliest.  Taking gates in list
// order instead lets a gate on new qubits in early and fills the group before
// the gates that would have fitted.  Gate counts per group on the 32-qubit
// depth-16 random circuit (768 gates): 89 groups in list order, 72 growing by
// fewest new qubits, 65 with the look-ahead (63 by ratio); a 24-qubit QFT
// 76 -> 55, a 20-qubit 6-layer ansatz 30 -> 21 (fewest new qubits ->
// look-ahead).
//
// With tile_q > 0 the groups are formed for passes of up to per_pass groups
// whose qubits and tile_low must fit tile_q qubits: a group that continues a
// pass grows only within that budget, and one whose first gate does not fit
// starts a new pass.
// Growth candidates whose look-ahead is evaluated per step: the first 24
// available gates in list order.  On the circuits measured (random layers,
// QFT, ansatz) the plans equal the unbounded search; a 32-qubit QFT plans in
// 30 ms instead of 112 (with 12 the plans lose 1-2 passes).
constexpr int kMaxCandidates = 24;

Groups closure_groups(const std::vector<size_t> &idx, const std::vector<uint64_t> &mask,
                      const std::vector<char> &diag, int k, bool ratio, uint64_t tile_low = 0, int tile_q = 0,
                      int per_pass = 1)
{
    Groups out;
    const size_t N = idx.size();
    std::vector<char> done(N, 0);
    size_t left = N, first = 0;
    // How many gates the closure of Q would take (and which, in *take when
    // take is non-null), gates marked in `trial` counting as placed: repeated
    // scans in list order; a scan stops once every qubit of Q is held by an
    // earlier unplaced non-diagonal gate.
    std::vector<char> trial(N, 0);
    auto closure = [&](uint64_t Q, std::vector<size_t> *take) {
        int n = 0;
        std::vector<size_t> touched;
        bool changed = true;
        while (changed) {
            changed = false;
            Blocker bl;
            for (size_t t = first; t < N && (Q & ~bl.any); ++t) {
                if (done[t] || trial[t]) continue;
                const uint64_t m = mask[idx[t]];
                const bool d = diag[idx[t]];
                if (bl.free(m, d) && !(m & ~Q)) {
                    trial[t] = 1;
                    touched.push_back(t);
                    ++n;
                    changed = true;
                } else {
                    bl.add(m, d);
                }
            }
        }
        for (size_t t : touched) trial[t] = 0;
        if (take) *take = std::move(touched);
        return n;
    };
    auto place = [&](size_t t, uint64_t &Q, std::vector<size_t> &mem) {
        done[t] = 1;
        --left;
        Q |= mask[idx[t]];
        mem.push_back(idx[t]);
    };
    uint64_t all_q = 0;                      // every qubit the gates touch
    for (size_t t = 0; t < N; ++t) all_q |= mask[idx[t]];
    uint64_t pass_T = tile_low;              // tile so far of the pass being filled (tile_q > 0)
    int in_pass = 0;
    while (left) {
        while (first < N && done[first]) ++first;
        if (tile_q > 0 && in_pass > 0 && __builtin_popcountll(pass_T | mask[idx[first]]) > tile_q) {
            pass_T = tile_low;               // the next gate does not fit this pass: start a new one
            in_pass = 0;
        }
        const uint64_t budget_T = tile_q > 0 && in_pass > 0 ? pass_T : 0;
        uint64_t Q = 0;
        std::vector<size_t> mem;
        place(first, Q, mem);                // seed: the first unplaced gate
        while (true) {
            std::vector<size_t> take;
            closure(Q, &take);
            for (size_t t : take) place(t, Q, mem);
            Blocker bl;                      // grow: available gates that fit
            int best_n = -1, best_add = 65;
            size_t best = N;
            int evaluated = 0;               // the first kMaxCandidates available gates are tried
            for (size_t t = first; t < N && (all_q & ~bl.any) && evaluated < kMaxCandidates; ++t) {
                if (done[t]) continue;
                const uint64_t m = mask[idx[t]];
                const bool d = diag[idx[t]];
                if (bl.free(m, d) && __builtin_popcountll(Q | m) <= k &&
                    (!budget_T || __builtin_popcountll(budget_T | Q | m) <= tile_q)) {
                    const int add = __builtin_popcountll(m & ~Q);
                    ++evaluated;
                    trial[t] = 1;
                    const int got = closure(Q | m, nullptr);
                    trial[t] = 0;
                    // by ratio: (got + 1) / max(add, 1) against the best's, cross-multiplied
                    const long lhs = (long)(got + 1) * (best_add > 1 ? best_add : 1);
                    const long rhs = (long)(best_n + 1) * (add > 1 ? add : 1);
                    const bool better = best == N || (ratio ? (lhs > rhs || (lhs == rhs && add < best_add))
                                                            : (got > best_n || (got == best_n && add < best_add)));
                    if (better) {
                        best_n = got;
                        best_add = add;
                        best = t;
                    }
                }
                bl.add(m, d);
            }
            if (best == N) break;
            place(best, Q, mem);
        }
        if (tile_q > 0) {
            pass_T |= Q;
            if (++in_pass == per_pass) {
                pass_T = tile_low;
                in_pass = 0;
            }
        }
        out.push_back(std::make_pair(Q, std::move(mem)));
    }
    return out;
}

// Block unitary: qubits q[0..4] ascending (global), gates applied in order.
// U starts as the identity and each gate acts on its rows, all 32 columns at
// once (column c gets exactly the operations the gates would apply to e_c), in
// plain real arithmetic: each gate's masks are mapped to the block once, and
// no complex multiply goes through the library's checked routine.
void block_unitary(PlanBlock &B, const std::vector<qs_prim> &prim)
{
    double re[32][32], im[32][32];
    for (int r = 0; r < 32; ++r)
        for (int c = 0; c < 32; ++c) {
            re[r][c] = r == c ? 1.0 : 0.0;
            im[r][c] = 0.0;
        }
    for (size_t gi : B.gates) {
        const qs_prim &p = prim[gi];
        const uint64_t holes = remap(p.holes, B.q, 5);
        if (p.kind == QS_PRIM_PHASE) {
            const double pr = p.m[0], pi = p.m[1];
            for (int r = 0; r < 32; ++r) {
                if ((r & holes) != holes) continue;
                for (int c = 0; c < 32; ++c) {
                    const double a = re[r][c], b = im[r][c];
                    re[r][c] = a * pr - b * pi;
                    im[r][c] = a * pi + b * pr;
                }
            }
            continue;
        }
        const uint64_t cmask = remap(p.cmask, B.q, 5), off0 = remap(p.off0, B.q, 5), off1 = remap(p.off1, B.q, 5);
        const double *m = p.m;                       // m00, m01, m10, m11 as (re, im)
        // a plain exchange of the two rows (NOT, CNOT, SWAP, Toffoli, CSWAP):
        // the products with 1 and 0 below would give exactly the swapped rows
        const bool exchange = m[0] == 0 && m[1] == 0 && m[6] == 0 && m[7] == 0 && m[2] == 1 && m[3] == 0 &&
                              m[4] == 1 && m[5] == 0;
        const bool diagonal = m[2] == 0 && m[3] == 0 && m[4] == 0 && m[5] == 0;
        for (int i = 0; i < 32; ++i) {
            if ((i & holes) != cmask) continue;
            double *ar = re[i | off0], *ai = im[i | off0], *br = re[i | off1], *bi = im[i | off1];
            if (exchange) {
                for (int c = 0; c < 32; ++c) {
                    std::swap(ar[c], br[c]);
                    std::swap(ai[c], bi[c]);
                }
                continue;
            }
            if (diagonal) {                          // RZ and the like: the zero products add nothing
                for (int c = 0; c < 32; ++c) {
                    const double xr = ar[c], xi = ai[c], yr = br[c], yi = bi[c];
                    ar[c] = m[0] * xr - m[1] * xi;
                    ai[c] = m[0] * xi + m[1] * xr;
                    br[c] = m[6] * yr - m[7] * yi;
                    bi[c] = m[6] * yi + m[7] * yr;
                }
                continue;
            }
            for (int c = 0; c < 32; ++c) {
                const double xr = ar[c], xi = ai[c], yr = br[c], yi = bi[c];
                ar[c] = (m[0] * xr - m[1] * xi) + (m[2] * yr - m[3] * yi);
                ai[c] = (m[0] * xi + m[1] * xr) + (m[2] * yi + m[3] * yr);
                br[c] = (m[4] * xr - m[5] * xi) + (m[6] * yr - m[7] * yi);
                bi[c] = (m[4] * xi + m[5] * xr) + (m[6] * yi + m[7] * yr);
            }
        }
    }
    B.U.resize(32 * 32);
    for (int r = 0; r < 32; ++r)
        for (int c = 0; c < 32; ++c) B.U[r * 32 + c] = cd(re[r][c], im[r][c]);
}

// Widen a mask to `want` qubits with the lowest free qubits of `pool`.
uint64_t widen(uint64_t Q, uint64_t pool, int want)
{
    for (int q = 0; q < 64 && __builtin_popcountll(Q) < want; ++q)
        if ((pool >> q) & 1ull) Q |= 1ull << q;
    return Q;
}

void mask_to_list(uint64_t Q, int *out)
{
    int k = 0;
    for (int q = 0; q < 64; ++q)
        if ((Q >> q) & 1ull) out[k++] = q;
}

// Lowered primitives, qubit masks and (when diag is non-null) which gates are
// diagonal: RZ and CR records, with or without controls - by kind, checked
// against their lowered matrices.
int lower_all(qs_plan *P, std::vector<qs_prim> &prim, std::vector<uint64_t> &mask, std::vector<char> *diag = nullptr)
{
    const size_t G = P->gates.size();
    prim.resize(G);
    mask.resize(G);
    if (diag) diag->assign(G, 0);
    for (size_t i = 0; i < G; ++i) {
        int r = qs_lower_gate(P->n, &P->gates[i], &prim[i]);
        if (r) return r;
        mask[i] = qs_gate_qubits(&P->gates[i]);
        if (diag) {
            const int op = P->gates[i].op;
            const qs_prim &q = prim[i];
            const bool diagonal_matrix = q.kind == QS_PRIM_PHASE ||
                                         (q.m[2] == 0 && q.m[3] == 0 && q.m[4] == 0 && q.m[5] == 0);
            (*diag)[i] = (op == QS_OP_RZ || op == QS_OP_CR) && diagonal_matrix;
        }
        if (__builtin_popcountll(mask[i]) > P->max_k)
            return qs_fail(QS_ERR_UNSUPPORTED, "plan: gate %zu touches %d qubits (fusion width %d)", i,
                           __builtin_popcountll(mask[i]), P->max_k);
    }
    return QS_OK;
}

// Single-block passes: every block is one pass of k_fused_tc.
int build_blocks(qs_plan *P)
{
    std::vector<qs_prim> prim;
    std::vector<uint64_t> mask;
    std::vector<char> diag;
    int r = lower_all(P, prim, mask, &diag);
    if (r) return r;
    std::vector<size_t> all(P->gates.size());
    for (size_t i = 0; i < all.size(); ++i) all[i] = i;
    const uint64_t every = P->n >= 64 ? ~0ull : ((1ull << P->n) - 1);
    Groups ga = greedy_groups(all, mask, diag, P->max_k), gb = closure_groups(all, mask, diag, P->max_k, false),
           gc = closure_groups(all, mask, diag, P->max_k, true);
    Groups &gbc = gc.size() < gb.size() ? gc : gb;
    for (auto &grp : gbc.size() < ga.size() ? gbc : ga) {
        PlanBlock B;
        B.gates = grp.second;
        mask_to_list(widen(grp.first, every, 5), B.q);
        B.k = 5;
        block_unitary(B, prim);
        P->blocks.push_back(std::move(B));
    }
    return QS_OK;
}

// Tiled passes.  A pass's tile holds the lowest low_qubits qubits (so that
// every row of the tile is a run of at least 2^low_qubits contiguous
// amplitudes) and the qubits of its blocks, at most tile_qubits in all; a
// pass applies up to max_sub blocks of 5 qubits.  Two drafts are built and
// the one with fewer passes is kept (the first on a tie):
//   tile-first: a pass takes gates in list order while its qubits stay
//     within the tile and its gates still fuse (greedy_groups) into at most
//     max_sub blocks;
//   blocks-first: all gates are fused into blocks (closure_groups, four
//     ways: two look-ahead scores, each free or keeping a pass's later
//     blocks within the tile), and consecutive blocks share a pass while
//     their qubits and the low qubits fit one tile.
// On the 32-qubit depth-16 random circuit the first gives 46 passes and the
// second 32; on a 28-qubit QFT 51 and 31.
struct DraftPass {
    uint64_t T;                          // tile qubits before widening
    Groups blocks;
};

std::vector<DraftPass> draft_tile_first(const std::vector<uint64_t> &mask, const std::vector<char> &diag, int TQ,
                                        int MS, uint64_t low)
{
    std::vector<DraftPass> out;
    const size_t G = mask.size();
    std::vector<char> done(G, 0);
    size_t left = G;
    while (left) {
        uint64_t T = low;
        std::vector<size_t> mem;
        bool changed = true;
        while (changed) {
            changed = false;
            Blocker bl;
            for (size_t i = 0; i < G; ++i) {
                if (done[i]) continue;
                const uint64_t m = mask[i];
                const bool d = diag[i];
                if (bl.free(m, d) && __builtin_popcountll(T | m) <= TQ) {
                    std::vector<size_t> trial = mem;
                    trial.push_back(i);
                    if ((int)greedy_groups(trial, mask, diag, 5, 0, MS).size() <= MS) {
                        done[i] = 1;
                        --left;
                        T |= m;
                        mem.push_back(i);
                        changed = true;
                        continue;
                    }
                }
                bl.add(m, d);
            }
        }
        if (mem.empty()) return {};
        out.push_back(DraftPass{T, greedy_groups(mem, mask, diag, 5)});
    }
    return out;
}

std::vector<DraftPass> draft_blocks_first(const std::vector<uint64_t> &mask, const std::vector<char> &diag, int TQ,
                                          int MS, uint64_t low)
{
    std::vector<size_t> all(mask.size());
    for (size_t i = 0; i < all.size(); ++i) all[i] = i;
    // four fusions: look-ahead by gates taken or by gates per qubit added,
    // free or with each pass's later blocks kept within the tile
    std::vector<DraftPass> best;
    for (int v = 0; v < 4; ++v) {
        Groups g = closure_groups(all, mask, diag, 5, v & 1, low, v & 2 ? TQ : 0, MS);
        std::vector<DraftPass> out;
        for (size_t i = 0; i < g.size();) {
            DraftPass d{low | g[i].first, {}};
            size_t c = 1;
            while ((int)c < MS && i + c < g.size() && __builtin_popcountll(d.T | g[i + c].first) <= TQ) {
                d.T |= g[i + c].first;
                ++c;
            }
            for (size_t j = i; j < i + c; ++j) d.blocks.push_back(std::move(g[j]));
            out.push_back(std::move(d));
            i += c;
        }
        if (v == 0 || out.size() < best.size()) best = std::move(out);
    }
    return best;
}

int build_passes(qs_plan *P)
{
    std::vector<qs_prim> prim;
    std::vector<uint64_t> mask;
    std::vector<char> diag;
    int r = lower_all(P, prim, mask, &diag);
    if (r) return r;
    const int TQ = P->opts.tile_qubits, MS = P->opts.max_sub;
    const uint64_t every = P->n >= 64 ? ~0ull : ((1ull << P->n) - 1);
    const uint64_t low = (1ull << P->opts.low_qubits) - 1;
    std::vector<DraftPass> a = draft_tile_first(mask, diag, TQ, MS, low);
    if (a.empty() && !mask.empty()) return qs_fail(QS_ERR_UNSUPPORTED, "plan: no gate fits a %d-qubit tile", TQ);
    std::vector<DraftPass> b = draft_blocks_first(mask, diag, TQ, MS, low);
    const std::vector<DraftPass> &d = b.size() < a.size() ? b : a;
    for (const DraftPass &dp : d) {
        PlanPass pass;
        const uint64_t T = widen(dp.T, every, TQ);
        mask_to_list(T, pass.T);
        pass.first = P->blocks.size();
        for (const auto &grp : dp.blocks) {
            PlanBlock B;
            B.gates = grp.second;
            mask_to_list(widen(grp.first, T, 5), B.q);
            B.k = 5;
            block_unitary(B, prim);
            P->blocks.push_back(std::move(B));
        }
        pass.count = P->blocks.size() - pass.first;
        int qpos[3][5];
        for (size_t k = 0; k < pass.count && k < 3; ++k)
            for (int j = 0; j < 5; ++j) qpos[k][j] = P->blocks[pass.first + k].q[j];
        if (P->n >= TQ && (r = qs_tile_row_orders(P->n, pass.T, (int)pass.count, qpos, pass.rows)))
            return r;                        // narrower states run the gates per gate
        P->passes.push_back(pass);
    }
    return QS_OK;
}

// R = [[Re U, -Im U], [Im U, Re U]] interleaved, split into bf16 hi and lo.
void block_bf16(const PlanBlock &B, uint16_t *out /* [2][64][64] */)
{
    for (int r = 0; r < 32; ++r)
        for (int c = 0; c < 32; ++c) {
            const cd u = B.U[r * 32 + c];
            const double R[2][2] = {{u.real(), -u.imag()}, {u.imag(), u.real()}};
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b) {
                    const int n = 2 * r + a, kk = 2 * c + b;
                    const float f = (float)R[a][b];
                    const uint16_t hi = bf16_bits(f);
                    const uint16_t lo = bf16_bits((float)(R[a][b] - (double)bf16_float(hi)));
                    out[n * 64 + kk] = hi;
                    out[64 * 64 + n * 64 + kk] = lo;
                }
        }
}

}  // namespace

extern "C" int qs_plan_apply_range(qs_state *s, qs_plan *P, size_t first, size_t count);

extern "C" int qs_plan_create(int n, const qs_gate *gates, size_t count, int max_k, qs_plan **out)
{
    qs_plan_opts o;
    o.block_qubits = max_k;
    o.tile_qubits = 12;
    o.max_sub = 1;
    o.low_qubits = 0;
    o.kernel = QS_PLAN_SINGLE;
    o.remap = 0;
    o.threads_per_row = 1;
    return qs_plan_create_ex(n, gates, count, &o, out);
}

extern "C" int qs_plan_default_opts(qs_plan_opts *o)
{
    if (!o) return qs_fail(QS_ERR_ARG, "qs_plan_default_opts: null");
    o->block_qubits = 5;
    o->tile_qubits = 12;
    o->max_sub = 2;              // passes of <= 2 blocks run three CTAs per SM (qs_fused2.cu)
    o->low_qubits = 3;
    o->kernel = QS_PLAN_TILED;
    o->remap = 0;
    o->threads_per_row = 1;
    o->tile_in_tmem = 1;
    return QS_OK;
}

extern "C" int qs_plan_create_ex(int n, const qs_gate *gates, size_t count, const qs_plan_opts *opts,
                                 qs_plan **out)
{
    if (!out) return qs_fail(QS_ERR_ARG, "qs_plan_create: null output");
    *out = nullptr;
    qs_plan_opts o;
    if (opts) o = *opts;
    else qs_plan_default_opts(&o);
    if (n < 1 || n > QS_MAX_QUBITS) return qs_fail(QS_ERR_ARG, "qs_plan_create: bad qubit count %d", n);
    if (o.block_qubits < 1 || o.block_qubits > 5)
        return qs_fail(QS_ERR_UNSUPPORTED, "qs_plan_create: fusion width %d (this build fuses up to 5 qubits)",
                       o.block_qubits);
    if (o.kernel != QS_PLAN_SINGLE && o.kernel != QS_PLAN_TILED)
        return qs_fail(QS_ERR_ARG, "qs_plan_create: unknown kernel %d", o.kernel);
    if (o.kernel == QS_PLAN_TILED &&
        (o.tile_qubits != 12 || o.max_sub < 1 || o.max_sub > 3 || o.low_qubits < 1 || o.low_qubits > 5))
        return qs_fail(QS_ERR_UNSUPPORTED,
                       "qs_plan_create: tiled passes need tile_qubits 12, max_sub 1..3, low_qubits 1..5");
    if (o.remap < 0 || o.remap > 2) return qs_fail(QS_ERR_ARG, "qs_plan_create: remap must be 0, 1 or 2");
    if (o.threads_per_row != 1 && o.threads_per_row != 2)
        return qs_fail(QS_ERR_ARG, "qs_plan_create: threads_per_row must be 1 or 2");
    if (count && !gates) return qs_fail(QS_ERR_ARG, "qs_plan_create: null gate list");
    qs_plan *P = new qs_plan();
    P->n = n;
    P->max_k = o.block_qubits;
    P->opts = o;
    P->gates.assign(gates, gates + count);
    // Below 12 qubits a state has fewer than one 128 x 32 tile: the plan keeps
    // the gate list only and runs it through the per-gate kernels.
    int r = n < 12 ? QS_OK : o.kernel == QS_PLAN_TILED ? build_passes(P) : build_blocks(P);
    if (r) { delete P; return r; }
    *out = P;
    return QS_OK;
}

extern "C" int qs_plan_destroy(qs_plan *P)
{
    if (!P) return QS_OK;
    if (P->mats) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(P->dev);
        if (P->mats_async) cudaFreeAsync(P->mats, P->mats_stream);
        else cudaFree(P->mats);
        cudaSetDevice(cur);
    }
    delete P;
    return QS_OK;
}

extern "C" int qs_plan_info(const qs_plan *P, size_t *n_blocks, size_t *n_gates)
{
    if (!P) return qs_fail(QS_ERR_ARG, "qs_plan_info: null plan");
    if (n_blocks) *n_blocks = P->blocks.size();
    if (n_gates) *n_gates = P->gates.size();
    return QS_OK;
}

extern "C" int qs_plan_block(const qs_plan *P, size_t i, int *k, int *qubits, double *matrix)
{
    if (!P || i >= P->blocks.size()) return qs_fail(QS_ERR_ARG, "qs_plan_block: no block %zu", i);
    const PlanBlock &B = P->blocks[i];
    if (k) *k = 5;
    if (qubits)
        for (int b = 0; b < 5; ++b) qubits[b] = B.q[b];
    if (matrix)
        for (int j = 0; j < 32 * 32; ++j) { matrix[2 * j] = B.U[j].real(); matrix[2 * j + 1] = B.U[j].imag(); }
    return QS_OK;
}

extern "C" int qs_plan_pass(const qs_plan *P, size_t i, int *n_blocks, int *tile_qubits, int *block_qubits)
{
    if (!P || i >= P->passes.size()) return qs_fail(QS_ERR_ARG, "qs_plan_pass: no tiled pass %zu", i);
    const PlanPass &S = P->passes[i];
    if (n_blocks) *n_blocks = (int)S.count;
    if (tile_qubits)
        for (int j = 0; j < 12; ++j) tile_qubits[j] = S.T[j];
    if (block_qubits)
        for (size_t b = 0; b < S.count; ++b)
            for (int j = 0; j < 5; ++j) block_qubits[5 * b + j] = P->blocks[S.first + b].q[j];
    return QS_OK;
}

// Block matrices to the state's device.  For a state with stream-ordered
// memory the matrices are too (allocated, copied and later freed in the
// state's stream order), so serving never synchronizes the device.
int qs_plan_upload(qs_plan *P, qs_state *s)
{
    if (P->mats && P->dev == s->device) return QS_OK;
    if (P->mats) {
        if (P->mats_async) cudaFreeAsync(P->mats, P->mats_stream);
        else cudaFree(P->mats);
        P->mats = nullptr;
    }
    const size_t per = 2 * 64 * 64;
    std::vector<uint16_t> host(per * (P->blocks.size() ? P->blocks.size() : 1));
    for (size_t b = 0; b < P->blocks.size(); ++b) block_bf16(P->blocks[b], host.data() + b * per);
    const size_t bytes = host.size() * sizeof(uint16_t);
    if (s->stream_alloc) {
        QS_CUDA_TRY(cudaMallocAsync(&P->mats, bytes, s->stream));
        QS_CUDA_TRY(cudaMemcpyAsync(P->mats, host.data(), bytes, cudaMemcpyHostToDevice, s->stream));
        QS_CUDA_TRY(cudaStreamSynchronize(s->stream));      // host buffer lifetime
        P->mats_async = true;
        P->mats_stream = s->stream;
    } else {
        QS_CUDA_TRY(cudaMalloc(&P->mats, bytes));
        QS_CUDA_TRY(cudaMemcpy(P->mats, host.data(), bytes, cudaMemcpyHostToDevice));
        P->mats_async = false;
    }
    P->dev = s->device;
    return QS_OK;
}

int qs_launch_prim(qs_state *s, const qs_prim &p);

static size_t plan_launches(const qs_plan *P)
{
    return P->opts.kernel == QS_PLAN_TILED ? P->passes.size() : P->blocks.size();
}

extern "C" int qs_plan_launches(const qs_plan *P, size_t *n)
{
    if (!P || !n) return qs_fail(QS_ERR_ARG, "qs_plan_launches: null argument");
    *n = plan_launches(P);
    return QS_OK;
}

extern "C" int qs_plan_apply(qs_state *s, qs_plan *P)
{
    return qs_plan_apply_range(s, P, 0, P ? plan_launches(P) : 0);
}

// Tiled pass u of a plan while its state is held with logical qubit q at
// position pos[q].  Every pass but the last of an application writes its
// tile as one contiguous run - the tile's qubits at positions 0..11, the
// others at 12.. in their current order - so that its stores stream through
// DRAM (stores scattered in short runs were the costlier half of a pass);
// the tile qubits that the next pass also uses go lowest, so that its loads
// come in runs of at least 2^low_qubits amplitudes.  The last pass writes the
// natural order back.  Updates pos to the layout the pass leaves.
static void tiled_pass_desc(const qs_plan *P, size_t u, bool last, int mode, std::vector<int> &pos,
                            qs_tiled_desc &d)
{
    const PlanPass &pp = P->passes[u];
    const int n = P->n;
    std::vector<int> at(n);                 // at[p] = logical qubit at position p
    for (int q = 0; q < n; ++q) at[pos[q]] = q;
    int phys[12], tq[12];
    uint64_t tmask = 0;
    for (int i = 0; i < 12; ++i) { phys[i] = pos[pp.T[i]]; tmask |= 1ull << phys[i]; }
    std::sort(phys, phys + 12);
    for (int i = 0; i < 12; ++i) { d.T[i] = phys[i]; tq[i] = at[phys[i]]; }
    d.nsub = (int)pp.count;
    d.first_block = pp.first;
    for (size_t b = 0; b < pp.count; ++b)
        for (int j = 0; j < 5; ++j) d.qpos[b][j] = pos[P->blocks[pp.first + b].q[j]];
    d.has_rows = 1;
    bool ident = true;
    for (int q = 0; q < n; ++q) ident = ident && pos[q] == q;
    // row orders: the plan's (chosen for the natural layout, written in
    // place); a permuted layout or write map gets its own at the end
    for (size_t b = 0; b < pp.count; ++b)
        for (int i = 0; i < 7; ++i) d.rows[b][i] = pos[pp.rows[b][i]];
    d.has_write = 0;
    if (last && ident) return;              // natural in, natural out: in place
    d.has_write = 1;
    std::vector<int> npos(n);
    if (last) {
        for (int l = 0; l < 12; ++l) d.wtile[l] = tq[l];
        for (int p = 0, i = 0; p < n; ++p)
            if (!((tmask >> p) & 1)) d.wpos[i++] = at[p];
        d.wmode = 2;
        for (int q = 0; q < n; ++q) npos[q] = q;
    } else if (mode == 2) {
        // contiguous loads for the next pass: its tile qubits at 0..11 (those
        // of this tile first, so that this pass's stores come in runs), every
        // other qubit at 12.. in its current order
        const PlanPass &nx = P->passes[u + 1];
        uint64_t next = 0, here = 0;
        for (int i = 0; i < 12; ++i) { next |= 1ull << nx.T[i]; here |= 1ull << tq[i]; }
        std::vector<int> order;
        const int c_next = P->blocks[nx.first].q[0];
        order.push_back(c_next);                       // the next loads move column pairs
        for (int i = 0; i < 12; ++i)
            if (nx.T[i] != c_next && ((here >> nx.T[i]) & 1)) order.push_back(nx.T[i]);
        for (int i = 0; i < 12; ++i)
            if (nx.T[i] != c_next && !((here >> nx.T[i]) & 1)) order.push_back(nx.T[i]);
        for (int k = 0; k < 12; ++k) npos[order[k]] = k;
        for (int p = 0, k = 12; p < n; ++p)
            if (!((next >> at[p]) & 1)) npos[at[p]] = k++;
        for (int l = 0; l < 12; ++l) d.wtile[l] = npos[tq[l]];
        for (int p = 0, i = 0; p < n; ++p)
            if (!((tmask >> p) & 1)) d.wpos[i++] = npos[at[p]];
        d.wmode = 2;
    } else {
        const PlanPass &nx = P->passes[u + 1];
        uint64_t next = 0;
        for (int i = 0; i < 12; ++i) next |= 1ull << nx.T[i];
        // position 0: the next pass's block-0 first column qubit (its loads
        // then move column pairs), else this pass's last-block first column
        // qubit (its stores then move column pairs), if shared
        const int c_next = P->blocks[nx.first].q[0];
        const int c_last = P->blocks[pp.first + pp.count - 1].q[0];
        auto in_tile = [&](int q) { return ((tmask >> pos[q]) & 1) != 0; };
        auto shared = [&](int q) { return ((next >> q) & 1) != 0; };
        std::vector<int> order;
        if (P->opts.tile_in_tmem) {
            // k_tile_tmem: position 0 a column of this pass's last block (its
            // results leave as 16-byte stores), shared with the next pass (whose
            // loads then start at 0) - one of its block-0 columns if possible; then the
            // shared qubits outside the last block, which become that block's
            // lanes (a warp's stores then cover consecutive positions), then
            // the other shared ones, then the rest, lanes before columns
            uint64_t lastcols = 0, nextcols = 0;
            for (int j = 0; j < 5; ++j) {
                lastcols |= 1ull << P->blocks[pp.first + pp.count - 1].q[j];
                nextcols |= 1ull << P->blocks[nx.first].q[j];
            }
            auto col = [&](int q) { return ((lastcols >> q) & 1) != 0; };
            auto ncol = [&](int q) { return ((nextcols >> q) & 1) != 0; };
            // position 0 in the last block's columns gives its 16-byte stores, in
            // the next pass's block-0 columns that pass's 16-byte gathers
            int head = -1;
            // a one-block pass reads and writes through one layout, whose
            // register bit 0 is either read position 0 (16-byte gathers) or
            // write position 0 (16-byte stores): when read position 0 is a
            // column, write it at 0 too, or - not shared with the next pass -
            // put a non-column there, so that the gather keeps its pairs
            if (pp.count == 1 && col(tq[0])) {
                if (shared(tq[0])) head = tq[0];
                for (int l = 1; l < 12 && head < 0; ++l)
                    if (shared(tq[l]) && !col(tq[l])) head = tq[l];
            }
            for (int l = 0; l < 12 && head < 0; ++l)
                if (shared(tq[l]) && col(tq[l]) && ncol(tq[l])) head = tq[l];
            for (int l = 0; l < 12 && head < 0; ++l)
                if (shared(tq[l]) && col(tq[l])) head = tq[l];
            if (head < 0 && in_tile(c_next) && shared(c_next)) head = c_next;
            if (head >= 0) order.push_back(head);
            for (int pass2 = 0; pass2 < 4; ++pass2)
                for (int l = 0; l < 12; ++l) {
                    const int q = tq[l];
                    if (q == head) continue;
                    const int cls = shared(q) ? (col(q) ? 1 : 0) : (col(q) ? 3 : 2);
                    if (cls == pass2) order.push_back(q);
                }
        } else {
            int head = -1;
            if (in_tile(c_next) && shared(c_next)) head = c_next;
            else if (in_tile(c_last) && shared(c_last)) head = c_last;
            if (head >= 0) order.push_back(head);
            for (int l = 0; l < 12; ++l)
                if (tq[l] != head && shared(tq[l])) order.push_back(tq[l]);
            for (int l = 0; l < 12; ++l)
                if (!shared(tq[l])) order.push_back(tq[l]);
        }
        for (int k = 0; k < 12; ++k) npos[order[k]] = k;
        for (int l = 0; l < 12; ++l) d.wtile[l] = npos[tq[l]];
        for (int p = 0, i = 0; p < n; ++p)
            if (!((tmask >> p) & 1)) { npos[at[p]] = 12 + i; d.wpos[i] = 12 + i; ++i; }
        d.wmode = 1;
    }
    // which tile bits are lowest - and so which lanes read and write what -
    // depends on the positions: choose the row orders for this layout
    int rows[3][7];
    if (qs_tile_row_orders(n, d.T, d.nsub, d.qpos, rows, d.wtile, 0) == QS_OK) memcpy(d.rows, rows, sizeof(rows));
    pos.swap(npos);
}

int qs_plan_tiled_schedule(const qs_plan *P, int n, size_t first, size_t count, int remap,
                           std::vector<qs_tiled_desc> &descs, std::vector<int> &dst)
{
    if (P->opts.kernel != QS_PLAN_TILED || n != P->n || first > P->passes.size() ||
        count > P->passes.size() - first)
        return qs_fail(QS_ERR_ARG, "tiled schedule: bad plan or range");
    descs.assign(count, qs_tiled_desc());
    dst.assign(count, 0);
    std::vector<int> pos(n);
    for (int q = 0; q < n; ++q) pos[q] = q;
    // Remapping ping-pongs between the state's buffer (0) and the spare one
    // (1); with an odd number of passes the first runs in place, so that the
    // last pass lands in the state's own buffer.
    if (count < 2) remap = 0;
    const size_t pong_from = remap ? (count & 1) : count;
    int cur = 0;
    for (size_t k = 0; k < count; ++k) {
        qs_tiled_desc &d = descs[k];
        memset(&d, 0, sizeof(d));
        if (k < pong_from) {
            std::vector<int> ident(pos);
            tiled_pass_desc(P, first + k, true, 0, ident, d);  // natural in, natural out, in place
            dst[k] = -1;
        } else {
            tiled_pass_desc(P, first + k, k + 1 == count, remap, pos, d);
            dst[k] = cur ^ 1;
            cur ^= 1;
        }
    }
    return QS_OK;
}

extern "C" int qs_plan_apply_range(qs_state *s, qs_plan *P, size_t first, size_t count)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (!P) return qs_fail(QS_ERR_ARG, "qs_plan_apply: null plan");
    if (P->n != s->n) return qs_fail(QS_ERR_ARG, "qs_plan_apply: plan for %d qubits, state has %d", P->n, s->n);
    if (s->dtype != QS_C64 || s->n < 12) {
        // No tensor-core form for complex128 or below 12 qubits: the gates of
        // the requested blocks (all gates when the plan has no blocks) through
        // the per-gate kernels.
        std::vector<size_t> idx;
        if (P->blocks.empty()) {
            for (size_t i = 0; i < P->gates.size(); ++i) idx.push_back(i);
        } else {
            const size_t nl = plan_launches(P);
            if (first > nl || count > nl - first)
                return qs_fail(QS_ERR_ARG, "qs_plan_apply_range: launches [%zu, +%zu) out of range", first, count);
            for (size_t u = first; u < first + count; ++u) {
                size_t b0 = u, b1 = u + 1;
                if (P->opts.kernel == QS_PLAN_TILED) { b0 = P->passes[u].first; b1 = b0 + P->passes[u].count; }
                for (size_t b = b0; b < b1; ++b)
                    idx.insert(idx.end(), P->blocks[b].gates.begin(), P->blocks[b].gates.end());
            }
        }
        for (size_t i : idx) {
            qs_prim p;
            if ((r = qs_lower_gate(s->n, &P->gates[i], &p)) || (r = qs_launch_prim(s, p))) return r;
        }
        return QS_OK;
    }
    if (first > plan_launches(P) || count > plan_launches(P) - first)
        return qs_fail(QS_ERR_ARG, "qs_plan_apply_range: launches [%zu, +%zu) out of range", first, count);
    if ((r = qs_plan_upload(P, s))) return r;
    // Norm partials live in their own per-state buffer, so that other calls
    // between two qs_plan_apply_range calls cannot overwrite them:
    // [0] input norm of block 0, [1]/[2] output norms of even/odd blocks.
    const int G = qs_fused_grid(s);
    if (!s->fused_norm) {
        void *p = nullptr;
        if ((r = qs_dev_alloc(s, 3 * (size_t)QS_SM_COUNT * 4 * sizeof(double), &p))) return r;
        s->fused_norm = static_cast<double *>(p);
    }
    double *norm = s->fused_norm;
    // watchdog flag (result area of scratch), cleared before the first block
    const size_t kFlagOff = 64 * 1024 + 192;
    int *flag = reinterpret_cast<int *>(static_cast<char *>(s->scratch) + kFlagOff);
    if (first == 0) QS_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), s->stream));
    const size_t per = 2 * 64 * 64 * sizeof(uint16_t);
    if (P->opts.kernel == QS_PLAN_TILED) {
        const int GT = qs_tiled_grid(s);
        const int remap = (count >= 2 && s->n >= 20) ? P->opts.remap : 0;
        if (remap && !s->spare) {
            void *p = nullptr;
            if ((r = qs_dev_alloc(s, s->amp_bytes(), &p))) return r;
            s->spare = p;
        }
        // the schedule (host work of ~0.5 ms per remapped pass) is kept with
        // the plan for its next application over the same range
        if (P->sched_remap != remap || P->sched_first != first || P->sched_count != count) {
            P->sched_remap = -1;
            if ((r = qs_plan_tiled_schedule(P, s->n, first, count, remap, P->sched, P->sched_dst))) return r;
            P->sched_remap = remap;
            P->sched_first = first;
            P->sched_count = count;
        }
        std::vector<qs_tiled_desc> descs(P->sched);
        const std::vector<int> &dst = P->sched_dst;
        void *buf[2] = {s->amp, s->spare};
        for (size_t u = first; u < first + count; ++u) {
            const PlanPass &pp = P->passes[u];
            qs_tiled_desc &d = descs[u - first];
            d.threads_per_row = P->opts.threads_per_row;
            if (dst[u - first] >= 0) {
                d.amp_out = buf[dst[u - first]];
                d.amp_in = buf[dst[u - first] ^ 1];
            }
            d.mat_dev = static_cast<const char *>(P->mats) + pp.first * per;
            d.norm0 = u ? norm : nullptr;
            d.prev_out = u ? norm + GT * (1 + (u - 1) % 2) : nullptr;
            d.in_parts = u ? nullptr : norm;
            d.out_parts = norm + GT * (1 + u % 2);
            r = QS_ERR_UNSUPPORTED;
            if (P->opts.tile_in_tmem) r = qs_launch_tiled_tmem(s, &d, flag);
            if (r == QS_ERR_UNSUPPORTED) r = qs_launch_tiled(s, &d, flag);
            if (r) return r;
        }
        // the rescale of each pass leaves only the last pass's drift
        if (count && first + count == plan_launches(P))
            return qs_launch_norm_fix(s, norm, norm + GT * (1 + (first + count - 1) % 2), GT);
        return QS_OK;
    }
    for (size_t b = first; b < first + count; ++b) {
        qs_fused_desc d;
        for (int j = 0; j < 5; ++j) d.qpos[j] = P->blocks[b].q[j];
        d.mat_dev = static_cast<const char *>(P->mats) + b * per;
        d.norm0 = b ? norm : nullptr;
        d.prev_out = b ? norm + G * (1 + (b - 1) % 2) : nullptr;
        d.in_parts = b ? nullptr : norm;
        d.out_parts = norm + G * (1 + b % 2);
        if ((r = qs_launch_fused(s, &d, flag))) return r;
    }
    if (count && first + count == plan_launches(P))
        return qs_launch_norm_fix(s, norm, norm + G * (1 + (first + count - 1) % 2), G);
    return QS_OK;
}

extern "C" int qs_release_spare(qs_state *s)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (s->spare) {
        if (s->stream_alloc) {
            qs_dev_free(s, s->spare);
        } else {
            QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
            QS_CUDA_TRY(cudaFree(s->spare));
        }
        s->spare = nullptr;
    }
    return QS_OK;
}

extern "C" int qs_plan_status(qs_state *s)
{
    int r = qs_check_state(s);
    if (r) return r;
    const size_t kFlagOff = 64 * 1024 + 192;
    int flag = 0;
    QS_CUDA_TRY(cudaMemcpyAsync(&flag, static_cast<char *>(s->scratch) + kFlagOff, sizeof(int),
                                cudaMemcpyDeviceToHost, s->stream));
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (flag == 2) return qs_fail(QS_ERR_STATE, "fused pass: dynamic shared memory not 1024-byte aligned");
    if (flag) return qs_fail(QS_ERR_STATE, "fused pass: a bounded wait in the tensor-core kernel expired");
    return QS_OK;
}

extern "C" int qs_plan_autotune(qs_state *s, const qs_gate *gates, size_t count, const qs_plan_opts *base,
                                int reps, qs_plan_opts *best, double *best_ms)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (!best) return qs_fail(QS_ERR_ARG, "qs_plan_autotune: null output");
    if (reps < 1 || reps > 100) return qs_fail(QS_ERR_ARG, "qs_plan_autotune: reps %d outside [1, 100]", reps);
    qs_plan_opts b0;
    if (base) b0 = *base;
    else qs_plan_default_opts(&b0);
    b0.kernel = QS_PLAN_TILED;
    *best = b0;
    if (best_ms) *best_ms = 0;
    if (s->n < 12) return QS_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    QS_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return qs_fail(QS_ERR_CUDA, "qs_plan_autotune: cudaEventCreate failed");
    }
    double best_t = -1;
    for (int tm = 1; tm >= 0 && !r; --tm)
        for (int ms = 2; ms <= 3 && !r; ++ms)
            for (int low = 3; low >= (b0.remap ? 1 : 2) && !r; --low) {
                qs_plan_opts o = b0;
                o.tile_in_tmem = tm;
                o.max_sub = ms;
                o.low_qubits = low;
                qs_plan *P = nullptr;
                if ((r = qs_plan_create_ex(s->n, gates, count, &o, &P))) break;
                r = qs_plan_apply(s, P);
                if (!r && cudaEventRecord(e0, s->stream) != cudaSuccess) r = qs_fail(QS_ERR_CUDA, "event record");
                for (int k = 0; k < reps && !r; ++k) r = qs_plan_apply(s, P);
                if (!r && cudaEventRecord(e1, s->stream) != cudaSuccess) r = qs_fail(QS_ERR_CUDA, "event record");
                if (!r && cudaEventSynchronize(e1) != cudaSuccess) r = qs_fail(QS_ERR_CUDA, "event sync");
                if (!r) r = qs_plan_status(s);
                float ms_t = 0;
                if (!r && cudaEventElapsedTime(&ms_t, e0, e1) != cudaSuccess) r = qs_fail(QS_ERR_CUDA, "event time");
                qs_plan_destroy(P);
                if (r) break;
                const double t = (double)ms_t / reps;
                if (best_t < 0 || t < best_t) {
                    best_t = t;
                    *best = o;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!r && best_ms) *best_ms = best_t;
    return r;
}

void qs_plan_block_bf16(const qs_plan *P, size_t b, uint16_t *out)
{
    block_bf16(P->blocks[b], out);
}

int qs_plan_rebind(const qs_plan *proto, const qs_gate *gates, size_t count, qs_plan **out)
{
    *out = nullptr;
    if (!proto || count != proto->gates.size()) return qs_fail(QS_ERR_ARG, "plan rebind: gate count differs");
    for (size_t i = 0; i < count; ++i) {
        const qs_gate &a = proto->gates[i], &g = gates[i];
        if (a.op != g.op || a.nctrl != g.nctrl || memcmp(a.q, g.q, sizeof(a.q)) ||
            memcmp(a.ctrl, g.ctrl, sizeof(int32_t) * (size_t)(a.nctrl > 0 ? a.nctrl : 0)))
            return qs_fail(QS_ERR_ARG, "plan rebind: gate %zu differs in operation or qubits", i);
    }
    qs_plan *P = new qs_plan();
    P->n = proto->n;
    P->max_k = proto->max_k;
    P->opts = proto->opts;
    P->gates.assign(gates, gates + count);
    P->passes = proto->passes;
    P->blocks.resize(proto->blocks.size());
    for (size_t b = 0; b < proto->blocks.size(); ++b) {    // the structure; unitaries are rebuilt below
        P->blocks[b].k = proto->blocks[b].k;
        std::copy(proto->blocks[b].q, proto->blocks[b].q + 5, P->blocks[b].q);
        P->blocks[b].gates = proto->blocks[b].gates;
    }
    std::vector<qs_prim> prim;
    std::vector<uint64_t> mask;
    int r = lower_all(P, prim, mask);
    if (r) { delete P; return r; }
    for (PlanBlock &B : P->blocks) block_unitary(B, prim);
    *out = P;
    return QS_OK;
}
