// qs_tile_layout.cu - host construction of a tiled pass's layout (see
// qs_tile_core.cuh): for each of the pass's blocks, which 5 tile bits are its
// columns and which 7 its rows, and the tables that route block b's results
// into block b+1's rows and columns.
#include <cstring>
#include <utility>
#include <vector>

#include "qs_tile_core.cuh"

namespace {

using qs_tile::kMaxSub;

// A block's 7 row bits may be listed in any order: rows are independent
// columns of the contraction.  The order decides which tile bits a warp's 32
// lanes (row bits 0..4) run over, and with it
//   * how many shared-memory wavefronts the block-0 input stores take
//     (convert_store: the lanes of a warp hold consecutive chunks, i.e. tile
//     bits 1..5, and write them at their rows and columns of the swizzled A
//     buffer - row bits 0..2 and column bits land on different bank bits);
//   * how many 32-byte sectors one warp-wide global store of the last block
//     touches: lanes on qubits 0 and 1 share sectors;
//   * how many shared-memory wavefronts one warp-wide 4-byte scatter store
//     into the next block's swizzled A buffer takes: the bank of a store is
//     offset bits 2..6 = the next block's column bits 0..1 and (column bits
//     2..4 XOR row bits 0..2); a lane bit that lands on none of them, or on
//     one another lane bit already took, doubles the wavefronts.
// Costs are warp-level transactions per tile, up to a common factor.
struct RowCfg {
    int t[3];                    // tile bits of row bits 0..2
    unsigned lanes;              // tile bits of row bits 0..4, as a mask
};

int glob_cost(unsigned lanes, int loc0, int loc1, bool vec)
{
    int k = 0;
    if (loc1 >= 0) k += (lanes >> loc1) & 1;
    if (!vec && loc0 >= 0) k += (lanes >> loc0) & 1;
    return (vec ? 16 : 32) * (32 >> k);
}

// 128-byte lines one warp-wide store of the last block touches, times the
// stores per thread: lanes whose tile bits are written at positions 1..3
// (0..3 without column pairs) share lines.
int store_cost(unsigned lanes, const int *W, bool vec)
{
    int k = 0;
    for (int b = 0; b < 12; ++b)
        if (((lanes >> b) & 1) && W[b] <= 3 && (W[b] >= 1 || !vec)) ++k;
    return (vec ? 16 : 32) * (32 >> (k > 5 ? 5 : k));
}

// Wavefronts of convert_store's stores for block 0 with columns Q0 and row
// bits 0..2 on tile bits t[0..2]: a lane's store lands at byte bits 2..6
// (4-byte stores) or 3..6 (8-byte column pairs) given by the lane's tile bits
// 1..5 (1..4): column c -> bit 2 + c (c < 2) or c + 2, XOR'd with row bits
// 0..2 -> bits 4..6; row bits 3.. land in the same banks.  Each lane bit that
// finds no bit of its own doubles the wavefronts.
int convert_cost(const int *Q0, const int *t)
{
    int col[12], rlo[12];
    for (int b = 0; b < 12; ++b) col[b] = rlo[b] = -1;
    for (int c = 0; c < 5; ++c) col[Q0[c]] = c;
    for (int r = 0; r < 3; ++r) rlo[t[r]] = r;
    const bool pair = col[0] == 0;
    const int nl = pair ? 4 : 5, lo = pair ? 3 : 2;
    unsigned hit = 0;
    for (int b = 1; b <= nl; ++b) {
        int a = -1;
        if (col[b] >= 0) a = col[b] < 2 ? 2 + col[b] : col[b] + 2;
        else if (rlo[b] >= 0) a = rlo[b] + 4;
        if (a >= lo && a <= 6) hit |= 1u << a;
    }
    return 64 << (nl - __builtin_popcount(hit));
}

int scatter_cost(unsigned lanes, const int *Qn, const int *t)
{
    unsigned hit = 0;
    for (int c = 0; c < 5; ++c) hit |= ((lanes >> Qn[c]) & 1u) << (2 + c);
    for (int r = 0; r < 3; ++r) hit |= ((lanes >> t[r]) & 1u) << (4 + r);
    return 64 << (5 - __builtin_popcount(hit));
}

// Row orders (tile bits) for each block minimising the costs above, by
// dynamic programming over the blocks; ascending order unless another order
// is strictly cheaper.
void choose_row_orders(const int *T, int nsub, const int (*Q)[5], int (*Cp)[7], const int *W, int input_mode)
{
    int loc0 = -1, loc1 = -1;
    for (int i = 0; i < 12; ++i) {
        if (T[i] == 0) loc0 = i;
        if (T[i] == 1) loc1 = i;
    }
    const bool vecl = W[Q[nsub - 1][0]] == 0, vec0 = T[Q[0][0]] == 0;
    // block 0's input: tile-order staging converted per chunk (k_fused_tile),
    // or one row per thread gathered from global memory (k_batch)
    auto in_cost = [&](const RowCfg &c) {
        return input_mode == 0 ? convert_cost(Q[0], c.t) : glob_cost(c.lanes, loc0, loc1, vec0);
    };
    // Configurations of block b: 210 ordered triples for row bits 0..2, each
    // with 6 choices of row bits 3..4 among the other four (index 6 t + u).
    // The input and scatter costs depend on a configuration through its
    // triple and the previous block's lane set only, so they are evaluated
    // once per triple.
    constexpr int kTriples = 210, kPer = 6, kCfg = kTriples * kPer;
    static_assert(kCfg == 1260, "7 x 6 x 5 triples x C(4, 2) lane pairs");
    std::vector<RowCfg> cfg[kMaxSub];
    for (int b = 0; b < nsub; ++b) {
        const int *C = Cp[b];
        cfg[b].reserve(kCfg);
        // configuration 0 is the ascending order
        for (int i = 0; i < 7; ++i)
            for (int j = 0; j < 7; ++j)
                for (int k = 0; k < 7; ++k) {
                    if (i == j || i == k || j == k) continue;
                    int rest[4], nr = 0;
                    for (int m = 0; m < 7; ++m)
                        if (m != i && m != j && m != k) rest[nr++] = C[m];
                    const unsigned m3 = (1u << C[i]) | (1u << C[j]) | (1u << C[k]);
                    for (int u = 0; u < 4; ++u)
                        for (int v = u + 1; v < 4; ++v)
                            cfg[b].push_back(RowCfg{{C[i], C[j], C[k]}, m3 | (1u << rest[u]) | (1u << rest[v])});
                }
    }
    std::vector<int> best[kMaxSub], from[kMaxSub];
    best[0].resize(kCfg);
    for (int t = 0; t < kTriples; ++t) {
        if (input_mode == 0) {
            const int c = convert_cost(Q[0], cfg[0][kPer * t].t);
            for (int u = 0; u < kPer; ++u) best[0][kPer * t + u] = c;
        } else {
            for (int u = 0; u < kPer; ++u) best[0][kPer * t + u] = in_cost(cfg[0][kPer * t + u]);
        }
    }
    std::vector<int> set_of(1u << 12);
    for (int b = 1; b < nsub; ++b) {
        // the previous block enters only through its lane set: keep its
        // cheapest configuration per set (first one on ties), sets in order of
        // first appearance
        std::vector<std::pair<unsigned, int>> sets;     // (lanes, configuration)
        std::fill(set_of.begin(), set_of.end(), -1);
        for (int p = 0; p < kCfg; ++p) {
            const unsigned ln = cfg[b - 1][p].lanes;
            int &s = set_of[ln];
            if (s < 0) { s = (int)sets.size(); sets.push_back({ln, p}); }
            else if (best[b - 1][p] < best[b - 1][sets[s].second]) sets[s].second = p;
        }
        best[b].assign(kCfg, 1 << 30);
        from[b].assign(kCfg, -1);
        for (int t = 0; t < kTriples; ++t) {
            int bc = 1 << 30, bf = -1;
            for (const auto &st : sets) {
                const int c = best[b - 1][st.second] + scatter_cost(st.first, Q[b], cfg[b][kPer * t].t);
                if (c < bc) { bc = c; bf = st.second; }
            }
            for (int u = 0; u < kPer; ++u) { best[b][kPer * t + u] = bc; from[b][kPer * t + u] = bf; }
        }
    }
    const int last = nsub - 1;
    int sel[kMaxSub] = {0, 0, 0}, bestc = 1 << 30;
    for (size_t i = 0; i < cfg[last].size(); ++i) {
        const int c = best[last][i] + store_cost(cfg[last][i].lanes, W, vecl);
        if (c < bestc) { bestc = c; sel[last] = (int)i; }
    }
    // cost of the ascending orders (configuration 0 everywhere)
    int base = in_cost(cfg[0][0]) + store_cost(cfg[last][0].lanes, W, vecl);
    for (int b = 1; b < nsub; ++b) base += scatter_cost(cfg[b - 1][0].lanes, Q[b], cfg[b][0].t);
    if (bestc >= base) return;
    for (int b = last; b > 0; --b) sel[b - 1] = from[b][sel[b]];
    for (int b = 0; b < nsub; ++b) {
        const RowCfg &c = cfg[b][sel[b]];
        int order[7], n = 0;
        for (int r = 0; r < 3; ++r) order[n++] = c.t[r];
        for (int m = 0; m < 7; ++m)          // row bits 3, 4: the other lanes, ascending
            if (((c.lanes >> Cp[b][m]) & 1) && Cp[b][m] != c.t[0] && Cp[b][m] != c.t[1] && Cp[b][m] != c.t[2])
                order[n++] = Cp[b][m];
        for (int m = 0; m < 7; ++m)          // row bits 5, 6
            if (!((c.lanes >> Cp[b][m]) & 1)) order[n++] = Cp[b][m];
        for (int m = 0; m < 7; ++m) Cp[b][m] = order[m];
    }
}

}  // namespace

int qs_tile_row_orders(int n, const int *T, int nsub, const int (*qpos)[5], int (*rows)[7], const int *wtile,
                       int input_mode)
{
    qs_tile::Layout L;
    int r = qs_tile_layout_build(n, T, nsub, qpos, nullptr, &L, nullptr, wtile);   // validates the pass
    if (r) return r;
    int W[12];
    for (int i = 0; i < 12; ++i) W[i] = wtile ? wtile[i] : T[i];
    int local[64];
    for (int i = 0; i < 64; ++i) local[i] = -1;
    for (int i = 0; i < 12; ++i) local[T[i]] = i;
    int Q[kMaxSub][5], Cp[kMaxSub][7];
    for (int b = 0; b < nsub; ++b) {
        uint32_t qm = 0;
        for (int i = 0; i < 5; ++i) { Q[b][i] = local[qpos[b][i]]; qm |= 1u << Q[b][i]; }
        for (int p = 0, c = 0; p < 12; ++p)
            if (!(qm & (1u << p))) Cp[b][c++] = p;
    }
    choose_row_orders(T, nsub, Q, Cp, W, input_mode);
    for (int b = 0; b < nsub; ++b)
        for (int i = 0; i < 7; ++i) rows[b][i] = T[Cp[b][i]];
    return QS_OK;
}

int qs_tile_layout_build(int n, const int *T, int nsub, const int (*qpos)[5], const int (*rows)[7],
                         qs_tile::Layout *L, qs_tile::LoadMap *M, const int *wtile)
{
    using qs_tile::kMaxSub;
    if (nsub < 1 || nsub > kMaxSub) return qs_fail(QS_ERR_ARG, "tiled pass: %d blocks", nsub);
    memset(L, 0, sizeof(*L));
    int local[64];
    for (int i = 0; i < 64; ++i) local[i] = -1;
    for (int i = 0; i < 12; ++i) {
        const int q = T[i];
        if (q < 0 || q >= n || (i && q <= T[i - 1]))
            return qs_fail(QS_ERR_ARG, "tiled pass: tile qubits must be ascending and in range");
        local[q] = i;
        L->tmask |= 1ull << q;
    }
    int Q[kMaxSub][5], Cp[kMaxSub][7];
    for (int b = 0; b < nsub; ++b) {
        uint32_t qm = 0;
        for (int i = 0; i < 5; ++i) {
            const int q = qpos[b][i];
            if (q < 0 || q >= n || local[q] < 0 || (qm & (1u << local[q])))
                return qs_fail(QS_ERR_ARG, "tiled pass: block qubits must be distinct tile qubits");
            Q[b][i] = local[q];
            qm |= 1u << local[q];
        }
        for (int p = 0, c = 0; p < 12; ++p)
            if (!(qm & (1u << p))) Cp[b][c++] = p;
        if (rows) {                              // a given order of the same row bits
            uint32_t rm = 0;
            for (int i = 0; i < 7; ++i) {
                const int q = rows[b][i];
                if (q < 0 || q >= n || local[q] < 0 || (qm & (1u << local[q])) || (rm & (1u << local[q])))
                    return qs_fail(QS_ERR_ARG, "tiled pass: row order must list the block's other tile qubits");
                rm |= 1u << local[q];
                Cp[b][i] = local[q];
            }
        }
    }
    int WT[12];                                  // write position of each tile bit
    uint64_t wseen = 0;
    for (int i = 0; i < 12; ++i) {
        WT[i] = wtile ? wtile[i] : T[i];
        if (WT[i] < 0 || WT[i] >= n || ((wseen >> WT[i]) & 1))
            return qs_fail(QS_ERR_ARG, "tiled pass: write positions must be distinct and in range");
        wseen |= 1ull << WT[i];
    }
    L->nsub = nsub;
    const int last = nsub - 1;
    for (int i = 0; i < 12; ++i) L->tpos[i] = (int8_t)T[i];
    for (int i = 0; i < 7; ++i) {
        L->c0_glob[i] = T[Cp[0][i]];
        L->cl_glob[i] = WT[Cp[last][i]];
        L->cl_loc[i] = (int8_t)Cp[last][i];
    }
    for (int j = 0; j < 32; ++j) {
        uint32_t t = 0;
        for (int i = 0; i < 5; ++i)
            if (j & (1 << i)) t |= 1u << Q[last][i];
        L->lout[j] = (uint16_t)t;
    }
    for (int j = 0; j < 32; ++j) {
        uint64_t a = 0, b = 0;
        for (int i = 0; i < 5; ++i)
            if (j & (1 << i)) { a |= 1ull << T[Q[0][i]]; b |= 1ull << WT[Q[last][i]]; }
        L->g0[j] = a;
        L->gl[j] = b;
    }
    L->vec0 = T[Q[0][0]] == 0;
    L->vecl = WT[Q[last][0]] == 0;
    if (M) {
        // block 0's view of each tile bit, and the tables of prefetch_tile
        memset(M, 0, sizeof(*M));
        for (int p = 0; p < 12; ++p) M->tpos[p] = (int8_t)T[p];
        for (int i = 0; i < 7; ++i) M->tmap0[Cp[0][i]] = (int8_t)i;
        for (int i = 0; i < 5; ++i) M->tmap0[Q[0][i]] = (int8_t)~i;
        const int m0 = M->tmap0[0];
        M->dr = (uint8_t)(m0 >= 0 ? 1u << m0 : 0);
        M->dj = (uint8_t)(m0 >= 0 ? 0 : 1u << (~m0));
        M->pair = (uint8_t)(m0 == ~0);
        for (int k = 0; k < 16; ++k) {
            uint64_t g = 0;
            uint32_t rr = 0, jj = 0;
            for (int t = 8; t < 12; ++t) {
                if (!((k >> (t - 8)) & 1)) continue;
                g |= 1ull << T[t];
                const int m = M->tmap0[t];
                if (m >= 0) rr |= 1u << m;
                else jj |= 1u << (~m);
            }
            M->gk[k] = g;
            M->rk[k] = (uint8_t)rr;
            M->jk[k] = (uint8_t)jj;
        }
    }
    for (int t = 0; t + 1 < nsub; ++t) {
        int rowbit[12], colbit[12];
        for (int p = 0; p < 12; ++p) rowbit[p] = colbit[p] = -1;
        for (int i = 0; i < 7; ++i) rowbit[Cp[t + 1][i]] = i;
        for (int i = 0; i < 5; ++i) colbit[Q[t + 1][i]] = i;
        for (int i = 0; i < 7; ++i) {
            const int p = Cp[t][i];
            L->rowmap[t][i] = (int8_t)(rowbit[p] >= 0 ? rowbit[p] : ~colbit[p]);
        }
        for (int j = 0; j < 32; ++j) {
            uint32_t rr = 0, jj = 0;
            for (int i = 0; i < 5; ++i) {
                if (!(j & (1 << i))) continue;
                const int p = Q[t][i];
                if (rowbit[p] >= 0) rr |= 1u << rowbit[p];
                else jj |= 1u << colbit[p];
            }
            L->tabR[t][j] = (uint8_t)rr;
            L->tabJ[t][j] = (uint8_t)jj;
            // swizzled offset bits contributed by column j (qs_tile::Layout::scat)
            L->scat[t][j] = (uint16_t)((rr << 7) | ((((jj >> 2) ^ (rr & 7)) & 7) << 4) | ((jj & 3) << 2));
        }
    }
    return QS_OK;
}
