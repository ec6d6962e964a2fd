// qs_tile_layout.cu - host construction of a tiled pass's layout (see
// qs_tile_core.cuh): for each of the pass's blocks, which 5 tile bits are its
// columns and which 7 its rows, and the tables that route block b's results
// into block b+1's rows and columns.
#include <cstring>

#include "qs_tile_core.cuh"

int qs_tile_layout_build(int n, const int *T, int nsub, const int (*qpos)[5], qs_tile::Layout *L)
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
            if (q < 0 || q >= n || local[q] < 0 || (i && q <= qpos[b][i - 1]))
                return qs_fail(QS_ERR_ARG, "tiled pass: block qubits must be ascending tile qubits");
            Q[b][i] = local[q];
            qm |= 1u << local[q];
        }
        for (int p = 0, c = 0; p < 12; ++p)
            if (!(qm & (1u << p))) Cp[b][c++] = p;
    }
    L->nsub = nsub;
    const int last = nsub - 1;
    for (int i = 0; i < 12; ++i) L->tpos[i] = (int8_t)T[i];
    for (int i = 0; i < 7; ++i) {
        L->c0_glob[i] = T[Cp[0][i]];
        L->cl_glob[i] = T[Cp[last][i]];
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
            if (j & (1 << i)) { a |= 1ull << T[Q[0][i]]; b |= 1ull << T[Q[last][i]]; }
        L->g0[j] = a;
        L->gl[j] = b;
    }
    L->vec0 = T[Q[0][0]] == 0;
    L->vecl = T[Q[last][0]] == 0;
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
