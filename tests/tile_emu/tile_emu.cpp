// tile_emu.cpp - CPU emulation of the tiled tensor-core passes, for tests.
//
// Runs a fused plan on a complex128 host state exactly the way k_fused_tile
// (qpanda_b200/csrc/qs_fused2.cu) moves data: the launch descriptors come
// from the library's own scheduler (qs_plan_tiled_schedule), the per-pass
// tables from its own layout builder (qs_tile_layout_build), and each tile
// goes through
//   * the tile-order staging copies of prefetch_tile_linear (LoadMap) and
//     convert_load / convert_store, which put each thread's chunks at their block-0 rows and
//     columns;
//   * each block's contraction (in FP64 here, on the block unitaries of the
//     plan, instead of split BF16 on the tensor cores);
//   * the scatter of a block's results into the next block's swizzled A
//     buffer by the kernel's XOR offsets (scatter_thread_part ^ scat), decoded
//     back to (row, column);
//   * the stores of the last block's results through StoreMap / gl / cl_glob,
//     in place or into the other buffer of the ping-pong.
// Every staging slot and every A slot must be written exactly once per tile
// and every output amplitude exactly once per pass; the result is compared
// with the oracle by the caller.  This checks all index arithmetic of the
// tiled path on the CPU; the GPU tests check the tensor-core arithmetic.
//
// Built by tests/test_tile_emulation.py against the library (host code only
// runs; nvcc because the shared headers hold device helpers):
//   nvcc -O2 -std=c++17 -x cu -shared -Xcompiler -fPIC tile_emu.cpp
//        -I<csrc> -I<include> -L<lib> -lqsb200
#include <algorithm>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "qs_fused.h"
#include "qs_plan_internal.h"
#include "qs_tile_core.cuh"
#include "qs_tile_tmem.cuh"

using qs_tile::Layout;
using qs_tile::LoadMap;
using qs_tile::StoreMap;
typedef std::complex<double> cd;

namespace {

char g_err[256];

uint64_t deposit_tile(uint64_t tile, const Layout &L)
{
    for (int j = 0; j < 12; ++j) {
        const uint64_t low = (1ull << L.tpos[j]) - 1;
        tile = ((tile & ~low) << 1) | (tile & low);
    }
    return tile;
}

uint32_t stage_off(int row, int chunk) { return row * 256 + ((chunk ^ (row & 15)) << 4); }

// same formula as qs_tile::scatter_thread_part
uint32_t emu_thread_part(const Layout &L, int t, int row)
{
    uint32_t r2 = 0, j2 = 0;
    for (int b = 0; b < 7; ++b) {
        const uint32_t bit = (row >> b) & 1;
        const int m = L.rowmap[t][b];
        if (m >= 0) r2 |= bit << m;
        else j2 |= bit << (~m);
    }
    return (r2 << 7) | ((((j2 >> 2) ^ (r2 & 7)) & 7) << 4) | ((j2 & 3) << 2);
}

// same formula as qs_tile::store_base
uint64_t emu_store_base(uint64_t tile, uint64_t read_base, const StoreMap &W)
{
    if (W.mode == 0) return read_base;
    if (W.mode == 1) return tile << 12;
    uint64_t b = 0;
    for (int i = 0; i < W.ntb; ++i) b |= ((tile >> i) & 1ull) << W.wpos[i];
    return b;
}

int fail(const char *msg, long long a = 0, long long b = 0)
{
    snprintf(g_err, sizeof(g_err), "%s (%lld, %lld)", msg, a, b);
    return 1;
}

}  // namespace

extern "C" const char *tile_emu_error(void) { return g_err; }

// Apply plan passes [0, all) to state (2^n complex128, interleaved re/im).
// *kinds_out (may be NULL) counts the passes whose chunk pairs are adjacent
// columns [0], other columns [1], two rows [2].
// Pass k (descriptor d, destination dst_k as qs_plan_tiled_schedule gives it)
// the way k_fused_tile moves data.
static int smem_pass(const qs_plan *P, int n, const qs_tiled_desc &d, int dst_k, size_t k, int tpr,
                     std::vector<cd> *bufs[2], std::vector<int> &hits, int *kinds_out)
{
    const uint64_t N = 1ull << n, tiles = N >> 12;
    std::vector<cd> &buf0 = *bufs[0];
    {
        const int dst[1] = {dst_k};
        Layout L;
        LoadMap M;
        if (qs_tile_layout_build(n, d.T, d.nsub, d.qpos, d.has_rows ? d.rows : nullptr, &L, &M,
                                 d.has_write ? d.wtile : nullptr))
            return fail("layout build failed", (long long)k);
        if (kinds_out) kinds_out[M.pair ? 0 : (M.dj ? 1 : 2)]++;
        StoreMap W;
        memset(&W, 0, sizeof(W));
        W.mode = d.has_write ? d.wmode : 0;
        W.ntb = n - 12;
        for (int i = 0; i < W.ntb && i < 52; ++i) W.wpos[i] = (int8_t)d.wpos[i];
        if (d.has_write && dst[0] < 0) return fail("remapped pass scheduled in place", (long long)k);
        const std::vector<cd> &in = dst[0] < 0 ? buf0 : *bufs[dst[0] ^ 1];
        std::vector<cd> in_copy;
        if (dst[0] < 0) in_copy = buf0;            // in place: tiles read and write the same set
        const std::vector<cd> &src = dst[0] < 0 ? in_copy : in;
        std::vector<cd> &out = dst[0] < 0 ? buf0 : *bufs[dst[0]];
        // block unitaries (row = output basis index, column = input)
        std::vector<std::vector<cd>> U(d.nsub, std::vector<cd>(32 * 32));
        for (int b = 0; b < d.nsub; ++b) {
            int kq = 0, qs[5];
            std::vector<double> m(2048);
            if (qs_plan_block(P, d.first_block + b, &kq, qs, m.data())) return fail("block", b);
            for (int e = 0; e < 1024; ++e) U[b][e] = cd(m[2 * e], m[2 * e + 1]);
        }
        std::fill(hits.begin(), hits.end(), 0);
        std::vector<cd> stage(4096), x(128 * 32), a(128 * 32);
        std::vector<int> sh(4096), ah(128 * 32);
        for (uint64_t t = 0; t < tiles; ++t) {
            const uint64_t tbase = deposit_tile(t, L);
            // ---- prefetch_tile_linear: chunk c = 128 k + thread (tile indices
            // 2c, 2c+1) into staging slot c, then convert_load / convert_store: each thread's
            // chunks into block 0's rows and columns
            std::fill(sh.begin(), sh.end(), 0);
            std::fill(ah.begin(), ah.end(), 0);
            for (int th = 0; th < 128 * tpr; ++th) {
                uint64_t g = 0;
                uint32_t r = 0, jj = 0;
                for (int tb = 1; tb < 7 + tpr; ++tb) {
                    if (!((th >> (tb - 1)) & 1)) continue;
                    g |= 1ull << M.tpos[tb];
                    const int mm = M.tmap0[tb];
                    if (mm >= 0) r |= 1u << mm;
                    else jj |= 1u << (~mm);
                }
                for (int kk = 0; kk < 16 / tpr; ++kk) {
                    const uint64_t s = tbase | g | M.gk[kk * tpr];
                    if (s + 1 >= N) return fail("load out of range", (long long)s);
                    const int c = 128 * tpr * kk + th;
                    stage[2 * c] = src[s];
                    stage[2 * c + 1] = src[s + 1];
                    sh[2 * c]++;
                    sh[2 * c + 1]++;
                    const uint32_t row = r ^ M.rk[kk * tpr], j = jj ^ M.jk[kk * tpr];
                    const uint32_t row1 = row | M.dr, j1 = j | M.dj;
                    if (row >= 128 || j >= 32 || row1 >= 128 || j1 >= 32 || row1 * 32 + j1 == row * 32 + j)
                        return fail("A slot out of range", row, j);
                    if (M.pair && !(M.dj == 1 && M.dr == 0 && (j & 1) == 0))
                        return fail("column pair not adjacent", row, j);
                    x[row * 32 + j] = stage[2 * c];
                    x[row1 * 32 + j1] = stage[2 * c + 1];
                    ah[row * 32 + j]++;
                    ah[row1 * 32 + j1]++;
                }
            }
            for (int o = 0; o < 4096; ++o)
                if (sh[o] != 1) return fail("staging slot not written exactly once", (long long)t, o);
            for (int o = 0; o < 4096; ++o)
                if (ah[o] != 1) return fail("block-0 A slot not written exactly once", (long long)t, o);
            // check against the per-row gather (block 0's rows and columns)
            for (int row = 0; row < 128; ++row) {
                uint64_t rb = 0;
                for (int b = 0; b < 7; ++b) if ((row >> b) & 1) rb |= 1ull << L.c0_glob[b];
                for (int j = 0; j < 32; ++j)
                    if (x[row * 32 + j] != src[tbase | rb | L.g0[j]]) return fail("staged value mismatch", row, j);
            }
            for (int b = 0; b < d.nsub; ++b) {
                // contraction: y[row][jo] = sum_ji U[jo][ji] x[row][ji]
                std::vector<cd> y(128 * 32);
                for (int row = 0; row < 128; ++row)
                    for (int jo = 0; jo < 32; ++jo) {
                        cd acc(0, 0);
                        for (int ji = 0; ji < 32; ++ji) acc += U[b][jo * 32 + ji] * x[row * 32 + ji];
                        y[row * 32 + jo] = acc;
                    }
                if (b + 1 < d.nsub) {
                    std::fill(ah.begin(), ah.end(), 0);
                    for (int row = 0; row < 128; ++row) {
                        const uint32_t tp = emu_thread_part(L, b, row);
                        for (int jo = 0; jo < 32; ++jo) {
                            const uint32_t off = tp ^ L.scat[b][jo];
                            if (off >= 128 * 128) return fail("scatter offset out of range", row, jo);
                            const uint32_t r2 = off >> 7, chunk = (off >> 4) & 7;
                            const uint32_t j2 = (((chunk ^ (r2 & 7)) & 7) << 2) | ((off >> 2) & 3);
                            a[r2 * 32 + j2] = y[row * 32 + jo];
                            ah[r2 * 32 + j2]++;
                        }
                    }
                    for (int e = 0; e < 128 * 32; ++e)
                        if (ah[e] != 1) return fail("A slot not written exactly once", (long long)t, e);
                    x.swap(a);
                } else {
                    const uint64_t ob = emu_store_base(t, tbase, W);
                    for (int row = 0; row < 128; ++row) {
                        uint64_t gcl = 0;
                        for (int bb = 0; bb < 7; ++bb) if ((row >> bb) & 1) gcl |= 1ull << L.cl_glob[bb];
                        for (int jo = 0; jo < 32; ++jo) {
                            const uint64_t o = ob | gcl | L.gl[jo];
                            if (o >= N) return fail("store out of range", (long long)o);
                            out[o] = y[row * 32 + jo];
                            hits[o]++;
                        }
                    }
                }
            }
        }
        for (uint64_t i = 0; i < N; ++i)
            if (hits[i] != 1) return fail("output amplitude not written exactly once", (long long)k, (long long)i);
    }
    return 0;
}

extern "C" int tile_emu_apply(const qs_plan *P, int n, double *state, int remap, int tpr, int *n_passes_out,
                              int *kinds_out)
{
    if (tpr != 1 && tpr != 2) return fail("threads per row must be 1 or 2");
    g_err[0] = 0;
    const size_t npass = P->passes.size();
    std::vector<qs_tiled_desc> descs;
    std::vector<int> dst;
    if (qs_plan_tiled_schedule(P, n, 0, npass, remap, descs, dst)) return fail("schedule failed");
    if (n_passes_out) *n_passes_out = (int)npass;
    const uint64_t N = 1ull << n;
    std::vector<cd> buf0(reinterpret_cast<cd *>(state), reinterpret_cast<cd *>(state) + N), buf1(N, cd(0, 0));
    std::vector<cd> *bufs[2] = {&buf0, &buf1};
    std::vector<int> hits(N);
    for (size_t k = 0; k < npass; ++k)
        if (smem_pass(P, n, descs[k], dst[k], k, tpr, bufs, hits, kinds_out)) return 1;
    memcpy(state, buf0.data(), N * sizeof(cd));
    return 0;
}

// One pass's block-0 input mapping for an arbitrary descriptor (columns in
// any order, so that tile bit 0 can be any column or row of block 0): with
// amplitude i of an n-qubit state set to i, every A slot (row, column) of
// every tile must receive exactly the amplitude at tile base | row bits |
// column bits.  Returns 0, or 1 with tile_emu_error() set; *kind = 0 adjacent
// column pair, 1 other column, 2 rows.
extern "C" int tile_emu_check_input(int n, const int *T, const int *qpos0, int tpr, int *kind)
{
    if (tpr != 1 && tpr != 2) return fail("threads per row must be 1 or 2");
    g_err[0] = 0;
    int qpos[3][5];
    for (int j = 0; j < 5; ++j) qpos[0][j] = qpos0[j];
    Layout L;
    LoadMap M;
    if (qs_tile_layout_build(n, T, 1, qpos, nullptr, &L, &M, nullptr)) return fail("layout build failed");
    *kind = M.pair ? 0 : (M.dj ? 1 : 2);
    const uint64_t N = 1ull << n, tiles = N >> 12;
    std::vector<int> ah(4096);
    std::vector<uint64_t> a(4096);
    for (uint64_t t = 0; t < tiles; t += (tiles > 64 ? tiles / 64 : 1)) {
        const uint64_t tbase = deposit_tile(t, L);
        std::fill(ah.begin(), ah.end(), 0);
        for (int th = 0; th < 128 * tpr; ++th) {
            uint64_t g = 0;
            uint32_t r = 0, jj = 0;
            for (int tb = 1; tb < 7 + tpr; ++tb) {
                if (!((th >> (tb - 1)) & 1)) continue;
                g |= 1ull << M.tpos[tb];
                const int mm = M.tmap0[tb];
                if (mm >= 0) r |= 1u << mm;
                else jj |= 1u << (~mm);
            }
            for (int kk = 0; kk < 16 / tpr; ++kk) {
                const uint64_t s0 = tbase | g | M.gk[kk * tpr];
                const uint32_t row = r ^ M.rk[kk * tpr], j = jj ^ M.jk[kk * tpr];
                const uint32_t row1 = row | M.dr, j1 = j | M.dj;
                if (row1 >= 128 || j1 >= 32) return fail("A slot out of range", row1, j1);
                a[row * 32 + j] = s0;
                a[row1 * 32 + j1] = s0 + 1;
                ah[row * 32 + j]++;
                ah[row1 * 32 + j1]++;
            }
        }
        for (int row = 0; row < 128; ++row) {
            uint64_t rb = 0;
            for (int b = 0; b < 7; ++b) if ((row >> b) & 1) rb |= 1ull << L.c0_glob[b];
            for (int j = 0; j < 32; ++j) {
                if (ah[row * 32 + j] != 1) return fail("A slot not written exactly once", row, j);
                if (a[row * 32 + j] != (tbase | rb | L.g0[j])) return fail("A slot holds the wrong amplitude", row, j);
            }
        }
    }
    return 0;
}

// The plan `proto` rebound to a gate list with the same operations on the
// same qubits (other angles), as the batched executor does; destroy with
// qs_plan_destroy.
extern "C" int tile_emu_rebind(const qs_plan *proto, const qs_gate *gates, size_t count, qs_plan **out)
{
    g_err[0] = 0;
    if (qs_plan_rebind(proto, gates, count, out)) return fail("rebind failed");
    return 0;
}

// ---------------------------------------------------------------- k_tile_tmem
// The same plans the way k_tile_tmem (qpanda_b200/csrc/qs_tile_tmem.cu) moves
// data, pass by pass where its layout builder takes the pass (the others as
// k_fused_tile above would, through the same tables):
//   * copy_tile: chunk c = 128 k + t of the tile, from g_t | gk[k], into stage
//     chunk  (t ^ cf_t) ^ (k << 7) ^ cf_k[k];
//   * the gather: thread (warp w, lane l) reads column j of its block-0 row at
//     stage slot  xrow(w, l) ^ s_col[j];
//   * each block's product with its matrix permuted to the kernel's column
//     order (tmem_matrix_index over mperm[b]) in FP64;
//   * the exchanges between blocks through the staging buffer (every slot
//     written once, then read once);
//   * the last block's stores at store_base | o_lane / o_warp | o_col.
// Every staging slot must be written once and read once per tile, every output
// amplitude written once per pass.  conflicts[0] counts shared-memory phases
// of the gather whose lanes share a bank slot, conflicts[1] those of the
// copies, conflicts[2] those of the exchanges between blocks; passes[0] / [1]
// count the passes the kernel took / left.
extern "C" int tmem_emu_apply(const qs_plan *P, int n, double *state, int remap, int *passes, long long *conflicts)
{
    g_err[0] = 0;
    const size_t npass = P->passes.size();
    std::vector<qs_tiled_desc> descs;
    std::vector<int> dst;
    if (qs_plan_tiled_schedule(P, n, 0, npass, remap, descs, dst)) return fail("schedule failed");
    const uint64_t N = 1ull << n, tiles = N >> 12;
    std::vector<cd> buf0(reinterpret_cast<cd *>(state), reinterpret_cast<cd *>(state) + N), buf1(N, cd(0, 0));
    std::vector<cd> *bufs[2] = {&buf0, &buf1};
    std::vector<int> hits(N);
    for (size_t k = 0; k < npass; ++k) {
        const qs_tiled_desc &d = descs[k];
        qs_tmem::TLayout T;
        const int rb = qs_tmem_layout_build(n, &d, &T);
        if (rb == QS_ERR_UNSUPPORTED) {             // the product runs it on k_fused_tile
            passes[1]++;
            if (smem_pass(P, n, d, dst[k], k, 1, bufs, hits, nullptr)) return 1;
            continue;
        }
        if (rb) return fail("tmem layout build failed", (long long)k);
        passes[0]++;
        StoreMap W;
        memset(&W, 0, sizeof(W));
        W.mode = d.has_write ? d.wmode : 0;
        W.ntb = n - 12;
        for (int i = 0; i < W.ntb && i < 52; ++i) W.wpos[i] = (int8_t)d.wpos[i];
        const std::vector<cd> &in = dst[k] < 0 ? buf0 : *bufs[dst[k] ^ 1];
        std::vector<cd> in_copy;
        if (dst[k] < 0) in_copy = buf0;
        const std::vector<cd> &src = dst[k] < 0 ? in_copy : in;
        std::vector<cd> &out = dst[k] < 0 ? buf0 : *bufs[dst[k]];
        // block matrices in the kernel's column order
        std::vector<std::vector<cd>> U(d.nsub, std::vector<cd>(32 * 32));
        for (int b = 0; b < d.nsub; ++b) {
            int kq = 0, qs[5];
            std::vector<double> m(2048);
            if (qs_plan_block(P, d.first_block + b, &kq, qs, m.data())) return fail("block", b);
            for (uint32_t i = 0; i < 32; ++i)
                for (uint32_t j = 0; j < 32; ++j) {
                    const uint32_t si = qs_tmem::tmem_matrix_index(i, T.mperm[b]);
                    const uint32_t sj = qs_tmem::tmem_matrix_index(j, T.mperm[b]);
                    U[b][i * 32 + j] = cd(m[2 * (si * 32 + sj)], m[2 * (si * 32 + sj) + 1]);
                }
        }
        // the tile base as tbase_of computes it
        Layout TL;
        memset(&TL, 0, sizeof(TL));
        for (int j = 0; j < 12; ++j) TL.tpos[j] = T.tpos[j];
        std::fill(hits.begin(), hits.end(), 0);
        std::vector<cd> stage(4096);
        std::vector<int> wr(4096), rd(4096);
        std::vector<cd> y(128 * 32), y2(128 * 32);
        for (uint64_t t = 0; t < tiles; ++t) {
            const uint64_t tbase = deposit_tile(t, TL);
            std::fill(wr.begin(), wr.end(), 0);
            std::fill(rd.begin(), rd.end(), 0);
            for (int lt = 0; lt < 128; ++lt) {
                uint64_t g_t = 0;
                uint32_t cs_t = (uint32_t)lt;
                for (int b = 0; b < 7; ++b)
                    if ((lt >> b) & 1) { g_t |= T.g_bit[b]; cs_t ^= T.cf_bit[b]; }
                for (int kk = 0; kk < 16; ++kk) {
                    const uint64_t s = tbase | g_t | T.gk[kk];
                    if (s + 1 >= N) return fail("load out of range", (long long)s);
                    const uint32_t c = cs_t ^ ((uint32_t)kk << 7) ^ T.cf_k[kk];
                    if (c >= 2048) return fail("stage chunk out of range", lt, kk);
                    stage[2 * c] = src[s];
                    stage[2 * c + 1] = src[s + 1];
                    wr[2 * c]++;
                    wr[2 * c + 1]++;
                }
            }
            // copies: the 8 lanes of a quarter warp must write 8 distinct 16-byte bank slots
            if (t == 0)
                for (int kk = 0; kk < 16; ++kk)
                    for (int q = 0; q < 16; ++q) {
                        unsigned seen = 0;
                        bool clash = false;
                        for (int l = 0; l < 8; ++l) {
                            const int lt = 8 * q + l;
                            uint32_t cs_t = (uint32_t)lt;
                            for (int b = 0; b < 7; ++b)
                                if ((lt >> b) & 1) cs_t ^= T.cf_bit[b];
                            const uint32_t c = cs_t ^ ((uint32_t)kk << 7) ^ T.cf_k[kk];
                            const unsigned bit = 1u << (c & 7);
                            if (seen & bit) clash = true;
                            seen |= bit;
                        }
                        if (clash) conflicts[1]++;
                    }
            for (int o = 0; o < 4096; ++o)
                if (wr[o] != 1) return fail("staging slot not written exactly once", (long long)t, o);
            // gather
            for (int w = 0; w < 4; ++w)
                for (int l = 0; l < 32; ++l) {
                    uint32_t x = 0;
                    for (int i = 0; i < 5; ++i)
                        if ((l >> i) & 1) x ^= T.s_lane[i];
                    for (int v = 0; v < 2; ++v)
                        if ((w >> v) & 1) x ^= T.s_warp[v];
                    for (int j = 0; j < 32; ++j) {
                        const uint32_t sl = x ^ T.s_col[j];
                        if (sl >= 4096) return fail("gather slot out of range", l, j);
                        if (T.pair_in && (j & 1) && sl != (x ^ T.s_col[j - 1]) + 1)
                            return fail("gathered column pair not adjacent", l, j);
                        y[(32 * w + l) * 32 + j] = stage[sl];
                        rd[sl]++;
                    }
                }
            for (int o = 0; o < 4096; ++o)
                if (rd[o] != 1) return fail("staging slot not gathered exactly once", (long long)t, o);
            if (t == 0) {
                // gather phases: 8 lanes (16-byte reads of column pairs) or 16
                // lanes (8-byte reads) must hit distinct bank slots
                const int ph = T.pair_in ? 8 : 16;
                for (int w = 0; w < 4; ++w)
                    for (int j = 0; j < 32; j += T.pair_in ? 2 : 1)
                        for (int p0 = 0; p0 < 32; p0 += ph) {
                            unsigned seen = 0;
                            bool clash = false;
                            for (int l = p0; l < p0 + ph; ++l) {
                                uint32_t x = 0;
                                for (int i = 0; i < 5; ++i)
                                    if ((l >> i) & 1) x ^= T.s_lane[i];
                                for (int v = 0; v < 2; ++v)
                                    if ((w >> v) & 1) x ^= T.s_warp[v];
                                const uint32_t sl = x ^ T.s_col[j];
                                const unsigned bit = T.pair_in ? 1u << ((sl >> 1) & 7) : 1u << (sl & 15);
                                if (seen & bit) clash = true;
                                seen |= bit;
                            }
                            if (clash) conflicts[0]++;
                        }
            }
            for (int b = 0; b < d.nsub; ++b) {
                for (int r = 0; r < 128; ++r)
                    for (int i = 0; i < 32; ++i) {
                        cd acc(0, 0);
                        for (int j = 0; j < 32; ++j) acc += U[b][i * 32 + j] * y[r * 32 + j];
                        y2[r * 32 + i] = acc;
                    }
                y.swap(y2);
                if (b + 1 < d.nsub) {
                    // through the staging buffer: every slot written once, read once
                    std::vector<cd> ex(4096);
                    std::vector<int> ew(4096, 0), er(4096, 0);
                    for (int w = 0; w < 4; ++w)
                        for (int l = 0; l < 32; ++l) {
                            uint32_t xw = 0, xr = 0;
                            for (int i = 0; i < 5; ++i)
                                if ((l >> i) & 1) { xw ^= T.xw_lane[b][i]; xr ^= T.xr_lane[b][i]; }
                            for (int v = 0; v < 2; ++v)
                                if ((w >> v) & 1) { xw ^= T.xw_warp[b][v]; xr ^= T.xr_warp[b][v]; }
                            for (int j = 0; j < 32; ++j) {
                                const uint32_t sl = xw ^ T.xw_col[b][j];
                                if (sl >= 4096) return fail("exchange write slot out of range", l, j);
                                ex[sl] = y[(32 * w + l) * 32 + j];
                                ew[sl]++;
                            }
                        }
                    for (int o = 0; o < 4096; ++o)
                        if (ew[o] != 1) return fail("exchange slot not written exactly once", (long long)t, o);
                    for (int w = 0; w < 4; ++w)
                        for (int l = 0; l < 32; ++l) {
                            uint32_t xr = 0;
                            for (int i = 0; i < 5; ++i)
                                if ((l >> i) & 1) xr ^= T.xr_lane[b][i];
                            for (int v = 0; v < 2; ++v)
                                if ((w >> v) & 1) xr ^= T.xr_warp[b][v];
                            for (int j = 0; j < 32; ++j) {
                                const uint32_t sl = xr ^ T.xr_col[b][j];
                                if (sl >= 4096) return fail("exchange read slot out of range", l, j);
                                y2[(32 * w + l) * 32 + j] = ex[sl];
                                er[sl]++;
                            }
                        }
                    for (int o = 0; o < 4096; ++o)
                        if (er[o] != 1) return fail("exchange slot not read exactly once", (long long)t, o);
                    y.swap(y2);
                    if (t == 0) {
                        // half warps of both phases: 16 distinct 8-byte bank slots
                        for (int ph = 0; ph < 2; ++ph)
                            for (int w = 0; w < 4; ++w)
                                for (int j = 0; j < 32; ++j)
                                    for (int h = 0; h < 2; ++h) {
                                        unsigned seen = 0;
                                        bool clash = false;
                                        for (int l = 16 * h; l < 16 * h + 16; ++l) {
                                            uint32_t x = 0;
                                            for (int i = 0; i < 5; ++i)
                                                if ((l >> i) & 1) x ^= ph ? T.xr_lane[b][i] : T.xw_lane[b][i];
                                            for (int v = 0; v < 2; ++v)
                                                if ((w >> v) & 1) x ^= ph ? T.xr_warp[b][v] : T.xw_warp[b][v];
                                            const uint32_t sl = x ^ (ph ? T.xr_col[b][j] : T.xw_col[b][j]);
                                            const unsigned bit = 1u << (sl & 15);
                                            if (seen & bit) clash = true;
                                            seen |= bit;
                                        }
                                        if (clash) conflicts[2]++;
                                    }
                    }
                } else {
                    const uint64_t ob = emu_store_base(t, tbase, W);
                    for (int w = 0; w < 4; ++w)
                        for (int l = 0; l < 32; ++l) {
                            uint64_t orow = 0;
                            for (int i = 0; i < 5; ++i)
                                if ((l >> i) & 1) orow |= T.o_lane[i];
                            for (int v = 0; v < 2; ++v)
                                if ((w >> v) & 1) orow |= T.o_warp[v];
                            for (int j = 0; j < 32; ++j) {
                                const uint64_t o = ob | orow | T.o_col[j];
                                if (o >= N) return fail("store out of range", (long long)o);
                                if (T.vec_out && (j & 1) && o != (ob | orow | T.o_col[j - 1]) + 1)
                                    return fail("stored column pair not adjacent", l, j);
                                out[o] = y[(32 * w + l) * 32 + j];
                                hits[o]++;
                            }
                        }
                }
            }
        }
        for (uint64_t i = 0; i < N; ++i)
            if (hits[i] != 1) return fail("output amplitude not written exactly once", (long long)k, (long long)i);
    }
    memcpy(state, buf0.data(), N * sizeof(cd));
    return 0;
}

// Memory shape of k_tile_tmem's accesses over a plan (no state needed): the
// passes whose last block stores 16-byte vectors, and per warp and tile the
// distinct 128-byte lines its store instructions and its copy instructions
// touch (8 KB each way: 64 lines at best), summed over the passes.
extern "C" int tmem_layout_stats(const qs_plan *P, int n, int remap, int *vec_out_passes, long long *store_lines,
                                 long long *copy_lines)
{
    g_err[0] = 0;
    const size_t npass = P->passes.size();
    std::vector<qs_tiled_desc> descs;
    std::vector<int> dst;
    if (qs_plan_tiled_schedule(P, n, 0, npass, remap, descs, dst)) return fail("schedule failed");
    *vec_out_passes = 0;
    *store_lines = *copy_lines = 0;
    for (size_t k = 0; k < npass; ++k) {
        qs_tmem::TLayout L;
        if (qs_tmem_layout_build(n, &descs[k], &L)) return fail("pass %lld: no tensor-memory layout", (long long)k);
        *vec_out_passes += L.vec_out ? 1 : 0;
        const int nj = L.vec_out ? 16 : 32;
        for (int w = 0; w < 4; ++w) {
            for (int j = 0; j < nj; ++j) {
                std::vector<uint64_t> lines;
                for (int l = 0; l < 32; ++l) {
                    uint64_t o = L.o_col[L.vec_out ? 2 * j : j];
                    for (int i = 0; i < 5; ++i)
                        if ((l >> i) & 1) o |= L.o_lane[i];
                    for (int v = 0; v < 2; ++v)
                        if ((w >> v) & 1) o |= L.o_warp[v];
                    lines.push_back(o >> 4);                     // 8-byte amplitudes, 128-byte lines
                }
                std::sort(lines.begin(), lines.end());
                *store_lines += std::unique(lines.begin(), lines.end()) - lines.begin();
            }
            for (int k2 = 0; k2 < 16; ++k2) {
                std::vector<uint64_t> lines;
                for (int l = 0; l < 32; ++l) {
                    const int t = 32 * w + l;
                    uint64_t g = L.gk[k2];
                    for (int b = 0; b < 7; ++b)
                        if ((t >> b) & 1) g |= L.g_bit[b];
                    lines.push_back(g >> 4);
                }
                std::sort(lines.begin(), lines.end());
                *copy_lines += std::unique(lines.begin(), lines.end()) - lines.begin();
            }
        }
    }
    *store_lines /= 4;
    *copy_lines /= 4;
    return 0;
}
