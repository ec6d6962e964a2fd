// qs_sharded.cpp - an n-qubit state over 2^g shards (one GPU each, or several
// in one process), host C++ over the single-GPU C ABI.
//
// Physical position p of the amplitude index is a local bit for p < L = n - g
// (each shard holds the 2^L amplitudes of its slice) and rank bit p - L above.
// Logical qubit q lives at physical position pos[q].  A gate whose qubits are
// all local runs on every shard with no communication; a gate on a global
// qubit first swaps it with a local position the gate does not use (the
// furthest-used one, highest first - the top position makes the half one
// contiguous block): the two shards that differ in that rank bit exchange half
// of their slices - the one with rank bit b gives the half with local bit
// p = 1 - b and receives the partner's half with local bit p = b into the same
// place.  The schedule is the one qpanda_b200/sharded.py computes.
//
// Transport: two local shards swap halves in place with one kernel
// (qs_swap.cu: each element pair read and written once, no staging); a
// partner whose shard this process can address (a peer GPU's buffer, or an
// IPC mapping of another process's shard, registered with
// qs_sharded_set_peer) is swapped with the same kernel over NVLink, each side
// taking half of the rows between two calls of the caller's barrier; any
// other partner's half goes through the caller's exchange function (NCCL
// send/receive, MPI ...): packed into a staging buffer in chunks of at most
// 256 MB, and what comes back unpacked.  The reference has no counterpart: it
// caps programs at 30 qubits (QPandaAPI.cpp:87).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "qs_common.cuh"
#include "qs_prim.h"
#include "qs_swap.h"

namespace {

constexpr size_t kChunkBytes = 256ull << 20;

struct Step {
    int swap = 0;                // 1: exchange rank bit j with local position p
    int j = 0, p = 0;
    std::vector<qs_gate> gates;  // swap == 0: gate records in physical positions
};

int gate_qubit_list(const qs_gate &g, int *q)
{
    int k = 2;
    if (g.op >= QS_OP_H && g.op <= QS_OP_RZ) k = 1;
    else if (g.op == QS_OP_TOFFOLI || g.op == QS_OP_CSWAP) k = 3;
    int c = 0;
    for (int i = 0; i < k; ++i) q[c++] = g.q[i];
    for (int i = 0; i < g.nctrl && i < QS_MAX_CTRL; ++i) q[c++] = g.ctrl[i];
    return c;
}

qs_gate relabel(const qs_gate &g, const std::vector<int> &pos)
{
    qs_gate h = g;
    int k = 2;
    if (g.op >= QS_OP_H && g.op <= QS_OP_RZ) k = 1;
    else if (g.op == QS_OP_TOFFOLI || g.op == QS_OP_CSWAP) k = 3;
    for (int i = 0; i < k; ++i) h.q[i] = pos[g.q[i]];
    for (int i = 0; i < g.nctrl && i < QS_MAX_CTRL; ++i) h.ctrl[i] = pos[g.ctrl[i]];
    return h;
}

// Steps for `gates` (logical qubits) from layout pos (updated in place).
int schedule(int n, int g, const qs_gate *gates, size_t count, std::vector<int> &pos, std::vector<Step> &steps)
{
    const int L = n - g;
    std::vector<int> at(n);
    for (int q = 0; q < n; ++q) at[pos[q]] = q;
    std::vector<std::vector<int>> uses(count);
    for (size_t i = 0; i < count; ++i) {
        int q[QS_MAX_CTRL + 3];
        const int k = gate_qubit_list(gates[i], q);
        for (int j = 0; j < k; ++j)
            if (q[j] < 0 || q[j] >= n) return qs_fail(QS_ERR_ARG, "sharded: gate %zu: qubit %d out of range", i, q[j]);
        if (k > L) return qs_fail(QS_ERR_ARG, "sharded: gate %zu has more qubits than a shard's %d local positions", i, L);
        uses[i].assign(q, q + k);
    }
    Step seg;
    for (size_t i = 0; i < count; ++i) {
        for (int q : uses[i]) {
            if (pos[q] < L) continue;
            std::vector<char> busy(L, 0);
            for (int x : uses[i])
                if (pos[x] < L) busy[pos[x]] = 1;
            auto next_use = [&](int p) {
                const int lq = at[p];
                for (size_t k = i; k < count; ++k)
                    if (std::find(uses[k].begin(), uses[k].end(), lq) != uses[k].end()) return k;
                return count;
            };
            size_t far = 0;
            int best = -1;
            for (int p = L - 1; p >= 0; --p) {
                if (busy[p]) continue;
                const size_t u = next_use(p);
                if (best < 0 || u > far) { far = u; best = p; }
            }
            if (best < 0) return qs_fail(QS_ERR_ARG, "sharded: no free local position for gate %zu", i);
            if (!seg.gates.empty()) {
                steps.push_back(seg);
                seg.gates.clear();
            }
            Step sw;
            sw.swap = 1;
            sw.j = pos[q] - L;
            sw.p = best;
            steps.push_back(sw);
            const int gp = pos[q], lq = at[best];
            pos[q] = best;
            pos[lq] = gp;
            at[best] = q;
            at[gp] = lq;
        }
        seg.gates.push_back(relabel(gates[i], pos));
    }
    if (!seg.gates.empty()) steps.push_back(seg);
    return QS_OK;
}

}  // namespace

struct qs_sharded_peer {
    int partner = -1;
    void *amp = nullptr;                     // the partner shard's amplitudes, addressable here
    qs_barrier_fn barrier = nullptr;
    void *ctx = nullptr;
};

struct qs_sharded {
    int n = 0, g = 0, L = 0, dtype = QS_C64;
    std::vector<qs_sharded_peer> peers;
    std::vector<int> ranks;                  // rank bits of the local shards
    std::vector<qs_state *> shards;
    std::vector<int> pos;
    qs_exchange_fn exchange = nullptr;
    void *ctx = nullptr;
    void *stage[2] = {nullptr, nullptr};     // staging buffers (device of shard 0)
    size_t stage_bytes = 0;
    size_t swaps = 0, bytes = 0;
};

namespace {

size_t amp_size(int dtype) { return dtype == QS_C64 ? 8 : 16; }

int ensure_stage(qs_sharded *S, size_t bytes)
{
    if (S->stage_bytes >= bytes) return QS_OK;
    for (void *&p : S->stage)
        if (p) { cudaFree(p); p = nullptr; }
    for (void *&p : S->stage) QS_CUDA_TRY(cudaMalloc(&p, bytes));
    S->stage_bytes = bytes;
    return QS_OK;
}

// The half of a shard's slice with local bit p == v, rows [r0, r0 + nr) of it:
// rows of 2^p amplitudes, 2^(p+1) apart.
struct Half {
    char *base;
    size_t width, pitch, rows;
};

Half half_of(const qs_sharded *S, qs_state *s, int p, int v)
{
    const size_t a = amp_size(S->dtype);
    Half h;
    h.width = (a << p);
    h.pitch = 2 * h.width;
    h.rows = (size_t)1 << (S->L - 1 - p);
    h.base = static_cast<char *>(s->amp) + (v ? h.width : 0);
    return h;
}

// A piece of a half: rows [r0, r0 + nr), bytes [c0, c0 + w) of each row.
// Pieces hold at most kChunkBytes: several whole rows, or part of one.
struct Piece {
    size_t r0, nr, c0, w;
};

void pieces_of(const Half &h, std::vector<Piece> &out)
{
    if (h.width <= kChunkBytes) {
        const size_t per = kChunkBytes / h.width;
        for (size_t r = 0; r < h.rows; r += per) out.push_back({r, std::min(per, h.rows - r), 0, h.width});
    } else {
        for (size_t r = 0; r < h.rows; ++r)
            for (size_t c = 0; c < h.width; c += kChunkBytes) out.push_back({r, 1, c, std::min(kChunkBytes, h.width - c)});
    }
}

size_t piece_bytes(const Piece &c) { return c.nr * c.w; }

char *piece_base(const Half &h, const Piece &c) { return h.base + c.r0 * h.pitch + c.c0; }

// a piece of a half to / from a contiguous buffer, or between two halves
int piece_copy(char *dst, size_t dpitch, const char *src, size_t spitch, const Piece &c, cudaStream_t st)
{
    QS_CUDA_TRY(cudaMemcpy2DAsync(dst, dpitch, src, spitch, c.w, c.nr, cudaMemcpyDeviceToDevice, st));
    return QS_OK;
}

int swap_local_pair(qs_sharded *S, qs_state *s0, qs_state *s1, int p)
{
    // s0 has rank bit 0: its half p = 1 trades places with s1's half p = 0
    const Half a = half_of(S, s0, p, 1), b = half_of(S, s1, p, 0);
    cudaStream_t st = s0->stream;
    QS_CUDA_TRY(cudaStreamSynchronize(s1->stream));
    int r = qs_launch_swap_halves(a.base, b.base, a.width, a.pitch, 0, a.rows, 0, a.width, st);
    if (r) return r;
    QS_CUDA_TRY(cudaStreamSynchronize(st));
    S->bytes += 2 * a.width * a.rows;
    return QS_OK;
}

// The partner's shard is addressable from here: this side swaps its share of
// the element pairs (the rank-bit-0 side the first half of the rows, or of the
// single row) in place, between two barriers with the partner.
int swap_peer(qs_sharded *S, size_t i, int j, int p, const qs_sharded_peer &peer)
{
    qs_state *s = S->shards[i];
    const int rank = S->ranks[i], partner = rank ^ (1 << j);
    const int b = (rank >> j) & 1;
    const Half mine = half_of(S, s, p, 1 - b);
    char *theirs = static_cast<char *>(peer.amp) + (b ? mine.width : 0);
    size_t r0 = 0, nr = mine.rows, c0 = 0, w = mine.width;
    if (mine.rows >= 2) {
        nr = mine.rows / 2;
        r0 = b ? nr : 0;
    } else {
        w = mine.width / 2;
        c0 = b ? w : 0;
    }
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (peer.barrier(peer.ctx, rank, partner))
        return qs_fail(QS_ERR_STATE, "sharded: barrier with shard %d before a swap failed", partner);
    int r = qs_launch_swap_halves(mine.base, theirs, mine.width, mine.pitch, r0, nr, c0, w, s->stream);
    if (r) return r;
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (peer.barrier(peer.ctx, rank, partner))
        return qs_fail(QS_ERR_STATE, "sharded: barrier with shard %d after a swap failed", partner);
    S->bytes += 2 * nr * w;
    return QS_OK;
}

const qs_sharded_peer *find_peer(const qs_sharded *S, int partner)
{
    for (const qs_sharded_peer &q : S->peers)
        if (q.partner == partner) return &q;
    return nullptr;
}

int swap_remote(qs_sharded *S, size_t i, int j, int p)
{
    qs_state *s = S->shards[i];
    const int rank = S->ranks[i], partner = rank ^ (1 << j);
    const int b = (rank >> j) & 1;
    const Half h = half_of(S, s, p, 1 - b);
    std::vector<Piece> pcs;
    pieces_of(h, pcs);
    int r = ensure_stage(S, std::min(kChunkBytes, h.width * h.rows));
    if (r) return r;
    cudaStream_t st = s->stream;
    char *out = static_cast<char *>(S->stage[0]), *in = static_cast<char *>(S->stage[1]);
    for (const Piece &c : pcs) {
        const size_t bytes = piece_bytes(c);
        if ((r = piece_copy(out, c.w, piece_base(h, c), h.pitch, c, st))) return r;
        QS_CUDA_TRY(cudaStreamSynchronize(st));
        const int rc = S->exchange(S->ctx, rank, partner, out, in, bytes, st);
        if (rc) return qs_fail(QS_ERR_STATE, "sharded: exchange with shard %d failed (%d)", partner, rc);
        if ((r = piece_copy(piece_base(h, c), h.pitch, in, c.w, c, st))) return r;
        S->bytes += 2 * bytes;
    }
    QS_CUDA_TRY(cudaStreamSynchronize(st));
    return QS_OK;
}

}  // namespace

extern "C" int qs_sharded_create(int n_qubits, int n_global, int dtype, const int *ranks, int n_ranks,
                                 qs_exchange_fn exchange, void *ctx, qs_sharded **out)
{
    if (!out) return qs_fail(QS_ERR_ARG, "qs_sharded_create: null output");
    *out = nullptr;
    if (dtype != QS_C64 && dtype != QS_C128) return qs_fail(QS_ERR_ARG, "qs_sharded_create: bad dtype %d", dtype);
    if (n_global < 0 || n_global > 16 || n_qubits - n_global < 2 || n_qubits > QS_MAX_QUBITS)
        return qs_fail(QS_ERR_ARG, "qs_sharded_create: %d qubits over 2^%d shards", n_qubits, n_global);
    if (!ranks || n_ranks < 1 || n_ranks > (1 << n_global))
        return qs_fail(QS_ERR_ARG, "qs_sharded_create: %d local shards", n_ranks);
    qs_sharded *S = new qs_sharded();
    S->n = n_qubits;
    S->g = n_global;
    S->L = n_qubits - n_global;
    S->dtype = dtype;
    S->exchange = exchange;
    S->ctx = ctx;
    S->pos.resize(n_qubits);
    for (int q = 0; q < n_qubits; ++q) S->pos[q] = q;
    for (int i = 0; i < n_ranks; ++i) {
        const int rk = ranks[i];
        if (rk < 0 || rk >= (1 << n_global) || std::count(ranks, ranks + i, rk)) {
            qs_sharded_destroy(S);
            return qs_fail(QS_ERR_ARG, "qs_sharded_create: shard %d listed twice or out of range", rk);
        }
        qs_state *s = nullptr;
        int r = qs_create(S->L, dtype, nullptr, &s);
        if (r) { qs_sharded_destroy(S); return r; }
        if (rk) {                                     // only shard 0 holds |0...0>
            r = cudaMemsetAsync(s->amp, 0, s->amp_bytes(), s->stream) == cudaSuccess ? QS_OK
                    : qs_fail(QS_ERR_CUDA, "qs_sharded_create: clearing a shard failed");
            if (r) { qs_destroy(s); qs_sharded_destroy(S); return r; }
        }
        S->ranks.push_back(rk);
        S->shards.push_back(s);
    }
    *out = S;
    return QS_OK;
}

extern "C" int qs_sharded_apply(qs_sharded *S, const qs_gate *gates, size_t count)
{
    if (!S) return qs_fail(QS_ERR_ARG, "qs_sharded_apply: null state");
    if (count && !gates) return qs_fail(QS_ERR_ARG, "qs_sharded_apply: null gate list");
    std::vector<int> pos = S->pos;
    std::vector<Step> steps;
    int r = schedule(S->n, S->g, gates, count, pos, steps);
    if (r) return r;
    for (const Step &st : steps) {
        if (!st.swap) {
            for (qs_state *s : S->shards)
                if ((r = qs_gates_apply(s, st.gates.data(), st.gates.size()))) return r;
            continue;
        }
        for (qs_state *s : S->shards) QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
        for (size_t i = 0; i < S->shards.size(); ++i) {
            const int rank = S->ranks[i], partner = rank ^ (1 << st.j);
            auto it = std::find(S->ranks.begin(), S->ranks.end(), partner);
            if (it != S->ranks.end()) {
                if (rank & (1 << st.j)) continue;      // the pair is handled from its rank-bit-0 member
                r = swap_local_pair(S, S->shards[i], S->shards[it - S->ranks.begin()], st.p);
            } else if (const qs_sharded_peer *pe = find_peer(S, partner)) {
                r = swap_peer(S, i, st.j, st.p, *pe);
            } else if (S->exchange) {
                r = swap_remote(S, i, st.j, st.p);
            } else {
                r = qs_fail(QS_ERR_ARG, "sharded: shard %d's partner %d is not local, not a peer, and no exchange "
                            "was given", rank, partner);
            }
            if (r) return r;
        }
        ++S->swaps;
    }
    S->pos = pos;
    return QS_OK;
}

extern "C" int qs_sharded_set_peer(qs_sharded *S, int partner, void *partner_amp, qs_barrier_fn barrier,
                                   void *ctx)
{
    if (!S || !partner_amp || !barrier) return qs_fail(QS_ERR_ARG, "qs_sharded_set_peer: null argument");
    if (partner < 0 || partner >= (1 << S->g))
        return qs_fail(QS_ERR_ARG, "qs_sharded_set_peer: shard %d out of range", partner);
    if (std::find(S->ranks.begin(), S->ranks.end(), partner) != S->ranks.end())
        return qs_fail(QS_ERR_ARG, "qs_sharded_set_peer: shard %d is local", partner);
    if ((uintptr_t)partner_amp % 16)
        return qs_fail(QS_ERR_ARG, "qs_sharded_set_peer: shard %d's amplitudes are not 16-byte aligned", partner);
    for (qs_sharded_peer &q : S->peers)
        if (q.partner == partner) {
            q.amp = partner_amp;
            q.barrier = barrier;
            q.ctx = ctx;
            return QS_OK;
        }
    qs_sharded_peer q;
    q.partner = partner;
    q.amp = partner_amp;
    q.barrier = barrier;
    q.ctx = ctx;
    S->peers.push_back(q);
    return QS_OK;
}

extern "C" int qs_sharded_shard(qs_sharded *S, int rank, qs_state **shard)
{
    if (!S || !shard) return qs_fail(QS_ERR_ARG, "qs_sharded_shard: null argument");
    auto it = std::find(S->ranks.begin(), S->ranks.end(), rank);
    if (it == S->ranks.end()) return qs_fail(QS_ERR_ARG, "qs_sharded_shard: shard %d is not local", rank);
    *shard = S->shards[it - S->ranks.begin()];
    return QS_OK;
}

extern "C" int qs_sharded_positions(const qs_sharded *S, int *pos)
{
    if (!S || !pos) return qs_fail(QS_ERR_ARG, "qs_sharded_positions: null argument");
    for (int q = 0; q < S->n; ++q) pos[q] = S->pos[q];
    return QS_OK;
}

extern "C" int qs_sharded_info(const qs_sharded *S, size_t *swaps, size_t *bytes_moved)
{
    if (!S) return qs_fail(QS_ERR_ARG, "qs_sharded_info: null state");
    if (swaps) *swaps = S->swaps;
    if (bytes_moved) *bytes_moved = S->bytes;
    return QS_OK;
}

extern "C" int qs_sharded_destroy(qs_sharded *S)
{
    if (!S) return QS_OK;
    for (qs_state *s : S->shards) qs_destroy(s);
    for (void *p : S->stage)
        if (p) cudaFree(p);
    delete S;
    return QS_OK;
}
