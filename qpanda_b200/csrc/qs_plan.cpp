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

struct PlanBlock {
    int k = 0;
    int q[5] = {0, 0, 0, 0, 0};          // ascending global qubits
    std::vector<cd> U;                   // 32 x 32 row-major
    std::vector<size_t> gates;           // indices into the gate list, in application order
};

struct qs_plan {
    int n = 0;
    int max_k = 5;
    std::vector<qs_gate> gates;
    std::vector<PlanBlock> blocks;
    int dev = -1;                        // device holding mats
    void *mats = nullptr;                // [blocks][2][64][64] bf16
};

namespace {

uint64_t remap(uint64_t mask, const int *q, int k)
{
    uint64_t r = 0;
    for (int b = 0; b < k; ++b)
        if (mask & (1ull << q[b])) r |= 1ull << b;
    return r;
}

// Apply a primitive (already remapped to local bit positions) to a k-qubit vector.
void apply_local(const qs_prim &p, cd *v, int k)
{
    const uint64_t N = 1ull << k;
    if (p.kind == QS_PRIM_PHASE) {
        cd ph(p.m[0], p.m[1]);
        for (uint64_t i = 0; i < N; ++i)
            if ((i & p.holes) == p.holes) v[i] *= ph;
        return;
    }
    cd m00(p.m[0], p.m[1]), m01(p.m[2], p.m[3]), m10(p.m[4], p.m[5]), m11(p.m[6], p.m[7]);
    for (uint64_t i = 0; i < N; ++i) {
        if ((i & p.holes) != p.cmask) continue;     // base: hole bits zero except controls
        cd a = v[i | p.off0], b = v[i | p.off1];
        v[i | p.off0] = m00 * a + m01 * b;
        v[i | p.off1] = m10 * a + m11 * b;
    }
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

int build_blocks(qs_plan *P)
{
    const size_t G = P->gates.size();
    std::vector<uint64_t> mask(G);
    std::vector<qs_prim> prim(G);
    for (size_t i = 0; i < G; ++i) {
        int r = qs_lower_gate(P->n, &P->gates[i], &prim[i]);
        if (r) return r;
        mask[i] = qs_gate_qubits(&P->gates[i]);
        if (__builtin_popcountll(mask[i]) > P->max_k)
            return qs_fail(QS_ERR_UNSUPPORTED, "plan: gate %zu touches %d qubits (fusion width %d)", i,
                           __builtin_popcountll(mask[i]), P->max_k);
    }
    std::vector<char> done(G, 0);
    size_t left = G, first = 0;
    while (left) {
        PlanBlock B;
        uint64_t Q = 0;
        bool changed = true;
        while (changed) {
            changed = false;
            uint64_t blocked = 0;
            while (first < G && done[first]) ++first;
            for (size_t i = first; i < G; ++i) {
                if (done[i]) continue;
                const uint64_t m = mask[i];
                if (!(m & blocked) && __builtin_popcountll(Q | m) <= P->max_k) {
                    done[i] = 1;
                    --left;
                    Q |= m;
                    B.gates.push_back(i);
                    changed = true;
                } else {
                    blocked |= m;
                }
            }
        }
        // widen to 5 qubits with the lowest free ones
        for (int q = 0; q < P->n && __builtin_popcountll(Q) < 5; ++q) Q |= 1ull << q;
        B.k = 0;
        for (int q = 0; q < P->n; ++q)
            if (Q & (1ull << q)) B.q[B.k++] = q;
        // U = product of the block's gates, column by column
        B.U.assign(32 * 32, cd(0, 0));
        std::vector<cd> col(32);
        for (int c = 0; c < 32; ++c) {
            std::fill(col.begin(), col.end(), cd(0, 0));
            col[c] = 1;
            for (size_t gi : B.gates) {
                qs_prim lp = prim[gi];
                lp.holes = remap(lp.holes, B.q, 5);
                lp.cmask = remap(lp.cmask, B.q, 5);
                lp.off0 = remap(lp.off0, B.q, 5);
                lp.off1 = remap(lp.off1, B.q, 5);
                apply_local(lp, col.data(), 5);
            }
            for (int r = 0; r < 32; ++r) B.U[r * 32 + c] = col[r];
        }
        P->blocks.push_back(std::move(B));
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
    if (!out) return qs_fail(QS_ERR_ARG, "qs_plan_create: null output");
    *out = nullptr;
    if (n < 1 || n > QS_MAX_QUBITS) return qs_fail(QS_ERR_ARG, "qs_plan_create: bad qubit count %d", n);
    if (max_k < 1 || max_k > 5)
        return qs_fail(QS_ERR_UNSUPPORTED, "qs_plan_create: fusion width %d (this build fuses up to 5 qubits)", max_k);
    if (count && !gates) return qs_fail(QS_ERR_ARG, "qs_plan_create: null gate list");
    qs_plan *P = new qs_plan();
    P->n = n;
    P->max_k = max_k;
    P->gates.assign(gates, gates + count);
    // Below 12 qubits a state has fewer than one 128 x 32 tile: the plan keeps
    // the gate list only and runs it through the per-gate kernels.
    int r = n >= 12 ? build_blocks(P) : QS_OK;
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
        cudaFree(P->mats);
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

int qs_plan_upload(qs_plan *P, int dev)
{
    if (P->mats && P->dev == dev) return QS_OK;
    if (P->mats) {
        cudaFree(P->mats);
        P->mats = nullptr;
    }
    const size_t per = 2 * 64 * 64;
    std::vector<uint16_t> host(per * (P->blocks.size() ? P->blocks.size() : 1));
    for (size_t b = 0; b < P->blocks.size(); ++b) block_bf16(P->blocks[b], host.data() + b * per);
    QS_CUDA_TRY(cudaMalloc(&P->mats, host.size() * sizeof(uint16_t)));
    QS_CUDA_TRY(cudaMemcpy(P->mats, host.data(), host.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    P->dev = dev;
    return QS_OK;
}

int qs_launch_prim(qs_state *s, const qs_prim &p);

extern "C" int qs_plan_apply(qs_state *s, qs_plan *P)
{
    return qs_plan_apply_range(s, P, 0, P ? P->blocks.size() : 0);
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
            if (first > P->blocks.size() || count > P->blocks.size() - first)
                return qs_fail(QS_ERR_ARG, "qs_plan_apply_range: blocks [%zu, +%zu) out of range", first, count);
            for (size_t b = first; b < first + count; ++b)
                idx.insert(idx.end(), P->blocks[b].gates.begin(), P->blocks[b].gates.end());
        }
        for (size_t i : idx) {
            qs_prim p;
            if ((r = qs_lower_gate(s->n, &P->gates[i], &p)) || (r = qs_launch_prim(s, p))) return r;
        }
        return QS_OK;
    }
    if (first > P->blocks.size() || count > P->blocks.size() - first)
        return qs_fail(QS_ERR_ARG, "qs_plan_apply_range: blocks [%zu, +%zu) out of range", first, count);
    if ((r = qs_plan_upload(P, s->device))) return r;
    // Norm partials live in their own per-state buffer, so that other calls
    // between two qs_plan_apply_range calls cannot overwrite them:
    // [0] input norm of block 0, [1]/[2] output norms of even/odd blocks.
    const int G = qs_fused_grid(s);
    if (!s->fused_norm) QS_CUDA_TRY(cudaMalloc(&s->fused_norm, 3 * (size_t)QS_SM_COUNT * 4 * sizeof(double)));
    double *norm = s->fused_norm;
    // watchdog flag (result area of scratch), cleared before the first block
    const size_t kFlagOff = 64 * 1024 + 192;
    int *flag = reinterpret_cast<int *>(static_cast<char *>(s->scratch) + kFlagOff);
    if (first == 0) QS_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), s->stream));
    const size_t per = 2 * 64 * 64 * sizeof(uint16_t);
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
    if (flag) return qs_fail(QS_ERR_STATE, "fused pass: a bounded wait in the tensor-core kernel expired");
    return QS_OK;
}
