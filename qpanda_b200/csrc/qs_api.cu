// qs_api.cu - C ABI: state lifetime, errors, and the lowering of reference
// gate records (QPandaSDK/QuantumInstructionHandle/QuantumGates.h methods)
// onto the generic kernels of qs_gates.cu.
//
// The reference conventions live in qs_lower.cpp (qs_lower_gate).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "qs_common.cuh"
#include "qs_lowstage.cuh"
#include "qs_prim.h"

int qs_copy_in(qs_state *s, const void *host, int host_dtype);
int qs_copy_out(qs_state *s, void *host, int host_dtype);

// ------------------------------------------------------------------ errors
static thread_local char g_err[512];

int qs_fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int qs_cuda_fail(cudaError_t e, const char *where)
{
    return qs_fail(e == cudaErrorMemoryAllocation ? QS_ERR_OOM : QS_ERR_CUDA, "%s: %s (%s)", where,
                   cudaGetErrorString(e), cudaGetErrorName(e));
}

void qs_clear_error() { g_err[0] = 0; }

extern "C" const char *qs_last_error(void) { return g_err; }

extern "C" const char *qs_version(void)
{
    return "qpanda_b200 0.1 (sm_100a; complex64/complex128 state vector)";
}

// ------------------------------------------------------------------ state
int qs_check_state(const qs_state *s)
{
    if (!s || !s->amp) return qs_fail(QS_ERR_ARG, "null or destroyed state handle");
    return QS_OK;
}

int qs_dev_alloc(qs_state *s, size_t bytes, void **p)
{
    *p = nullptr;
    if (s->stream_alloc) QS_CUDA_TRY(cudaMallocAsync(p, bytes, s->stream));
    else QS_CUDA_TRY(cudaMalloc(p, bytes));
    return QS_OK;
}

void qs_dev_free(qs_state *s, void *p)
{
    if (!p) return;
    if (s->stream_alloc) cudaFreeAsync(p, s->stream);
    else cudaFree(p);
}

int qs_ensure_scratch(qs_state *s, size_t bytes)
{
    if (bytes <= s->scratch_bytes) return QS_OK;
    size_t nb = 1 << 20;
    while (nb < bytes) nb <<= 1;
    void *p = nullptr;
    // The stream may still be using the old buffer (stream-ordered frees wait
    // for it by construction).
    if (!s->stream_alloc) QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    int r = qs_dev_alloc(s, nb, &p);
    if (r) return r;
    qs_dev_free(s, s->scratch);
    s->scratch = p;
    s->scratch_bytes = nb;
    return QS_OK;
}

static int create_impl(int n_qubits, int dtype, void *stream, bool stream_alloc, qs_state **out);

extern "C" int qs_create(int n_qubits, int dtype, void *stream, qs_state **out)
{
    return create_impl(n_qubits, dtype, stream, false, out);
}

extern "C" int qs_create_async(int n_qubits, int dtype, void *stream, qs_state **out)
{
    return create_impl(n_qubits, dtype, stream, true, out);
}

static int create_impl(int n_qubits, int dtype, void *stream, bool stream_alloc, qs_state **out)
{
    if (!out) return qs_fail(QS_ERR_ARG, "qs_create: null output");
    *out = nullptr;
    if (n_qubits < 1 || n_qubits > QS_MAX_QUBITS)
        return qs_fail(QS_ERR_ARG, "qs_create: qubit count %d outside [1, %d]", n_qubits, QS_MAX_QUBITS);
    if (dtype != QS_C64 && dtype != QS_C128) return qs_fail(QS_ERR_ARG, "qs_create: bad dtype %d", dtype);
    qs_state *s = new qs_state();
    s->n = n_qubits;
    s->dtype = dtype;
    s->N = 1ull << n_qubits;
    s->stream = static_cast<cudaStream_t>(stream);
    s->stream_alloc = stream_alloc;
    const size_t ab = s->amp_bytes() < 16 ? 16 : s->amp_bytes();
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess) e = stream_alloc ? cudaMallocAsync(&s->amp, ab, s->stream) : cudaMalloc(&s->amp, ab);
    if (e == cudaSuccess) {
        if (stream_alloc) s->pinned = malloc(4096);
        else e = cudaMallocHost(&s->pinned, 4096);
    }
    if (e != cudaSuccess) {
        int r = qs_cuda_fail(e, "qs_create");
        if (s->amp) qs_dev_free(s, s->amp);
        if (stream_alloc) free(s->pinned);
        delete s;
        cudaGetLastError();
        return r;
    }
    int r = qs_ensure_scratch(s, 1 << 20);
    if (!r) r = launch_fill_zero_state(s);
    if (r) { qs_destroy(s); return r; }
    *out = s;
    return QS_OK;
}

extern "C" int qs_destroy(qs_state *s)
{
    if (!s) return QS_OK;
    if (s->stream_alloc) {
        // stream-ordered: the frees run after the work queued on the stream
        qs_dev_free(s, s->amp);
        qs_dev_free(s, s->scratch);
        qs_dev_free(s, s->fused_norm);
        qs_dev_free(s, s->spare);
        free(s->pinned);
    } else {
        cudaStreamSynchronize(s->stream);
        if (s->amp) cudaFree(s->amp);
        if (s->scratch) cudaFree(s->scratch);
        if (s->pinned) cudaFreeHost(s->pinned);
        if (s->fused_norm) cudaFree(s->fused_norm);
        if (s->spare) cudaFree(s->spare);
    }
    s->amp = nullptr;
    delete s;
    return QS_OK;
}

extern "C" int qs_num_qubits(const qs_state *s, int *n)
{
    int r = qs_check_state(s);
    if (r) return r;
    *n = s->n;
    return QS_OK;
}

extern "C" int qs_dtype(const qs_state *s, int *dtype)
{
    int r = qs_check_state(s);
    if (r) return r;
    *dtype = s->dtype;
    return QS_OK;
}

extern "C" int qs_device_ptr(const qs_state *s, void **p)
{
    int r = qs_check_state(s);
    if (r) return r;
    *p = s->amp;
    return QS_OK;
}

extern "C" int qs_set_stream(qs_state *s, void *stream)
{
    int r = qs_check_state(s);
    if (r) return r;
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->stream = static_cast<cudaStream_t>(stream);
    return QS_OK;
}

extern "C" int qs_synchronize(qs_state *s)
{
    int r = qs_check_state(s);
    if (r) return r;
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    QS_CUDA_TRY(cudaGetLastError());
    return QS_OK;
}

extern "C" int qs_reset_zero(qs_state *s)
{
    int r = qs_check_state(s);
    if (r) return r;
    return launch_fill_zero_state(s);
}

extern "C" int qs_set_state(qs_state *s, const void *host, int host_dtype)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (!host) return qs_fail(QS_ERR_ARG, "qs_set_state: null buffer");
    if (host_dtype != QS_C64 && host_dtype != QS_C128) return qs_fail(QS_ERR_ARG, "qs_set_state: bad dtype");
    return qs_copy_in(s, host, host_dtype);
}

extern "C" int qs_get_state(qs_state *s, void *host, int host_dtype)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (!host) return qs_fail(QS_ERR_ARG, "qs_get_state: null buffer");
    if (host_dtype != QS_C64 && host_dtype != QS_C128) return qs_fail(QS_ERR_ARG, "qs_get_state: bad dtype");
    return qs_copy_out(s, host, host_dtype);
}

// ------------------------------------------------------------------ generic unitaries
static int check_q(const qs_state *s, int q, const char *who)
{
    if (q < 0 || q >= s->n) return qs_fail(QS_ERR_ARG, "%s: qubit %d out of range [0,%d)", who, q, s->n);
    return QS_OK;
}

static int check_mask(const qs_state *s, uint64_t mask, const char *who)
{
    if (s->n < 64 && (mask >> s->n)) return qs_fail(QS_ERR_ARG, "%s: control mask has qubits >= %d", who, s->n);
    return QS_OK;
}

extern "C" int qs_apply_1q(qs_state *s, int q, const double m[8], uint64_t cmask)
{
    int r = qs_check_state(s);
    if (r || (r = check_q(s, q, "qs_apply_1q")) || (r = check_mask(s, cmask, "qs_apply_1q"))) return r;
    if (cmask & (1ull << q)) return qs_fail(QS_ERR_ARG, "qs_apply_1q: target %d is also a control", q);
    return launch_pair(s, cmask | (1ull << q), cmask, 0, 1ull << q, m);
}

extern "C" int qs_apply_unitary_1q(qs_state *s, int q, const double m[8])
{
    // det = m00*m11 - m01*m10; the reference rejects |det| off 1 by > 1e-6.
    double dr = (m[0] * m[6] - m[1] * m[7]) - (m[2] * m[4] - m[3] * m[5]);
    double di = (m[0] * m[7] + m[1] * m[6]) - (m[2] * m[5] + m[3] * m[4]);
    if (fabs(hypot(dr, di) - 1) > 0.000001)
        return qs_fail(QS_ERR_NOT_UNITARY, "qs_apply_unitary_1q: |det| = %.9g", hypot(dr, di));
    return qs_apply_1q(s, q, m, 0);
}

extern "C" int qs_apply_2q(qs_state *s, int q0, int q1, const double m[32], uint64_t cmask)
{
    int r = qs_check_state(s);
    if (r || (r = check_q(s, q0, "qs_apply_2q")) || (r = check_q(s, q1, "qs_apply_2q")) ||
        (r = check_mask(s, cmask, "qs_apply_2q")))
        return r;
    if (q0 == q1) return qs_fail(QS_ERR_ARG, "qs_apply_2q: qubits coincide (%d)", q0);
    if (cmask & ((1ull << q0) | (1ull << q1))) return qs_fail(QS_ERR_ARG, "qs_apply_2q: target is also a control");
    return launch_quad(s, q0, q1, cmask, m);
}

extern "C" int qs_apply_exchange(qs_state *s, int a, int b, const double m[8], uint64_t cmask)
{
    int r = qs_check_state(s);
    if (r || (r = check_q(s, a, "qs_apply_exchange")) || (r = check_q(s, b, "qs_apply_exchange")) ||
        (r = check_mask(s, cmask, "qs_apply_exchange")))
        return r;
    if (a == b) return qs_fail(QS_ERR_ARG, "qs_apply_exchange: qubits coincide (%d)", a);
    uint64_t ab = (1ull << a) | (1ull << b);
    if (cmask & ab) return qs_fail(QS_ERR_ARG, "qs_apply_exchange: target is also a control");
    return launch_pair(s, cmask | ab, cmask, 1ull << a, 1ull << b, m);
}

extern "C" int qs_apply_phase(qs_state *s, uint64_t mask, double re, double im)
{
    int r = qs_check_state(s);
    if (r || (r = check_mask(s, mask, "qs_apply_phase"))) return r;
    return launch_phase(s, mask, re, im);
}

// ------------------------------------------------------------------ gate records
int qs_launch_prim(qs_state *s, const qs_prim &p)
{
    if (p.kind == QS_PRIM_PHASE) return launch_phase(s, p.holes, p.m[0], p.m[1]);
    return launch_pair(s, p.holes, p.cmask, p.off0, p.off1, p.m);
}

extern "C" int qs_gate_apply(qs_state *s, const qs_gate *g)
{
    int r = qs_check_state(s);
    if (r) return r;
    qs_prim p;
    if ((r = qs_lower_gate(s->n, g, &p))) return r;
    return qs_launch_prim(s, p);
}

// qs_lowstage.cu
int qs_lowstage_bits(int n);
void qs_lowstage_passes(const std::vector<qs_prim> &prims, int n, int dtype, bool stage_all,
                        std::vector<qs_low::Pass> &out);
int qs_launch_lowstage(qs_state *s, const std::vector<qs_prim> &run, uint64_t qmask);

// Gate by gate, except that runs of consecutive gates whose targets lie
// within one tile's 10 qubits go through shared memory and registers in one
// pass each (qs_lowstage.cu) when that moves fewer bytes than the gates would
// one by one: same arithmetic per amplitude, fewer passes over HBM.
extern "C" int qs_gates_apply(qs_state *s, const qs_gate *g, size_t count)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (count && !g) return qs_fail(QS_ERR_ARG, "qs_gates_apply: null gate list");
    std::vector<qs_prim> prims(count);
    for (size_t i = 0; i < count; ++i)
        if ((r = qs_lower_gate(s->n, &g[i], &prims[i]))) return r;
    std::vector<qs_low::Pass> passes;
    qs_lowstage_passes(prims, s->n, s->dtype, false, passes);
    std::vector<qs_prim> run;
    for (const qs_low::Pass &ps : passes) {
        if (ps.qmask) {
            run.assign(prims.begin() + ps.first, prims.begin() + ps.first + ps.count);
            r = qs_launch_lowstage(s, run, ps.qmask);
        } else {
            r = qs_launch_prim(s, prims[ps.first]);
        }
        if (r) return r;
    }
    return QS_OK;
}

extern "C" int qs_pmeasure(qs_state *s, const int *qubits, int m, uint64_t *idx_out, double *p_out, int *count)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (m < 0 || m > 30) return qs_fail(QS_ERR_ARG, "qs_pmeasure: %d qubits (at most 30)", m);
    std::vector<double> probs(1ull << m);
    if ((r = qs_probs(s, qubits, m, probs.data()))) return r;
    // Descending probability; ties keep ascending index (the reference's
    // std::sort leaves their order unspecified).
    std::vector<uint64_t> order(probs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    size_t keep = order.size() < 10 ? order.size() : 10;
    std::partial_sort(order.begin(), order.begin() + keep, order.end(), [&](uint64_t a, uint64_t b) {
        return probs[a] > probs[b] || (probs[a] == probs[b] && a < b);
    });
    for (size_t i = 0; i < keep; ++i) { idx_out[i] = order[i]; p_out[i] = probs[order[i]]; }
    *count = (int)keep;
    return QS_OK;
}
