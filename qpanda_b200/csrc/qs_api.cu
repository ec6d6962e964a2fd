// qs_api.cu - C ABI: state lifetime, errors, and the lowering of reference
// gate records (QPandaSDK/QuantumInstructionHandle/QuantumGates.h methods)
// onto the generic kernels of qs_gates.cu.
//
// The matrices below restate the conventions of CPUQuantumGates.cpp:
//   H       (alpha+beta)*SQ2, (alpha-beta)*SQ2, SQ2 = 0.707106781186548  (:92-117, :36)
//   RX      [[c, -is], [-is, c]], dagger +is, c = cos(t/2), s = sin(t/2) (:271-309)
//   RY      [[c, -s], [s, c]], dagger transposed                        (:473-511)
//   RZ      diag(c - is, c + is), dagger conjugated                     (:524-570)
//   CR      |11> times (cos t + i sin t), dagger conjugated             (:773-825)
//   iSWAP   |01> <-> |10> with factor +i, dagger -i                     (:838-899)
//   sqiSWAP [[SQ2, i SQ2], [i SQ2, SQ2]] on {|01>,|10>}, dagger -i      (:978-1039)
//   NOT/CNOT/Toffoli: X on the target where every control is 1          (:668-737, :1277-1435)
//   controlSwap(c, a, b): exchange |a=1,b=0> and |a=0,b=1> where c = 1  (:934-965)
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "qs_common.cuh"

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

int qs_ensure_scratch(qs_state *s, size_t bytes)
{
    if (bytes <= s->scratch_bytes) return QS_OK;
    size_t nb = 1 << 20;
    while (nb < bytes) nb <<= 1;
    void *p = nullptr;
    // The stream may still be using the old buffer.
    QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
    QS_CUDA_TRY(cudaMalloc(&p, nb));
    if (s->scratch) cudaFree(s->scratch);
    s->scratch = p;
    s->scratch_bytes = nb;
    return QS_OK;
}

extern "C" int qs_create(int n_qubits, int dtype, void *stream, qs_state **out)
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
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess) e = cudaMalloc(&s->amp, s->amp_bytes() < 16 ? 16 : s->amp_bytes());
    if (e == cudaSuccess) e = cudaMallocHost(&s->pinned, 4096);
    if (e != cudaSuccess) {
        int r = qs_cuda_fail(e, "qs_create");
        if (s->amp) cudaFree(s->amp);
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
    if (s->stream || s->amp) cudaStreamSynchronize(s->stream);
    if (s->amp) cudaFree(s->amp);
    if (s->scratch) cudaFree(s->scratch);
    if (s->pinned) cudaFreeHost(s->pinned);
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
static const double kSQ2 = 0.707106781186548;     // CPUQuantumGates.cpp:36

static int gate_ctrl_mask(const qs_state *s, const qs_gate *g, uint64_t *mask)
{
    *mask = 0;
    if (g->nctrl < 0 || g->nctrl > QS_MAX_CTRL) return qs_fail(QS_ERR_ARG, "gate: bad control count %d", g->nctrl);
    for (int j = 0; j < g->nctrl; ++j) {
        int c = g->ctrl[j];
        if (c < 0 || c >= s->n) return qs_fail(QS_ERR_ARG, "gate: control %d out of range", c);
        if (*mask & (1ull << c)) return qs_fail(QS_ERR_ARG, "gate: control %d listed twice", c);
        *mask |= 1ull << c;
    }
    return QS_OK;
}

static int add_ctrl(const qs_state *s, uint64_t *mask, int q)
{
    if (q < 0 || q >= s->n) return qs_fail(QS_ERR_ARG, "gate: qubit %d out of range", q);
    if (*mask & (1ull << q)) return qs_fail(QS_ERR_ARG, "gate: qubit %d used twice", q);
    *mask |= 1ull << q;
    return QS_OK;
}

// Fill the 2x2 matrix of a 1-qubit reference gate.
int qs_gate_matrix_1q(const qs_gate *g, double m[8])
{
    const double t = g->theta;
    memset(m, 0, 8 * sizeof(double));
    switch (g->op) {
    case QS_OP_H:
        m[0] = kSQ2; m[2] = kSQ2; m[4] = kSQ2; m[6] = -kSQ2;
        return 1;
    case QS_OP_X:
    case QS_OP_CNOT:
    case QS_OP_TOFFOLI:
        m[2] = 1; m[4] = 1;
        return 1;
    case QS_OP_RX: {
        double c = cos(t / 2), sn = sin(t / 2), sg = g->dagger ? 1.0 : -1.0;
        m[0] = c; m[3] = sg * sn; m[5] = sg * sn; m[6] = c;
        return 1;
    }
    case QS_OP_RY: {
        double c = cos(t / 2), sn = sin(t / 2);
        if (g->dagger) { m[0] = c; m[2] = sn; m[4] = -sn; m[6] = c; }
        else { m[0] = c; m[2] = -sn; m[4] = sn; m[6] = c; }
        return 1;
    }
    case QS_OP_RZ: {
        double c = cos(t / 2), sn = sin(t / 2), sg = g->dagger ? -1.0 : 1.0;
        m[0] = c; m[1] = -sg * sn; m[6] = c; m[7] = sg * sn;
        return 1;
    }
    default:
        return 0;
    }
}

extern "C" int qs_gate_apply(qs_state *s, const qs_gate *g)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (!g) return qs_fail(QS_ERR_ARG, "qs_gate_apply: null gate");
    uint64_t cm;
    if ((r = gate_ctrl_mask(s, g, &cm))) return r;
    double m[8];
    switch (g->op) {
    case QS_OP_H: case QS_OP_X: case QS_OP_RX: case QS_OP_RY: case QS_OP_RZ: {
        int t = g->q[0];
        if ((r = check_q(s, t, "gate"))) return r;
        if (cm & (1ull << t)) return qs_fail(QS_ERR_ARG, "gate: target %d is also a control", t);
        qs_gate_matrix_1q(g, m);
        return launch_pair(s, cm | (1ull << t), cm, 0, 1ull << t, m);
    }
    case QS_OP_CNOT: case QS_OP_TOFFOLI: {
        int nc = g->op == QS_OP_CNOT ? 1 : 2, t = g->q[nc];
        for (int j = 0; j < nc; ++j)
            if ((r = add_ctrl(s, &cm, g->q[j]))) return r;
        if ((r = check_q(s, t, "gate"))) return r;
        if (cm & (1ull << t)) return qs_fail(QS_ERR_ARG, "gate: target %d is also a control", t);
        qs_gate_matrix_1q(g, m);
        return launch_pair(s, cm | (1ull << t), cm, 0, 1ull << t, m);
    }
    case QS_OP_CR: {
        uint64_t mask = cm;
        if ((r = add_ctrl(s, &mask, g->q[0])) || (r = add_ctrl(s, &mask, g->q[1]))) return r;
        double sn = g->dagger ? -sin(g->theta) : sin(g->theta);
        return launch_phase(s, mask, cos(g->theta), sn);
    }
    case QS_OP_ISWAP: case QS_OP_SQISWAP: case QS_OP_SWAP: case QS_OP_CSWAP: {
        int a = g->q[0], b = g->q[1];
        if (g->op == QS_OP_CSWAP) {
            if ((r = add_ctrl(s, &cm, g->q[0]))) return r;
            a = g->q[1]; b = g->q[2];
        }
        uint64_t ab = 0;
        if ((r = add_ctrl(s, &ab, a)) || (r = add_ctrl(s, &ab, b))) return r;
        if (cm & ab) return qs_fail(QS_ERR_ARG, "gate: exchanged qubit is also a control");
        memset(m, 0, sizeof(m));
        double sg = g->dagger ? -1.0 : 1.0;
        if (g->op == QS_OP_ISWAP) { m[3] = sg; m[5] = sg; }
        else if (g->op == QS_OP_SQISWAP) { m[0] = kSQ2; m[3] = sg * kSQ2; m[5] = sg * kSQ2; m[6] = kSQ2; }
        else { m[2] = 1; m[4] = 1; }
        return launch_pair(s, cm | ab, cm, 1ull << a, 1ull << b, m);
    }
    default:
        return qs_fail(QS_ERR_ARG, "qs_gate_apply: unknown op %d", g->op);
    }
}

extern "C" int qs_gates_apply(qs_state *s, const qs_gate *g, size_t count)
{
    for (size_t i = 0; i < count; ++i) {
        int r = qs_gate_apply(s, &g[i]);
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
