// GPUEmulatorShim.cpp - libGPUEmulator.so over the B200 C ABI (see
// include/qpanda_b200_gpuemu.h for the contract).  Every entry point takes the
// reference's QState record, draws the generator like the CPU backend, and
// forwards one gate record to qs_gate_apply (or qs_measure, qs_pmeasure,
// qs_get_state) on a complex128 state.
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

#include "qpanda_b200.h"
#include "qpanda_b200_gpuemu.h"

namespace {

double (*g_rng)(void) = nullptr;
int g_seed = 0;

// Park-Miller minimal standard generator (multiplier 16807, modulus 2^31 - 1,
// Schrage's decomposition), the generator the reference seeds from the clock
// (QPandaSDK/QuantumInstructionHandle/QuantumGates.cpp:46-85); never returns 0.
// Unless qs_gpuemu_seed set one, the seed is the time of the first draw.
double own_rng()
{
    if (!g_seed) g_seed = (int)(time(nullptr) % 2147483646) + 1;
    const int a = 16807, m = 2147483647, q = 127773, r = 2836;
    int x = a * (g_seed % q) - r * (g_seed / q);
    if (x < 0) x += m;
    g_seed = x;
    return (double)x / m;
}

double draw() { return g_rng ? g_rng() : own_rng(); }

qs_state *handle(const GATEGPU::QState &s) { return reinterpret_cast<qs_state *>(s.real); }

// One gate on the subspace where every control is 1 (targets removed from the
// control list, as the controlled overloads receive them appended).
bool gate(GATEGPU::QState &s, int op, std::initializer_list<size_t> q, double theta, int dagger,
          const std::vector<size_t> &ctrl, double error_rate)
{
    qs_state *h = handle(s);
    if (!h) return false;
    if (!(draw() > error_rate)) return true;
    qs_gate g;
    memset(&g, 0, sizeof(g));
    g.op = op;
    g.dagger = dagger;
    g.theta = theta;
    int nq = 0;
    for (size_t x : q) g.q[nq++] = (int32_t)x;
    for (size_t c : ctrl) {
        bool skip = false;
        for (int j = 0; j < nq; ++j) skip |= (size_t)g.q[j] == c;
        for (int j = 0; j < g.nctrl; ++j) skip |= (size_t)g.ctrl[j] == c;
        if (skip) continue;
        if (g.nctrl == QS_MAX_CTRL) return false;
        g.ctrl[g.nctrl++] = (int32_t)c;
    }
    return qs_gate_apply(h, &g) == QS_OK;
}

bool controlled(GATEGPU::QState &s, int op, qs_emu_qnum &qnum, double theta, int dagger, double error_rate)
{
    if (qnum.empty()) return false;
    const size_t target = qnum.back();
    return gate(s, op, {target}, theta, dagger, qnum, error_rate);
}

const std::vector<size_t> kNone;

int log2_exact(size_t block)
{
    if (!block || (block & (block - 1))) return -1;
    int q = 0;
    while (!((block >> q) & 1)) ++q;
    return q;
}

bool pmeasure_list(GATEGPU::QState &s, qs_emu_probs &vprob, const std::vector<int> &qs)
{
    qs_state *h = handle(s);
    if (!h) return false;
    uint64_t idx[10];
    double p[10];
    int cnt = 0;
    if (qs_pmeasure(h, qs.data(), (int)qs.size(), idx, p, &cnt) != QS_OK) return false;
    vprob.clear();
    for (int i = 0; i < cnt; ++i) vprob.push_back(std::make_pair((size_t)idx[i], p[i]));
    return true;
}

}  // namespace

extern "C" {

void qs_gpuemu_set_rng(double (*fn)(void)) { g_rng = fn; }
void qs_gpuemu_seed(int seed) { g_seed = seed ? seed : 1; }

bool qs_emu_initstate(GATEGPU::QState &psi, GATEGPU::QState &psigpu, int qnum)
{
    if (qnum < 1 || qnum > 40) return false;
    qs_state *h = nullptr;
    if (qs_create(qnum, QS_C128, nullptr, &h) != QS_OK) return false;
    const size_t dim = (size_t)1 << qnum;
    psi.real = static_cast<double *>(calloc(dim, sizeof(double)));
    psi.imag = static_cast<double *>(calloc(dim, sizeof(double)));
    if (!psi.real || !psi.imag) {
        free(psi.real);
        free(psi.imag);
        psi.real = psi.imag = nullptr;
        qs_destroy(h);
        return false;
    }
    psi.real[0] = 1.0;
    psi.qnum = qnum;
    psigpu.real = reinterpret_cast<double *>(h);
    psigpu.imag = nullptr;
    psigpu.qnum = qnum;
    return true;
}

bool destroyState(GATEGPU::QState &psi, GATEGPU::QState &psigpu, size_t)
{
    if (!handle(psigpu)) return false;
    qs_destroy(handle(psigpu));
    free(psi.real);
    free(psi.imag);
    psi.real = psi.imag = psigpu.real = psigpu.imag = nullptr;
    return true;
}

bool clearState(GATEGPU::QState &, GATEGPU::QState &psigpu, size_t)
{
    return handle(psigpu) && qs_reset_zero(handle(psigpu)) == QS_OK;
}

bool Hadamard(GATEGPU::QState &s, size_t qn, double e) { return gate(s, QS_OP_H, {qn}, 0, 0, kNone, e); }
bool Hadamardnew(GATEGPU::QState &s, size_t qn, double e) { return gate(s, QS_OP_H, {qn}, 0, 0, kNone, e); }
bool Hadamarddagger(GATEGPU::QState &s, size_t qn, double e) { return gate(s, QS_OP_H, {qn}, 0, 1, kNone, e); }
bool RX(GATEGPU::QState &s, size_t qn, double t, double e) { return gate(s, QS_OP_RX, {qn}, t, 0, kNone, e); }
bool RXdagger(GATEGPU::QState &s, size_t qn, double t, double e) { return gate(s, QS_OP_RX, {qn}, t, 1, kNone, e); }
bool RY(GATEGPU::QState &s, size_t qn, double t, double e) { return gate(s, QS_OP_RY, {qn}, t, 0, kNone, e); }
bool RYdagger(GATEGPU::QState &s, size_t qn, double t, double e) { return gate(s, QS_OP_RY, {qn}, t, 1, kNone, e); }
bool RZ(GATEGPU::QState &s, size_t qn, double t, double e) { return gate(s, QS_OP_RZ, {qn}, t, 0, kNone, e); }
bool RZdagger(GATEGPU::QState &s, size_t qn, double t, double e) { return gate(s, QS_OP_RZ, {qn}, t, 1, kNone, e); }
bool NOT(GATEGPU::QState &s, size_t qn, double e) { return gate(s, QS_OP_X, {qn}, 0, 0, kNone, e); }
bool NOTdagger(GATEGPU::QState &s, size_t qn, double e) { return gate(s, QS_OP_X, {qn}, 0, 1, kNone, e); }
bool CNOT(GATEGPU::QState &s, size_t c, size_t t, double e) { return gate(s, QS_OP_CNOT, {c, t}, 0, 0, kNone, e); }
bool CNOTdagger(GATEGPU::QState &s, size_t c, size_t t, double e)
{
    return gate(s, QS_OP_CNOT, {c, t}, 0, 1, kNone, e);
}
bool CR(GATEGPU::QState &s, size_t a, size_t b, double t, double e) { return gate(s, QS_OP_CR, {a, b}, t, 0, kNone, e); }
bool CRdagger(GATEGPU::QState &s, size_t a, size_t b, double t, double e)
{
    return gate(s, QS_OP_CR, {a, b}, t, 1, kNone, e);
}
bool pCRdagger(GATEGPU::QState &s, size_t a, size_t b, double t, double e) { return CRdagger(s, a, b, t, e); }
bool iSWAP(GATEGPU::QState &s, size_t a, size_t b, double e) { return gate(s, QS_OP_ISWAP, {a, b}, 0, 0, kNone, e); }
bool iSWAPdagger(GATEGPU::QState &s, size_t a, size_t b, double e)
{
    return gate(s, QS_OP_ISWAP, {a, b}, 0, 1, kNone, e);
}
bool sqiSWAP(GATEGPU::QState &s, size_t a, size_t b, double e)
{
    return gate(s, QS_OP_SQISWAP, {a, b}, 0, 0, kNone, e);
}
bool sqiSWAPdagger(GATEGPU::QState &s, size_t a, size_t b, double e)
{
    return gate(s, QS_OP_SQISWAP, {a, b}, 0, 1, kNone, e);
}

int qubitmeasure(GATEGPU::QState &s, size_t block)
{
    qs_state *h = handle(s);
    const int q = log2_exact(block);
    if (!h || q < 0) return -1;
    const double u = draw();
    int out = 0;
    if (qs_measure(h, q, u, &out) != QS_OK) return -1;
    return out;
}

bool controlHadamard(GATEGPU::QState &s, qs_emu_qnum &q, double e) { return controlled(s, QS_OP_H, q, 0, 0, e); }
bool controlHadamarddagger(GATEGPU::QState &s, qs_emu_qnum &q, double e) { return controlled(s, QS_OP_H, q, 0, 1, e); }
bool controlRX(GATEGPU::QState &s, qs_emu_qnum &q, double t, double e) { return controlled(s, QS_OP_RX, q, t, 0, e); }
bool controlRXdagger(GATEGPU::QState &s, qs_emu_qnum &q, double t, double e)
{
    return controlled(s, QS_OP_RX, q, t, 1, e);
}
bool controlRY(GATEGPU::QState &s, qs_emu_qnum &q, double t, double e) { return controlled(s, QS_OP_RY, q, t, 0, e); }
bool controlRYdagger(GATEGPU::QState &s, qs_emu_qnum &q, double t, double e)
{
    return controlled(s, QS_OP_RY, q, t, 1, e);
}
bool controlRZ(GATEGPU::QState &s, qs_emu_qnum &q, double t, double e) { return controlled(s, QS_OP_RZ, q, t, 0, e); }
bool controlRZdagger(GATEGPU::QState &s, qs_emu_qnum &q, double t, double e)
{
    return controlled(s, QS_OP_RZ, q, t, 1, e);
}

bool toffoli(GATEGPU::QState &s, size_t c0, size_t c1, size_t t, double e)
{
    return gate(s, QS_OP_TOFFOLI, {c0, c1, t}, 0, 0, kNone, e);
}
bool toffolidagger(GATEGPU::QState &s, size_t c0, size_t c1, size_t t, double e)
{
    return gate(s, QS_OP_TOFFOLI, {c0, c1, t}, 0, 1, kNone, e);
}

// CPUQuantumGates::Reset: measure, then flip a 1 back to 0 (the flip is a gate
// and draws like one).
bool qbReset(GATEGPU::QState &s, size_t qn, double)
{
    const int o = qubitmeasure(s, (size_t)1 << qn);
    if (o < 0) return false;
    return o ? NOT(s, qn, 0) : true;
}

bool pMeasure(GATEGPU::QState &s, qs_emu_probs &vprob, size_t *block, size_t m)
{
    if (!block && m) return false;
    std::vector<int> qs;
    for (size_t j = 0; j < m; ++j) {
        const int q = log2_exact(block[j]);
        if (q < 0) return false;
        qs.push_back(q);
    }
    return pmeasure_list(s, vprob, qs);
}

bool pMeasurenew(GATEGPU::QState &s, qs_emu_probs &vprob, qs_emu_qnum &qnum)
{
    std::vector<int> qs(qnum.begin(), qnum.end());
    return pmeasure_list(s, vprob, qs);
}

bool getState(GATEGPU::QState &psi, GATEGPU::QState &psigpu, int qnum)
{
    qs_state *h = handle(psigpu);
    if (!h || !psi.real || !psi.imag || qnum != psigpu.qnum) return false;
    const size_t dim = (size_t)1 << qnum;
    std::vector<double> v(2 * dim);
    if (qs_get_state(h, v.data(), QS_C128) != QS_OK) return false;
    for (size_t i = 0; i < dim; ++i) {
        psi.real[i] = v[2 * i];
        psi.imag[i] = v[2 * i + 1];
    }
    return true;
}

}  // extern "C"
