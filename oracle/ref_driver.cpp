// ref_driver.cpp - extern "C" driver around the reference CPU backend
// (QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp), compiled from the
// reference's own sources into oracle/_ref/.  TEST INFRASTRUCTURE ONLY: the
// tests use it to pin the C restatement (oracle/qs_oracle.c) and to generate
// the golden fixtures; bench.py --impl reference times it on the host cores.
//
// Gate records are dispatched the way Instruction.cpp does it: a non-empty
// control list gets the target appended and goes to the controlled overload
// (Instruction.cpp:52-58, 132-150, 359-371), CNOT with controls goes through
// NOT (CPUQuantumGates.cpp:750-757), Toffoli with controls pushes both controls
// and the target (Instruction.cpp:464-478).  iSWAP without controls calls the
// four-argument method directly (the dispatcher's branches for it are
// swapped, Instruction.cpp:558-577, which would make it a no-op).
#include <algorithm>
#include <cstring>
#include <vector>

#include "CPUQuantumGates.h"
#include "../include/qpanda_b200.h"

extern "C" void ref_rng_set_next(double u);

struct RefState {
    CPUQuantumGates g;
    QuantumGateParam param;
};

extern "C" {

void *ref_create(int n)
{
    RefState *s = new RefState();
    s->param.setQBitNum(n);
    if (s->g.initState(&s->param) != qErrorNone) { delete s; return nullptr; }
    return s;
}

void ref_destroy(void *h) { delete static_cast<RefState *>(h); }

double *ref_data(void *h)
{
    return reinterpret_cast<double *>(static_cast<RefState *>(h)->g.mvQuantumStat.data());
}

size_t ref_size(void *h) { return static_cast<RefState *>(h)->g.getQStateSize(); }

void ref_end_gate(void *h)
{
    RefState *s = static_cast<RefState *>(h);
    s->g.endGate(&s->param, &s->g);
}

// Returns 0 on success, 1 when the reference has no implementation for the
// request (controlled iSWAP / sqiSWAP / CR / controlSwap, SWAP), -1 on error.
int ref_gate(void *h, const qs_gate *gt)
{
    RefState *s = static_cast<RefState *>(h);
    CPUQuantumGates &g = s->g;
    size_t n = (size_t)s->param.mQuantumBitNumber;
    Qnum ctl;
    for (int j = 0; j < gt->nctrl; ++j) ctl.push_back((size_t)gt->ctrl[j]);
    bool c = !ctl.empty();
    QError r = qErrorNone;
    size_t q0 = (size_t)gt->q[0], q1 = (size_t)gt->q[1], q2 = (size_t)gt->q[2];
    switch (gt->op) {
    case QS_OP_H:
        if (c) { ctl.push_back(q0); r = g.Hadamard(q0, 0, ctl, n); }
        else r = g.Hadamard(q0, 0);
        break;
    case QS_OP_X:
        if (c) { ctl.push_back(q0); r = g.NOT(q0, 0, ctl, (int)n); }
        else r = g.NOT(q0, 0);
        break;
    case QS_OP_RX:
        if (c) { ctl.push_back(q0); r = g.RX(q0, gt->theta, 0, ctl, n, gt->dagger); }
        else r = g.RX(q0, gt->theta, 0, gt->dagger);
        break;
    case QS_OP_RY:
        if (c) { ctl.push_back(q0); r = g.RY(q0, gt->theta, 0, ctl, n, gt->dagger); }
        else r = g.RY(q0, gt->theta, 0, gt->dagger);
        break;
    case QS_OP_RZ:
        if (c) { ctl.push_back(q0); r = g.RZ(q0, gt->theta, 0, ctl, n, gt->dagger); }
        else r = g.RZ(q0, gt->theta, 0, gt->dagger);
        break;
    case QS_OP_CNOT:
        if (c) { ctl.push_back(q0); ctl.push_back(q1); r = g.CNOT(q0, q1, 0, ctl, (int)n); }
        else r = g.CNOT(q0, q1, 0);
        break;
    case QS_OP_CR:
        if (c) return 1;
        r = g.CR(q0, q1, gt->theta, 0, gt->dagger);
        break;
    case QS_OP_ISWAP:
        if (c) return 1;
        r = g.iSWAP(q0, q1, 0, gt->dagger);
        break;
    case QS_OP_SQISWAP:
        if (c) return 1;
        r = g.sqiSWAP(q0, q1, 0, gt->dagger);
        break;
    case QS_OP_TOFFOLI:
        if (c) { ctl.push_back(q0); ctl.push_back(q1); ctl.push_back(q2); r = g.NOT(q2, 0, ctl, (int)n); }
        else r = g.toffoli(q0, q1, q2, 0, (int)n);
        break;
    case QS_OP_CSWAP:
        if (c) return 1;
        r = g.controlSwap(q0, q1, q2, 0);
        break;
    case QS_OP_SWAP:
        // QRunes has no SWAP; a program writes it as three CNOTs.
        if (c) return 1;
        g.CNOT(q0, q1, 0); g.CNOT(q1, q0, 0); r = g.CNOT(q0, q1, 0);
        break;
    default:
        return -1;
    }
    return r == qErrorNone ? 0 : -1;
}

int ref_gates(void *h, const qs_gate *g, size_t count)
{
    for (size_t i = 0; i < count; ++i) {
        int r = ref_gate(h, &g[i]);
        if (r) return r;
    }
    return 0;
}

// qubitMeasure with the next uniform forced to u.
int ref_measure(void *h, int q, double u)
{
    ref_rng_set_next(u);
    return static_cast<RefState *>(h)->g.qubitMeasure((size_t)q);
}

// pMeasure as the reference returns it (sorted, cut to 10): returns the count.
int ref_pmeasure(void *h, const int *qubits, int m, size_t *idx, double *p)
{
    Qnum qn;
    for (int j = 0; j < m; ++j) qn.push_back((size_t)qubits[j]);
    std::vector<std::pair<size_t, double>> res;
    if (static_cast<RefState *>(h)->g.pMeasure(qn, res) != qErrorNone) return -1;
    for (size_t i = 0; i < res.size(); ++i) { idx[i] = res[i].first; p[i] = res[i].second; }
    return (int)res.size();
}

// Shots by re-measuring a fresh copy of the state per shot (QPandaAPI.cpp:173-182).
int ref_sample(void *h, const int *qubits, int m, const double *u, size_t shots, uint64_t *out)
{
    RefState *s = static_cast<RefState *>(h);
    QStat saved = s->g.mvQuantumStat;
    for (size_t sh = 0; sh < shots; ++sh) {
        s->g.mvQuantumStat = saved;
        uint64_t bits = 0;
        for (int k = 0; k < m; ++k) {
            int o = ref_measure(h, qubits[k], u[sh * (size_t)m + k]);
            if (o < 0) return -1;
            bits |= (uint64_t)o << k;
        }
        out[sh] = bits;
    }
    s->g.mvQuantumStat = saved;
    return 0;
}

// The reference's getQState text (CPUQuantumGates.cpp:64-82) into buf (cap
// bytes, NUL-terminated).  Returns its length, or -(length + 1) when buf is
// too small, or -1 on failure.
long ref_qstate_text(void *h, char *buf, size_t cap)
{
    RefState *s = static_cast<RefState *>(h);
    std::string t;
    if (!s->g.getQState(t, &s->param)) return -1;
    if (t.size() + 1 > cap) return -(long)(t.size() + 1);
    memcpy(buf, t.c_str(), t.size() + 1);
    return (long)t.size();
}

}  // extern "C"
