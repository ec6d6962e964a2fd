// qs_lower.cpp - reference gate records -> primitive operations.
//
// The matrices restate the conventions of
// QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp:
//   H       (alpha+beta)*SQ2, (alpha-beta)*SQ2, SQ2 = 0.707106781186548  (:92-117, :36)
//   RX      [[c, -is], [-is, c]], dagger +is, c = cos(t/2), s = sin(t/2) (:271-309)
//   RY      [[c, -s], [s, c]], dagger transposed                        (:473-511)
//   RZ      diag(c - is, c + is), dagger conjugated                     (:524-570)
//   CR      |11> times (cos t + i sin t), dagger conjugated             (:773-825)
//   iSWAP   |01> <-> |10> with factor +i, dagger -i                     (:838-899)
//   sqiSWAP [[SQ2, i SQ2], [i SQ2, SQ2]] on {|01>,|10>}, dagger -i      (:978-1039)
//   NOT/CNOT/Toffoli: X on the target where every control is 1          (:668-737, :1277-1435)
//   controlSwap(c, a, b): exchange |a=1,b=0> and |a=0,b=1> where c = 1  (:934-965)
#include <cmath>
#include <cstring>

#include "qs_prim.h"

static const double kSQ2 = 0.707106781186548;

static int add_bit(int n, uint64_t *mask, int q)
{
    if (q < 0 || q >= n) return qs_fail(QS_ERR_ARG, "gate: qubit %d out of range [0,%d)", q, n);
    if (*mask & (1ull << q)) return qs_fail(QS_ERR_ARG, "gate: qubit %d used twice", q);
    *mask |= 1ull << q;
    return QS_OK;
}

uint64_t qs_gate_qubits(const qs_gate *g)
{
    uint64_t m = 0;
    int nt = 2;
    if (g->op >= QS_OP_H && g->op <= QS_OP_RZ) nt = 1;
    else if (g->op == QS_OP_TOFFOLI || g->op == QS_OP_CSWAP) nt = 3;
    for (int j = 0; j < nt; ++j) m |= 1ull << g->q[j];
    for (int j = 0; j < g->nctrl && j < QS_MAX_CTRL; ++j) m |= 1ull << g->ctrl[j];
    return m;
}

static void matrix_1q(const qs_gate *g, double m[8])
{
    const double t = g->theta;
    memset(m, 0, 8 * sizeof(double));
    switch (g->op) {
    case QS_OP_H:
        m[0] = kSQ2; m[2] = kSQ2; m[4] = kSQ2; m[6] = -kSQ2;
        break;
    case QS_OP_RX: {
        double c = cos(t / 2), sn = sin(t / 2), sg = g->dagger ? 1.0 : -1.0;
        m[0] = c; m[3] = sg * sn; m[5] = sg * sn; m[6] = c;
        break;
    }
    case QS_OP_RY: {
        double c = cos(t / 2), sn = sin(t / 2);
        if (g->dagger) { m[0] = c; m[2] = sn; m[4] = -sn; m[6] = c; }
        else { m[0] = c; m[2] = -sn; m[4] = sn; m[6] = c; }
        break;
    }
    case QS_OP_RZ: {
        double c = cos(t / 2), sn = sin(t / 2), sg = g->dagger ? -1.0 : 1.0;
        m[0] = c; m[1] = -sg * sn; m[6] = c; m[7] = sg * sn;
        break;
    }
    default:    // X and the X-type controlled gates
        m[2] = 1; m[4] = 1;
        break;
    }
}

int qs_lower_gate(int n, const qs_gate *g, qs_prim *p)
{
    if (!g) return qs_fail(QS_ERR_ARG, "gate: null record");
    memset(p, 0, sizeof(*p));
    if (g->nctrl < 0 || g->nctrl > QS_MAX_CTRL) return qs_fail(QS_ERR_ARG, "gate: bad control count %d", g->nctrl);
    uint64_t cm = 0;
    int r;
    for (int j = 0; j < g->nctrl; ++j)
        if ((r = add_bit(n, &cm, g->ctrl[j]))) return r;
    switch (g->op) {
    case QS_OP_H: case QS_OP_X: case QS_OP_RX: case QS_OP_RY: case QS_OP_RZ:
    case QS_OP_CNOT: case QS_OP_TOFFOLI: {
        int nc = g->op == QS_OP_CNOT ? 1 : g->op == QS_OP_TOFFOLI ? 2 : 0;
        for (int j = 0; j < nc; ++j)
            if ((r = add_bit(n, &cm, g->q[j]))) return r;
        uint64_t all = cm;
        int t = g->q[nc];
        if ((r = add_bit(n, &all, t))) return r;
        p->kind = QS_PRIM_PAIR;
        p->holes = all;
        p->cmask = cm;
        p->off0 = 0;
        p->off1 = 1ull << t;
        matrix_1q(g, p->m);
        return QS_OK;
    }
    case QS_OP_CR: {
        uint64_t mask = cm;
        if ((r = add_bit(n, &mask, g->q[0])) || (r = add_bit(n, &mask, g->q[1]))) return r;
        p->kind = QS_PRIM_PHASE;
        p->holes = mask;
        p->cmask = mask;
        p->m[0] = cos(g->theta);
        p->m[1] = g->dagger ? -sin(g->theta) : sin(g->theta);
        return QS_OK;
    }
    case QS_OP_ISWAP: case QS_OP_SQISWAP: case QS_OP_SWAP: case QS_OP_CSWAP: {
        int a = g->q[0], b = g->q[1];
        if (g->op == QS_OP_CSWAP) {
            if ((r = add_bit(n, &cm, g->q[0]))) return r;
            a = g->q[1];
            b = g->q[2];
        }
        uint64_t all = cm;
        if ((r = add_bit(n, &all, a)) || (r = add_bit(n, &all, b))) return r;
        p->kind = QS_PRIM_PAIR;
        p->holes = all;
        p->cmask = cm;
        p->off0 = 1ull << a;
        p->off1 = 1ull << b;
        double sg = g->dagger ? -1.0 : 1.0;
        if (g->op == QS_OP_ISWAP) { p->m[3] = sg; p->m[5] = sg; }
        else if (g->op == QS_OP_SQISWAP) { p->m[0] = kSQ2; p->m[3] = sg * kSQ2; p->m[5] = sg * kSQ2; p->m[6] = kSQ2; }
        else { p->m[2] = 1; p->m[4] = 1; }
        return QS_OK;
    }
    default:
        return qs_fail(QS_ERR_ARG, "gate: unknown op %d", g->op);
    }
}
