/*
 * qs_oracle.c - CPU restatement of the QPanda 2018 CPU state-vector backend.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the B200 kernels:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product path (qpanda_b200/) never links or calls it.
 *
 * It restates, function by function, the arithmetic of
 * QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp in plain C over an
 * interleaved complex128 array.  Every product keeps the reference's operand
 * order, so with IEEE double arithmetic and no FMA contraction
 * (-ffp-contract=off) the results are bit-identical to the reference compiled
 * from its own sources (oracle/Makefile, target ref); tests check that.
 *
 * Where the reference multiplies std::complex values the expansion used by
 * libstdc++ is (a+ib)(c+id) = (ac-bd) + i(ad+bc); products by a real scalar
 * scale both parts.  std::abs(complex<double>) is hypot(re, im).
 *
 * Large states: the per-amplitude loops of the gates run on OpenMP threads
 * (-fopenmp).  Every amplitude is still computed by the same expression from
 * the same inputs, so results do not depend on the thread count; sums
 * (probabilities, norms) stay serial, in the reference's order.
 *
 * Differences from the reference, on purpose:
 *  - measurements take the uniform u as an argument instead of drawing it
 *    from the global 16807 generator (QuantumGates.cpp:46-85);
 *  - pmeasure returns the full 2^m vector; the top-10 cut is done by callers;
 *  - controlled iSWAP / sqiSWAP act on the control=1 subspace (the reference
 *    returns without doing anything, CPUQuantumGates.cpp:914-922, 1054-1062);
 *  - the generic 2x2 unitary uses stride 2^q (the reference uses 2^(q-1),
 *    CPUQuantumGates.cpp:1188, which is wrong for every q).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/qpanda_b200.h"

#define SQ2 0.707106781186548          /* CPUQuantumGates.cpp:36 */
#define POW2(n) (1ull << (n))
#define PAR_MIN (1ll << 16)            /* loops shorter than this stay on one thread */

typedef struct orc_state {
    int n;
    uint64_t N;
    double *a;                           /* 2*N doubles: re0, im0, re1, im1, ... */
} orc_state;

/* ---------------------------------------------------------------- lifetime */
orc_state *orc_create(int n)
{
    orc_state *s = (orc_state *)calloc(1, sizeof(orc_state));
    if (!s) return NULL;
    s->n = n;
    s->N = POW2(n);
    s->a = (double *)calloc(2 * s->N, sizeof(double));
    if (!s->a) { free(s); return NULL; }
    s->a[0] = 1.0;                       /* initState: CPUQuantumGates.cpp:1136-1157 */
    return s;
}

void orc_destroy(orc_state *s)
{
    if (!s) return;
    free(s->a);
    free(s);
}

double *orc_data(orc_state *s) { return s->a; }
uint64_t orc_size(orc_state *s) { return s->N; }

/* endGate: CPUQuantumGates.cpp:1445-1453 */
void orc_reset(orc_state *s)
{
    memset(s->a, 0, 2 * s->N * sizeof(double));
    s->a[0] = 1.0;
}

/* ------------------------------------------------------------ index helpers */
/* Insert a zero bit at every position of the ascending list pos[0..k). */
static uint64_t insert_zeros(uint64_t x, const int *pos, int k)
{
    for (int j = 0; j < k; ++j) {
        uint64_t lo = x & (POW2(pos[j]) - 1);
        x = ((x >> pos[j]) << (pos[j] + 1)) | lo;
    }
    return x;
}

static int sort_unique(int *v, int k)
{
    for (int i = 1; i < k; ++i) {        /* insertion sort, k is small */
        int t = v[i], j = i - 1;
        while (j >= 0 && v[j] > t) { v[j + 1] = v[j]; --j; }
        v[j + 1] = t;
    }
    for (int i = 1; i < k; ++i)
        if (v[i] == v[i - 1]) return -1;
    return 0;
}

/* Enumerate the pairs (i0, i0 + 2^t) where every control bit is 1.  The
 * reference builds the same index set by bit insertion over the sorted list
 * "controls + target" and adds the control bits
 * (CPUQuantumGates.cpp:221-254, 337-381, 1331-1363). */
typedef void (*pair_fn)(double *a0, double *a1, const double *p);

static int for_each_pair(orc_state *s, int t, const int *ctrl, int nctrl,
                         pair_fn fn, const double *p)
{
    int holes[QS_MAX_CTRL + 1];
    uint64_t block = 0;
    if (nctrl > QS_MAX_CTRL || t < 0 || t >= s->n) return -1;
    for (int j = 0; j < nctrl; ++j) {
        if (ctrl[j] < 0 || ctrl[j] >= s->n) return -1;
        holes[j] = ctrl[j];
        block |= POW2(ctrl[j]);
    }
    holes[nctrl] = t;
    if (sort_unique(holes, nctrl + 1)) return -1;
    long long M = (long long)(s->N >> (nctrl + 1));
    uint64_t st = POW2(t);
#pragma omp parallel for schedule(static) if (M >= PAR_MIN)
    for (long long i = 0; i < M; ++i) {
        uint64_t idx = insert_zeros((uint64_t)i, holes, nctrl + 1) | block;
        fn(&s->a[2 * idx], &s->a[2 * (idx + st)], p);
    }
    return 0;
}

/* ------------------------------------------------------------- pair bodies */
/* Hadamard: (alpha+beta)*SQ2, (alpha-beta)*SQ2   CPUQuantumGates.cpp:108-111 */
static void body_h(double *x, double *y, const double *p)
{
    (void)p;
    double ar = x[0], ai = x[1], br = y[0], bi = y[1];
    x[0] = (ar + br) * SQ2; x[1] = (ai + bi) * SQ2;
    y[0] = (ar - br) * SQ2; y[1] = (ai - bi) * SQ2;
}

/* RX, p = {c, s, sigma}: alpha*c + (sigma*i*s)*beta  CPUQuantumGates.cpp:283-305
 * (sigma = -1 for the gate, +1 for its dagger). */
static void body_rx(double *x, double *y, const double *p)
{
    double c = p[0], s = p[1], sg = p[2];
    double ar = x[0], ai = x[1], br = y[0], bi = y[1];
    double ss = sg * s;                       /* imaginary part of compll*s */
    x[0] = ar * c + (-(ss * bi));             /* re: 0*br - ss*bi */
    x[1] = ai * c + ss * br;                  /* im: 0*bi + ss*br */
    y[0] = br * c + (-(ss * ai));
    y[1] = bi * c + ss * ar;
}

/* RY, p = {c, s, dagger}                        CPUQuantumGates.cpp:490-506 */
static void body_ry(double *x, double *y, const double *p)
{
    double c = p[0], s = p[1];
    double ar = x[0], ai = x[1], br = y[0], bi = y[1];
    if (p[2] != 0.0) {
        x[0] = ar * c + s * br; x[1] = ai * c + s * bi;
        y[0] = br * c - s * ar; y[1] = bi * c - s * ai;
    } else {
        x[0] = ar * c - s * br; x[1] = ai * c - s * bi;
        y[0] = br * c + s * ar; y[1] = bi * c + s * ai;
    }
}

/* RZ, p = {c, s1, c, s2}: x *= (c + i s2) [compl2], y *= (c + i s1) [compll]
 * (compl2 * a expands to (c*ar - s2*ai, c*ai + s2*ar))  CPUQuantumGates.cpp:533-566 */
static void body_rz(double *x, double *y, const double *p)
{
    double c = p[0], s1 = p[1], s2 = p[3];
    double ar = x[0], ai = x[1], br = y[0], bi = y[1];
    x[0] = c * ar - s2 * ai; x[1] = c * ai + s2 * ar;
    y[0] = c * br - s1 * bi; y[1] = c * bi + s1 * br;
}

/* NOT / CNOT / Toffoli: swap                      CPUQuantumGates.cpp:1296-1299 */
static void body_x(double *x, double *y, const double *p)
{
    (void)p;
    double t0 = x[0], t1 = x[1];
    x[0] = y[0]; x[1] = y[1];
    y[0] = t0; y[1] = t1;
}

/* Generic 2x2, p = {m00r, m00i, m01r, m01i, m10r, m10i, m11r, m11i}:
 * x' = x*m00 + y*m01, y' = x*m10 + y*m11        CPUQuantumGates.cpp:1198-1205 */
static void body_u(double *x, double *y, const double *p)
{
    double ar = x[0], ai = x[1], br = y[0], bi = y[1];
    double t0r = ar * p[0] - ai * p[1], t0i = ar * p[1] + ai * p[0];
    double t1r = br * p[2] - bi * p[3], t1i = br * p[3] + bi * p[2];
    double t2r = ar * p[4] - ai * p[5], t2i = ar * p[5] + ai * p[4];
    double t3r = br * p[6] - bi * p[7], t3i = br * p[7] + bi * p[6];
    x[0] = t0r + t1r; x[1] = t0i + t1i;
    y[0] = t2r + t3r; y[1] = t2i + t3i;
}

/* ------------------------------------------------------- reference methods */
int orc_h(orc_state *s, int q, const int *ctrl, int nctrl)
{
    return for_each_pair(s, q, ctrl, nctrl, body_h, NULL);
}

int orc_x(orc_state *s, int q, const int *ctrl, int nctrl)
{
    return for_each_pair(s, q, ctrl, nctrl, body_x, NULL);
}

int orc_rx(orc_state *s, int q, double theta, int dagger, const int *ctrl, int nctrl)
{
    double p[3] = {cos(theta / 2), sin(theta / 2), dagger ? 1.0 : -1.0};
    return for_each_pair(s, q, ctrl, nctrl, body_rx, p);
}

int orc_ry(orc_state *s, int q, double theta, int dagger, const int *ctrl, int nctrl)
{
    double p[3] = {cos(theta / 2), sin(theta / 2), dagger ? 1.0 : 0.0};
    return for_each_pair(s, q, ctrl, nctrl, body_ry, p);
}

int orc_rz(orc_state *s, int q, double theta, int dagger, const int *ctrl, int nctrl)
{
    double c = cos(theta / 2), sn = sin(theta / 2);
    /* compll = c + i*s (|1>), compl2 = c - i*s (|0>); swapped for the dagger */
    double p[4] = {c, dagger ? -sn : sn, c, dagger ? sn : -sn};
    return for_each_pair(s, q, ctrl, nctrl, body_rz, p);
}

int orc_u1q(orc_state *s, int q, const double m[8], const int *ctrl, int nctrl)
{
    return for_each_pair(s, q, ctrl, nctrl, body_u, m);
}

/* CNOT(c, t) = X on t where bit c is 1 (CPUQuantumGates.cpp:668-737). */
int orc_cnot(orc_state *s, int c, int t, const int *ctrl, int nctrl)
{
    int all[QS_MAX_CTRL + 1];
    if (nctrl >= QS_MAX_CTRL) return -1;
    memcpy(all, ctrl, sizeof(int) * (size_t)nctrl);
    all[nctrl] = c;
    return for_each_pair(s, t, all, nctrl + 1, body_x, NULL);
}

/* toffoli(c1, c2, t) (CPUQuantumGates.cpp:1378-1435). */
int orc_toffoli(orc_state *s, int c1, int c2, int t, const int *ctrl, int nctrl)
{
    int all[QS_MAX_CTRL + 2];
    if (nctrl + 2 > QS_MAX_CTRL + 1) return -1;
    memcpy(all, ctrl, sizeof(int) * (size_t)nctrl);
    all[nctrl] = c1;
    all[nctrl + 1] = c2;
    return for_each_pair(s, t, all, nctrl + 2, body_x, NULL);
}

/* Amplitudes whose index has every bit of {q...} U ctrl equal to the pattern
 * "bits of set1 = 1, the rest of the listed bits = 0".  Used for CR, iSWAP,
 * sqiSWAP and controlSwap, whose reference loops visit these subspaces
 * (CPUQuantumGates.cpp:807-819, 877-893, 950-962, 1017-1031). */
static int subspace_setup(orc_state *s, const int *q, int nq, const int *ctrl, int nctrl,
                          int *holes, uint64_t *cmask)
{
    int k = 0;
    *cmask = 0;
    if (nctrl > QS_MAX_CTRL) return -1;
    for (int j = 0; j < nq; ++j) {
        if (q[j] < 0 || q[j] >= s->n) return -1;
        holes[k++] = q[j];
    }
    for (int j = 0; j < nctrl; ++j) {
        if (ctrl[j] < 0 || ctrl[j] >= s->n) return -1;
        holes[k++] = ctrl[j];
        *cmask |= POW2(ctrl[j]);
    }
    return sort_unique(holes, k) ? -1 : k;
}

/* CR: amplitudes with both bits set times (cos th + i*sigma*sin th), a*compll
 * (CPUQuantumGates.cpp:787-819). */
int orc_cr(orc_state *s, int q1, int q2, double theta, int dagger, const int *ctrl, int nctrl)
{
    int holes[QS_MAX_CTRL + 3], q[2] = {q1, q2};
    uint64_t cmask;
    int k = subspace_setup(s, q, 2, ctrl, nctrl, holes, &cmask);
    if (k < 0) return -1;
    double c = cos(theta), sn = dagger ? -sin(theta) : sin(theta);
    uint64_t set = cmask | POW2(q1) | POW2(q2);
    long long M = (long long)(s->N >> k);
#pragma omp parallel for schedule(static) if (M >= PAR_MIN)
    for (long long i = 0; i < M; ++i) {
        uint64_t idx = insert_zeros((uint64_t)i, holes, k) | set;
        double ar = s->a[2 * idx], ai = s->a[2 * idx + 1];
        s->a[2 * idx] = ar * c - ai * sn;
        s->a[2 * idx + 1] = ar * sn + ai * c;
    }
    return 0;
}

/* iSWAP: k = |q_hi=0, q_lo=1>, k' = |q_hi=1, q_lo=0>:
 * a_k' <- compll*a_k, a_k <- compll*a_k', compll = (0, +-1)
 * (CPUQuantumGates.cpp:851-893). */
int orc_iswap(orc_state *s, int q1, int q2, int dagger, const int *ctrl, int nctrl)
{
    int holes[QS_MAX_CTRL + 3], q[2] = {q1, q2};
    uint64_t cmask;
    int k = subspace_setup(s, q, 2, ctrl, nctrl, holes, &cmask);
    if (k < 0) return -1;
    double sg = dagger ? -1.0 : 1.0;
    long long M = (long long)(s->N >> k);
#pragma omp parallel for schedule(static) if (M >= PAR_MIN)
    for (long long i = 0; i < M; ++i) {
        uint64_t base = insert_zeros((uint64_t)i, holes, k) | cmask;
        uint64_t i1 = base | POW2(q1), i2 = base | POW2(q2);
        double ar = s->a[2 * i1], ai = s->a[2 * i1 + 1];
        double br = s->a[2 * i2], bi = s->a[2 * i2 + 1];
        /* compll*beta = (0*br - sg*bi, 0*bi + sg*br) */
        s->a[2 * i1] = -(sg * bi); s->a[2 * i1 + 1] = sg * br;
        s->a[2 * i2] = -(sg * ai); s->a[2 * i2 + 1] = sg * ar;
    }
    return 0;
}

/* sqiSWAP: a_k <- a_k*SQ2 + (compll*a_k')*SQ2, a_k' <- (compll*a_k)*SQ2 + a_k'*SQ2
 * (CPUQuantumGates.cpp:1001-1031). */
int orc_sqiswap(orc_state *s, int q1, int q2, int dagger, const int *ctrl, int nctrl)
{
    int holes[QS_MAX_CTRL + 3], q[2] = {q1, q2};
    uint64_t cmask;
    int k = subspace_setup(s, q, 2, ctrl, nctrl, holes, &cmask);
    if (k < 0) return -1;
    double sg = dagger ? -1.0 : 1.0;
    long long M = (long long)(s->N >> k);
#pragma omp parallel for schedule(static) if (M >= PAR_MIN)
    for (long long i = 0; i < M; ++i) {
        uint64_t base = insert_zeros((uint64_t)i, holes, k) | cmask;
        uint64_t i1 = base | POW2(q1), i2 = base | POW2(q2);
        double ar = s->a[2 * i1], ai = s->a[2 * i1 + 1];
        double br = s->a[2 * i2], bi = s->a[2 * i2 + 1];
        s->a[2 * i1]     = ar * SQ2 + (-(sg * bi)) * SQ2;
        s->a[2 * i1 + 1] = ai * SQ2 + (sg * br) * SQ2;
        s->a[2 * i2]     = (-(sg * ai)) * SQ2 + br * SQ2;
        s->a[2 * i2 + 1] = (sg * ar) * SQ2 + bi * SQ2;
    }
    return 0;
}

/* controlSwap(c, a, b): where bit c = 1, swap |a=1,b=0> and |a=0,b=1>
 * (CPUQuantumGates.cpp:934-965).  SWAP is the same without c. */
int orc_cswap(orc_state *s, int c, int qa, int qb, const int *ctrl, int nctrl)
{
    int holes[QS_MAX_CTRL + 4], q[2] = {qa, qb}, all[QS_MAX_CTRL + 1];
    uint64_t cmask;
    int na = nctrl;
    memcpy(all, ctrl, sizeof(int) * (size_t)nctrl);
    if (c >= 0) all[na++] = c;
    int k = subspace_setup(s, q, 2, all, na, holes, &cmask);
    if (k < 0) return -1;
    long long M = (long long)(s->N >> k);
#pragma omp parallel for schedule(static) if (M >= PAR_MIN)
    for (long long i = 0; i < M; ++i) {
        uint64_t base = insert_zeros((uint64_t)i, holes, k) | cmask;
        uint64_t i1 = base | POW2(qa), i2 = base | POW2(qb);
        double t0 = s->a[2 * i1], t1 = s->a[2 * i1 + 1];
        s->a[2 * i1] = s->a[2 * i2]; s->a[2 * i1 + 1] = s->a[2 * i2 + 1];
        s->a[2 * i2] = t0; s->a[2 * i2 + 1] = t1;
    }
    return 0;
}

/* Apply one gate record (the dispatch of QuantumInstructionGet::transmit,
 * QuantumInstructionGet.cpp:104-124, with the Instruction.cpp argument
 * conventions). */
int orc_gate(orc_state *s, const qs_gate *g)
{
    const int *c = g->ctrl;
    int nc = g->nctrl;
    switch (g->op) {
    case QS_OP_H:       return orc_h(s, g->q[0], c, nc);
    case QS_OP_X:       return orc_x(s, g->q[0], c, nc);
    case QS_OP_RX:      return orc_rx(s, g->q[0], g->theta, g->dagger, c, nc);
    case QS_OP_RY:      return orc_ry(s, g->q[0], g->theta, g->dagger, c, nc);
    case QS_OP_RZ:      return orc_rz(s, g->q[0], g->theta, g->dagger, c, nc);
    case QS_OP_CNOT:    return orc_cnot(s, g->q[0], g->q[1], c, nc);
    case QS_OP_CR:      return orc_cr(s, g->q[0], g->q[1], g->theta, g->dagger, c, nc);
    case QS_OP_ISWAP:   return orc_iswap(s, g->q[0], g->q[1], g->dagger, c, nc);
    case QS_OP_SQISWAP: return orc_sqiswap(s, g->q[0], g->q[1], g->dagger, c, nc);
    case QS_OP_TOFFOLI: return orc_toffoli(s, g->q[0], g->q[1], g->q[2], c, nc);
    case QS_OP_CSWAP:   return orc_cswap(s, g->q[0], g->q[1], g->q[2], c, nc);
    case QS_OP_SWAP:    return orc_cswap(s, -1, g->q[0], g->q[1], c, nc);
    default:            return -1;
    }
}

int orc_gates(orc_state *s, const qs_gate *g, uint64_t count)
{
    for (uint64_t i = 0; i < count; ++i)
        if (orc_gate(s, &g[i])) return -1 - (int)i;
    return 0;
}

/* --------------------------------------------------------- measurement */
static double amp_p(const double *a)      /* abs(a)*abs(a) */
{
    double m = hypot(a[0], a[1]);
    return m * m;
}

/* qubitMeasure with an explicit uniform (CPUQuantumGates.cpp:1071-1126). */
int orc_prob_zero(orc_state *s, int q, double *p0)
{
    if (q < 0 || q >= s->n) return -1;
    uint64_t st = POW2(q);
    double d = 0;
    for (uint64_t i = 0; i < s->N; i += 2 * st)
        for (uint64_t j = i; j < i + st; ++j)
            d += amp_p(&s->a[2 * j]);
    *p0 = d;
    return 0;
}

int orc_measure(orc_state *s, int q, double u)
{
    double d;
    if (orc_prob_zero(s, q, &d)) return -1;
    uint64_t st = POW2(q);
    float fi = (float)u;
    int out = ((double)fi > d) ? 1 : 0;
    double sc = out ? 1 / sqrt(1 - d) : 1 / sqrt(d);
    for (uint64_t i = 0; i < s->N; i += 2 * st)
        for (uint64_t j = i; j < i + st; ++j) {
            double *keep = &s->a[2 * (out ? j + st : j)];
            double *zero = &s->a[2 * (out ? j : j + st)];
            keep[0] *= sc; keep[1] *= sc;
            zero[0] = 0; zero[1] = 0;
        }
    return out;
}

/* Full marginal (CPUQuantumGates.cpp:161-176), before the sort and cut. */
int orc_pmeasure(orc_state *s, const int *qubits, int m, double *out)
{
    for (int j = 0; j < m; ++j)
        if (qubits[j] < 0 || qubits[j] >= s->n) return -1;
    memset(out, 0, sizeof(double) * POW2(m));
    for (uint64_t i = 0; i < s->N; ++i) {
        uint64_t idx = 0;
        for (int j = 0; j < m; ++j)
            idx += ((i >> qubits[j]) % 2) << j;
        out[idx] += amp_p(&s->a[2 * i]);
    }
    return 0;
}

/* Shots by literal re-measurement of a copy of the state per shot: the
 * QPandaSDK::run loop with terminal MEASUREs (QPandaAPI.cpp:173-182). */
int orc_sample(orc_state *s, const int *qubits, int m, const double *u,
               uint64_t shots, uint64_t *out)
{
    int bad = 0;
    /* shots are independent: each thread re-measures its own copy */
#pragma omp parallel reduction(| : bad)
    {
        orc_state *w = orc_create(s->n);
        if (!w) bad = 1;
#pragma omp for schedule(dynamic, 4)
        for (long long sh = 0; sh < (long long)shots; ++sh) {
            if (!w) continue;
            memcpy(w->a, s->a, 2 * s->N * sizeof(double));
            uint64_t bits = 0;
            for (int k = 0; k < m; ++k) {
                int o = orc_measure(w, qubits[k], u[(uint64_t)sh * (uint64_t)m + k]);
                if (o < 0) { bad = 1; break; }
                bits |= (uint64_t)o << k;
            }
            out[sh] = bits;
        }
        orc_destroy(w);
    }
    return bad ? -1 : 0;
}

double orc_norm2(orc_state *s)
{
    double d = 0;
    for (uint64_t i = 0; i < s->N; ++i) d += s->a[2 * i] * s->a[2 * i] + s->a[2 * i + 1] * s->a[2 * i + 1];
    return d;
}

/* The reference's 16807 generator (QuantumGates.cpp:46-85) with an explicit
 * seed, for tests that want its stream. */
double orc_rand16807(int *seed)
{
    const int ia = 16807, im = 2147483647, iq = 127773, ir = 2836;
    int x = ia * (*seed % iq) - ir * (*seed / iq);
    if (x < 0) x += im;
    *seed = x;
    return (double)x / im;
}
