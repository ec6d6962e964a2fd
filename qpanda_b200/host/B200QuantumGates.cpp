// B200QuantumGates.cpp - QuantumGates methods forwarded to the B200 C ABI.
// Reference behaviour cited per method (QPandaSDK/QuantumInstructionHandle/).
#include "B200QuantumGates.h"

#include <algorithm>
#include <cstring>
#include <sstream>

B200QuantumGates::B200QuantumGates(int dtype) : mDtype(dtype == QS_C64 ? QS_C64 : QS_C128)
{
    sCalculationUnitType = "B200";
}

B200QuantumGates::~B200QuantumGates()
{
    if (mState) qs_destroy(mState);
}

QError B200QuantumGates::fromStatus(int rc) const
{
    switch (rc) {
    case QS_OK: return qErrorNone;
    case QS_ERR_ARG: return qParameterError;
    default: return undefineError;           // CPUQuantumGates.cpp:1185 for a non-unitary matrix
    }
}

// One gate: draw the generator like every CPUQuantumGates method does, then
// hand the record to the device.  `controls` may hold the gate's own qubits
// (the dispatcher appends the targets, Instruction.cpp:52-58, 359-360,
// 470-472); those are not controls.
QError B200QuantumGates::apply(int op, const size_t *q, int nq, double theta, int dagger,
                               const Qnum &controls, double error_rate)
{
    if (!mState) return undefineError;
    if (mMode != kNormal) {
        uint64_t m = 0;
        for (int j = 0; j < nq; ++j) m |= 1ull << q[j];
        for (size_t c : controls) m |= 1ull << c;
        touch(m);
    }
    if (!(draw() > error_rate) || mMode == kProbe) return qErrorNone;
    qs_gate g;
    memset(&g, 0, sizeof(g));
    g.op = op;
    g.dagger = dagger ? 1 : 0;
    g.theta = theta;
    for (int j = 0; j < nq; ++j) g.q[j] = (int32_t)q[j];
    for (size_t c : controls) {
        bool own = false;
        for (int j = 0; j < nq; ++j) own |= (c == q[j]);
        bool dup = false;
        for (int j = 0; j < g.nctrl; ++j) dup |= ((size_t)g.ctrl[j] == c);
        if (own || dup) continue;
        if (g.nctrl == QS_MAX_CTRL) return qParameterError;
        g.ctrl[g.nctrl++] = (int32_t)c;
    }
    return fromStatus(qs_gate_apply(mState, &g));
}

size_t B200QuantumGates::getQStateSize()
{
    return mState ? (size_t)1 << mQubits : 0;
}

// CPUQuantumGates.cpp:64-82: one line per amplitude, default stream precision.
bool B200QuantumGates::getQState(string &sState, QuantumGateParam *)
{
    if (!mState) return false;
    if (mMode != kNormal && mMeasured) mTerminal = false;
    vector<complex<double>> v((size_t)1 << mQubits);
    if (qs_get_state(mState, v.data(), QS_C128) != QS_OK) return false;
    std::stringstream ss;
    int i = 0;
    for (auto &a : v) {
        ss << "state[" << i << "].real = " << a.real() << " " << "state[" << i << "].imag = " << a.imag() << "\n";
        ++i;
    }
    sState.append(ss.str());
    return true;
}

QError B200QuantumGates::Hadamard(size_t qn, double error_rate)
{
    return apply(QS_OP_H, &qn, 1, 0, 0, Qnum(), error_rate);
}

QError B200QuantumGates::Hadamard(size_t qn, double error_rate, Qnum vControlBit, size_t)
{
    return apply(QS_OP_H, &qn, 1, 0, 0, vControlBit, error_rate);
}

// CPUQuantumGates.cpp:126-136: measure, then flip if the outcome was 1.
QError B200QuantumGates::Reset(size_t qn)
{
    if (mMode != kNormal) mTerminal = false;     // its flip depends on the outcome
    if (mMode == kProbe) return qErrorNone;
    int o = qubitMeasure(qn);
    if (o < 0) return undefineError;
    if (o) return NOT(qn, 0);
    return qErrorNone;
}

QError B200QuantumGates::pMeasure(Qnum &qnum, vector<pair<size_t, double>> &mResult)
{
    if (!mState) return undefineError;
    if (mMode != kNormal && mMeasured) mTerminal = false;
    if (mMode == kProbe) return mResult.clear(), qErrorNone;
    vector<int> qs(qnum.begin(), qnum.end());
    uint64_t idx[10];
    double p[10];
    int cnt = 0;
    int rc = qs_pmeasure(mState, qs.data(), (int)qs.size(), idx, p, &cnt);
    if (rc) return fromStatus(rc);
    mResult.clear();
    for (int i = 0; i < cnt; ++i) mResult.push_back(std::make_pair((size_t)idx[i], p[i]));
    return qErrorNone;
}

QError B200QuantumGates::RX(size_t qn, double theta, double error_rate, int iDagger)
{
    return apply(QS_OP_RX, &qn, 1, theta, iDagger, Qnum(), error_rate);
}

QError B200QuantumGates::RX(size_t qn, double theta, double error_rate, Qnum ctl, size_t, int iDagger)
{
    return apply(QS_OP_RX, &qn, 1, theta, iDagger, ctl, error_rate);
}

QError B200QuantumGates::RY(size_t qn, double theta, double error_rate, int iDagger)
{
    return apply(QS_OP_RY, &qn, 1, theta, iDagger, Qnum(), error_rate);
}

// The reference takes the target from vControlBit.back() (CPUQuantumGates.cpp:408).
QError B200QuantumGates::RY(size_t qn, double theta, double error_rate, Qnum ctl, size_t, int iDagger)
{
    size_t t = ctl.empty() ? qn : ctl.back();
    return apply(QS_OP_RY, &t, 1, theta, iDagger, ctl, error_rate);
}

QError B200QuantumGates::RZ(size_t qn, double theta, double error_rate, int iDagger)
{
    return apply(QS_OP_RZ, &qn, 1, theta, iDagger, Qnum(), error_rate);
}

QError B200QuantumGates::RZ(size_t qn, double theta, double error_rate, Qnum ctl, size_t, int iDagger)
{
    return apply(QS_OP_RZ, &qn, 1, theta, iDagger, ctl, error_rate);
}

QError B200QuantumGates::CNOT(size_t qn_1, size_t qn_2, double error_rate)
{
    size_t q[2] = {qn_1, qn_2};
    return apply(QS_OP_CNOT, q, 2, 0, 0, Qnum(), error_rate);
}

// CPUQuantumGates.cpp:750-757: NOT on qn_2 with the list (which holds qn_1).
QError B200QuantumGates::CNOT(size_t qn_1, size_t qn_2, double error_rate, Qnum ctl, int)
{
    size_t q[2] = {qn_1, qn_2};
    return apply(QS_OP_CNOT, q, 2, 0, 0, ctl, error_rate);
}

QError B200QuantumGates::CR(size_t qn_1, size_t qn_2, double theta, double error_rate, int iDagger)
{
    size_t q[2] = {qn_1, qn_2};
    return apply(QS_OP_CR, q, 2, theta, iDagger, Qnum(), error_rate);
}

QError B200QuantumGates::iSWAP(size_t qn_1, size_t qn_2, double error_rate, int iDagger)
{
    size_t q[2] = {qn_1, qn_2};
    return apply(QS_OP_ISWAP, q, 2, 0, iDagger, Qnum(), error_rate);
}

QError B200QuantumGates::iSWAP(size_t qn_1, size_t qn_2, double error_rate, Qnum ctl, int, int iDagger)
{
    size_t q[2] = {qn_1, qn_2};
    return apply(QS_OP_ISWAP, q, 2, 0, iDagger, ctl, error_rate);
}

QError B200QuantumGates::sqiSWAP(size_t qn_1, size_t qn_2, double error_rate, int iDagger)
{
    size_t q[2] = {qn_1, qn_2};
    return apply(QS_OP_SQISWAP, q, 2, 0, iDagger, Qnum(), error_rate);
}

QError B200QuantumGates::sqiSWAP(size_t qn_1, size_t qn_2, double error_rate, Qnum ctl, int, int iDagger)
{
    size_t q[2] = {qn_1, qn_2};
    return apply(QS_OP_SQISWAP, q, 2, 0, iDagger, ctl, error_rate);
}

QError B200QuantumGates::controlSwap(size_t qn_1, size_t qn_2, size_t qn_3, double error_rate)
{
    if (qn_2 == qn_3) return draw(), qErrorNone;              // the reference's loop is a no-op then
    size_t q[3] = {qn_1, qn_2, qn_3};
    return apply(QS_OP_CSWAP, q, 3, 0, 0, Qnum(), error_rate);
}

// CPUQuantumGates.cpp:1071-1126.  Returns -1 on failure (Instruction.cpp:710).
int B200QuantumGates::qubitMeasure(size_t qn)
{
    if (!mState) return -1;
    if (mMode != kNormal) {
        if (qn >= (size_t)mQubits) return -1;
        const size_t pos = mDraws;
        mRec.push_back(Recorded{(int)qn, pos, draw()});
        mMeasured |= 1ull << qn;
        return 0;
    }
    double u = randGenerator();
    int out = 0;
    if (qs_measure(mState, (int)qn, u, &out) != QS_OK) return -1;
    return out;
}

// CPUQuantumGates.cpp:1170-1212: matrix is a QStat* of 4 entries {m00, m01,
// m10, m11}; |det| must be 1 within 1e-6.
QError B200QuantumGates::unitarySingleQubitGate(size_t qn, void *matrix, double error_rate)
{
    if (!mState || !matrix) return undefineError;
    const QStat &M = *static_cast<QStat *>(matrix);
    if (M.size() < 4) return qParameterError;
    if (mMode != kNormal) touch(1ull << qn);
    if (!(draw() > error_rate) || mMode == kProbe) return qErrorNone;
    double m[8];
    for (int j = 0; j < 4; ++j) { m[2 * j] = M[j].real(); m[2 * j + 1] = M[j].imag(); }
    return fromStatus(qs_apply_unitary_1q(mState, (int)qn, m));
}

// CPUQuantumGates.cpp:1136-1157: 2^n amplitudes, |0...0>.
QError B200QuantumGates::initState(QuantumGateParam *param)
{
    if (!param) return undefineError;
    int n = param->mQuantumBitNumber;
    if (mState && n == mQubits) return fromStatus(qs_reset_zero(mState));
    if (mState) {
        qs_destroy(mState);
        mState = nullptr;
        mQubits = 0;
    }
    if (qs_create(n, mDtype, nullptr, &mState) != QS_OK) {
        mState = nullptr;
        return undefineError;
    }
    mQubits = n;
    return qErrorNone;
}

bool B200QuantumGates::compareCalculationUnitType(string &s)
{
    return 0 == s.compare(sCalculationUnitType);
}

QError B200QuantumGates::NOT(size_t qn, double error_rate)
{
    return apply(QS_OP_X, &qn, 1, 0, 0, Qnum(), error_rate);
}

// The reference takes the target from vControlBit.back() (CPUQuantumGates.cpp:1328).
QError B200QuantumGates::NOT(size_t qn, double error_rate, Qnum ctl, int)
{
    size_t t = ctl.empty() ? qn : ctl.back();
    return apply(QS_OP_X, &t, 1, 0, 0, ctl, error_rate);
}

QError B200QuantumGates::toffoli(size_t c1, size_t c2, size_t t, double errorRate, int)
{
    size_t q[3] = {c1, c2, t};
    return apply(QS_OP_TOFFOLI, q, 3, 0, 0, Qnum(), errorRate);
}

QError B200QuantumGates::destroyState(size_t)
{
    if (mState) qs_destroy(mState);
    mState = nullptr;
    mQubits = 0;
    return qErrorNone;
}

// CPUQuantumGates.cpp:1445-1453: back to |0...0> (sent before every run).
QError B200QuantumGates::endGate(QuantumGateParam *, QuantumGates *)
{
    if (!mState) return undefineError;
    if (mMode == kProbe) return qErrorNone;
    return fromStatus(qs_reset_zero(mState));
}

// Swap the middle two rows and columns of a 4x4 (CPUQuantumGates.cpp:1223-1250).
QError B200QuantumGates::matReverse(COMPLEX (*mat)[4], COMPLEX (*mat_rev)[4])
{
    static const int perm[4] = {0, 2, 1, 3};
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) mat_rev[r][c] = mat[perm[r]][perm[c]];
    return qErrorNone;
}

// A uniform from the generator, counted in a deferred pass; a probe pass
// counts without drawing (and reports 1, so that every gate "applies").
double B200QuantumGates::draw()
{
    if (mMode == kNormal) return randGenerator();
    ++mDraws;
    return mMode == kProbe ? 1.0 : randGenerator();
}

void B200QuantumGates::touch(uint64_t qubit_mask)
{
    if (qubit_mask & mMeasured) mTerminal = false;
}

void B200QuantumGates::beginProbe()
{
    mMode = kProbe;
    mTerminal = true;
    mDraws = 0;
    mMeasured = 0;
    mRec.clear();
}

bool B200QuantumGates::endProbe()
{
    mMode = kNormal;
    return mTerminal && !mRec.empty();
}

void B200QuantumGates::beginDeferredMeasure()
{
    mMode = kDeferred;
    mTerminal = true;
    mDraws = 0;
    mMeasured = 0;
    mRec.clear();
}

QError B200QuantumGates::sampleDeferred(size_t shots, vector<uint64_t> &out)
{
    mMode = kNormal;
    out.assign(shots, 0);
    if (!mState || !mTerminal) return undefineError;
    const size_t m = mRec.size();
    if (shots == 0 || m == 0) return qErrorNone;
    // distinct qubits in the order first measured: slot[k] = the distinct qubit
    // of measurement k, lead[j] = the measurement that first measures qubit j
    vector<int> qubits;
    vector<size_t> slot(m), lead;
    for (size_t k = 0; k < m; ++k) {
        size_t j = 0;
        while (j < qubits.size() && qubits[j] != mRec[k].qubit) ++j;
        if (j == qubits.size()) {
            qubits.push_back(mRec[k].qubit);
            lead.push_back(k);
        }
        slot[k] = j;
    }
    const size_t mu = qubits.size();
    vector<double> u(shots * mu), pass(mDraws);
    for (size_t j = 0; j < mu; ++j) u[j] = mRec[lead[j]].u;         // shot 0: the pass's own draws
    for (size_t s = 1; s < shots; ++s) {                             // then a pass's worth per shot
        for (size_t d = 0; d < mDraws; ++d) pass[d] = randGenerator();
        for (size_t j = 0; j < mu; ++j) u[s * mu + j] = pass[mRec[lead[j]].draw];
    }
    vector<uint64_t> raw(shots);
    int rc = qs_sample(mState, qubits.data(), (int)mu, u.data(), shots, raw.data());
    if (rc) return fromStatus(rc);
    // the state the loop leaves: the last shot's measurements, in order
    uint64_t last = 0;
    for (size_t j = 0; j < mu; ++j) {
        int o = 0;
        if ((rc = qs_measure(mState, qubits[j], u[(shots - 1) * mu + j], &o))) return fromStatus(rc);
        last |= (uint64_t)o << j;
    }
    raw[shots - 1] = last;
    for (size_t s = 0; s < shots; ++s) {
        uint64_t bits = 0;
        for (size_t k = 0; k < m; ++k) bits |= ((raw[s] >> slot[k]) & 1ull) << k;
        out[s] = bits;
    }
    return qErrorNone;
}
