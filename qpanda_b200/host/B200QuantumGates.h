// B200QuantumGates.h - the B200 backend behind the reference gate interface.
//
// A subclass of QuantumGates (QPandaSDK/QuantumInstructionHandle/QuantumGates.h:31-474),
// the abstract class that QuantumInstructionGet::transmit drives gate by gate
// (QuantumInstructionGet.cpp:104-124).  It takes the place of CPUQuantumGates /
// GPUQuantumGates: QuantumInstructionHandleAPI::setComputeUnit can construct
// it like the other two (QuantumInstructionHandleAPI.cpp:194-229), and QRunes
// programs then run unchanged through the reference's parser and dispatcher.
//
// Every method forwards to the C ABI of include/qpanda_b200.h; the state
// lives in HBM for the object's lifetime.  Semantics follow CPUQuantumGates:
//  - each gate first draws randGenerator() and applies only if the draw
//    exceeds error_rate (CPUQuantumGates.cpp:98 and every gate), so the
//    generator's stream - and with it every later measurement - stays aligned
//    with the reference backend for the same program and seed;
//  - controlled overloads receive the control list with the target(s)
//    appended (Instruction.cpp:52-58); the targets are removed from it here;
//  - qubitMeasure draws one uniform and uses qubitMeasure's float-cast rule;
//  - pMeasure returns the 10 most probable outcomes (CPUQuantumGates.cpp:178-189);
//  - getQState prints the reference's text format (CPUQuantumGates.cpp:64-82).
// Deliberate differences: the controlled iSWAP / sqiSWAP overloads, which the
// reference leaves empty (CPUQuantumGates.cpp:914-922, 1054-1062), apply the
// gate on the control=1 subspace (an empty control list gives the plain gate);
// unitarySingleQubitGate uses stride 2^qn (the reference's 2^(qn-1) at
// :1188 is a bug).
#ifndef B200_QUANTUM_GATES_H
#define B200_QUANTUM_GATES_H

#include "QuantumGates.h"
#include "qpanda_b200.h"

class B200QuantumGates : public QuantumGates
{
public:
    // dtype: QS_C128 (default; the reference's precision) or QS_C64.
    explicit B200QuantumGates(int dtype = QS_C128);
    ~B200QuantumGates();

    size_t getQStateSize();
    bool getQState(string &sState, QuantumGateParam *pQuantumProParam);
    QError Hadamard(size_t qn, double error_rate);
    QError Reset(size_t qn);
    QError pMeasure(Qnum &qnum, vector<pair<size_t, double>> &mResult);
    QError Hadamard(size_t qn, double error_rate, Qnum vControlBit, size_t stQuantumBitNumber);
    QError RX(size_t qn, double theta, double error_rate, int iDagger);
    QError RX(size_t qn, double theta, double error_rate, Qnum vControlBitNumber,
              size_t stQuantumBitNumber, int iDagger);
    QError RY(size_t qn, double theta, double error_rate, int iDagger);
    QError RY(size_t qn, double theta, double error_rate, Qnum vControlBit, size_t stQuantumBitNumber,
              int iDagger);
    QError RZ(size_t qn, double theta, double error_rate, int iDagger);
    QError RZ(size_t qn, double theta, double error_rate, Qnum vControlBitNumber,
              size_t stQuantumBitNumber, int iDagger);
    QError CNOT(size_t qn_1, size_t qn_2, double error_rate);
    QError CNOT(size_t qn_1, size_t qn_2, double error_rate, Qnum vControlBitNumber, int stQuantumBitNumber);
    QError CR(size_t qn_1, size_t qn_2, double theta, double error_rate, int iDagger);
    QError iSWAP(size_t qn_1, size_t qn_2, double error_rate, int iDagger);
    QError iSWAP(size_t qn_1, size_t qn_2, double error_rate, Qnum vControlBitNumber, int stQuantumBitNumber,
                 int iDagger);
    QError sqiSWAP(size_t qn_1, size_t qn_2, double error_rate, int iDagger);
    QError sqiSWAP(size_t qn_1, size_t qn_2, double error_rate, Qnum vControlBitNumber, int stQuantumBitNumber,
                   int iDagger);
    QError controlSwap(size_t qn_1, size_t qn_2, size_t qn_3, double error_rate);
    int qubitMeasure(size_t qn);
    QError unitarySingleQubitGate(size_t qn, void *matrix, double error_rate);
    QError initState(QuantumGateParam *pQuantumProParam);
    bool compareCalculationUnitType(string &sCalculationUnitType);
    QError NOT(size_t qn, double error_rate);
    QError NOT(size_t qn, double error_rate, Qnum vControlBit, int stQuantumBitNumber);
    QError toffoli(size_t stControlBit1, size_t stControlBit2, size_t stQuantumBit, double errorRate,
                   int stQuantumBitNumber);
    QError destroyState(size_t stQNum);
    QError endGate(QuantumGateParam *pQuantumProParam, QuantumGates *pQGate);

    // ---- shots of a program whose measurements are terminal --------------
    // QPandaSDK::run re-runs a MEASURE program once per shot, resetting the
    // state each time (QPandaAPI.cpp:169-182).  When no gate, Reset or
    // pMeasure touches the state after a measurement, one run plus sampling
    // gives the same outcomes from the same generator stream.  Use:
    //   beginProbe(); one pass of the program; endProbe() - a dry pass that
    //     launches nothing and draws nothing, and tells whether every
    //     measurement is terminal (false: run the per-shot loop as before);
    //   beginDeferredMeasure(); one pass of the program (endGate, then every
    //     node), in which qubitMeasure draws its uniform and records it with
    //     the qubit and its position in the pass's draws, returns 0 and leaves
    //     the state alone;  then sampleDeferred(shots, out).
    void beginProbe();
    bool endProbe();
    void beginDeferredMeasure();
    // True after a pass unless something touched the state after a
    // measurement.
    bool deferredTerminal() const { return mTerminal; }
    // Measurements recorded in the pass, in program order.
    size_t deferredCount() const { return mRec.size(); }
    // out[s] bit k = outcome of the k-th recorded measurement in shot s.  Shot
    // 0 uses the uniforms drawn in the pass; shot s > 0 draws a whole pass's
    // worth (one per gate and per measurement, in program order) from
    // randGenerator() and uses the draws at the measurements' positions - the
    // draws the per-shot loop would give them.  Outcomes follow qubitMeasure's
    // rule with sequential collapse (qs_sample); a qubit measured again gets
    // its first outcome.  Afterwards the state is collapsed as the last shot
    // left it and the generator stands where the loop would leave it.  Ends
    // deferred mode.
    QError sampleDeferred(size_t shots, vector<uint64_t> &out);

    // Direct access for callers that want the C ABI's extra entry points
    // (fused plans, shot sampling) on the same state.
    qs_state *state() { return mState; }
    // Message of the last failing C-ABI call.
    const char *lastError() const { return qs_last_error(); }

protected:
    QError matReverse(COMPLEX (*mat)[4], COMPLEX (*mat_rev)[4]);

private:
    QError apply(int op, const size_t *q, int nq, double theta, int dagger, const Qnum &controls,
                 double error_rate);
    QError fromStatus(int rc) const;

    // draw one uniform, counting the pass's draws in deferred mode
    double draw();
    void touch(uint64_t qubit_mask);

    qs_state *mState = nullptr;
    int mQubits = 0;
    int mDtype;
    // deferred measurements
    struct Recorded {
        int qubit;
        size_t draw;                     // position among the pass's draws
        double u;
    };
    enum Mode { kNormal, kProbe, kDeferred };
    Mode mMode = kNormal;
    bool mTerminal = true;
    size_t mDraws = 0;
    uint64_t mMeasured = 0;              // qubits measured so far in the pass
    vector<Recorded> mRec;
};

#endif
