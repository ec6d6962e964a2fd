/*
 * qpanda_b200_gpuemu.h - libGPUEmulator.so: the B200 backend behind the
 * reference's own GPU compute unit.
 *
 * The reference's GPUQuantumGates (QPandaSDK/QuantumInstructionHandle/
 * GPUQuantumGates.cpp:36-48) opens "libGPUEmulator.so" with dlopen and looks
 * up each gate function by name with dlsym; the names and signatures are the
 * function-pointer types of QPandaSDK/GPUEmulator/GPUGatesDecl.h:38-75, C
 * linkage with C++ reference arguments.  This header declares the same
 * entry points, implemented over the C ABI of qpanda_b200.h
 * (qpanda_b200/host/GPUEmulatorShim.cpp, built into
 * qpanda_b200/_lib/libGPUEmulator.so), so the unmodified reference - the
 * command line's `run -gpu` included - runs its programs on the B200 kernels.
 *
 * The state handle travels in the reference's own QState record
 * (QPandaSDK/GPUEmulator/GPUStruct.h:13-18, same layout here): for the device
 * state ("psigpu") `real` holds the qs_state handle and `imag` is NULL; the
 * host state ("psi") holds the split real/imaginary arrays that getState
 * fills for GPUQuantumGates::getQState.
 *
 * Semantics are those of the reference's CPU backend (CPUQuantumGates.cpp,
 * the parity target of this library), not of its old GPU kernels
 * (QPandaSDK/GPUEmulator/GPUGates.cu), where they differ: RZ is
 * diag(e^{-i theta/2}, e^{+i theta/2}) (GPUGates.cu:331-345 applies
 * diag(1, e^{i theta})), iSWAP is +i (GPUGates.cu uses -i), measurement uses
 * the CPU's float-cast comparison, qbReset measures and flips (GPUGates.cu's
 * projects onto |0> without a draw), pMeasure reads the qubits in the order
 * given (GPUGates.cu sorts them) and clears the output first.  Every gate
 * draws one uniform first and applies when it exceeds error_rate, like the
 * CPU backend, so a program's measurement stream matches the CPU backend's
 * for the same generator.  CRdagger is also exported as "pCRdagger", the name
 * GPUQuantumGates looks up for CR with dagger (GPUQuantumGates.cpp:633).
 * Functions return false (or -1) on failure; the message is qs_last_error().
 */
#ifndef QPANDA_B200_GPUEMU_H
#define QPANDA_B200_GPUEMU_H

#include <stddef.h>

#include <utility>
#include <vector>

namespace GATEGPU {
struct QState {                 /* layout of QPandaSDK/GPUEmulator/GPUStruct.h:13-18 */
    double *real;
    double *imag;
    int qnum;
};
}  // namespace GATEGPU

extern "C" {
typedef std::vector<size_t> qs_emu_qnum;
typedef std::vector<std::pair<size_t, double>> qs_emu_probs;

/* GPUGatesDecl.h:42-44.  The C library declares a different initstate()
 * (<stdlib.h>); the C++ name here is qs_emu_initstate and the exported
 * symbol, which the reference looks up, is "initstate". */
bool qs_emu_initstate(GATEGPU::QState &psi, GATEGPU::QState &psigpu, int qnum) __asm__("initstate");
bool destroyState(GATEGPU::QState &psi, GATEGPU::QState &psigpu, size_t qnum);
bool clearState(GATEGPU::QState &psi, GATEGPU::QState &psigpu, size_t qnum);
/* GPUGatesDecl.h:45-62: single- and two-qubit gates */
bool Hadamard(GATEGPU::QState &psigpu, size_t qn, double error_rate);
bool Hadamardnew(GATEGPU::QState &psigpu, size_t qn, double error_rate);
bool Hadamarddagger(GATEGPU::QState &psigpu, size_t qn, double error_rate);
bool RX(GATEGPU::QState &psigpu, size_t qn, double theta, double error_rate);
bool RXdagger(GATEGPU::QState &psigpu, size_t qn, double theta, double error_rate);
bool RY(GATEGPU::QState &psigpu, size_t qn, double theta, double error_rate);
bool RYdagger(GATEGPU::QState &psigpu, size_t qn, double theta, double error_rate);
bool RZ(GATEGPU::QState &psigpu, size_t qn, double theta, double error_rate);
bool RZdagger(GATEGPU::QState &psigpu, size_t qn, double theta, double error_rate);
bool NOT(GATEGPU::QState &psigpu, size_t qn, double error_rate);
bool NOTdagger(GATEGPU::QState &psigpu, size_t qn, double error_rate);
bool CNOT(GATEGPU::QState &psigpu, size_t control, size_t target, double error_rate);
bool CNOTdagger(GATEGPU::QState &psigpu, size_t control, size_t target, double error_rate);
bool CR(GATEGPU::QState &psigpu, size_t q0, size_t q1, double theta, double error_rate);
bool CRdagger(GATEGPU::QState &psigpu, size_t q0, size_t q1, double theta, double error_rate);
bool pCRdagger(GATEGPU::QState &psigpu, size_t q0, size_t q1, double theta, double error_rate);
bool iSWAP(GATEGPU::QState &psigpu, size_t q0, size_t q1, double error_rate);
bool iSWAPdagger(GATEGPU::QState &psigpu, size_t q0, size_t q1, double error_rate);
bool sqiSWAP(GATEGPU::QState &psigpu, size_t q0, size_t q1, double error_rate);
bool sqiSWAPdagger(GATEGPU::QState &psigpu, size_t q0, size_t q1, double error_rate);
/* GPUGatesDecl.h:63: measure qubit log2(block); returns 0/1, -1 on failure */
int qubitmeasure(GATEGPU::QState &psigpu, size_t block);
/* GPUGatesDecl.h:64-71: controlled gates; qnum = controls with the target last */
bool controlHadamard(GATEGPU::QState &psigpu, qs_emu_qnum &qnum, double error_rate);
bool controlHadamarddagger(GATEGPU::QState &psigpu, qs_emu_qnum &qnum, double error_rate);
bool controlRX(GATEGPU::QState &psigpu, qs_emu_qnum &qnum, double theta, double error_rate);
bool controlRXdagger(GATEGPU::QState &psigpu, qs_emu_qnum &qnum, double theta, double error_rate);
bool controlRY(GATEGPU::QState &psigpu, qs_emu_qnum &qnum, double theta, double error_rate);
bool controlRYdagger(GATEGPU::QState &psigpu, qs_emu_qnum &qnum, double theta, double error_rate);
bool controlRZ(GATEGPU::QState &psigpu, qs_emu_qnum &qnum, double theta, double error_rate);
bool controlRZdagger(GATEGPU::QState &psigpu, qs_emu_qnum &qnum, double theta, double error_rate);
/* GPUGatesDecl.h:72-75 */
bool toffoli(GATEGPU::QState &psigpu, size_t c0, size_t c1, size_t target, double error_rate);
bool toffolidagger(GATEGPU::QState &psigpu, size_t c0, size_t c1, size_t target, double error_rate);
bool qbReset(GATEGPU::QState &psigpu, size_t qn, double error_rate);
/* pMeasure over the qubits log2(block[0..m)) and pMeasurenew over qnum: the
 * 10 most probable outcomes, descending, index bit j = qubit j of the list */
bool pMeasure(GATEGPU::QState &psigpu, qs_emu_probs &vprob, size_t *block, size_t m);
bool pMeasurenew(GATEGPU::QState &psigpu, qs_emu_probs &vprob, qs_emu_qnum &qnum);
/* copy the device state into psi.real / psi.imag */
bool getState(GATEGPU::QState &psi, GATEGPU::QState &psigpu, int qnum);

/* No reference counterpart.  The generator the gates draw from: a function
 * handed in here (e.g. one that calls the program's
 * QuantumGates::randGenerator, so that the shim and the CPU backend share one
 * stream; NULL restores the default), else the shim's own Park-Miller 16807
 * generator, seeded from the clock like the reference's unless
 * qs_gpuemu_seed sets the seed. */
void qs_gpuemu_set_rng(double (*fn)(void));
void qs_gpuemu_seed(int seed);
}

#endif /* QPANDA_B200_GPUEMU_H */
