// qs_prim.h - the two primitive operations every reference gate lowers to.
// Host-only; shared by the per-gate path (qs_api.cu) and the fusion planner
// (qs_plan.cpp), so both apply exactly the same matrices.
#pragma once
#include <stdint.h>

#include "../../include/qpanda_b200.h"

enum { QS_PRIM_PAIR = 1, QS_PRIM_PHASE = 2 };

struct qs_prim {
    int kind;
    uint64_t holes;      // PAIR: target/exchanged bits + control bits; PHASE: the mask
    uint64_t cmask;      // PAIR: control bits (1 in every touched amplitude)
    uint64_t off0, off1; // PAIR: the two amplitudes are base|off0 and base|off1
    double m[8];         // PAIR: 2x2 row-major complex; PHASE: m[0] + i*m[1]
};

// Lower one gate record on an n-qubit register; QS_OK or a QS_ERR_* code
// (the message is recorded for qs_last_error()).
int qs_lower_gate(int n, const qs_gate *g, qs_prim *p);
// All qubits (targets and controls) a gate touches.
uint64_t qs_gate_qubits(const qs_gate *g);

int qs_fail(int code, const char *fmt, ...);
