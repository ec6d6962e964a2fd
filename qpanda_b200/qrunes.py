"""Gate records -> QRunes program text (the input language of the reference's
parser, QPandaSDK/QRunesParser), for running the same circuit through the
reference's own toolchain.

Controls become (nested, one qubit each) CONTROL/ENDCONTROL blocks and dagger flags DAGGER/ENDDAGGER
blocks (the parser copies the control stack into each node and toggles the
dagger flag, LinkedListController.cpp:289-398).  QRunes has no SWAP or
controlSwap keyword: SWAP is written as three CNOTs and controlSwap as three
CNOTs inside a CONTROL block.  Angles are written in fixed notation with 17
decimals (the lexer reads them with atof, lex.yy.cpp:944).
"""
import numpy as np

from .capi import OP

_NAMES = {OP["H"]: "H", OP["X"]: "NOT", OP["RX"]: "RX", OP["RY"]: "RY", OP["RZ"]: "RZ",
          OP["CNOT"]: "CNOT", OP["CR"]: "CR", OP["ISWAP"]: "ISWAP", OP["SQISWAP"]: "SQISWAP",
          OP["TOFFOLI"]: "TOFFOLI"}


def _angle(t):
    return '"' + format(float(t), ".17f") + '"'


def _gate_lines(g):
    op = int(g["op"])
    q = [int(x) for x in g["q"]]
    t = float(g["theta"])
    if op in (OP["H"], OP["X"]):
        return [f"{_NAMES[op]} {q[0]}"]
    if op in (OP["RX"], OP["RY"], OP["RZ"]):
        return [f"{_NAMES[op]} {q[0]},{_angle(t)}"]
    if op == OP["CNOT"]:
        return [f"CNOT {q[0]},{q[1]}"]
    if op == OP["CR"]:
        return [f"CR {q[0]},{q[1]},{_angle(t)}"]
    if op == OP["ISWAP"]:
        return [f"ISWAP {q[0]},{q[1]},{_angle(0.0)}"]     # the keyword takes an (unused) angle
    if op == OP["SQISWAP"]:
        return [f"SQISWAP {q[0]},{q[1]}"]
    if op == OP["TOFFOLI"]:
        return [f"TOFFOLI {q[0]},{q[1]},{q[2]}"]
    if op == OP["SWAP"]:
        a, b = q[0], q[1]
        return [f"CNOT {a},{b}", f"CNOT {b},{a}", f"CNOT {a},{b}"]
    if op == OP["CSWAP"]:
        c, a, b = q
        return [f"CONTROL {c}", f"CNOT {a},{b}", f"CNOT {b},{a}", f"CNOT {a},{b}", f"ENDCONTROL {c}"]
    raise ValueError(f"op {op} has no QRunes form")


def to_qrunes(n, gates, measure=None, pmeasure=None):
    """QRunes text for `gates` on n qubits.  measure: list of (qubit, creg)
    pairs appended as MEASURE lines; pmeasure: list of qubits for a final
    PMEASURE line."""
    ncreg = max([c for _, c in measure], default=-1) + 1 if measure else 1
    out = [f"QINIT {n}", f"CREG {ncreg}"]
    for g in np.atleast_1d(gates):
        lines = _gate_lines(g)
        if int(g["dagger"]):
            lines = ["DAGGER"] + lines + ["ENDDAGGER"]
        nc = int(g["nctrl"])
        # one qubit per CONTROL line (the grammar takes a single qubit);
        # several controls are nested blocks
        for c in reversed([int(c) for c in g["ctrl"][:nc]]):
            lines = [f"CONTROL {c}"] + lines + [f"ENDCONTROL {c}"]
        out.extend(lines)
    for q, c in (measure or []):
        out.append(f"MEASURE {q},${c}")
    if pmeasure is not None:
        out.append("PMEASURE " + ",".join(str(q) for q in pmeasure))
    return "\n".join(out) + "\n"
