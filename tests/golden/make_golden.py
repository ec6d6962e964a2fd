"""Generate the golden fixtures from the reference's own CPU backend.

Runs QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp, compiled from the
reference sources by `make -C oracle ref` (oracle/_ref/libqpanda_ref.so), on
small seeded cases and stores inputs and outputs in tests/golden/*.npz.
Run from the repository root:  python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.pyoracle import RefState, ref_available  # noqa: E402
from qpanda_b200 import circuits  # noqa: E402
from qpanda_b200.capi import GATE_DTYPE, OP  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")


def gate(op, q, theta=0.0, dagger=0, ctrl=()):
    g = np.zeros((), dtype=GATE_DTYPE)
    g["op"] = OP[op]
    g["q"] = list(q) + [0] * (3 - len(q))
    g["theta"] = theta
    g["dagger"] = dagger
    g["nctrl"] = len(ctrl)
    g["ctrl"][:len(ctrl)] = list(ctrl)
    return g


def every_gate_circuit(n, seed):
    """Every gate kind the reference implements, with and without daggers and
    control lists, on seeded qubits (qubit 0 and the top qubit included)."""
    rng = np.random.default_rng(seed)
    gs = []
    for q in range(n):
        gs.append(gate("H", (q,)))
    for _ in range(6):
        for op in ("RX", "RY", "RZ"):
            for dag in (0, 1):
                gs.append(gate(op, (int(rng.integers(n)),), float(rng.uniform(0, 2 * math.pi)), dag))
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        gs.append(gate("CNOT", (a, b)))
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        gs.append(gate("CR", (a, b), float(rng.uniform(0, 2 * math.pi)), int(rng.integers(2))))
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        gs.append(gate("ISWAP", (a, b), 0.0, int(rng.integers(2))))
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        gs.append(gate("SQISWAP", (a, b), 0.0, int(rng.integers(2))))
        a, b, c = (int(x) for x in rng.choice(n, 3, replace=False))
        gs.append(gate("TOFFOLI", (a, b, c)))
        a, b, c = (int(x) for x in rng.choice(n, 3, replace=False))
        gs.append(gate("CSWAP", (a, b, c)))
        gs.append(gate("X", (int(rng.integers(n)),)))
        # controlled single-qubit gates (QRunes CONTROL blocks)
        for op in ("H", "X", "RX", "RY", "RZ"):
            qs = [int(x) for x in rng.choice(n, 3, replace=False)]
            gs.append(gate(op, (qs[0],), float(rng.uniform(0, 2 * math.pi)), int(rng.integers(2)), ctrl=qs[1:]))
        qs = [int(x) for x in rng.choice(n, 4, replace=False)]
        gs.append(gate("CNOT", (qs[0], qs[1]), ctrl=qs[2:]))
        gs.append(gate("H", (0,)))
        gs.append(gate("RY", (n - 1,), 0.7))
    return np.array(gs, dtype=GATE_DTYPE)


def main():
    if not ref_available():
        sys.exit("oracle/_ref/libqpanda_ref.so missing: run `make -C oracle ref` first")
    cases = {}
    # 1) every gate kind, n = 7 and 10
    for n, seed in ((7, 11), (10, 12)):
        g = every_gate_circuit(n, seed)
        r = RefState(n)
        r.apply(g)
        cases[f"gates_n{n}"] = dict(n=n, gates=g, state=r.state())
    # 2) config-0 structure at small n: random layers, pMeasure, shots
    for n, layers, seed in ((10, 20, 100), (12, 8, 101)):
        g = circuits.random_layers(n, layers, seed)
        r = RefState(n)
        r.apply(g)
        st = r.state()
        rng = np.random.default_rng(seed + 1)
        qs = np.arange(n, dtype=np.int32)
        shots = 256
        u = rng.uniform(size=(shots, n))
        u = np.where(u == 0.0, 0.5, u)
        sh = r.sample(qs, u)
        pm_q = np.array([n - 1, 0, 3], dtype=np.int32)
        pm = r.pmeasure(pm_q)
        cases[f"layers_n{n}"] = dict(n=n, gates=g, state=st, shot_qubits=qs, uniforms=u, shots=sh,
                                     pm_qubits=pm_q, pm_idx=np.array([a for a, _ in pm], dtype=np.int64),
                                     pm_p=np.array([b for _, b in pm]))
    # 3) iSWAP-mixed layers (config-2 structure) and QFT on a Gaussian state
    g = circuits.random_layers(9, 6, 102, iswap_frac=0.1)
    r = RefState(9)
    r.apply(g)
    cases["iswap_layers_n9"] = dict(n=9, gates=g, state=r.state())
    n = 9
    rng = np.random.default_rng(103)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    g = circuits.qft(n)
    r = RefState(n)
    r.set_state(v)
    r.apply(g)
    cases["qft_n9"] = dict(n=n, gates=g, init=v, state=r.state())
    # 4) sequential measurements with known uniforms (qubitMeasure semantics)
    n = 8
    g = circuits.random_layers(n, 5, 104)
    r = RefState(n)
    r.apply(g)
    mq = np.array([3, 0, 7, 5], dtype=np.int32)
    mu = np.array([0.31, 0.77, 0.5, 0.93])
    outs = np.array([r.measure(int(q), float(u)) for q, u in zip(mq, mu)], dtype=np.int32)
    cases["measure_n8"] = dict(n=n, gates=g, mqubits=mq, muniforms=mu, outcomes=outs, state=r.state())
    for name, d in cases.items():
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)
        print("wrote", name)
    # 5) the reference's getQState text of the gates_n7 state: the .fullstate
    #    file format (QCommand.cpp:402-428 writes this text verbatim)
    r = RefState(7)
    r.apply(cases["gates_n7"]["gates"])
    with open(os.path.join(OUT, "qstate_n7.txt"), "w") as f:
        f.write(r.qstate_text())
    print("wrote qstate_n7.txt")


if __name__ == "__main__":
    main()
