"""Seeded synthetic circuits, as arrays of qs_gate records.

The workloads are the ones the reference's benchmarks would be quoted on:
  random_layers  - n qubits, L layers; per layer an RX/RY/RZ on every qubit
                   (axis uniform, angle uniform in [0, 2pi)), then a two-qubit
                   gate on each pair of a seeded random perfect matching: CNOT
                   (control = first of the pair) or, with probability
                   iswap_frac, iSWAP.
  qft            - the gate order of QRunesGenerator/src/QRLib.cpp:45-66 (qft):
                   for j = 0..n-1: CR(j, i, pi/2^(j-i)) for i < j, then H(j);
                   then the qubit-reversal SWAPs.  Full-precision pi.
  vqe_ansatz     - per layer RY then RZ on every qubit, then CNOT(i, i+1) for
                   i = 0..n-2 (hardware-efficient ansatz).
"""
import math

import numpy as np

from .capi import GATE_DTYPE, OP


def _gate(op, q, theta=0.0, dagger=0):
    g = np.zeros((), dtype=GATE_DTYPE)
    g["op"] = OP[op]
    qq = list(q) + [0] * (3 - len(q))
    g["q"] = qq
    g["theta"] = theta
    g["dagger"] = dagger
    return g


def make_gates(spec):
    """spec: list of (op, qubits, theta) tuples -> gate record array."""
    out = np.zeros(len(spec), dtype=GATE_DTYPE)
    for i, s in enumerate(spec):
        op, q = s[0], s[1]
        theta = s[2] if len(s) > 2 else 0.0
        out[i] = _gate(op, q, theta, s[3] if len(s) > 3 else 0)
    return out


def random_layers(n, layers, seed, iswap_frac=0.0):
    rng = np.random.default_rng(seed)
    spec = []
    for _ in range(layers):
        axes = rng.integers(0, 3, size=n)
        angles = rng.uniform(0.0, 2 * math.pi, size=n)
        for q in range(n):
            spec.append((("RX", "RY", "RZ")[axes[q]], (q,), float(angles[q])))
        perm = rng.permutation(n)
        kinds = rng.uniform(size=n // 2)
        for p in range(n // 2):
            a, b = int(perm[2 * p]), int(perm[2 * p + 1])
            spec.append(("ISWAP" if kinds[p] < iswap_frac else "CNOT", (a, b)))
    return make_gates(spec)


def qft(n, with_swaps=True):
    spec = []
    for j in range(n):
        for i in range(j):
            spec.append(("CR", (j, i), math.pi / 2 ** (j - i)))
        spec.append(("H", (j,)))
    if with_swaps:
        for k in range(n // 2):
            spec.append(("SWAP", (k, n - 1 - k)))
    return make_gates(spec)


def vqe_ansatz(n, layers, seed=None, angles=None):
    rng = np.random.default_rng(seed)
    if angles is None:
        angles = rng.uniform(0.0, 2 * math.pi, size=(layers, 2, n))
    spec = []
    for l in range(layers):
        for q in range(n):
            spec.append(("RY", (q,), float(angles[l, 0, q])))
        for q in range(n):
            spec.append(("RZ", (q,), float(angles[l, 1, q])))
        for q in range(n - 1):
            spec.append(("CNOT", (q, q + 1)))
    return make_gates(spec)


def gate_bytes(gates, n, amp_bytes):
    """Algorithmic HBM bytes of the plain per-gate path: 2 * S * (amplitudes the
    gate changes) per gate."""
    N = 1 << n
    tot = 0
    for g in np.atleast_1d(gates):
        op = int(g["op"])
        c = int(g["nctrl"])
        if op in (OP["H"], OP["X"], OP["RX"], OP["RY"], OP["RZ"]):
            amps = N
        elif op in (OP["CNOT"], OP["SWAP"], OP["ISWAP"], OP["SQISWAP"]):
            amps = N // 2
        elif op == OP["CR"]:
            amps = N // 4
        elif op in (OP["TOFFOLI"], OP["CSWAP"]):
            amps = N // 4
        else:
            amps = N
        tot += 2 * amp_bytes * (amps >> c)
    return tot


def vqe_sweep(n_circuits, seed, qmin=10, qmax=22, lmin=4, lmax=12):
    """Batched variational sweep: circuit k has q ~ U{qmin..qmax} qubits and
    L ~ U{lmin..lmax} layers of the hardware-efficient ansatz (vqe_ansatz),
    angles uniform in [0, 2pi).  Returns [(q, gates), ...]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_circuits):
        q = int(rng.integers(qmin, qmax + 1))
        L = int(rng.integers(lmin, lmax + 1))
        out.append((q, vqe_ansatz(q, L, angles=rng.uniform(0.0, 2 * math.pi, size=(L, 2, q)))))
    return out


def request_trace(n_requests, seed, rate=2000.0, qmin=8, qmax=30, dmin=4, dmax=32):
    """Request-loop workload: arrivals of a Poisson process with `rate` per
    second; each request has q ~ U{qmin..qmax} qubits, a random_layers circuit
    of depth ~ U{dmin..dmax} (its own seed) and asks for shots or the full
    probability vector with equal odds.  Returns a list of dicts."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    out = []
    for k in range(n_requests):
        out.append({"arrival": float(t[k]), "qubits": int(rng.integers(qmin, qmax + 1)),
                    "depth": int(rng.integers(dmin, dmax + 1)), "kind": "shots" if rng.uniform() < 0.5 else "probs",
                    "seed": int(rng.integers(1 << 31))})
    return out
