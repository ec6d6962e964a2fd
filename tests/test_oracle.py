"""The CPU oracle (oracle/qs_oracle.c) pinned against the reference.

1. against the golden fixtures, which tests/golden/make_golden.py produced by
   running the reference's own CPUQuantumGates.cpp (bit-exact);
2. against the reference compiled from its sources here (oracle/_ref), on
   fresh seeded cases, when that library has been built;
3. the known-answer tests of QPandaSDK/testMain/testCPUQuantumGates.cpp,
   restated with fixed angles (the reference draws them from its
   time-seeded generator).
"""
import glob
import math
import os

import numpy as np
import pytest

from oracle.pyoracle import OracleState, RefState, ref_available
from qpanda_b200 import circuits
from qpanda_b200.capi import GATE_DTYPE, OP

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
ZERO = 1e-12     # testCPUQuantumGates.cpp:6
SQ2 = 0.707106781186548


def bits(a):
    return np.ascontiguousarray(a, dtype=np.complex128).view(np.uint64)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(path):
    d = np.load(path)
    n = int(d["n"])
    o = OracleState(n)
    if "init" in d:
        o.set_state(d["init"])
    o.apply(d["gates"])
    if "mqubits" in d:
        outs = [o.measure(int(q), float(u)) for q, u in zip(d["mqubits"], d["muniforms"])]
        assert outs == d["outcomes"].tolist()
    assert np.array_equal(bits(o.state()), bits(d["state"])), "state differs from the reference"
    if "shots" in d:
        sh = o.sample(d["shot_qubits"], d["uniforms"])
        assert np.array_equal(sh, d["shots"])
        p = o.probs(d["pm_qubits"])
        order = sorted(range(len(p)), key=lambda i: (-p[i], i))[:10]
        assert np.allclose(p[order], d["pm_p"], rtol=0, atol=1e-15)
        # the top-10 set agrees (ties may be ordered differently by std::sort)
        assert set(np.array(order)[p[order] > 1e-14].tolist()) == set(
            d["pm_idx"][d["pm_p"] > 1e-14].tolist())


needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (no reference tree)")


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_reference_random(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 12))
    from tests.golden.make_golden import every_gate_circuit
    g = np.concatenate([every_gate_circuit(n, seed + 1000),
                        circuits.random_layers(n, 3, seed, iswap_frac=0.5)])
    o, r = OracleState(n), RefState(n)
    o.apply(g)
    r.apply(g)
    assert np.array_equal(bits(o.state()), bits(r.state()))
    for q in rng.permutation(n)[:3]:
        u = float(rng.uniform())
        assert o.measure(int(q), u) == r.measure(int(q), u)
        assert np.array_equal(bits(o.state()), bits(r.state()))


@needs_ref
def test_oracle_shots_match_reference():
    n = 9
    g = circuits.random_layers(n, 6, 5)
    o, r = OracleState(n), RefState(n)
    o.apply(g)
    r.apply(g)
    qs = np.array([4, 0, 8, 2, 1, 3, 5, 6, 7], dtype=np.int32)
    u = np.random.default_rng(9).uniform(size=(200, n))
    assert np.array_equal(o.sample(qs, u), r.sample(qs, u))


# ---------------------------------------------------------------- known answers
def one(op, q, theta=0.0, dagger=0, ctrl=()):
    g = np.zeros(1, dtype=GATE_DTYPE)
    g["op"] = OP[op]
    g["q"][0, :len(q)] = q
    g["theta"] = theta
    g["dagger"] = dagger
    g["nctrl"] = len(ctrl)
    g["ctrl"][0, :len(ctrl)] = ctrl
    return g


def test_kat_rx_ry_rz():
    th = 1.234
    for q in range(4):
        o = OracleState(4)
        o.apply(one("RX", (q,), th))                      # testRX :93-118
        s = o.state()
        assert abs(s[0] - math.cos(th / 2)) < ZERO and abs(s[1 << q] - (-1j * math.sin(th / 2))) < ZERO
        o = OracleState(4)
        o.apply(one("RY", (q,), th))                      # testRY :120-145
        s = o.state()
        assert abs(s[0] - math.cos(th / 2)) < ZERO and abs(s[1 << q] - math.sin(th / 2)) < ZERO
        o = OracleState(4)
        o.apply(one("RZ", (q,), th))                      # testRZ :147-176: RZ|0> = e^{-i th/2}|0>
        assert abs(o.state()[0] - np.exp(-0.5j * th)) < ZERO
        o.apply(one("X", (q,)))
        o.apply(one("RZ", (q,), th))                      # RZ|1> = e^{+i th/2}|1>
        assert abs(o.state()[1 << q] - np.exp(-0.5j * th) * np.exp(0.5j * th)) < ZERO


def test_kat_hadamard_not():
    o = OracleState(5)
    for q in range(5):
        o.apply(one("H", (q,)))                           # testHadamard :66-91
        s = o.state()
        assert abs(s[0] - SQ2) < ZERO and abs(s[1 << q] - SQ2) < ZERO
        o.apply(one("H", (q,)))
        o.apply(one("X", (q,)))                           # testNOT :50-64
        assert abs(o.state()[1 << q] - 1) < ZERO
        o.apply(one("X", (q,)))


def test_kat_cnot_cr_iswap_sqiswap():
    n = 4
    for c in range(n):
        for t in range(n):
            if c == t:
                continue
            o = OracleState(n)
            o.apply(one("X", (c,)))
            o.apply(one("CNOT", (c, t)))                  # testCNOT :178-210
            assert abs(o.state()[(1 << c) | (1 << t)] - 1) < ZERO
            th = 0.77
            o.apply(one("CR", (c, t), th))                # testCR :212-248: |11> -> e^{i th}|11>
            assert abs(o.state()[(1 << c) | (1 << t)] - np.exp(1j * th)) < ZERO
            o = OracleState(n)
            o.apply(one("X", (c,)))
            o.apply(one("ISWAP", (c, t)))                 # testISWAP :250-289: +i
            assert abs(o.state()[1 << t] - 1j) < ZERO
            o = OracleState(n)
            o.apply(one("X", (c,)))
            o.apply(one("SQISWAP", (c, t)))               # testSqiSWAP :291-333: +i/sqrt2
            s = o.state()
            assert abs(s[1 << c] - SQ2) < ZERO and abs(s[1 << t] - 1j * SQ2) < ZERO


def test_kat_toffoli_and_controlled():
    o = OracleState(4)
    o.apply(one("X", (0,)))
    o.apply(one("X", (2,)))
    o.apply(one("TOFFOLI", (0, 2, 3)))                    # testToffoli :380-446
    assert abs(o.state()[0b1101] - 1) < ZERO
    o = OracleState(4)
    o.apply(one("X", (1,)))
    o.apply(one("RZ", (3,), 0.5, 0, ctrl=(1,)))           # testControledRZ :634-683
    assert abs(o.state()[0b0010] - np.exp(-0.25j)) < ZERO


def test_kat_measure_and_pmeasure():
    o = OracleState(3)
    for q in range(3):
        o.apply(one("H", (q,)))
    p = o.probs([2, 1, 0])                                 # testPMeasure :360-378 (1/8 each)
    assert np.all(np.abs(p - 0.125) < 1e-12)
    # testQubitMeasure :335-358 - statistical
    rng = np.random.default_rng(0)
    ones = 0
    for _ in range(2000):
        o = OracleState(1)
        o.apply(one("H", (0,)))
        ones += o.measure(0, rng.uniform())
    assert abs(ones / 2000 - 0.5) < 0.05


def test_rng16807_matches_reference_stream():
    import ctypes as C
    from oracle.pyoracle import oracle_lib
    s = C.c_int(1)
    v = [oracle_lib().orc_rand16807(C.byref(s)) for _ in range(3)]
    assert s.value == 1622650073    # Park-Miller: 16807^3 mod (2^31 - 1)
    assert all(0 < x < 1 for x in v)
