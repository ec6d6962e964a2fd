"""GPU parity of the plain per-gate path against the oracle (C-ABI calls).

Tolerances (max |amplitude difference|, states of norm 1): 1e-12 for
complex128, 1e-5 for complex64, against the FP64 oracle.
"""
import glob
import math
import os

import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import StateVector, circuits
from qpanda_b200.capi import GATE_DTYPE, OP, QSError

pytestmark = pytest.mark.gpu
TOL = {"c128": 1e-12, "c64": 1e-5}
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def gate(op, q, theta=0.0, dagger=0, ctrl=()):
    g = np.zeros(1, dtype=GATE_DTYPE)
    g["op"] = OP[op]
    g["q"][0, :len(q)] = q
    g["theta"] = theta
    g["dagger"] = dagger
    g["nctrl"] = len(ctrl)
    g["ctrl"][0, :len(ctrl)] = ctrl
    return g


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def run_both(n, gates, dt, init=None):
    sv = StateVector(n, dt)
    o = OracleState(n)
    if init is not None:
        sv.set_state(init.astype(np.complex64) if dt == "c64" else init)
        o.set_state(init.astype(np.complex64).astype(np.complex128) if dt == "c64" else init)
    sv.apply(gates)
    o.apply(gates)
    got = sv.get_state()
    sv.close()
    return got, o.state()


def inverse(gates):
    inv = gates[::-1].copy()
    flip = np.isin(inv["op"], [OP[k] for k in ("RX", "RY", "RZ", "CR", "ISWAP", "SQISWAP")])
    inv["dagger"][flip] = 1 - inv["dagger"][flip]
    return inv


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("n", [1, 2, 5, 13])
def test_single_qubit_gates_every_target(need_gpu, dt, n):
    init = random_state(n, n)
    for q in range(n):
        for op, th, dag in (("H", 0, 0), ("X", 0, 0), ("RX", 0.3, 0), ("RX", 1.1, 1), ("RY", 2.2, 0),
                            ("RY", 0.4, 1), ("RZ", 5.0, 0), ("RZ", 0.9, 1)):
            got, ref = run_both(n, gate(op, (q,), th, dag), dt, init)
            assert np.abs(got - ref).max() < TOL[dt], (op, q, dag)


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("n", [2, 6, 12])
def test_two_qubit_gates_every_pair(need_gpu, dt, n):
    init = random_state(n, 100 + n)
    pairs = [(a, b) for a in range(n) for b in range(n) if a != b]
    if n > 6:
        pairs = [p for p in pairs if 0 in p or n - 1 in p or p == (3, 5)]
    for a, b in pairs:
        for op, th, dag in (("CNOT", 0, 0), ("CR", 0.7, 0), ("CR", 0.7, 1), ("ISWAP", 0, 0),
                            ("ISWAP", 0, 1), ("SQISWAP", 0, 0), ("SQISWAP", 0, 1), ("SWAP", 0, 0)):
            got, ref = run_both(n, gate(op, (a, b), th, dag), dt, init)
            assert np.abs(got - ref).max() < TOL[dt], (op, a, b, dag)


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_three_qubit_and_controlled(need_gpu, dt):
    n = 7
    init = random_state(n, 7)
    rng = np.random.default_rng(1)
    for _ in range(40):
        a, b, c, d, e = (int(x) for x in rng.choice(n, 5, replace=False))
        for g in (gate("TOFFOLI", (a, b, c)), gate("CSWAP", (a, b, c)),
                  gate("H", (a,), ctrl=(b, c)), gate("X", (a,), ctrl=(b,)),
                  gate("RX", (a,), 0.4, int(rng.integers(2)), ctrl=(b, c, d)),
                  gate("RY", (a,), 1.4, int(rng.integers(2)), ctrl=(0 if a else 1,)),
                  gate("RZ", (a,), 2.4, int(rng.integers(2)), ctrl=(b,)),
                  gate("CNOT", (a, b), ctrl=(c, d)), gate("TOFFOLI", (a, b, c), ctrl=(d, e)),
                  gate("CR", (a, b), 0.3, ctrl=(c,)), gate("ISWAP", (a, b), ctrl=(c,)),
                  gate("SQISWAP", (a, b), 0, 1, ctrl=(c, d))):
            got, ref = run_both(n, g, dt, init)
            assert np.abs(got - ref).max() < TOL[dt], g


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_golden_fixtures(need_gpu, path, dt):
    """The GPU path against outputs of the reference's own CPU backend."""
    d = np.load(path)
    n = int(d["n"])
    sv = StateVector(n, dt)
    if "init" in d:
        sv.set_state(d["init"])
    sv.apply(d["gates"])
    if "mqubits" in d:
        outs = [sv.measure(int(q), float(u)) for q, u in zip(d["mqubits"], d["muniforms"])]
        assert outs == d["outcomes"].tolist()
    assert np.abs(sv.get_state() - d["state"]).max() < TOL[dt]
    if "shots" in d and dt == "c128":
        assert np.array_equal(sv.sample(d["shot_qubits"], d["uniforms"]), d["shots"])
        pm = sv.pmeasure(d["pm_qubits"])
        assert np.allclose([p for _, p in pm], d["pm_p"], atol=1e-12)


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_random_circuit_n20_config0(need_gpu, dt):
    """The 20-qubit, 20-layer random circuit, amplitude by amplitude."""
    g = circuits.random_layers(20, 20, 2024)
    got, ref = run_both(20, g, dt)
    assert np.abs(got - ref).max() < TOL[dt]


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_qft_gaussian_input(need_gpu, dt):
    n = 16
    init = random_state(n, 16)
    got, ref = run_both(n, circuits.qft(n), dt, init)
    assert np.abs(got - ref).max() < TOL[dt]


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_generic_unitaries_vs_numpy(need_gpu, dt):
    n = 6
    rng = np.random.default_rng(5)
    init = random_state(n, 6)

    def rand_u(k):
        z = rng.normal(size=(k, k)) + 1j * rng.normal(size=(k, k))
        q, r = np.linalg.qr(z)
        return q * (np.diag(r) / np.abs(np.diag(r)))

    T = init.reshape([2] * n)          # axis n-1-q is qubit q
    for q0, q1, cm in ((0, 1, 0), (1, 0, 0), (4, 2, 0b1), (5, 0, 0b100), (2, 3, 0b110001)):
        U = rand_u(4)
        sv = StateVector(n, dt)
        sv.set_state(init)
        sv.apply_2q(q0, q1, U, cm)
        got = sv.get_state()
        ref = init.copy()
        for i in range(1 << n):
            if (i & cm) != cm or (i >> q0) & 1 or (i >> q1) & 1:
                continue
            idx = [i, i | 1 << q0, i | 1 << q1, i | 1 << q0 | 1 << q1]
            ref[idx] = U @ init[idx]
        assert np.abs(got - ref).max() < TOL[dt] * 4
    for q, cm in ((0, 0), (3, 0b10), (5, 0b11)):
        U = rand_u(2)
        sv = StateVector(n, dt)
        sv.set_state(init)
        sv.apply_1q(q, U, cm)
        ref = init.copy()
        for i in range(1 << n):
            if (i & cm) != cm or (i >> q) & 1:
                continue
            idx = [i, i | 1 << q]
            ref[idx] = U @ init[idx]
        assert np.abs(sv.get_state() - ref).max() < TOL[dt] * 2
    del T


def test_unitary_check_and_errors(need_gpu):
    sv = StateVector(4, "c128")
    with pytest.raises(QSError) as e:
        sv.apply_unitary_1q(0, [[1, 0], [0, 2]])
    assert e.value.code == -5
    with pytest.raises(QSError):
        sv.apply(gate("CNOT", (1, 1)))
    with pytest.raises(QSError):
        sv.apply(gate("H", (4,)))
    with pytest.raises(QSError):
        sv.apply(gate("RX", (0,), 0.1, ctrl=(0,)))
    sv.apply_unitary_1q(1, [[0, 1], [1, 0]])
    assert abs(sv.get_state()[2] - 1) < 1e-15


@pytest.mark.parametrize("dt", ["c64", "c128"])
def test_round_trip_28q(need_gpu, dt):
    """Full size property check: a random circuit followed by its inverse
    returns |0...0>; the norm stays 1 throughout."""
    n = 28 if dt == "c64" else 27
    g = circuits.random_layers(n, 2, 77, iswap_frac=0.3)
    g = np.concatenate([g, circuits.qft(n)[:60]])
    sv = StateVector(n, dt)
    sv.apply(g)
    assert abs(sv.norm2() - 1) < (1e-5 if dt == "c64" else 1e-12)
    sv.apply(inverse(g))
    p0 = sv.probs([0, 1, 2, n - 1])
    assert abs(p0[0] - 1) < (1e-5 if dt == "c64" else 1e-12)
    assert abs(sv.norm2() - 1) < (1e-5 if dt == "c64" else 1e-12)


def _one_by_one(sv, gates):
    import ctypes as C

    from qpanda_b200 import lib
    from qpanda_b200.capi import check
    g = np.ascontiguousarray(gates)
    for i in range(len(g)):
        check(lib().qs_gate_apply(sv.handle, C.c_void_p(g[i:i + 1].ctypes.data)))


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("n", [5, 6, 9, 10, 12, 18, 20])
def test_staged_runs_match_gate_by_gate(need_gpu, dt, n):
    """qs_gates_apply runs consecutive gates whose targets share one tile's
    10 qubits (any qubits, with the lowest ones) through shared memory and
    registers in one pass (qs_lowstage.cu): the same state as the gates one
    by one on the streaming kernels, and the oracle's within the usual bar.
    Random layers (rotations on every qubit, CNOT / iSWAP on random pairs),
    the QFT (long runs of controlled phases) and every gate kind with control
    lists."""
    from tests.golden.make_golden import every_gate_circuit
    for g in (circuits.random_layers(n, 4, 70 + n, iswap_frac=0.3), circuits.qft(n),
              every_gate_circuit(n, 5 + n)):
        init = random_state(n, n)
        a, b = StateVector(n, dt), StateVector(n, dt)
        a.set_state(init)
        b.set_state(init)
        a.apply(g)
        _one_by_one(b, g)
        mx, _ = a.diff(b)
        # FP32 rounding level (a few ulps of amplitudes up to ~0.5 on the
        # narrow states; the two kernels may contract multiply-adds differently)
        assert mx <= (1e-15 if dt == "c128" else 5e-7), mx
        o = OracleState(n)
        o.set_state(init)
        o.apply(g)
        assert np.abs(a.get_state() - o.state()).max() < TOL[dt]
        a.close()
        b.close()
