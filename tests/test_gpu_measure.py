"""GPU parity of probabilities, measurement collapse, pMeasure and shots."""
import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import StateVector, circuits
from qpanda_b200.capi import QSError

pytestmark = pytest.mark.gpu
TOL = {"c128": 1e-12, "c64": 1e-5}


def prepared(n, dt, seed, layers=6):
    g = circuits.random_layers(n, layers, seed, iswap_frac=0.2)
    sv = StateVector(n, dt)
    sv.apply(g)
    o = OracleState(n)
    o.apply(g)
    return sv, o


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("n", [1, 3, 9, 14])
def test_prob_zero_every_qubit(need_gpu, dt, n):
    sv, o = prepared(n, dt, n)
    for q in range(n):
        assert abs(sv.prob_zero(q) - o.prob_zero(q)) < TOL[dt]


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_measure_sequence(need_gpu, dt):
    n = 12
    sv, o = prepared(n, dt, 3)
    rng = np.random.default_rng(4)
    for q in rng.permutation(n)[:8]:
        u = float(rng.uniform())
        assert sv.measure(int(q), u) == o.measure(int(q), u)
        assert np.abs(sv.get_state() - o.state()).max() < TOL[dt] * 10


def test_measure_deterministic_outcome_and_zero_probability(need_gpu):
    sv = StateVector(3, "c128")
    assert sv.measure(1, 0.999) == 0          # |000>: p0 = 1, (float)u <= 1
    with pytest.raises(QSError):
        sv.measure(1, 2.0)        # (float)u > 1 selects outcome 1, whose probability is 0


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("n", [4, 13, 16])
def test_probs_subsets(need_gpu, dt, n):
    sv, o = prepared(n, dt, 10 + n)
    rng = np.random.default_rng(n)
    subsets = [list(range(n)), list(range(n))[::-1], [0], [n - 1], [n - 1, 0],
               list(rng.permutation(n)[: n // 2]), list(rng.permutation(n)[: max(1, n - 2)])]
    for qs in subsets:
        p = sv.probs(qs)
        assert np.abs(p - o.probs(qs)).max() < TOL[dt], qs
        assert abs(p.sum() - 1) < TOL[dt] * 10


def test_probs_large_state_subsets(need_gpu):
    """Marginals of a 26-qubit state: sums over many chunks and slices."""
    n = 26
    g = circuits.random_layers(n, 1, 8)
    sv = StateVector(n, "c128")
    sv.apply(g)
    full = sv.probs(list(range(n)))
    assert abs(full.sum() - 1) < 1e-12
    P = full.reshape([2] * n)               # axis n-1-q is qubit q
    for qs in ([25], [0, 25], [3, 17, 24], [1, 2, 13, 20, 21, 22]):
        axes = tuple(n - 1 - q for q in range(n) if q not in qs)
        marg = P.sum(axis=axes)             # remaining axes ordered by descending qubit
        kept = sorted(qs, reverse=True)
        perm = [kept.index(q) for q in qs[::-1]]
        ref = np.transpose(marg, perm).reshape(-1)
        assert np.abs(sv.probs(qs) - ref).max() < 1e-12


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_pmeasure_top10(need_gpu, dt):
    n = 10
    sv, o = prepared(n, dt, 21)
    qs = [2, 7, 0, 9, 4]
    p = o.probs(qs)
    order = sorted(range(len(p)), key=lambda i: (-p[i], i))[:10]
    got = sv.pmeasure(qs)
    assert [i for i, _ in got] == order
    assert np.allclose([v for _, v in got], p[order], atol=TOL[dt])


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_shots_match_sequential_measurement(need_gpu, dt):
    """Bitstrings equal the oracle's per-shot re-measurement, given the same
    uniforms (1024 shots at 14 qubits; 64 shots of the 20-qubit circuit)."""
    for n, layers, shots in ((14, 8, 1024), (20, 20, 64)):
        g = circuits.random_layers(n, layers, 500 + n)
        sv = StateVector(n, dt)
        sv.apply(g)
        o = OracleState(n)
        if dt == "c64":
            o.set_state(np.zeros(1 << n))
            o.set_state(sv.get_state(np.complex64).astype(np.complex128))
        else:
            o.apply(g)
        qs = np.arange(n, dtype=np.int32)
        u = np.random.default_rng(n).uniform(size=(shots, n))
        assert np.array_equal(sv.sample(qs, u), o.sample(qs, u))


def test_shots_subset_and_order(need_gpu):
    n = 11
    sv, o = prepared(n, "c128", 77)
    qs = np.array([5, 0, 10, 3], dtype=np.int32)
    u = np.random.default_rng(1).uniform(size=(500, 4))
    assert np.array_equal(sv.sample(qs, u), o.sample(qs, u))


def test_shots_deep_levels(need_gpu):
    """More than 20 measured qubits: levels past the materialised tree sum
    amplitudes directly."""
    n = 23
    g = circuits.random_layers(n, 3, 99)
    sv = StateVector(n, "c128")
    sv.apply(g)
    o = OracleState(n)
    o.apply(g)
    qs = np.array(list(range(n))[::-1], dtype=np.int32)
    u = np.random.default_rng(2).uniform(size=(6, n))
    assert np.array_equal(sv.sample(qs, u), o.sample(qs, u))


def test_norm_and_inner(need_gpu):
    n = 15
    g = circuits.random_layers(n, 4, 1)
    a, b = StateVector(n, "c64"), StateVector(n, "c128")
    a.apply(g)
    b.apply(g)
    assert abs(b.norm2() - 1) < 1e-12
    ip = a.inner(b)
    assert abs(abs(ip) ** 2 - 1) < 1e-6
    ref = np.vdot(a.get_state(), b.get_state())
    assert abs(ip - ref) < 1e-12


def test_probs_and_shots_with_scratch_growth(need_gpu):
    """22 qubits with 20+ measured: the partial slices outgrow the initial
    scratch, which must be sized before any pointer into it is taken."""
    n = 22
    g = circuits.random_layers(n, 2, 31)
    sv = StateVector(n, "c128")
    sv.apply(g)
    o = OracleState(n)
    o.apply(g)
    qs = list(range(2, 22))
    assert np.abs(sv.probs(qs) - o.probs(qs)).max() < 1e-12
    qa = np.arange(n, dtype=np.int32)[::-1].copy()
    u = np.random.default_rng(3).uniform(size=(12, n))
    assert np.array_equal(sv.sample(qa, u), o.sample(qa, u))
