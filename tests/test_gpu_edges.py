"""Edge cases of the GPU paths against the oracle: empty gate lists, the
smallest states (1 qubit; 11 and 12 qubits around the tiled kernels' lower
limit), a measurement whose outcome is certain, the smallest batches and a
request loop that is closed without requests."""
import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import Batch, FusionPlan, Server, StateVector, circuits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dt", ["c64", "c128"])
def test_empty_gate_list_leaves_the_state(need_gpu, dt):
    n = 14
    rng = np.random.default_rng(3)
    init = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    init /= np.linalg.norm(init)
    npdt = np.complex64 if dt == "c64" else np.complex128
    sv = StateVector(n, dt)
    sv.set_state(init.astype(npdt))
    before = sv.get_state()
    sv.apply(circuits.make_gates([]))
    assert np.array_equal(sv.get_state(), before)
    p = FusionPlan(n, circuits.make_gates([]))
    assert p.num_launches() == 0
    p.apply(sv)
    assert np.array_equal(sv.get_state(), before)
    p.close()
    sv.close()


@pytest.mark.parametrize("dt,tol", [("c64", 1e-6), ("c128", 1e-14)])
def test_one_qubit_state(need_gpu, dt, tol):
    g = circuits.make_gates([("H", (0,)), ("RY", (0,), 0.7), ("RZ", (0,), 1.3), ("X", (0,)), ("RX", (0,), 2.1, 1)])
    sv = StateVector(1, dt)
    sv.apply(g)
    o = OracleState(1)
    o.apply(g)
    assert np.abs(sv.get_state() - o.state()).max() < tol
    assert np.abs(sv.probs() - o.probs()).max() < tol
    if dt == "c128":             # the reference's precision: shots bit-exact
        u = np.random.default_rng(1).uniform(size=(64, 1))
        qs = np.array([0], dtype=np.int32)
        assert np.array_equal(sv.sample(qs, u), o.sample(qs, u))
    assert sv.measure(0, 0.4) == o.measure(0, 0.4)
    assert np.abs(sv.get_state() - o.state()).max() < tol
    sv.close()


@pytest.mark.parametrize("n", [11, 12])
def test_plans_at_the_tiled_kernels_lower_limit(need_gpu, n):
    """11 qubits: the plan's gates run on the per-gate kernels; 12: one tile,
    the tensor-core passes (a single tile per pass)."""
    g = circuits.random_layers(n, 6, 400 + n, iswap_frac=0.2)
    sv = StateVector(n, "c64")
    p = FusionPlan(n, g)
    p.apply(sv)
    p.status(sv)
    o = OracleState(n)
    o.apply(g)
    assert np.abs(sv.get_state() - o.state()).max() < 1e-5
    assert abs(sv.norm2() - 1) < 1e-6
    one = circuits.make_gates([("RY", (n - 1,), 0.3)])
    q = FusionPlan(n, one)
    q.apply(sv)
    o.apply(one)
    assert np.abs(sv.get_state() - o.state()).max() < 1e-5
    p.close()
    q.close()
    sv.close()


@pytest.mark.parametrize("dt", ["c64", "c128"])
def test_measurement_of_a_certain_outcome(need_gpu, dt):
    """A basis state: P(0) of each qubit is 0 or 1, and any uniform in (0, 1)
    gives the certain outcome, the state unchanged (a renormalisation by 1)."""
    n = 13
    g = circuits.make_gates([("X", (q,)) for q in (0, 5, 12)])
    sv = StateVector(n, dt)
    sv.apply(g)
    o = OracleState(n)
    o.apply(g)
    for q, u in ((0, 0.01), (5, 0.99), (7, 0.5), (12, 0.5)):
        assert sv.prob_zero(q) == o.prob_zero(q)
        assert sv.measure(q, u) == o.measure(q, u) == (1 if q in (0, 5, 12) else 0)
    assert np.array_equal(sv.get_state(), o.state())
    sv.close()


def test_smallest_batches(need_gpu):
    """One circuit; and circuits narrower than a tile (1 and 3 qubits, padded
    with idle qubits in |0>) beside a wider one."""
    for sweep in ([(12, circuits.vqe_ansatz(12, 2, seed=1))],
                  [(1, circuits.make_gates([("RY", (0,), 0.4), ("RZ", (0,), 0.2)])),
                   (3, circuits.vqe_ansatz(3, 2, seed=2)), (13, circuits.vqe_ansatz(13, 3, seed=3))]):
        b = Batch(sweep)
        b.run()
        zz = b.zz()
        for z, (q, g) in zip(zz, sweep):
            o = OracleState(q)
            o.apply(g)
            ref = [float(p[0] - p[1] - p[2] + p[3]) for p in (o.probs([i, i + 1]) for i in range(q - 1))]
            assert len(z) == q - 1
            if ref:
                assert np.abs(np.asarray(z) - ref).max() < 1e-5, q
        b.close()


def test_request_loop_closed_without_requests(need_gpu):
    srv = Server(slots=2)
    srv.close()
