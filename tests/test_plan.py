"""The fusion planner (host C++), checked on the CPU: applying its FP64 block
matrices to a state must reproduce the oracle's gate-by-gate result."""
import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import FusionPlan, circuits
from qpanda_b200.capi import QSError


def apply_block(v, n, qubits, U):
    """v' = U on the given qubits (row/col bit b = qubits[b])."""
    T = v.reshape([2] * n)                      # axis n-1-q is qubit q
    axes = [n - 1 - q for q in qubits[::-1]]    # most significant block bit first
    T = np.moveaxis(T, axes, list(range(5)))
    sh = T.shape
    T = (U @ T.reshape(32, -1)).reshape(sh)
    return np.moveaxis(T, list(range(5)), axes).reshape(-1)


@pytest.mark.parametrize("kernel", ["single", "tiled"])
@pytest.mark.parametrize("case", ["layers", "qft", "every_gate", "vqe"])
def test_plan_blocks_reproduce_oracle(case, kernel):
    n = 13
    if case == "layers":
        g = circuits.random_layers(n, 6, 3, iswap_frac=0.3)
    elif case == "qft":
        g = circuits.qft(n)
    elif case == "vqe":
        g = circuits.vqe_ansatz(n, 3, seed=4)
    else:
        from tests.golden.make_golden import every_gate_circuit
        g = every_gate_circuit(n, 5)
    rng = np.random.default_rng(1)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    o = OracleState(n)
    o.set_state(v)
    o.apply(g)
    p = FusionPlan(n, g, kernel=kernel)
    nb = p.num_blocks()
    assert 0 < nb < len(g)
    assert 0 < p.num_launches() <= nb
    w = v.copy()
    for i in range(nb):
        q, U = p.block(i)
        assert q == sorted(q) and len(set(q)) == 5
        assert np.abs(U.conj().T @ U - np.eye(32)).max() < 1e-12
        w = apply_block(w, n, q, U)
    assert np.abs(w - o.state()).max() < 1e-12


def test_plan_pass_count_32q():
    g = circuits.random_layers(32, 16, 20240601, iswap_frac=0.1)
    p = FusionPlan(32, g, kernel="single")
    # closure-first fusion with look-ahead: 63 blocks (89 in plain gate order)
    assert p.num_blocks() <= 64 and p.num_launches() == p.num_blocks()   # vs ~640 per-gate passes
    t3 = FusionPlan(32, g, kernel="tiled", max_sub=3)
    assert t3.num_launches() <= 38        # up to 3 blocks per pass within 12 tile qubits
    t2 = FusionPlan(32, g, kernel="tiled")  # default: up to 2 blocks per pass
    assert t3.num_launches() <= t2.num_launches() <= 32
    assert FusionPlan(32, g, kernel="tiled", low_qubits=2).num_launches() <= 32
    for T, blocks in t2.passes():
        assert 1 <= len(blocks) <= 2 and T[:3] == [0, 1, 2] and T == sorted(T)
        assert all(set(q) <= set(T) for q in blocks)


def test_plan_rejects_wide_gates_and_bad_width():
    g = circuits.make_gates([("TOFFOLI", (0, 1, 2))])
    g["nctrl"] = 3
    g["ctrl"][0, :3] = [3, 4, 5]
    with pytest.raises(QSError):
        FusionPlan(12, g)
    with pytest.raises(QSError):
        FusionPlan(12, circuits.qft(12), max_k=6)


def test_plan_rejects_bad_tiled_options():
    """remap must be 0..2 and threads_per_row 1 or 2; both valid values build."""
    g = circuits.qft(12)
    for kw in ({"remap": 3}, {"threads_per_row": 0}, {"threads_per_row": 3}):
        with pytest.raises(QSError):
            FusionPlan(12, g, **kw)
    for kw in ({"remap": 2}, {"threads_per_row": 2}):
        FusionPlan(12, g, **kw).close()
