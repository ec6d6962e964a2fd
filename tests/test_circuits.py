import math

import numpy as np

from qpanda_b200 import circuits
from qpanda_b200.capi import OP


def test_random_layers_structure():
    g = circuits.random_layers(20, 20, 0)
    assert len(g) == 20 * (20 + 10)
    two = g[np.isin(g["op"], [OP["CNOT"], OP["ISWAP"]])]
    assert len(two) == 200
    lay = g[:30]
    assert sorted(np.concatenate([lay[20:]["q"][:, 0], lay[20:]["q"][:, 1]]).tolist()) == list(range(20))
    assert np.all((g["theta"] >= 0) & (g["theta"] < 2 * math.pi))


def test_random_layers_iswap_fraction():
    g = circuits.random_layers(32, 16, 1, iswap_frac=0.1)
    n_isw = int(np.sum(g["op"] == OP["ISWAP"]))
    assert 20 < n_isw < 80          # 10% of 256 pairs


def test_qft_counts():
    g = circuits.qft(28)
    assert np.sum(g["op"] == OP["H"]) == 28
    assert np.sum(g["op"] == OP["CR"]) == 378
    assert np.sum(g["op"] == OP["SWAP"]) == 14


def test_vqe_counts():
    g = circuits.vqe_ansatz(10, 4, seed=0)
    assert len(g) == 4 * (10 + 10 + 9)


def test_gate_bytes():
    g = circuits.make_gates([("H", (0,)), ("CNOT", (0, 1)), ("CR", (0, 1), 0.3)])
    N = 1 << 10
    assert circuits.gate_bytes(g, 10, 8) == 2 * 8 * (N + N // 2 + N // 4)
