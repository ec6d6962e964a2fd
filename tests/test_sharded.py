"""Sharded state (no GPU): the swap schedule against the oracle, and the half
exchange between gloo ranks (world sizes 2 and 4) on CPU tensors.

The ranks' local engine here is the oracle on each shard (a stand-in for the
GPU shards, which tests/test_gpu_sharded.py runs); the check is the oracle on
the whole state."""
import os
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle.pyoracle import OracleState
from qpanda_b200 import circuits
from qpanda_b200.capi import GATE_DTYPE, OP
from qpanda_b200.sharded import (LocalExchanger, NcclExchanger, ShardedState, gather_logical, gate_qubits,
                                 schedule, schedule_from)


def swap_gate(a, b):
    g = np.zeros((), dtype=GATE_DTYPE)
    g["op"] = OP["SWAP"]
    g["q"] = [a, b, 0]
    return g


def full_reference(n, gates):
    o = OracleState(n)
    o.apply(gates)
    return o.state()


def run_schedule_on_full(n, g_bits, gates, pos0=None):
    """Replay schedule steps on one full state: local steps as given, a swap of
    rank bit j with local position p as SWAP of physical bits L+j and p."""
    L = n - g_bits
    o = OracleState(n)
    if pos0 is None:
        steps, pos = schedule(n, g_bits, gates)
    else:
        steps, pos = schedule_from(n, g_bits, gates, pos0)
    for st in steps:
        if st[0] == "local":
            for rec in st[1]:
                assert all(q < L for q in gate_qubits(rec))
            o.apply(st[1])
        else:
            _, j, p = st
            assert 0 <= j < g_bits and 0 <= p < L
            o.apply(np.array([swap_gate(L + j, p)], dtype=GATE_DTYPE))
    return o.state(), pos, steps


@pytest.mark.parametrize("n,g_bits", [(8, 1), (10, 2), (11, 3), (9, 4)])
def test_schedule_reproduces_circuit(n, g_bits):
    gates = circuits.random_layers(n, 5, 50 + n + g_bits, iswap_frac=0.3)
    st, pos, steps = run_schedule_on_full(n, g_bits, gates)
    got = gather_logical([st], n, 0, pos)
    assert np.abs(got - full_reference(n, gates)).max() < 1e-12
    assert any(s[0] == "swap" for s in steps)


def test_schedule_every_gate_kind_and_controls():
    from tests.golden.make_golden import every_gate_circuit
    n, g_bits = 8, 2
    gates = every_gate_circuit(n, 5)
    st, pos, _ = run_schedule_on_full(n, g_bits, gates)
    assert np.abs(gather_logical([st], n, 0, pos) - full_reference(n, gates)).max() < 1e-12


def test_schedule_prefers_contiguous_halves():
    """Single-qubit gates on the top (global) qubits swap with the top local
    position, whose half of a shard is one contiguous block."""
    n, g_bits = 10, 2
    spec = [("H", (9,)), ("H", (8,)), ("RX", (9,), 0.3)]
    steps, _ = schedule(n, g_bits, circuits.make_gates(spec))
    swaps = [s for s in steps if s[0] == "swap"]
    assert swaps and swaps[0][2] == n - g_bits - 1


def test_local_exchanger_on_host_matches():
    """All shards in one process on CPU tensors (the exchanger the single-GPU
    test uses on device tensors)."""
    n, g_bits = 10, 2
    L = n - g_bits
    gates = circuits.random_layers(n, 4, 8, iswap_frac=0.2)
    engines = [OracleShard(L, r) for r in range(1 << g_bits)]
    s = ShardedState(n, g_bits, engines, LocalExchanger(1 << g_bits))
    s.run(gates)
    got = gather_logical([e.o.state() for e in engines], n, g_bits, s.pos)
    assert np.abs(got - full_reference(n, gates)).max() < 1e-12
    assert s.swaps > 0


class OracleShard:
    """Test engine: the oracle on one shard's 2^L amplitudes."""

    def __init__(self, L, rank_bits):
        self.o = OracleState(L)
        if rank_bits:
            self.o.view()[:] = 0

    def apply(self, records):
        self.o.apply(records)

    def synchronize(self):
        pass

    def tensor(self):
        return torch.from_numpy(self.o.view())


def _rank_main(rank, world, port, n, out_dir, chunk_amps=1 << 26):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    g_bits = world.bit_length() - 1
    L = n - g_bits
    gates = circuits.random_layers(n, 4, 123 + world, iswap_frac=0.3)
    eng = OracleShard(L, rank)
    x = NcclExchanger(chunk_amps=chunk_amps)
    s = ShardedState(n, g_bits, [eng], x)
    s.run(gates)
    if x.stage is not None:                   # one staging buffer, bounded, for every swap
        assert x.stage.numel() <= chunk_amps
    np.save(os.path.join(out_dir, f"shard{rank}.npy"), eng.o.state())
    if rank == 0:
        np.save(os.path.join(out_dir, "pos.npy"), np.array(s.pos))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,chunk", [(2, 1 << 26), (4, 1 << 26), (2, 32), (4, 8)])
def test_gloo_ranks_exchange_halves(world, chunk):
    """Swaps in one piece, and in many chunks through a small staging buffer
    (down to pieces of one row of a strided half)."""
    import socket
    n = 10
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, port, n, d, chunk), nprocs=world, join=True,
                           start_method="spawn")
        shards = [np.load(os.path.join(d, f"shard{r}.npy")) for r in range(world)]
        pos = list(np.load(os.path.join(d, "pos.npy")))
    g_bits = world.bit_length() - 1
    gates = circuits.random_layers(n, 4, 123 + world, iswap_frac=0.3)
    got = gather_logical(shards, n, g_bits, pos)
    assert np.abs(got - full_reference(n, gates)).max() < 1e-12
