"""GPU: a sharded state with its shards in one process on one GPU (the
exchange as device copies), against the oracle on the whole state.  Ranks on
separate GPUs exchange through NCCL with the same code (NcclExchanger), which
tests/test_sharded.py runs on gloo ranks; this pool gives one GPU per run."""
import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import circuits
from qpanda_b200.sharded import GpuShard, LocalExchanger, ShardedState, gather_logical

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,tol,fused", [("c128", 1e-12, False), ("c64", 1e-5, False), ("c64", 1e-5, True)])
@pytest.mark.parametrize("n,g_bits", [(16, 1), (18, 2)])
def test_sharded_matches_oracle(need_gpu, n, g_bits, dtype, tol, fused):
    L = n - g_bits
    gates = circuits.random_layers(n, 6, 700 + n + g_bits, iswap_frac=0.2)
    engines = [GpuShard(L, dtype, r, fused=fused) for r in range(1 << g_bits)]
    s = ShardedState(n, g_bits, engines, LocalExchanger(1 << g_bits))
    s.run(gates)
    got = gather_logical([e.host() for e in engines], n, g_bits, s.pos)
    o = OracleState(n)
    o.apply(gates)
    assert np.abs(got - o.state()).max() < tol
    assert s.swaps > 0
    for e in engines:
        e.close()


def test_sharded_runs_continue_from_the_layout(need_gpu):
    """Two runs in a row: the second starts from the permuted layout the first
    left (no swap back in between)."""
    n, g_bits = 16, 2
    L = n - g_bits
    g1 = circuits.random_layers(n, 3, 1)
    g2 = circuits.qft(n)
    engines = [GpuShard(L, "c128", r) for r in range(4)]
    s = ShardedState(n, g_bits, engines, LocalExchanger(4))
    s.run(g1)
    s.run(g2)
    got = gather_logical([e.host() for e in engines], n, g_bits, s.pos)
    o = OracleState(n)
    o.apply(g1)
    o.apply(g2)
    assert np.abs(got - o.state()).max() < 1e-12
    for e in engines:
        e.close()
