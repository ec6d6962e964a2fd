"""Batched circuits in one persistent launch (qs_batch_*), against the oracle.

<Z_i Z_{i+1}> = P00 + P11 - P01 - P10 of the marginal on (i, i+1), which the
reference computes with pMeasure (CPUQuantumGates.cpp:159-190).  Tolerance
1e-5 (complex64 state, fused tensor-core passes) against the FP64 oracle.
"""
import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import Batch, autotune_batch, circuits
from qpanda_b200.capi import QSError

pytestmark = pytest.mark.gpu
TOL = 1e-5


def oracle_zz(n, g):
    o = OracleState(n)
    o.apply(g)
    zz = []
    for i in range(n - 1):
        p = o.probs([i, i + 1])
        zz.append(p[0] - p[1] - p[2] + p[3])
    return np.array(zz), o.state()


def small_sweep(seed, count=20):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        q = int(rng.choice([3, 8, 10, 11, 12, 13, 15, 16]))
        L = int(rng.integers(1, 6))
        out.append((q, circuits.vqe_ansatz(q, L, seed=seed * 1000 + k)))
    return out


def test_batch_zz_and_states_match_oracle(need_gpu):
    sweep = small_sweep(1)
    b = Batch(sweep)
    b.run()
    zz = b.zz()
    for k, (q, g) in enumerate(sweep):
        ref_zz, ref_state = oracle_zz(q, g)
        assert np.abs(zz[k] - ref_zz).max() < TOL, (k, q)
        assert np.abs(b.state(k) - ref_state).max() < TOL, (k, q)


def test_batch_replay_and_options_agree(need_gpu):
    sweep = small_sweep(2, count=12)
    base = Batch(sweep)
    base.run()
    z0 = base.zz()
    base.run()                               # graph replay
    z1 = base.zz()
    for a, c in zip(z0, z1):
        assert np.array_equal(a, c)
    for ms in (1, 2, 3):
        for lq in (3, 5):
            for order in (0, 1):
                b = Batch(sweep, max_sub=ms, low_qubits=lq, order=order, use_graph=0)
                b.run()
                for a, c in zip(z0, b.zz()):
                    assert np.abs(a - c).max() < 2 * TOL


def test_batch_general_circuits(need_gpu):
    """Any gate mix (random layers with iSWAP, QFT), not only the ansatz."""
    sweep = [(13, circuits.random_layers(13, 4, 5, iswap_frac=0.3)), (12, circuits.qft(12)),
             (9, circuits.random_layers(9, 6, 6))]
    b = Batch(sweep)
    b.run()
    zz = b.zz()
    for k, (q, g) in enumerate(sweep):
        ref_zz, ref_state = oracle_zz(q, g)
        assert np.abs(zz[k] - ref_zz).max() < TOL
        assert np.abs(b.state(k) - ref_state).max() < TOL


def test_batch_autotune_and_limits(need_gpu):
    sweep = small_sweep(3, count=16)
    opts, ms = autotune_batch(sweep, stride=2)
    assert 1 <= opts.max_sub <= 3 and opts.low_qubits in (3, 5) and ms > 0
    b = Batch(sweep, opts=opts)
    b.run()
    assert len(b.zz()) == 16
    with pytest.raises(QSError):
        Batch([(25, circuits.vqe_ansatz(25, 1, seed=0))])


def test_fusion_width_4_and_tuning_cache(need_gpu, tmp_path):
    """Blocks of at most 4 qubits (one of the autotuner's fusion widths) give
    the same <ZZ> as the oracle; the cached autotuner tunes once, then
    returns the same options from its file without timing."""
    import ctypes as C

    from qpanda_b200.capi import BatchOpts, check, lib
    sweep = small_sweep(3, count=10)
    o = BatchOpts()
    check(lib().qs_batch_default_opts(C.byref(o)))
    o.block_qubits = 4
    b = Batch(sweep, opts=o)
    b.run()
    for zz, (q, g) in zip(b.zz(), sweep):
        ref, _ = oracle_zz(q, g)
        assert np.abs(zz - ref).max() < TOL, q
    b.close()
    cache = tmp_path / "tune.txt"
    o1, ms1, hit1 = autotune_batch(sweep, stride=2, cache=cache)
    o2, ms2, hit2 = autotune_batch(sweep, stride=2, cache=cache)
    assert not hit1 and hit2
    assert (o1.block_qubits, o1.max_sub, o1.low_qubits, o1.order) == (o2.block_qubits, o2.max_sub, o2.low_qubits,
                                                                      o2.order)
    assert o1.block_qubits in (4, 5)
    assert len(cache.read_text().splitlines()) == 1


@pytest.mark.parametrize("tmem", [1, 0])
def test_batch_tile_in_tensor_or_shared_memory(need_gpu, tmem):
    """The batched kernels with the tile in tensor memory (k_batch_tmem, the
    default for passes of up to two blocks) and in shared memory (k_batch)
    both give the oracle's <ZZ> and states, with both fusion widths."""
    sweep = small_sweep(4, count=16)
    for bq in (5, 4):
        b = Batch(sweep, tile_in_tmem=tmem, block_qubits=bq)
        b.run()
        zz = b.zz()
        for k, (q, g) in enumerate(sweep):
            ref_zz, ref_state = oracle_zz(q, g)
            assert np.abs(zz[k] - ref_zz).max() < TOL, (k, q, bq)
            assert np.abs(b.state(k) - ref_state).max() < TOL, (k, q, bq)
        b.close()
