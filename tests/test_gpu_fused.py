"""GPU parity of the fused tensor-core path (qs_plan_apply, complex64).

Bar: max |amplitude error| <= 1e-5 against the FP64 oracle and state
fidelity |<oracle|fused>|^2 >= 1 - 1e-6.
"""
import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import FusionPlan, StateVector, circuits

pytestmark = pytest.mark.gpu
AMP_TOL, FID_TOL = 1e-5, 1e-6


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


# "tiled": the default tiled passes (the tile in tensor memory, k_tile_tmem,
# where a pass fits it); "tiled-smem": every pass on k_fused_tile.
KERNELS = ["single", "tiled", "tiled-smem"]


def make_plan(n, g, kernel="tiled", **kw):
    if kernel == "tiled-smem":
        return FusionPlan(n, g, kernel="tiled", tile_in_tmem=0, **kw)
    return FusionPlan(n, g, kernel=kernel, **kw)


def check_fused(n, g, init=None, kernel="tiled", **kw):
    sv = StateVector(n, "c64")
    o = OracleState(n)
    if init is not None:
        sv.set_state(init.astype(np.complex64))
        o.set_state(init.astype(np.complex64).astype(np.complex128))
    p = make_plan(n, g, kernel=kernel, **kw)
    p.apply(sv)
    p.status(sv)
    o.apply(g)
    got, ref = sv.get_state(), o.state()
    err = np.abs(got - ref).max()
    fid = abs(np.vdot(ref, got)) ** 2 / (np.vdot(got, got).real * np.vdot(ref, ref).real)
    assert err < AMP_TOL, err
    assert fid > 1 - FID_TOL, fid
    return p.num_blocks()


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("n", [12, 13, 17])
def test_fused_random_layers(need_gpu, n, kernel):
    nb = check_fused(n, circuits.random_layers(n, 8, 40 + n, iswap_frac=0.1), kernel=kernel)
    assert nb > 0


@pytest.mark.parametrize("kernel", KERNELS)
def test_fused_qft_gaussian(need_gpu, kernel):
    check_fused(14, circuits.qft(14), init=random_state(14, 2), kernel=kernel)


@pytest.mark.parametrize("kernel", KERNELS)
def test_fused_every_gate_kind(need_gpu, kernel):
    from tests.golden.make_golden import every_gate_circuit
    check_fused(12, every_gate_circuit(12, 9), init=random_state(12, 3), kernel=kernel)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("max_k", [3, 4])
def test_fusion_width_below_five(need_gpu, kernel, max_k):
    """Blocks of at most 3 or 4 qubits (fusion width 4 is the batch
    autotuner's other choice), applied as widened 5-qubit blocks."""
    n = 17
    g = np.concatenate([circuits.random_layers(n, 6, 600 + max_k, iswap_frac=0.2),
                        circuits.vqe_ansatz(n, 2, seed=max_k)])
    check_fused(n, g, init=random_state(n, 50 + max_k), kernel=kernel, max_k=max_k)


@pytest.mark.parametrize("max_sub", [1, 2, 3])
@pytest.mark.parametrize("low", [1, 3, 5])
def test_tiled_options(need_gpu, max_sub, low):
    """Every blocks-per-pass count and tile shape of the tiled kernel."""
    n = 15
    check_fused(n, circuits.random_layers(n, 6, 70 + max_sub + 10 * low, iswap_frac=0.2),
                init=random_state(n, max_sub), kernel="tiled")


def test_fused_block_positions(need_gpu):
    """Blocks on the lowest qubits (paired 16-byte loads), on the highest
    qubits, and straddling: one dense random 2-qubit-gate layer per case."""
    n = 15
    rng = np.random.default_rng(0)
    for qs in ([0, 1, 2, 3, 4], [10, 11, 12, 13, 14], [0, 5, 9, 13, 14], [1, 2, 3, 4, 5], [3, 7, 8, 11, 12]):
        spec = []
        for q in qs:
            spec.append(("RY", (q,), float(rng.uniform(0, 6.28))))
            spec.append(("RZ", (q,), float(rng.uniform(0, 6.28))))
        for a, b in zip(qs[:-1], qs[1:]):
            spec.append(("CNOT", (a, b)))
            spec.append(("SQISWAP", (b, a)))
        g = circuits.make_gates(spec)
        for kernel in KERNELS:
            p = make_plan(n, g, kernel=kernel)
            assert p.num_blocks() == 1 and p.block(0)[0] == sorted(qs)
            check_fused(n, g, init=random_state(n, qs[0] + 7), kernel=kernel)


@pytest.mark.parametrize("kernel", KERNELS)
def test_fused_vqe_and_reuse(need_gpu, kernel):
    n = 16
    g = circuits.vqe_ansatz(n, 4, seed=5)
    p = make_plan(n, g, kernel=kernel)
    a = StateVector(n, "c64")
    p.apply(a)
    p.apply(a)               # a plan applies repeatedly
    o = OracleState(n)
    o.apply(g)
    o.apply(g)
    assert np.abs(a.get_state() - o.state()).max() < AMP_TOL


@pytest.mark.parametrize("tmem", [1, 0])
@pytest.mark.parametrize("remap", [1, 2])
@pytest.mark.parametrize("max_sub", [1, 2, 3])
@pytest.mark.parametrize("n", [20, 21])
def test_tiled_remap(need_gpu, n, max_sub, remap, tmem):
    """Remapped passes (ping-pong through a second buffer, contiguous tile
    writes, natural order back at the end) at an even and an odd count of
    passes; a second application reuses the spare buffer, and releasing it
    leaves the state intact."""
    g = circuits.random_layers(n, 6, 90 + n + max_sub, iswap_frac=0.2)
    init = random_state(n, n + max_sub)
    check_fused(n, g, init=init, kernel="tiled", max_sub=max_sub, remap=remap, tile_in_tmem=tmem)
    sv = StateVector(n, "c64")
    sv.set_state(init.astype(np.complex64))
    p = FusionPlan(n, g, max_sub=max_sub, remap=remap, tile_in_tmem=tmem)
    p.apply(sv)
    p.apply(sv)
    p.status(sv)
    o = OracleState(n)
    o.set_state(init.astype(np.complex64).astype(np.complex128))
    o.apply(g)
    o.apply(g)
    sv.release_spare()
    assert np.abs(sv.get_state() - o.state()).max() < AMP_TOL


@pytest.mark.parametrize("remap", [0, 1])
@pytest.mark.parametrize("max_sub", [1, 2, 3])
@pytest.mark.parametrize("n", [13, 20])
def test_tiled_two_threads_per_row(need_gpu, n, max_sub, remap):
    """The 256-threads-per-lane variant of the tiled kernel (two threads per
    tile row, 16 columns each) in place and remapped."""
    g = circuits.random_layers(n, 6, 130 + n + max_sub, iswap_frac=0.2)
    check_fused(n, g, init=random_state(n, n + 7 * max_sub), kernel="tiled", max_sub=max_sub, remap=remap,
                threads_per_row=2)


@pytest.mark.parametrize("kernel,remap,tpr", [("single", 0, 1), ("tiled", 0, 1), ("tiled", 1, 1), ("tiled", 2, 1),
                                              ("tiled", 1, 2), ("tiled-smem", 1, 1)])
def test_fused_fidelity_26q_vs_fp64_gpu(need_gpu, kernel, remap, tpr):
    """26 qubits, 12 layers: fused complex64 against the complex128 per-gate
    path (itself pinned to the oracle by the other tests)."""
    n = 26
    g = circuits.random_layers(n, 12, 7, iswap_frac=0.1)
    f = StateVector(n, "c64")
    p = make_plan(n, g, kernel=kernel, remap=remap, threads_per_row=tpr)
    p.apply(f)
    p.status(f)
    d = StateVector(n, "c128")
    d.apply(g)
    ip = f.inner(d)
    fid = abs(ip) ** 2 / f.norm2()
    assert fid > 1 - FID_TOL, fid
    # the per-pass rescale and the plan's closing one keep the norm
    assert abs(f.norm2() - 1) < 1e-6, f.norm2()


def inverse(gates):
    """The circuit undone: gates reversed, each with its dagger flag flipped
    (the reference's isConjugate argument)."""
    inv = np.array(gates[::-1], copy=True)
    inv["dagger"] ^= 1
    return inv


@pytest.mark.parametrize("kernel,remap", [("single", 0), ("tiled", 0), ("tiled", 1), ("tiled-smem", 1)])
def test_round_trip_returns_to_zero_with_its_norm(need_gpu, kernel, remap):
    """A plan, then the plan of the inverse circuit, on |0...0>: the state comes
    back with |<0|psi>|^2 >= 1 - 1e-6.  In such a round trip the split
    products' rounding in the last passes is coherent with the state (the
    inverse block's entries are conjugates of the amplitudes it maps back):
    the last pass alone can drift the norm by 1e-5 (32 qubits), which no later
    pass rescales; the plan's closing rescale (k_norm_fix) keeps it within
    1e-6."""
    n = 26
    g = circuits.random_layers(n, 16, 20240601, iswap_frac=0.1)
    a, z = StateVector(n, "c64"), StateVector(n, "c64")
    for gates in (g, inverse(g)):
        p = make_plan(n, gates, kernel=kernel, remap=remap, low_qubits=2)
        p.apply(a)
        p.status(a)
        p.close()
        assert abs(a.norm2() - 1) < 1e-6, a.norm2()
    back = abs(a.inner(z)) ** 2
    assert back > 1 - FID_TOL, back


@pytest.mark.parametrize("kernel", KERNELS)
def test_fused_range_with_interleaved_probs(need_gpu, kernel):
    """Passes applied one at a time with a marginal computed in between give
    the same state as the whole plan (norm partials survive other calls)."""
    n = 20
    g = circuits.random_layers(n, 6, 11, iswap_frac=0.1)
    p = make_plan(n, g, kernel=kernel)
    a, b = StateVector(n, "c64"), StateVector(n, "c64")
    p.apply(a)
    for i in range(p.num_launches()):
        p.apply_range(b, i, 1)
        b.probs(list(range(n)))
    mx, _ = a.diff(b)
    assert mx == 0.0


def test_small_state_plan_runs_per_gate(need_gpu):
    n = 8
    g = circuits.random_layers(n, 5, 2)
    sv = StateVector(n, "c128")
    FusionPlan(n, g).apply(sv)
    o = OracleState(n)
    o.apply(g)
    assert np.abs(sv.get_state() - o.state()).max() < 1e-12


@pytest.mark.parametrize("remap", [0, 1])
def test_tile_in_tmem_matches_shared_memory_kernel(need_gpu, remap):
    """The two tiled kernels apply the same passes with the same split-BF16
    products: their results agree to FP32 accumulation-order differences,
    and each is within the bar of the oracle (checked above)."""
    n = 22
    g = circuits.random_layers(n, 10, 4242, iswap_frac=0.1)
    init = random_state(n, 5).astype(np.complex64)
    out = []
    for tmem in (1, 0):
        sv = StateVector(n, "c64")
        sv.set_state(init)
        p = FusionPlan(n, g, remap=remap, tile_in_tmem=tmem)
        p.apply(sv)
        p.status(sv)
        out.append(sv)
    mx, _ = out[0].diff(out[1])
    assert mx < 1e-6, mx


def test_bounded_wait_expires_and_reports(need_gpu):
    """The waits of the tensor-core kernels give up after a limit: a kernel
    that waits on an mbarrier nothing arrives on (qs_watchdog_selftest, 50 ms)
    returns, qs_plan_status reports it, and the context stays usable - a fused
    plan runs correctly right after."""
    import time

    from qpanda_b200 import lib
    from qpanda_b200.capi import QSError, check
    n = 14
    sv = StateVector(n, "c64")
    t0 = time.perf_counter()
    check(lib().qs_watchdog_selftest(sv.handle, 50000))
    with pytest.raises(QSError) as e:
        check(lib().qs_plan_status(sv.handle))
    assert "bounded wait" in str(e.value)
    assert time.perf_counter() - t0 < 5.0
    g = circuits.random_layers(n, 4, 3, iswap_frac=0.1)
    p = FusionPlan(n, g)
    p.apply(sv)
    p.status(sv)                               # cleared by the next application
    o = OracleState(n)
    o.apply(g)
    assert np.abs(sv.get_state() - o.state()).max() < AMP_TOL


def test_plan_autotune_picks_a_valid_plan(need_gpu):
    """qs_plan_autotune times the candidate options on the state and returns
    the fastest; a plan built with them gives the oracle's state."""
    from qpanda_b200 import autotune_plan
    n = 20
    g = circuits.random_layers(n, 6, 777, iswap_frac=0.1)
    sv = StateVector(n, "c64")
    best, ms = autotune_plan(sv, g, remap=True)
    assert ms > 0
    assert best.tile_in_tmem in (0, 1) and best.max_sub in (2, 3) and best.low_qubits in (1, 2, 3)
    assert best.remap == 1 and best.block_qubits == 5
    sv.reset()
    p = FusionPlan(n, g, remap=best.remap, max_sub=best.max_sub, low_qubits=best.low_qubits,
                   tile_in_tmem=best.tile_in_tmem)
    p.apply(sv)
    p.status(sv)
    o = OracleState(n)
    o.apply(g)
    assert np.abs(sv.get_state() - o.state()).max() < AMP_TOL
