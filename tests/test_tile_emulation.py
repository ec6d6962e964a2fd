"""CPU check of the tiled passes' index arithmetic (no GPU).

tests/tile_emu/tile_emu.cpp replays a fused plan on the host exactly as
k_fused_tile moves data - the library's own pass scheduler and layout tables,
the warp-contiguous staging copies, the swizzled scatter between blocks, the
in-place or remapped (ping-pong, contiguous tile writes) stores - with FP64
block contractions in place of the tensor cores.  The result must match the
FP64 oracle to rounding, and every staging slot, A slot and output amplitude
must be written exactly once.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import FusionPlan, circuits
from qpanda_b200.capi import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "qpanda_b200", "csrc")
LIBDIR = os.path.join(ROOT, "qpanda_b200", "_lib")
SRC = os.path.join(ROOT, "tests", "tile_emu", "tile_emu.cpp")


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    lib()                                     # the library must be built
    out = str(tmp_path_factory.mktemp("tile_emu") / "libtile_emu.so")
    cmd = ["/usr/local/cuda/bin/nvcc", "-O2", "-std=c++17", "-x", "cu", "-shared", "-Xcompiler", "-fPIC",
           "-gencode", "arch=compute_100a,code=sm_100a", SRC, "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
           "-L" + LIBDIR, "-lqsb200", "-Xlinker", "-rpath=" + LIBDIR, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    E = C.CDLL(out)
    E.tile_emu_apply.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)]
    E.tile_emu_apply.restype = C.c_int
    E.tile_emu_error.restype = C.c_char_p
    E.tile_emu_check_input.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int,
                                       C.POINTER(C.c_int)]
    E.tile_emu_check_input.restype = C.c_int
    E.tmem_emu_apply.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_longlong)]
    E.tmem_emu_apply.restype = C.c_int
    return E


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def run_emu(E, n, g, init, remap, kinds=None, tpr=1, **kw):
    """tpr: the kernel's threads per tile row (1: 128 threads per lane, 2: 256)."""
    p = FusionPlan(n, g, remap=remap, **kw)
    st = np.ascontiguousarray(init.astype(np.complex128))
    npass = C.c_int()
    k = (C.c_int * 3)()
    rc = E.tile_emu_apply(p.handle, n, st.ctypes.data, int(remap), int(tpr), C.byref(npass), k)
    if kinds is not None:
        for i in range(3):
            kinds[i] += k[i]
    assert rc == 0, E.tile_emu_error().decode()
    o = OracleState(n)
    o.set_state(init)
    o.apply(g)
    err = np.abs(st - o.state()).max()
    p.close()
    return err, npass.value


@pytest.mark.parametrize("tpr", [1, 2])
@pytest.mark.parametrize("remap", [0, 1, 2])
@pytest.mark.parametrize("max_sub,low", [(1, 3), (2, 3), (3, 3), (2, 1), (2, 5), (3, 4)])
def test_tiled_index_math_random_layers(emu, remap, max_sub, low, tpr):
    n = 16
    g = circuits.random_layers(n, 6, 300 + 10 * max_sub + low, iswap_frac=0.2)
    err, npass = run_emu(emu, n, g, random_state(n, 1), remap, tpr=tpr, max_sub=max_sub, low_qubits=low)
    assert npass >= 2
    assert err < 1e-10, err


@pytest.mark.parametrize("tpr", [1, 2])
@pytest.mark.parametrize("remap", [0, 1, 2])
@pytest.mark.parametrize("n", [12, 13, 17])
def test_tiled_index_math_sizes(emu, remap, n, tpr):
    """One tile (12 qubits), two tiles, and an odd count of passes."""
    g = circuits.random_layers(n, 5, 40 + n, iswap_frac=0.1)
    err, _ = run_emu(emu, n, g, random_state(n, n), remap, tpr=tpr)
    assert err < 1e-10, err


@pytest.mark.parametrize("remap", [0, 1, 2])
def test_tiled_index_math_qft_and_ansatz(emu, remap):
    n = 15
    err, _ = run_emu(emu, n, circuits.qft(n), random_state(n, 2), remap)
    assert err < 1e-10, err
    err, _ = run_emu(emu, n, circuits.vqe_ansatz(n, 3, seed=4), random_state(n, 3), remap)
    assert err < 1e-10, err


def test_tiled_index_math_chunk_pairings_in_plans(emu):
    """In-place and remapped plans meet both common pairings (tile bit 0 as
    block 0's column 0, or as a row bit) and reproduce the oracle."""
    kinds = [0, 0, 0]
    for seed in range(12):
        n = 14 + seed % 3
        g = circuits.random_layers(n, 5, 900 + seed, iswap_frac=0.2)
        for remap in (0, 1, 2):
            err, _ = run_emu(emu, n, g, random_state(n, seed), remap, kinds=kinds, tpr=1 + seed % 2)
            assert err < 1e-10, (seed, remap, err)
    assert kinds[0] > 0 and kinds[2] > 0, kinds


def test_block0_input_mapping_any_column_order(emu):
    """Arbitrary passes: tile bit 0 as column 0, as a later column (block
    columns in any order - remapped layouts can give this) and as a row; every
    A slot of every tile gets exactly its amplitude."""
    rng = np.random.default_rng(3)
    kinds = [0, 0, 0]
    for it in range(300):
        n = 12 + int(rng.integers(0, 9))
        rest = rng.permutation(np.arange(1, n))[:11]
        T = np.sort(np.concatenate([[0], rest])).astype(np.int32)
        q = rng.permutation(T)[:5].astype(np.int32)
        if it % 3 == 0 and 0 not in q:
            q[int(rng.integers(1, 5))] = 0           # tile bit 0 as a later column
        for tpr in (1, 2):
            kind = C.c_int(-1)
            rc = emu.tile_emu_check_input(n, T.ctypes.data_as(C.POINTER(C.c_int)),
                                          q.ctypes.data_as(C.POINTER(C.c_int)), tpr, C.byref(kind))
            assert rc == 0, (it, tpr, emu.tile_emu_error().decode())
        kinds[kind.value] += 1
    assert all(k > 0 for k in kinds), kinds


@pytest.mark.parametrize("seed", range(6))
def test_planner_every_gate_kind_random_mix(emu, seed):
    """Plans of mixed circuits - every gate kind, 3-qubit gates, control
    lists, QFT and ansatz pieces concatenated - from both pass drafts
    (gate-order tiles and closure-first blocks) reproduce the oracle."""
    from tests.golden.make_golden import every_gate_circuit
    n = 13 + seed % 4
    g = np.concatenate([every_gate_circuit(n, 50 + seed), circuits.qft(n),
                        circuits.random_layers(n, 3, 60 + seed, iswap_frac=0.3),
                        circuits.vqe_ansatz(n, 2, seed=seed)])
    for remap, low in ((0, 3), (1, 2), (2, 1)):
        err, _ = run_emu(emu, n, g, random_state(n, seed), remap, low_qubits=low)
        assert err < 1e-10, (seed, remap, low, err)


def test_rebound_plans_keep_a_valid_order(emu):
    """A plan built for one set of angles, rebound to another (as the batch
    executor shares plans between circuits of one gate pattern), applies the
    new circuit exactly - also when the first set has zero angles, which make
    RX / RY gates diagonal numerically: the planner lets only gates that are
    diagonal by kind (RZ, CR) pass each other."""
    from qpanda_b200 import lib
    n = 14
    base = np.concatenate([circuits.vqe_ansatz(n, 3, seed=4), circuits.qft(n),
                           circuits.random_layers(n, 3, 8, iswap_frac=0.2)])
    zero = base.copy()
    zero["theta"] = 0.0
    other = base.copy()
    other["theta"] = np.random.default_rng(5).uniform(0, 6.28, len(base))
    emu.tile_emu_rebind.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p)]
    for proto_gates in (zero, base):
        p = FusionPlan(n, proto_gates, remap=1, low_qubits=2)
        g = np.ascontiguousarray(other)
        h = C.c_void_p()
        assert emu.tile_emu_rebind(p.handle, g.ctypes.data, len(g), C.byref(h)) == 0, emu.tile_emu_error().decode()
        init = random_state(n, 9)
        st = np.ascontiguousarray(init.astype(np.complex128))
        npass = C.c_int()
        k = (C.c_int * 3)()
        rc = emu.tile_emu_apply(h, n, st.ctypes.data, 1, 1, C.byref(npass), k)
        lib().qs_plan_destroy(h)
        p.close()
        assert rc == 0, emu.tile_emu_error().decode()
        o = OracleState(n)
        o.set_state(init)
        o.apply(g)
        assert np.abs(st - o.state()).max() < 1e-10


# ------------------------------------------------------------- k_tile_tmem
def run_tmem_emu(E, n, g, init, remap, **kw):
    """The plan as k_tile_tmem runs it (passes it does not take as
    k_fused_tile does).  Returns (max error vs the oracle, passes taken,
    passes left, bank clashes of the gather, of the copies, of the exchanges
    between blocks)."""
    p = FusionPlan(n, g, remap=remap, **kw)
    st = np.ascontiguousarray(init.astype(np.complex128).copy())
    ps = (C.c_int * 2)()
    cf = (C.c_longlong * 3)()
    rc = E.tmem_emu_apply(p.handle, n, st.ctypes.data, int(remap), ps, cf)
    p.close()
    assert rc == 0, E.tile_emu_error().decode()
    o = OracleState(n)
    o.set_state(init)
    o.apply(g)
    return np.abs(st - o.state()).max(), ps[0], ps[1], cf[0], cf[1], cf[2]


@pytest.mark.parametrize("remap", [0, 1, 2])
@pytest.mark.parametrize("max_sub,low", [(1, 3), (2, 3), (3, 3), (2, 1), (2, 2), (2, 5)])
def test_tmem_index_math_random_layers(emu, remap, max_sub, low):
    """Staging swizzle, row gather, the exchanges between blocks through the
    staging buffer, the permuted block matrices and the stores reproduce the
    oracle; no phase of the copies or of an exchange clashes on a bank, nor of
    the gather in passes of two or three blocks (a one-block pass whose
    column written at position 0 is not tile bit 0 gives register bit 0 to
    16-byte stores, and its 8-byte gather then has three bank bits); every
    pass runs on this kernel."""
    n = 16
    g = circuits.random_layers(n, 6, 300 + 10 * max_sub + low, iswap_frac=0.2)
    err, took, left, gclash, cclash, xclash = run_tmem_emu(emu, n, g, random_state(n, 1), remap,
                                                           max_sub=max_sub, low_qubits=low)
    assert err < 1e-10, err
    assert took > 0 and left == 0
    assert cclash == 0 and xclash == 0, (cclash, xclash)
    if max_sub > 1:
        assert gclash == 0, gclash


@pytest.mark.parametrize("remap", [0, 1])
@pytest.mark.parametrize("n", [12, 13, 17])
def test_tmem_index_math_sizes(emu, remap, n):
    g = circuits.random_layers(n, 5, 40 + n, iswap_frac=0.1)
    err, took, _, _, _, _ = run_tmem_emu(emu, n, g, random_state(n, n), remap)
    assert err < 1e-10 and took > 0, err


@pytest.mark.parametrize("seed", range(4))
def test_tmem_index_math_mixed_circuits(emu, seed):
    from tests.golden.make_golden import every_gate_circuit
    n = 13 + seed % 4
    g = np.concatenate([every_gate_circuit(n, 50 + seed), circuits.qft(n),
                        circuits.random_layers(n, 3, 60 + seed, iswap_frac=0.3),
                        circuits.vqe_ansatz(n, 2, seed=seed)])
    for remap, low, ms in ((0, 3, 2), (1, 2, 3), (2, 1, 2)):
        err, took, _, _, _, xclash = run_tmem_emu(emu, n, g, random_state(n, seed), remap, low_qubits=low,
                                                  max_sub=ms)
        assert err < 1e-10 and took > 0, (seed, remap, low, err)
        assert xclash == 0


def test_tmem_conflict_free_on_the_bench_layouts(emu):
    """The benchmark's circuit structure at 18 qubits, in place and remapped:
    no bank clash in any shared-memory phase of any pass."""
    n = 18
    g = circuits.random_layers(n, 8, 20240601, iswap_frac=0.1)
    for remap in (0, 1):
        err, took, left, gclash, cclash, xclash = run_tmem_emu(emu, n, g, random_state(n, 7), remap)
        assert err < 1e-10 and left == 0
        assert (gclash, cclash, xclash) == (0, 0, 0), (remap, gclash, cclash, xclash)


def test_tmem_layout_shape_of_the_32q_bench_plan(emu):
    """The remapped plan of the 32-qubit benchmark circuit (2 low qubits, the
    tuned choice) puts a column of each pass's last block at write position 0
    and its lanes just above, so that most passes store 16-byte vectors and a
    warp's stores touch few 128-byte lines; the next pass's copies keep their
    contiguous runs.  8 KB per warp and tile each way: 64 lines at best."""
    E = emu
    E.tmem_layout_stats.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                    C.POINTER(C.c_longlong)]
    E.tmem_layout_stats.restype = C.c_int
    n = 32
    g = circuits.random_layers(n, 16, 20240601, iswap_frac=0.1)
    p = FusionPlan(n, g, remap=1, low_qubits=2)
    vec, st, cp = C.c_int(), C.c_longlong(), C.c_longlong()
    assert E.tmem_layout_stats(p.handle, n, 1, C.byref(vec), C.byref(st), C.byref(cp)) == 0, \
        E.tile_emu_error().decode()
    passes = p.num_launches()
    p.close()
    assert passes == 32
    assert vec.value >= 20, vec.value                       # 11 before the write order favoured the stores
    assert st.value / passes <= 80, st.value / passes       # 120 lines per warp and tile before
    assert cp.value / passes <= 72, cp.value / passes


@pytest.mark.parametrize("remap", [0, 1])
@pytest.mark.parametrize("max_k", [2, 3, 4])
def test_fusion_width_below_five(emu, max_k, remap):
    """Blocks of at most 2, 3 or 4 qubits (4 is the batch autotuner's other
    fusion width), widened to 5-qubit blocks: both tiled kernels' index math
    with the widened block unitaries reproduces the oracle."""
    n = 16
    g = np.concatenate([circuits.random_layers(n, 6, 500 + max_k, iswap_frac=0.2), circuits.vqe_ansatz(n, 2, seed=max_k)])
    init = random_state(n, 40 + max_k)
    err, npass = run_emu(emu, n, g, init, remap, max_k=max_k)
    assert npass >= 2 and err < 1e-10, err
    err, took, left, _, cclash, xclash = run_tmem_emu(emu, n, g, init, remap, max_k=max_k)
    assert err < 1e-10 and took > 0 and left == 0, err
    assert cclash == 0 and xclash == 0
