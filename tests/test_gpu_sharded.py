"""GPU: a sharded state with its shards in one process on one GPU (the
exchange as device copies), against the oracle on the whole state.  Ranks on
separate GPUs exchange through NCCL with the same code (NcclExchanger), which
tests/test_sharded.py runs on gloo ranks; this pool gives one GPU per run.
The C ABI's driver is tested with all shards local (in-place swap kernel),
with one qs_sharded per host thread exchanging through a caller function,
and with peer swaps over the partner's memory (one in-place kernel per side,
the partner's buffer standing in for a peer GPU's)."""
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


# ------------------------------------------------ the C ABI's sharded driver
def _sharded_reference(n, gates):
    o = OracleState(n)
    o.apply(gates)
    return o.state()


def _circuit(n, seed):
    return np.concatenate([circuits.random_layers(n, 5, seed, iswap_frac=0.3), circuits.qft(n)])


@pytest.mark.parametrize("dt,tol", [("c128", 1e-12), ("c64", 1e-5)])
@pytest.mark.parametrize("n,g_bits", [(14, 1), (15, 2)])
def test_c_abi_sharded_all_shards_local(need_gpu, n, g_bits, dt, tol):
    """qs_sharded_* with every shard in this process: the C++ schedule (the
    same swaps and final layout as qpanda_b200.sharded.schedule) and the
    device-copy swaps of strided and contiguous halves, against the oracle."""
    import ctypes as C

    from qpanda_b200 import lib
    from qpanda_b200.capi import QS_C64, QS_C128, check
    from qpanda_b200.sharded import schedule
    gates = _circuit(n, 40 + n)
    code = QS_C64 if dt == "c64" else QS_C128
    ranks = np.arange(1 << g_bits, dtype=np.int32)
    h = C.c_void_p()
    check(lib().qs_sharded_create(n, g_bits, code, ranks.ctypes.data_as(C.POINTER(C.c_int)), len(ranks), None,
                                  None, C.byref(h)))
    g = np.ascontiguousarray(gates)
    check(lib().qs_sharded_apply(h, g.ctypes.data, len(g)))
    shards = []
    for r in ranks:
        s = C.c_void_p()
        check(lib().qs_sharded_shard(h, int(r), C.byref(s)))
        out = np.empty(1 << (n - g_bits), dtype=np.complex128)
        check(lib().qs_get_state(s, out.ctypes.data, QS_C128))
        shards.append(out)
    pos = np.empty(n, dtype=np.int32)
    check(lib().qs_sharded_positions(h, pos.ctypes.data_as(C.POINTER(C.c_int))))
    swaps, moved = C.c_size_t(), C.c_size_t()
    check(lib().qs_sharded_info(h, C.byref(swaps), C.byref(moved)))
    lib().qs_sharded_destroy(h)
    steps, pos_py = schedule(n, g_bits, gates)
    assert list(pos) == list(pos_py)
    assert swaps.value == sum(1 for st in steps if st[0] == "swap") > 0
    got = gather_logical(shards, n, g_bits, list(pos))
    assert np.abs(got - _sharded_reference(n, gates)).max() < tol


@pytest.fixture(scope="module")
def mailbox(tmp_path_factory):
    import ctypes as C
    import os
    import subprocess

    from qpanda_b200 import lib
    lib()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "qpanda_b200", "_lib")
    out = str(tmp_path_factory.mktemp("mailbox") / "libmailbox.so")
    cmd = ["/usr/local/cuda/bin/nvcc", "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           os.path.join(root, "tests", "sharded_emu", "mailbox.cpp"), "-I" + os.path.join(root, "include"),
           "-L" + libdir, "-lqsb200", "-Xlinker", "-rpath=" + libdir, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    E = C.CDLL(out)
    E.mailbox_run.restype = C.c_int
    E.mailbox_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p,
                              C.POINTER(C.c_int), C.POINTER(C.c_size_t)]
    E.peer_run.restype = C.c_int
    E.peer_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p,
                           C.POINTER(C.c_int), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    return E


@pytest.mark.parametrize("dt,tol", [("c128", 1e-12), ("c64", 1e-5)])
@pytest.mark.parametrize("n,g_bits", [(14, 1), (15, 2)])
def test_c_abi_sharded_exchange_function(need_gpu, mailbox, n, g_bits, dt, tol):
    """One qs_sharded per shard, each in its own host thread, swapping halves
    through the caller's exchange function (here a host mailbox and a device
    copy; NCCL send/receive in a multi-GPU job): packed halves in 256 MB
    pieces, the same result as the oracle."""
    import ctypes as C

    from qpanda_b200.capi import QS_C64, QS_C128
    gates = np.ascontiguousarray(_circuit(n, 90 + n))
    code = QS_C64 if dt == "c64" else QS_C128
    npdt = np.complex64 if dt == "c64" else np.complex128
    out = np.empty((1 << g_bits) << (n - g_bits), dtype=npdt)
    pos = np.empty(n, dtype=np.int32)
    swaps = C.c_size_t()
    rc = mailbox.mailbox_run(n, g_bits, code, gates.ctypes.data, len(gates), out.ctypes.data,
                             pos.ctypes.data_as(C.POINTER(C.c_int)), C.byref(swaps))
    assert rc == 0, rc
    assert swaps.value > 0
    shards = np.split(out.astype(np.complex128), 1 << g_bits)
    got = gather_logical(shards, n, g_bits, list(pos))
    assert np.abs(got - _sharded_reference(n, gates)).max() < tol


@pytest.mark.parametrize("dt,tol", [("c128", 1e-12), ("c64", 1e-5)])
@pytest.mark.parametrize("n,g_bits", [(14, 1), (15, 2), (13, 3)])
def test_c_abi_sharded_peer_swaps(need_gpu, mailbox, n, g_bits, dt, tol):
    """One qs_sharded per shard in its own host thread, every other shard
    registered as a peer (qs_sharded_set_peer): each swap is one in-place
    kernel per side over the partner's memory (a peer GPU's, or an IPC mapping,
    in a multi-GPU job; another buffer of this GPU here), the rank-bit-0 side
    taking the first half of the rows, or of the single row when the swapped
    position is the top local one.  The result equals the oracle's and, bit for
    bit, the exchange-function path's; each side moves half of its half-slice
    per swap, both ways."""
    import ctypes as C

    from qpanda_b200.capi import QS_C64, QS_C128
    gates = np.ascontiguousarray(_circuit(n, 190 + n))
    code = QS_C64 if dt == "c64" else QS_C128
    npdt = np.complex64 if dt == "c64" else np.complex128
    outs = []
    for run in ("peer", "mailbox"):
        out = np.empty((1 << g_bits) << (n - g_bits), dtype=npdt)
        pos = np.empty(n, dtype=np.int32)
        swaps, moved = C.c_size_t(), C.c_size_t()
        if run == "peer":
            rc = mailbox.peer_run(n, g_bits, code, gates.ctypes.data, len(gates), out.ctypes.data,
                                  pos.ctypes.data_as(C.POINTER(C.c_int)), C.byref(swaps), C.byref(moved))
            assert rc == 0, rc
            assert swaps.value > 0
            amp = 8 if dt == "c64" else 16
            assert moved.value == swaps.value * (amp << (n - g_bits)) // 2, (moved.value, swaps.value)
        else:
            rc = mailbox.mailbox_run(n, g_bits, code, gates.ctypes.data, len(gates), out.ctypes.data,
                                     pos.ctypes.data_as(C.POINTER(C.c_int)), C.byref(swaps))
            assert rc == 0, rc
        outs.append((out, list(pos)))
    (a, pa), (b, pb) = outs
    assert pa == pb and np.array_equal(a, b)
    shards = np.split(a.astype(np.complex128), 1 << g_bits)
    got = gather_logical(shards, n, g_bits, pa)
    assert np.abs(got - _sharded_reference(n, gates)).max() < tol
