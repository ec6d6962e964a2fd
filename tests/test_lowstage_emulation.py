"""CPU check of the staged runs' index arithmetic (no GPU).

tests/lowstage_emu/lowstage_emu.cpp moves every run of a gate list exactly as
k_lowstage does - the library's own passes and planner (tile qubits, register
layouts, op kinds), the tile bases and copy offsets in the state, the
swizzled 16-byte copies, each thread's register slots, the round trips
through shared memory at every layout switch - with FP64 arithmetic.  The
result must match the oracle to rounding, every shared-memory slot must be
written and read exactly once per phase, and no access phase may hit a bank
twice (the swizzle and lane-order claim of qs_lowstage.cuh).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import circuits
from qpanda_b200.capi import lib
from tests.golden.make_golden import every_gate_circuit

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "qpanda_b200", "csrc")
LIBDIR = os.path.join(ROOT, "qpanda_b200", "_lib")
SRC = os.path.join(ROOT, "tests", "lowstage_emu", "lowstage_emu.cpp")
C64, C128 = 0, 1


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    lib()                                     # the library must be built
    out = str(tmp_path_factory.mktemp("lowstage_emu") / "liblowstage_emu.so")
    cmd = ["/usr/local/cuda/bin/nvcc", "-O2", "-std=c++17", "-x", "cu", "-shared", "-Xcompiler", "-fPIC",
           "-gencode", "arch=compute_100a,code=sm_100a", SRC, "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
           "-L" + LIBDIR, "-lqsb200", "-Xlinker", "-rpath=" + LIBDIR, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    E = C.CDLL(out)
    E.lowstage_emu_apply.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_longlong)]
    E.lowstage_emu_apply.restype = C.c_int
    E.lowstage_emu_error.restype = C.c_char_p
    E.lowstage_emu_passes.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_longlong)]
    E.lowstage_emu_passes.restype = C.c_int
    return E


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


def run_emu(E, n, gates, dtype):
    init = random_state(n, 7 * n + dtype)
    st = np.ascontiguousarray(init.copy())
    g = np.ascontiguousarray(gates)
    stats = (C.c_longlong * 4)()
    r = E.lowstage_emu_apply(st.ctypes.data, n, g.ctypes.data, len(g), dtype, stats)
    assert r == 0, E.lowstage_emu_error().decode()
    o = OracleState(n)
    o.set_state(init)
    o.apply(gates)
    return np.abs(st - o.state()).max(), list(stats)


# the plan holds the matrices in the state's precision: FP32 for complex64
TOL = {C64: 1e-6, C128: 1e-12}


@pytest.mark.parametrize("dtype", [C64, C128])
@pytest.mark.parametrize("n", [5, 7, 9, 10, 12])
def test_runs_match_oracle_without_bank_conflicts(emu, n, dtype):
    """Bank-conflict freedom is claimed for the full 10-bit tile (n >= 10);
    narrower tiles (whole states below 10 qubits) have too few thread bits
    to always find independent bank images and are checked for results and
    slot coverage only."""
    for k, g in enumerate((circuits.random_layers(n, 4, 90 + n, iswap_frac=0.3), circuits.qft(n),
                           every_gate_circuit(n, 11 + n))):
        err, (reg_conf, copy_conf, switches, runs) = run_emu(emu, n, g, dtype)
        assert err < TOL[dtype], (k, err)
        assert runs > 0, k
        assert copy_conf == 0, (k, copy_conf)
        if n >= 10:
            assert reg_conf == 0, (k, reg_conf)


def test_rotation_layer_needs_three_layout_switches(emu):
    """The rotations of one layer on qubits 0..9 (one run): three register
    bits per layout, so the run switches layouts three times (0-2, 3-5, 6-8,
    then 9)."""
    n = 12
    g = circuits.random_layers(n, 1, 3)[:10]
    assert list(g["q"][:, 0]) == list(range(10))
    err, (reg_conf, copy_conf, switches, runs) = run_emu(emu, n, g, C64)
    assert err < TOL[C64] and reg_conf == 0 and copy_conf == 0
    assert runs == 1 and switches == 3, (runs, switches)


@pytest.mark.parametrize("dtype", [C64, C128])
def test_runs_on_any_qubits(emu, dtype):
    """Runs whose gates act on high qubits stage tiles of those qubits plus
    the lowest ones: every amplitude copied in and out exactly once per run,
    the oracle's state, no bank conflicts."""
    n = 14
    for k, g in enumerate((circuits.random_layers(n, 3, 500 + dtype, iswap_frac=0.3),
                           every_gate_circuit(n, 77 + dtype))):
        err, (reg_conf, copy_conf, switches, runs) = run_emu(emu, n, g, dtype)
        assert err < TOL[dtype], (k, err)
        assert runs > 0 and copy_conf == 0 and reg_conf == 0, (k, runs, copy_conf, reg_conf)


def passes_of(E, n, g, dtype):
    g = np.ascontiguousarray(g)
    out = (C.c_longlong * 3)()
    assert E.lowstage_emu_passes(n, g.ctypes.data, len(g), dtype, out) == 0, E.lowstage_emu_error().decode()
    return list(out)


def test_benchmark_circuits_run_in_few_passes(emu):
    """The per-gate path's passes over the state (qs_gates_apply): the
    20-qubit complex128 circuit (600 gates), the 32-qubit complex64 circuit
    (768 gates) and the 28-qubit QFT (420 gates) each stage nearly every gate,
    in runs of up to 24 whose targets share one tile."""
    for n, g, dtype, most in ((20, circuits.random_layers(20, 20, 20240601), C128, 70),
                              (32, circuits.random_layers(32, 16, 20240601, iswap_frac=0.1), C64, 110),
                              (28, circuits.qft(28), C64, 25)):
        staged, single, in_staged = passes_of(emu, n, g, dtype)
        assert staged + single <= most, (n, staged, single)
        assert in_staged >= 0.99 * len(g), (n, in_staged, len(g))
