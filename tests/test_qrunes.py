"""QRunes programs through the reference's own parser and dispatcher.

CPU part: the harness with the reference CPU backend reproduces the oracle and
the reference's own fixture programs (read from the reference tree when it is
present).  GPU part: the B200 backend (B200QuantumGates over the C ABI) gives
the same PMEASURE probabilities and - with the same generator seed - the same
MEASURE counts as the reference backend."""
import os

import numpy as np
import pytest

from oracle.pyoracle import OracleState
from qpanda_b200 import circuits
from qpanda_b200.qrunes import to_qrunes
from tests import qrunes_harness as H

needs_runner = pytest.mark.skipif(not H.available(), reason="tests/qrunes not built (needs the reference tree)")


def _ref_sdk():
    """The reference's QPandaSDK directory: QPANDA_REF, or where build()
    found the reference tree ("" when neither is there)."""
    ref = os.environ.get("QPANDA_REF", "")
    rec = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qrunes", "_build", "qpanda_ref.txt")
    if not ref and os.path.exists(rec):
        with open(rec) as f:
            ref = f.read().strip()
    return os.path.join(ref, "QPandaSDK") if ref else ""


REF_SDK = _ref_sdk()


def programs(tmp_path):
    progs = {}
    n = 9
    g = circuits.random_layers(n, 6, 77)
    progs["layers_pmeasure"] = to_qrunes(n, g, pmeasure=[0, 3, 8, 5])
    progs["layers_measure"] = to_qrunes(n, g, measure=[(q, q) for q in range(n)])
    from tests.golden.make_golden import every_gate_circuit
    eg = every_gate_circuit(7, 21)
    # plain ISWAP lines are a no-op on the reference path (swapped dispatch
    # branches, Instruction.cpp:558-577): keep them inside CONTROL blocks only
    keep = [i for i in range(len(eg)) if not (eg[i]["op"] == 8 and eg[i]["nctrl"] == 0)]
    eg = eg[keep]
    # and controlled sqiSWAP / iSWAP / CR / CSWAP are no-ops or uncontrolled on
    # the reference path: drop the controls from those
    for i in range(len(eg)):
        if int(eg[i]["op"]) in (7, 8, 9, 11):
            eg[i]["nctrl"] = 0
    progs["every_gate_pmeasure"] = to_qrunes(7, eg, pmeasure=[0, 1, 2, 3, 4, 5, 6])
    qft = circuits.qft(8)
    progs["qft_pmeasure"] = to_qrunes(8, np.concatenate([circuits.random_layers(8, 1, 5), qft]), pmeasure=[7, 6, 5])
    paths = {}
    for k, text in progs.items():
        p = tmp_path / f"{k}.txt"
        p.write_text(text)
        paths[k] = str(p)
    return paths


@needs_runner
def test_cpu_harness_matches_oracle(tmp_path):
    n = 9
    g = circuits.random_layers(n, 6, 77)
    path = programs(tmp_path)["layers_pmeasure"]
    kind, res, nq = H.run(path, H.CPU)
    assert kind == "PMEASURE" and nq == n
    o = OracleState(n)
    o.apply(g)
    p = o.probs([0, 3, 8, 5])
    top = sorted(range(16), key=lambda i: (-p[i], i))[:10]
    for i in top:
        assert abs(res[format(i, "04b")] - p[i]) < 1e-12


@needs_runner
@pytest.mark.skipif(not REF_SDK or not os.path.isdir(REF_SDK), reason="reference fixture programs not present")
def test_cpu_harness_reference_fixtures():
    kind, res, _ = H.run(os.path.join(REF_SDK, "shor.txt"), H.CPU)
    assert kind == "PMEASURE"
    assert abs(res["100"] - 0.5) < 1e-12 and abs(res["101"] - 0.5) < 1e-12
    kind, res, _ = H.run(os.path.join(REF_SDK, "testMain", "shor_15.txt"), H.CPU, seed=7, repeat=200)
    assert kind == "MEASURE" and abs(sum(res.values()) - 1) < 1e-12


@needs_runner
@pytest.mark.gpu
@pytest.mark.parametrize("backend,tol", [(H.B200_C128, 1e-12), (H.B200_C64, 1e-5)])
def test_b200_backend_pmeasure(need_gpu, tmp_path, backend, tol):
    for name, path in programs(tmp_path).items():
        if "pmeasure" not in name:
            continue
        k0, r0, _ = H.run(path, H.CPU)
        k1, r1, _ = H.run(path, backend)
        assert k0 == k1 == "PMEASURE"
        assert set(r0) == set(r1), name
        for b in r0:
            assert abs(r0[b] - r1[b]) < tol, (name, b)


@needs_runner
@pytest.mark.gpu
def test_b200_backend_measure_counts_bit_exact(need_gpu, tmp_path):
    path = programs(tmp_path)["layers_measure"]
    k0, r0, _ = H.run(path, H.CPU, seed=4242, repeat=64)
    k1, r1, _ = H.run(path, H.B200_C128, seed=4242, repeat=64)
    assert k0 == k1 == "MEASURE"
    assert r0 == r1


def gpu_unit_programs(tmp_path):
    """Programs within what the reference GPU compute unit implements: its
    controlled NOT / CNOT / iSWAP / sqiSWAP overloads and controlSwap return
    without doing anything (GPUQuantumGates.cpp:587-594, 729-733, 975-983)."""
    paths = programs(tmp_path)
    from tests.golden.make_golden import every_gate_circuit
    eg = every_gate_circuit(7, 33)
    keep = [i for i in range(len(eg))
            if not (int(eg[i]["op"]) in (2, 6, 8, 9) and eg[i]["nctrl"] > 0)
            and not (int(eg[i]["op"]) == 8 and eg[i]["nctrl"] == 0) and int(eg[i]["op"]) != 11]
    eg = eg[keep]
    for i in range(len(eg)):
        if int(eg[i]["op"]) == 7:
            eg[i]["nctrl"] = 0
    p = tmp_path / "gpu_unit_every_gate.txt"
    p.write_text(to_qrunes(7, eg, pmeasure=[6, 0, 3, 1]))
    paths["gpu_unit_every_gate_pmeasure"] = str(p)
    del paths["every_gate_pmeasure"]
    return paths


@needs_runner
@pytest.mark.gpu
def test_reference_gpu_unit_over_shim_pmeasure(need_gpu, tmp_path):
    """The reference's own GPUQuantumGates (compiled from its sources,
    unmodified) over libGPUEmulator.so gives the CPU backend's PMEASURE
    results."""
    for name, path in gpu_unit_programs(tmp_path).items():
        if "pmeasure" not in name:
            continue
        k0, r0, _ = H.run(path, H.CPU)
        k1, r1, _ = H.run(path, H.GPU_UNIT)
        assert k0 == k1 == "PMEASURE"
        assert set(r0) == set(r1), name
        for b in r0:
            assert abs(r0[b] - r1[b]) < 1e-12, (name, b)


@needs_runner
@pytest.mark.gpu
def test_reference_gpu_unit_over_shim_measure_counts(need_gpu, tmp_path):
    """Same generator seed: the same MEASURE counts as the CPU backend, shot
    by shot (each gate and measurement draws like the CPU backend)."""
    path = programs(tmp_path)["layers_measure"]
    k0, r0, _ = H.run(path, H.CPU, seed=99, repeat=64)
    k1, r1, _ = H.run(path, H.GPU_UNIT, seed=99, repeat=64)
    assert k0 == k1 == "MEASURE"
    assert r0 == r1


@needs_runner
def test_cpu_harness_every_gate_program_matches_oracle(tmp_path):
    """The generated every-gate program (nested CONTROL and DAGGER blocks)
    through the reference parser and CPU backend equals the oracle."""
    from tests.golden.make_golden import every_gate_circuit
    eg = every_gate_circuit(7, 21)
    keep = [i for i in range(len(eg)) if not (eg[i]["op"] == 8 and eg[i]["nctrl"] == 0)]
    eg = eg[keep]
    for i in range(len(eg)):
        if int(eg[i]["op"]) in (7, 8, 9, 11):
            eg[i]["nctrl"] = 0
    o = OracleState(7)
    o.apply(eg)
    p = o.probs(list(range(7)))
    path = programs(tmp_path)["every_gate_pmeasure"]
    kind, res, _ = H.run(path, H.CPU)
    top = sorted(range(128), key=lambda i: (-p[i], i))[:10]
    for i in top:
        assert abs(res[format(i, "07b")] - p[i]) < 1e-12


# ------------------------------------------------ shots, RESET, getQState text
def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


@needs_runner
@pytest.mark.gpu
def test_terminal_measures_one_run_plus_sampling(need_gpu, tmp_path):
    """QPandaSDK::run re-simulates a MEASURE program once per shot
    (QPandaAPI.cpp:169-182).  With every MEASURE terminal, the B200 backend
    runs it once and samples the shots, drawing each shot's uniforms from the
    same 16807 stream at the positions the loop would: the counts equal the
    reference CPU backend's per-shot loop, shot for shot; classical registers
    in scrambled order, one qubit measured twice."""
    n = 10
    g = circuits.random_layers(n, 5, 31)
    order = (3, 0, 9, 5, 1, 8, 2, 7, 4, 6)
    measure = [(q, (7 * q + 3) % n) for q in order] + [(order[0], n)]
    path = _write(tmp_path, "terminal.txt", to_qrunes(n, g, measure=measure))
    k0, r0, _ = H.run(path, H.CPU, seed=4242, repeat=300)
    runs = []
    k1, r1, _ = H.run(path, H.B200_C128, seed=4242, repeat=300, sample=True, runs_out=runs)
    assert k0 == k1 == "MEASURE" and runs == [1]
    assert r0 == r1


@needs_runner
@pytest.mark.gpu
def test_measure_followed_by_a_gate_runs_the_loop(need_gpu, tmp_path):
    """A gate after a MEASURE on the measured qubit: the probe pass sees it,
    and the shots come from the per-shot loop (one run per shot)."""
    text = "\n".join(["QINIT 4", "CREG 3", "H 0", "CNOT 0,1", 'RY 2,"0.9"', "MEASURE 0,$0", "H 0",
                      'RX 1,"0.3"', "MEASURE 0,$1", "MEASURE 1,$2"]) + "\n"
    path = _write(tmp_path, "nonterminal.txt", text)
    k0, r0, _ = H.run(path, H.CPU, seed=11, repeat=120)
    runs = []
    k1, r1, _ = H.run(path, H.B200_C128, seed=11, repeat=120, sample=True, runs_out=runs)
    assert runs == [120]
    assert r0 == r1


@needs_runner
@pytest.mark.gpu
def test_reset_matches_cpu_backend(need_gpu, tmp_path):
    """RESET (CPUQuantumGates.cpp:126-136: a measurement, then NOT when it gave
    1; its draws shift the generator stream by one or two): the per-shot
    counts of a program with two RESETs equal the CPU backend's; with
    sampling asked for, RESET keeps the loop."""
    text = "\n".join(["QINIT 5", "CREG 5", "H 0", "CNOT 0,1", 'RY 2,"1.1"', "RESET 1", "CNOT 2,1", "H 3",
                      "RESET 3", 'RX 3,"0.7"'] + [f"MEASURE {q},${q}" for q in range(5)]) + "\n"
    path = _write(tmp_path, "reset.txt", text)
    k0, r0, _ = H.run(path, H.CPU, seed=5, repeat=200)
    for backend in (H.B200_C128, H.B200_C64):
        runs = []
        k1, r1, _ = H.run(path, backend, seed=5, repeat=200, sample=True, runs_out=runs)
        assert runs == [200]
        assert r0 == r1, backend


@needs_runner
@pytest.mark.gpu
def test_getqstate_text_matches_cpu_backend(need_gpu, tmp_path):
    """B200QuantumGates::getQState prints the state as CPUQuantumGates::getQState
    does (CPUQuantumGates.cpp:64-82), byte for byte, for a program whose
    amplitudes sit well inside their printed digits."""
    text = "\n".join(["QINIT 4", "CREG 1", "H 0", "H 1", "CNOT 1,2", 'RZ 2,"0.5"', 'RX 3,"1.25"',
                      'CR 0,3,"0.75"']) + "\n"
    path = _write(tmp_path, "qstate.txt", text)
    t0 = H.qstate_text(path, H.CPU)
    t1 = H.qstate_text(path, H.B200_C128)
    assert t0.count("\n") == 16
    assert t0 == t1
