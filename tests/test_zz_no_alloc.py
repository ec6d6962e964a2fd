"""qs_measure_noalloc: qubit measurement for callers that cannot allocate.

Some callers hold a state vector in memory they allocated themselves (or in a
pool whose allocator must not be bypassed) and cannot call cudaMalloc at the
moment they measure.  The entry point takes the amplitudes and two device
output words and keeps its partial sums in a fixed array inside the library.
This test calls it through the C ABI and compares it with qs_measure - the
entry point that uses allocated scratch - on the same state, for two
measurements in a row: same outcomes, P(0) and collapsed amplitudes within the
tolerances of the other GPU tests (1e-12 for complex128, 1e-5 for complex64).
This file is collected last so that a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from qpanda_b200 import StateVector, circuits, lib
from qpanda_b200.capi import QS_C64, QS_C128, QSError, check

pytestmark = pytest.mark.gpu
TOL = {"c128": 1e-12, "c64": 1e-5}


@pytest.mark.parametrize("dt", ["c128", "c64"])
@pytest.mark.parametrize("n", [3, 17, 21])
def test_noalloc_measure_matches_qs_measure(need_gpu, dt, n):
    import torch
    g = circuits.random_layers(n, 5, 900 + n, iswap_frac=0.2)
    ref, tgt = StateVector(n, dt), StateVector(n, dt)
    ref.apply(g)
    tgt.apply(g)
    amp = C.c_void_p()
    check(lib().qs_device_ptr(tgt.handle, C.byref(amp)))
    out = torch.zeros(2, dtype=torch.int32, device="cuda")
    p0 = torch.zeros(2, dtype=torch.float64, device="cuda")
    tgt.synchronize()
    rng = np.random.default_rng(n)
    for k, q in enumerate((n - 1, 0)):           # two calls in a row
        u = float(rng.uniform())
        p_ref = ref.prob_zero(q)
        o_ref = ref.measure(q, u)
        check(lib().qs_measure_noalloc(amp, n, QS_C64 if dt == "c64" else QS_C128, q, u,
                                       C.c_void_p(out.data_ptr() + 4 * k), C.c_void_p(p0.data_ptr() + 8 * k),
                                       None))
        torch.cuda.synchronize()
        assert int(out[k]) == o_ref
        assert abs(float(p0[k]) - p_ref) < TOL[dt]
        assert np.abs(tgt.get_state() - ref.get_state()).max() < TOL[dt]


def test_noalloc_rejects_oversize_and_bad_args(need_gpu):
    dummy = C.c_void_p(1 << 20)
    out = C.c_void_p(1 << 21)
    with pytest.raises(QSError) as e:
        check(lib().qs_measure_noalloc(dummy, 33, QS_C64, 0, 0.5, out, out, None))
    assert "32 qubits" in str(e.value) or "1..32" in str(e.value)
    with pytest.raises(QSError):
        check(lib().qs_measure_noalloc(dummy, 10, QS_C64, 10, 0.5, out, out, None))
    with pytest.raises(QSError):
        check(lib().qs_measure_noalloc(None, 10, QS_C64, 0, 0.5, out, out, None))
    # amplitudes must sit on their element size (checked before any launch)
    with pytest.raises(QSError) as e:
        check(lib().qs_measure_noalloc(C.c_void_p((1 << 20) + 4), 10, QS_C64, 0, 0.5, out, out, None))
    assert "aligned" in str(e.value)
    with pytest.raises(QSError):
        check(lib().qs_measure_noalloc(C.c_void_p((1 << 20) + 8), 10, QS_C128, 0, 0.5, out, out, None))


def _ptr(sv):
    amp = C.c_void_p()
    check(lib().qs_device_ptr(sv.handle, C.byref(amp)))
    return amp


@pytest.mark.parametrize("dt", ["c128", "c64"])
def test_noalloc_outcome_of_probability_zero(need_gpu, dt):
    """A uniform that selects an outcome of probability 0 (only a uniform
    outside (0, 1] can): outcome -1, P(0) reported, state untouched - where
    qs_measure reports QS_ERR_STATE and also leaves the state."""
    import torch
    n = 5
    code = QS_C64 if dt == "c64" else QS_C128
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    p0 = torch.zeros(1, dtype=torch.float64, device="cuda")
    for basis, u in ((0, 2.0), (1 << 3, -1.0)):          # |0> with u > 1; |q=1> with u < 0
        init = np.zeros(1 << n, dtype=np.complex128)
        init[basis] = 1.0
        sv = StateVector(n, dt)
        sv.set_state(init)
        check(lib().qs_measure_noalloc(_ptr(sv), n, code, 3, u, C.c_void_p(out.data_ptr()),
                                       C.c_void_p(p0.data_ptr()), None))
        torch.cuda.synchronize()
        assert int(out[0]) == -1
        assert float(p0[0]) == (1.0 if basis == 0 else 0.0)
        assert np.array_equal(sv.get_state(), init)
        ref = StateVector(n, dt)
        ref.set_state(init)
        with pytest.raises(QSError):
            ref.measure(3, u)
        assert np.array_equal(ref.get_state(), init)


def test_noalloc_8_byte_aligned_complex64_on_a_caller_stream(need_gpu):
    """complex64 amplitudes that start 8 bytes into a buffer (the per-amplitude
    load path), measured twice on a stream of the caller's."""
    import torch
    n = 18
    g = circuits.random_layers(n, 4, 77, iswap_frac=0.2)
    ref = StateVector(n, "c64")
    ref.apply(g)
    host = ref.get_state(np.complex64)
    buf = torch.zeros(2 * (1 << n) + 2, dtype=torch.float32, device="cuda")
    view = buf[2:]
    view.copy_(torch.from_numpy(host.view(np.float32)).to("cuda"))
    assert (view.data_ptr() % 16) == 8
    st = torch.cuda.Stream()
    out = torch.zeros(2, dtype=torch.int32, device="cuda")
    p0 = torch.zeros(2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rng = np.random.default_rng(3)
    for k, q in enumerate((0, 13)):
        u = float(rng.uniform())
        o_ref = ref.measure(q, u)
        check(lib().qs_measure_noalloc(C.c_void_p(view.data_ptr()), n, QS_C64, q, u,
                                       C.c_void_p(out.data_ptr() + 4 * k), C.c_void_p(p0.data_ptr() + 8 * k),
                                       C.c_void_p(st.cuda_stream)))
        st.synchronize()
        assert int(out[k]) == o_ref
        got = view.cpu().numpy().view(np.complex64)
        assert np.abs(got - ref.get_state()).max() < TOL["c64"]


def test_noalloc_at_the_32_qubit_maximum(need_gpu):
    """The documented maximum: a 32-qubit complex64 state (32 GiB, 65536
    partial sums), a qubit above the 2^16-amplitude chunks and one inside
    them, against qs_measure on a copy."""
    import torch
    n = 32
    spec = [("H", (q,)) for q in (0, 3, 16, 20, 31)] + [("RY", (5,), 0.7), ("CNOT", (31, 2)), ("RX", (17,), 1.9)]
    g = circuits.make_gates(spec)
    ref, tgt = StateVector(n, "c64"), StateVector(n, "c64")
    ref.apply(g)
    tgt.apply(g)
    tgt.synchronize()
    out = torch.zeros(2, dtype=torch.int32, device="cuda")
    p0 = torch.zeros(2, dtype=torch.float64, device="cuda")
    for k, (q, u) in enumerate(((31, 0.61), (3, 0.27))):
        p_ref = ref.prob_zero(q)
        o_ref = ref.measure(q, u)
        check(lib().qs_measure_noalloc(_ptr(tgt), n, QS_C64, q, u, C.c_void_p(out.data_ptr() + 4 * k),
                                       C.c_void_p(p0.data_ptr() + 8 * k), None))
        torch.cuda.synchronize()
        assert int(out[k]) == o_ref
        assert abs(float(p0[k]) - p_ref) < TOL["c64"]
        mx, _ = tgt.diff(ref)
        assert mx < TOL["c64"], mx
    ref.close()
    tgt.close()
