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
