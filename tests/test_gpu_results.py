"""GPU: the .fullstate writers against the reference's getQState text."""
import os

import numpy as np
import pytest

from qpanda_b200 import StateVector, circuits

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_fullstate_text_and_binary_match_reference(need_gpu, tmp_path):
    """The gates_n7 state set exactly: the text file equals the reference's
    getQState text byte for byte; the binary file holds the amplitudes."""
    st = np.load(os.path.join(GOLDEN, "gates_n7.npz"))["state"]
    with open(os.path.join(GOLDEN, "qstate_n7.txt")) as f:
        golden = f.read()
    sv = StateVector(7, "c128")
    sv.set_state(st)
    prefix = str(tmp_path / "prog")
    sv.write_fullstate(prefix)
    sv.write_fullstate(prefix, binary=True)
    with open(prefix + ".fullstate") as f:
        assert f.read() == golden
    got = np.fromfile(prefix + ".fullstate.binary", dtype=np.complex128)
    assert np.array_equal(got, st)


@pytest.mark.parametrize("dtype", ["c64", "c128"])
def test_fullstate_streams_in_chunks(need_gpu, tmp_path, dtype):
    """A state larger than one device-to-host chunk (2^21 amplitudes)."""
    n = 21
    sv = StateVector(n, dtype)
    sv.apply(circuits.random_layers(n, 2, 3))
    prefix = str(tmp_path / "big")
    sv.write_fullstate(prefix, binary=True)
    got = np.fromfile(prefix + ".fullstate.binary", dtype=np.complex128)
    ref = sv.get_state(np.complex64 if dtype == "c64" else np.complex128).astype(np.complex128)
    assert np.array_equal(got, ref)
    sv.write_fullstate(prefix)
    with open(prefix + ".fullstate") as f:
        lines = f.read().splitlines()
    assert len(lines) == 1 << n
    k = (1 << 20) + 7
    assert lines[k] == f"state[{k}].real = {ref[k].real:g} state[{k}].imag = {ref[k].imag:g}"
