"""Result formats (no GPU): the .fullstate text pinned to the reference's own
getQState output, and the QPandaSDK::getResult outcome text."""
import os

import numpy as np
import pytest

from qpanda_b200 import QSError, format_outcomes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def qstate_text(state):
    """CPUQuantumGates.cpp:64-82: one line per amplitude, default C++ stream
    formatting of a double (printf %g)."""
    return "".join(f"state[{i}].real = {a.real:g} state[{i}].imag = {a.imag:g}\n" for i, a in enumerate(state))


def test_golden_qstate_text_format():
    """The reference's getQState text for the gates_n7 state (written by
    tests/golden/make_golden.py from the reference backend) is the %g format
    that qs_write_fullstate produces."""
    st = np.load(os.path.join(GOLDEN, "gates_n7.npz"))["state"]
    with open(os.path.join(GOLDEN, "qstate_n7.txt")) as f:
        golden = f.read()
    assert golden == qstate_text(st)


def ref_result_text(keys, values, width):
    """QPandaSDK::getResult over a std::map<string, double> keyed by
    integerToBinary(key, width) (QPandaAPI.cpp:220-238, 295-305)."""
    m = {format(int(k), f"0{width}b"): float(v) for k, v in zip(keys, values)}
    return "".join(f"{k} {m[k]:g}\n" for k in sorted(m))


def test_format_outcomes_matches_getresult():
    rng = np.random.default_rng(5)
    for width in (1, 3, 10, 33):
        keys = np.unique(rng.integers(0, 2 ** width, size=min(10, 2 ** width), dtype=np.uint64))
        vals = rng.uniform(size=keys.size)
        perm = rng.permutation(keys.size)
        assert format_outcomes(keys[perm], vals[perm], width) == ref_result_text(keys, vals, width)
    assert format_outcomes([], [], 4) == ""
    # PMEASURE-style values of a uniform 2-qubit state
    assert format_outcomes([3, 0, 2, 1], [0.25] * 4, 2) == "00 0.25\n01 0.25\n10 0.25\n11 0.25\n"


def test_format_outcomes_rejects_bad_input():
    with pytest.raises(QSError):
        format_outcomes([1, 1], [0.5, 0.5], 2)        # a map holds each key once
    with pytest.raises(QSError):
        format_outcomes([4], [1.0], 2)                # key wider than the width
    with pytest.raises(QSError):
        format_outcomes([0], [1.0], 0)
