"""ctypes access to the CPU checkers.  TEST INFRASTRUCTURE ONLY.

OracleState wraps oracle/_build/liboracle.so (the C restatement of
QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp).  RefState wraps
oracle/_ref/libqpanda_ref.so, the reference's own CPU backend compiled from its
sources, when it has been built.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqpanda_ref.so")
REF_OMP_SO = os.path.join(HERE, "_ref", "libqpanda_ref_omp.so")

_vp, _i, _d, _u64, _sz = C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_size_t
_dp, _ip = C.POINTER(C.c_double), C.POINTER(C.c_int)


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def _load_oracle():
    if not os.path.exists(ORACLE_SO):
        build_oracle()
    L = C.CDLL(ORACLE_SO)
    sig = {
        "orc_create": (_vp, [_i]), "orc_destroy": (None, [_vp]), "orc_data": (_dp, [_vp]),
        "orc_size": (_u64, [_vp]), "orc_reset": (None, [_vp]),
        "orc_gate": (_i, [_vp, _vp]), "orc_gates": (_i, [_vp, _vp, _u64]),
        "orc_u1q": (_i, [_vp, _i, _dp, _ip, _i]),
        "orc_prob_zero": (_i, [_vp, _i, _dp]), "orc_measure": (_i, [_vp, _i, _d]),
        "orc_pmeasure": (_i, [_vp, _ip, _i, _dp]),
        "orc_sample": (_i, [_vp, _ip, _i, _dp, _u64, C.POINTER(C.c_uint64)]),
        "orc_norm2": (_d, [_vp]), "orc_rand16807": (_d, [_ip]),
    }
    for k, (r, a) in sig.items():
        f = getattr(L, k)
        f.restype = r
        f.argtypes = a
    return L


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = _load_oracle()
    return _oracle


def _as_gates(g):
    from qpanda_b200.capi import GATE_DTYPE
    return np.ascontiguousarray(g, dtype=GATE_DTYPE)


class OracleState:
    """FP64 CPU restatement of the reference backend."""

    def __init__(self, n):
        self.L = oracle_lib()
        self.n = n
        self.h = self.L.orc_create(n)
        if not self.h:
            raise MemoryError(f"oracle: cannot allocate {n} qubits")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def view(self):
        """Live complex128 view of the amplitudes."""
        p = self.L.orc_data(self.h)
        a = np.ctypeslib.as_array(p, shape=(2 << self.n,))
        return a.view(np.complex128)

    def state(self):
        return self.view().copy()

    def set_state(self, amps):
        self.view()[:] = np.asarray(amps, dtype=np.complex128)

    def reset(self):
        self.L.orc_reset(self.h)

    def apply(self, gates):
        g = _as_gates(gates)
        r = self.L.orc_gates(self.h, g.ctypes.data, g.size)
        if r:
            raise ValueError(f"oracle rejected gate {-1 - r}")

    def apply_u1q(self, q, m, ctrl=()):
        m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(2, 2)).view(np.float64)
        c = np.asarray(ctrl, dtype=np.int32)
        if self.L.orc_u1q(self.h, q, m.ctypes.data_as(_dp), c.ctypes.data_as(_ip), len(c)):
            raise ValueError("oracle rejected u1q")

    def prob_zero(self, q):
        p = C.c_double()
        self.L.orc_prob_zero(self.h, q, C.byref(p))
        return p.value

    def measure(self, q, u):
        return self.L.orc_measure(self.h, q, float(u))

    def probs(self, qubits=None):
        qs = np.arange(self.n, dtype=np.int32) if qubits is None else np.asarray(qubits, dtype=np.int32)
        out = np.empty(1 << len(qs))
        self.L.orc_pmeasure(self.h, qs.ctypes.data_as(_ip), len(qs), out.ctypes.data_as(_dp))
        return out

    def sample(self, qubits, u):
        qs = np.asarray(qubits, dtype=np.int32)
        u = np.ascontiguousarray(u, dtype=np.float64)
        shots = u.size // len(qs)
        out = np.empty(shots, dtype=np.uint64)
        r = self.L.orc_sample(self.h, qs.ctypes.data_as(_ip), len(qs), u.ctypes.data_as(_dp), shots,
                              out.ctypes.data_as(C.POINTER(C.c_uint64)))
        if r:
            raise ValueError("oracle sample failed")
        return out

    def norm2(self):
        return self.L.orc_norm2(self.h)


def ref_available(omp=False):
    return os.path.exists(REF_OMP_SO if omp else REF_SO)


_ref = {}


def ref_lib(omp=False):
    key = bool(omp)
    if key in _ref:
        return _ref[key]
    path = REF_OMP_SO if omp else REF_SO
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built (make -C oracle ref, needs the reference tree)")
    L = C.CDLL(path)
    sig = {
        "ref_create": (_vp, [_i]), "ref_destroy": (None, [_vp]), "ref_data": (_dp, [_vp]),
        "ref_size": (_sz, [_vp]), "ref_end_gate": (None, [_vp]),
        "ref_gate": (_i, [_vp, _vp]), "ref_gates": (_i, [_vp, _vp, _sz]),
        "ref_measure": (_i, [_vp, _i, _d]),
        "ref_pmeasure": (_i, [_vp, _ip, _i, C.POINTER(C.c_size_t), _dp]),
        "ref_sample": (_i, [_vp, _ip, _i, _dp, _sz, C.POINTER(C.c_uint64)]),
        "ref_rng_seed": (None, [_i]), "ref_rng_set_next": (None, [_d]),
        "ref_qstate_text": (C.c_long, [_vp, C.c_char_p, _sz]),
    }
    for k, (r, a) in sig.items():
        f = getattr(L, k)
        f.restype = r
        f.argtypes = a
    _ref[key] = L
    return L


class RefState:
    """The reference's own CPUQuantumGates, compiled from its sources."""

    def __init__(self, n, omp=False):
        self.L = ref_lib(omp)
        self.n = n
        self.h = self.L.ref_create(n)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def view(self):
        p = self.L.ref_data(self.h)
        return np.ctypeslib.as_array(p, shape=(2 << self.n,)).view(np.complex128)

    def state(self):
        return self.view().copy()

    def set_state(self, amps):
        self.view()[:] = np.asarray(amps, dtype=np.complex128)

    def apply(self, gates):
        g = _as_gates(gates)
        r = self.L.ref_gates(self.h, g.ctypes.data, g.size)
        if r < 0:
            raise ValueError("reference rejected a gate")
        return r

    def measure(self, q, u):
        return self.L.ref_measure(self.h, q, float(u))

    def pmeasure(self, qubits):
        qs = np.asarray(qubits, dtype=np.int32)
        idx = np.zeros(max(10, 1 << len(qs)), dtype=np.uintp)
        p = np.zeros(idx.size)
        cnt = self.L.ref_pmeasure(self.h, qs.ctypes.data_as(_ip), len(qs),
                                  idx.ctypes.data_as(C.POINTER(C.c_size_t)), p.ctypes.data_as(_dp))
        return list(zip(idx[:cnt].tolist(), p[:cnt].tolist()))

    def qstate_text(self):
        """The reference's getQState text (CPUQuantumGates.cpp:64-82)."""
        need = -self.L.ref_qstate_text(self.h, None, 0)
        buf = C.create_string_buffer(int(need))
        r = self.L.ref_qstate_text(self.h, buf, need)
        if r < 0:
            raise RuntimeError("reference getQState failed")
        return buf.value.decode()

    def sample(self, qubits, u):
        qs = np.asarray(qubits, dtype=np.int32)
        u = np.ascontiguousarray(u, dtype=np.float64)
        shots = u.size // len(qs)
        out = np.empty(shots, dtype=np.uint64)
        self.L.ref_sample(self.h, qs.ctypes.data_as(_ip), len(qs), u.ctypes.data_as(_dp), shots,
                          out.ctypes.data_as(C.POINTER(C.c_uint64)))
        return out
