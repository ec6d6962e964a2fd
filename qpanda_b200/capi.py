"""ctypes binding of the C ABI in include/qpanda_b200.h.

This is the Python view of the same entry points the C++ QuantumGates
subclass calls.  It loads the in-tree library qpanda_b200/_lib/libqsb200.so and
raises if it is missing: there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libqsb200.so")

QS_OK = 0
QS_C64 = 0
QS_C128 = 1

OP = dict(H=1, X=2, RX=3, RY=4, RZ=5, CNOT=6, CR=7, ISWAP=8, SQISWAP=9, TOFFOLI=10, CSWAP=11, SWAP=12)
MAX_CTRL = 16

# struct qs_gate (96 bytes)
GATE_DTYPE = np.dtype([("op", "<i4"), ("dagger", "<i4"), ("q", "<i4", (3,)), ("nctrl", "<i4"),
                       ("ctrl", "<i4", (MAX_CTRL,)), ("theta", "<f8")], align=True)
assert GATE_DTYPE.itemsize == 96


class QSError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"qpanda_b200 error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded library (loads on first use, raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m qpanda_b200.build` "
                          "(the CUDA extension is required; there is no CPU path)")
    L = C.CDLL(LIB_PATH)
    vp, i, d, u64, sz = C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_size_t
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    sig = {
        "qs_last_error": (C.c_char_p, []),
        "qs_version": (C.c_char_p, []),
        "qs_create": (i, [i, i, vp, C.POINTER(vp)]),
        "qs_destroy": (i, [vp]),
        "qs_num_qubits": (i, [vp, ip]),
        "qs_dtype": (i, [vp, ip]),
        "qs_device_ptr": (i, [vp, C.POINTER(vp)]),
        "qs_set_stream": (i, [vp, vp]),
        "qs_synchronize": (i, [vp]),
        "qs_reset_zero": (i, [vp]),
        "qs_set_state": (i, [vp, vp, i]),
        "qs_get_state": (i, [vp, vp, i]),
        "qs_gate_apply": (i, [vp, vp]),
        "qs_gates_apply": (i, [vp, vp, sz]),
        "qs_apply_1q": (i, [vp, i, dp, u64]),
        "qs_apply_unitary_1q": (i, [vp, i, dp]),
        "qs_apply_2q": (i, [vp, i, i, dp, u64]),
        "qs_apply_exchange": (i, [vp, i, i, dp, u64]),
        "qs_apply_phase": (i, [vp, u64, d, d]),
        "qs_prob_zero": (i, [vp, i, dp]),
        "qs_measure": (i, [vp, i, d, ip]),
        "qs_probs": (i, [vp, ip, i, dp]),
        "qs_pmeasure": (i, [vp, ip, i, C.POINTER(C.c_uint64), dp, ip]),
        "qs_sample": (i, [vp, ip, i, dp, sz, C.POINTER(C.c_uint64)]),
        "qs_norm2": (i, [vp, dp]),
        "qs_inner": (i, [vp, vp, dp, dp]),
        "qs_plan_create": (i, [i, vp, sz, i, C.POINTER(vp)]),
        "qs_create_async": (i, [i, i, vp, C.POINTER(vp)]),
        "qs_probs_device": (i, [vp, ip, i, vp]),
        "qs_server_default_opts": (i, [vp]),
        "qs_server_create": (i, [vp, C.POINTER(vp)]),
        "qs_server_submit": (i, [vp, i, vp, sz, i, dp, sz, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "qs_server_wait": (i, [vp, C.c_uint64, dp, dp]),
        "qs_server_fetch_probs": (i, [vp, C.c_uint64, dp]),
        "qs_server_release": (i, [vp, C.c_uint64]),
        "qs_server_stats": (i, [vp, C.POINTER(sz), C.POINTER(sz), C.POINTER(sz)]),
        "qs_server_destroy": (i, [vp]),
        "qs_batch_default_opts": (i, [vp]),
        "qs_batch_create": (i, [i, ip, vp, C.POINTER(sz), vp, C.POINTER(vp)]),
        "qs_batch_run": (i, [vp, vp]),
        "qs_batch_zz": (i, [vp, dp, C.POINTER(sz)]),
        "qs_batch_zz_offsets": (i, [vp, C.POINTER(sz)]),
        "qs_batch_state": (i, [vp, i, vp, i]),
        "qs_batch_info": (i, [vp, C.POINTER(sz), C.POINTER(sz)]),
        "qs_batch_destroy": (i, [vp]),
        "qs_batch_autotune": (i, [i, ip, vp, C.POINTER(sz), i, vp, dp]),
        "qs_batch_autotune_cached": (i, [i, ip, vp, C.POINTER(sz), i, C.c_char_p, vp, dp, ip]),
        "qs_plan_create_ex": (i, [i, vp, sz, vp, C.POINTER(vp)]),
        "qs_plan_default_opts": (i, [vp]),
        "qs_plan_autotune": (i, [vp, vp, sz, vp, i, vp, C.POINTER(C.c_double)]),
        "qs_plan_launches": (i, [vp, C.POINTER(sz)]),
        "qs_plan_destroy": (i, [vp]),
        "qs_plan_info": (i, [vp, C.POINTER(sz), C.POINTER(sz)]),
        "qs_plan_block": (i, [vp, sz, ip, ip, dp]),
        "qs_plan_pass": (i, [vp, sz, ip, ip, ip]),
        "qs_plan_apply": (i, [vp, vp]),
        "qs_plan_apply_range": (i, [vp, vp, sz, sz]),
        "qs_diff": (i, [vp, vp, dp, dp]),
        "qs_measure_noalloc": (i, [vp, i, i, i, d, vp, vp, vp]),
        "qs_plan_status": (i, [vp]),
        "qs_watchdog_selftest": (i, [vp, C.c_uint]),
        "qs_sharded_create": (i, [i, i, i, ip, i, vp, vp, C.POINTER(vp)]),
        "qs_sharded_apply": (i, [vp, vp, sz]),
        "qs_sharded_shard": (i, [vp, i, C.POINTER(vp)]),
        "qs_sharded_positions": (i, [vp, ip]),
        "qs_sharded_set_peer": (i, [vp, i, vp, vp, vp]),
        "qs_sharded_info": (i, [vp, C.POINTER(sz), C.POINTER(sz)]),
        "qs_sharded_destroy": (i, [vp]),
        "qs_release_spare": (i, [vp]),
        "qs_write_fullstate": (i, [vp, C.c_char_p, i]),
        "qs_format_outcomes": (i, [C.POINTER(C.c_uint64), dp, sz, i, C.c_char_p, sz, C.POINTER(sz)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(code):
    if code != QS_OK:
        raise QSError(code, lib().qs_last_error().decode(errors="replace"))


def format_outcomes(keys, values, width):
    """QPandaSDK::getResult text of an outcome map (qs_format_outcomes)."""
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    v = np.ascontiguousarray(values, dtype=np.float64)
    need = C.c_size_t()
    check(lib().qs_format_outcomes(k.ctypes.data_as(C.POINTER(C.c_uint64)), _dptr(v), k.size, int(width),
                                   None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    check(lib().qs_format_outcomes(k.ctypes.data_as(C.POINTER(C.c_uint64)), _dptr(v), k.size, int(width),
                                   buf, need.value, C.byref(need)))
    return buf.value.decode()


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class StateVector:
    """One state vector resident in HBM, driven through the C ABI."""

    def __init__(self, n, dtype="c64", stream=None):
        self.n = int(n)
        self.dtype = QS_C64 if dtype in ("c64", QS_C64, np.complex64) else QS_C128
        h = C.c_void_p()
        check(lib().qs_create(self.n, self.dtype, stream, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().qs_destroy(self._h)
            self._h = None

    def release_spare(self):
        """Free the second buffer that remapping plans keep with the state."""
        check(lib().qs_release_spare(self._h))

    def write_fullstate(self, path_prefix, binary=False):
        """Write <prefix>.fullstate (getQState text) or <prefix>.fullstate.binary."""
        check(lib().qs_write_fullstate(self._h, os.fsencode(path_prefix), 1 if binary else 0))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state
    def reset(self):
        check(lib().qs_reset_zero(self._h))

    def set_state(self, amps):
        a = np.ascontiguousarray(amps)
        dt = QS_C64 if a.dtype == np.complex64 else QS_C128
        if dt == QS_C128:
            a = np.ascontiguousarray(a, dtype=np.complex128)
        assert a.size == (1 << self.n)
        check(lib().qs_set_state(self._h, a.ctypes.data, dt))

    def get_state(self, dtype=np.complex128):
        out = np.empty(1 << self.n, dtype=dtype)
        check(lib().qs_get_state(self._h, out.ctypes.data, QS_C64 if dtype == np.complex64 else QS_C128))
        return out

    def synchronize(self):
        check(lib().qs_synchronize(self._h))

    # -- gates
    def apply(self, gates):
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        check(lib().qs_gates_apply(self._h, g.ctypes.data, g.size))

    def apply_1q(self, q, m, ctrl_mask=0):
        m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(2, 2)).view(np.float64)
        check(lib().qs_apply_1q(self._h, q, _dptr(m), ctrl_mask))

    def apply_unitary_1q(self, q, m):
        m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(2, 2)).view(np.float64)
        check(lib().qs_apply_unitary_1q(self._h, q, _dptr(m)))

    def apply_2q(self, q0, q1, m, ctrl_mask=0):
        m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(4, 4)).view(np.float64)
        check(lib().qs_apply_2q(self._h, q0, q1, _dptr(m), ctrl_mask))

    def apply_exchange(self, a, b, m, ctrl_mask=0):
        m = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(2, 2)).view(np.float64)
        check(lib().qs_apply_exchange(self._h, a, b, _dptr(m), ctrl_mask))

    def apply_phase(self, mask, phase):
        check(lib().qs_apply_phase(self._h, mask, float(np.real(phase)), float(np.imag(phase))))

    # -- measurement
    def prob_zero(self, q):
        p = C.c_double()
        check(lib().qs_prob_zero(self._h, q, C.byref(p)))
        return p.value

    def measure(self, q, u):
        o = C.c_int()
        check(lib().qs_measure(self._h, q, float(u), C.byref(o)))
        return o.value

    def probs(self, qubits=None):
        qs = np.arange(self.n, dtype=np.int32) if qubits is None else np.asarray(qubits, dtype=np.int32)
        out = np.empty(1 << len(qs), dtype=np.float64)
        check(lib().qs_probs(self._h, _iptr(qs), len(qs), _dptr(out)))
        return out

    def pmeasure(self, qubits):
        qs = np.asarray(qubits, dtype=np.int32)
        idx = np.zeros(10, dtype=np.uint64)
        p = np.zeros(10, dtype=np.float64)
        cnt = C.c_int()
        check(lib().qs_pmeasure(self._h, _iptr(qs), len(qs), idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                _dptr(p), C.byref(cnt)))
        return list(zip(idx[:cnt.value].tolist(), p[:cnt.value].tolist()))

    def sample(self, qubits, u):
        qs = np.asarray(qubits, dtype=np.int32)
        u = np.ascontiguousarray(u, dtype=np.float64)
        shots = u.size // len(qs)
        out = np.empty(shots, dtype=np.uint64)
        check(lib().qs_sample(self._h, _iptr(qs), len(qs), _dptr(u), shots,
                              out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def norm2(self):
        d = C.c_double()
        check(lib().qs_norm2(self._h, C.byref(d)))
        return d.value

    def diff(self, other):
        """(max |a_i - b_i|, sum |a_i - b_i|^2), computed on the device."""
        m, s2 = C.c_double(), C.c_double()
        check(lib().qs_diff(self._h, other._h, C.byref(m), C.byref(s2)))
        return m.value, s2.value

    def inner(self, other):
        re, im = C.c_double(), C.c_double()
        check(lib().qs_inner(self._h, other._h, C.byref(re), C.byref(im)))
        return complex(re.value, im.value)


class PlanOpts(C.Structure):
    _fields_ = [("block_qubits", C.c_int), ("tile_qubits", C.c_int), ("max_sub", C.c_int),
                ("low_qubits", C.c_int), ("kernel", C.c_int), ("remap", C.c_int), ("threads_per_row", C.c_int),
                ("tile_in_tmem", C.c_int)]


PLAN_SINGLE, PLAN_TILED = 1, 2


class FusionPlan:
    """Gate list fused into dense 5-qubit blocks (qs_plan_*).  kernel="tiled"
    (default) applies up to max_sub blocks per pass over the state;
    kernel="single" one block per pass.  remap=1: tiled passes write their
    tiles as contiguous runs into a second state-size buffer kept with the
    state (twice the memory; faster passes on large states); remap=2: the
    next pass's tiles contiguous instead (qs_plan_opts.remap).
    threads_per_row=2: tiled passes with two threads per tile row
    (qs_plan_opts.threads_per_row; measured slightly slower than 1).
    tile_in_tmem=0: keep every pass's tile in shared memory instead of tensor
    memory (qs_plan_opts.tile_in_tmem)."""

    def __init__(self, n, gates, max_k=5, kernel="tiled", max_sub=2, low_qubits=3, remap=False, threads_per_row=1,
                 tile_in_tmem=1):
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        self._keep = g
        h = C.c_void_p()
        if kernel == "single":
            check(lib().qs_plan_create(int(n), g.ctypes.data, g.size, int(max_k), C.byref(h)))
        else:
            o = PlanOpts()
            check(lib().qs_plan_default_opts(C.byref(o)))
            o.block_qubits, o.max_sub, o.low_qubits = int(max_k), int(max_sub), int(low_qubits)
            o.remap = int(remap)
            o.threads_per_row = int(threads_per_row)
            o.tile_in_tmem = int(tile_in_tmem)
            check(lib().qs_plan_create_ex(int(n), g.ctypes.data, g.size, C.byref(o), C.byref(h)))
        self._h = h
        self.n = int(n)
        self.kernel = kernel

    def num_launches(self):
        nl = C.c_size_t()
        check(lib().qs_plan_launches(self._h, C.byref(nl)))
        return nl.value

    def close(self):
        if self._h:
            lib().qs_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def num_blocks(self):
        nb, ng = C.c_size_t(), C.c_size_t()
        check(lib().qs_plan_info(self._h, C.byref(nb), C.byref(ng)))
        return nb.value

    def block(self, i):
        k = C.c_int()
        q = np.zeros(5, dtype=np.int32)
        m = np.zeros(2 * 32 * 32)
        check(lib().qs_plan_block(self._h, i, C.byref(k), _iptr(q), _dptr(m)))
        return q.tolist(), m.view(np.complex128).reshape(32, 32)

    def passes(self):
        """Tiled plans: [(tile_qubits, [block qubits, ...]), ...] per pass."""
        out = []
        for i in range(self.num_launches()):
            nb = C.c_int()
            T = np.zeros(12, dtype=np.int32)
            Q = np.zeros(15, dtype=np.int32)
            check(lib().qs_plan_pass(self._h, i, C.byref(nb), _iptr(T), _iptr(Q)))
            out.append((T.tolist(), [Q[5 * b:5 * b + 5].tolist() for b in range(nb.value)]))
        return out

    def apply(self, sv):
        check(lib().qs_plan_apply(sv.handle, self._h))

    def apply_range(self, sv, first, count):
        check(lib().qs_plan_apply_range(sv.handle, self._h, first, count))

    def status(self, sv):
        check(lib().qs_plan_status(sv.handle))


class BatchOpts(C.Structure):
    _fields_ = [("max_sub", C.c_int), ("low_qubits", C.c_int), ("order", C.c_int), ("use_graph", C.c_int),
                ("block_qubits", C.c_int), ("tile_in_tmem", C.c_int)]


def _concat(circuits_list):
    nq = np.array([n for n, _ in circuits_list], dtype=np.int32)
    offs = np.zeros(len(circuits_list) + 1, dtype=np.uint64)
    for k, (_, g) in enumerate(circuits_list):
        offs[k + 1] = offs[k] + len(g)
    gates = np.ascontiguousarray(np.concatenate([np.asarray(g, dtype=GATE_DTYPE) for _, g in circuits_list]),
                                 dtype=GATE_DTYPE)
    return nq, gates, offs


def autotune_plan(sv, gates, remap=False, reps=1):
    """Fastest tiled-plan options for this circuit on this state
    (qs_plan_autotune: tile in tensor or shared memory, 2 or 3 blocks per
    pass, 2 or 3 low qubits, or 1 with remap) and its time per application
    in ms.  Overwrites the state."""
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    base, best, ms = PlanOpts(), PlanOpts(), C.c_double()
    check(lib().qs_plan_default_opts(C.byref(base)))
    base.remap = int(remap)
    check(lib().qs_plan_autotune(sv.handle, g.ctypes.data, g.size, C.byref(base), int(reps), C.byref(best),
                                 C.byref(ms)))
    return best, ms.value


def autotune_batch(circuits_list, stride=8, cache=None):
    """Fastest BatchOpts for these circuits (timed on every stride-th one) and
    its time per run in ms.  cache: a file that keeps tunings by device and
    gate pattern (qs_batch_autotune_cached); then returns (opts, ms, hit)."""
    nq, gates, offs = _concat(circuits_list)
    best, ms = BatchOpts(), C.c_double()
    if cache is None:
        check(lib().qs_batch_autotune(len(nq), _iptr(nq), gates.ctypes.data,
                                      offs.ctypes.data_as(C.POINTER(C.c_size_t)), int(stride), C.byref(best),
                                      C.byref(ms)))
        return best, ms.value
    hit = C.c_int()
    check(lib().qs_batch_autotune_cached(len(nq), _iptr(nq), gates.ctypes.data,
                                         offs.ctypes.data_as(C.POINTER(C.c_size_t)), int(stride),
                                         str(cache).encode(), C.byref(best), C.byref(ms), C.byref(hit)))
    return best, ms.value, bool(hit.value)


class Batch:
    """Many circuits run from |0...0> in one persistent launch (qs_batch_*).
    circuits_list: [(n_qubits, gate records), ...]."""

    def __init__(self, circuits_list, opts=None, **kw):
        nq, gates, offs = _concat(circuits_list)
        self.nq = nq
        o = BatchOpts()
        if opts is not None:
            o = opts
        else:
            check(lib().qs_batch_default_opts(C.byref(o)))
        for k, v in kw.items():
            setattr(o, k, int(v))
        h = C.c_void_p()
        check(lib().qs_batch_create(len(nq), _iptr(nq), gates.ctypes.data,
                                    offs.ctypes.data_as(C.POINTER(C.c_size_t)), C.byref(o), C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().qs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, stream=None):
        check(lib().qs_batch_run(self._h, stream))

    def zz(self):
        """List of arrays: <Z_i Z_{i+1}> for each circuit."""
        cnt = C.c_size_t()
        check(lib().qs_batch_zz(self._h, None, C.byref(cnt)))
        out = np.empty(cnt.value)
        check(lib().qs_batch_zz(self._h, _dptr(out), C.byref(cnt)))
        offs = np.empty(len(self.nq) + 1, dtype=np.uint64)
        check(lib().qs_batch_zz_offsets(self._h, offs.ctypes.data_as(C.POINTER(C.c_size_t))))
        return [out[int(offs[k]):int(offs[k + 1])] for k in range(len(self.nq))]

    def state(self, c, dtype=np.complex128):
        out = np.empty(1 << int(self.nq[c]), dtype=dtype)
        check(lib().qs_batch_state(self._h, int(c), out.ctypes.data, QS_C64 if dtype == np.complex64 else QS_C128))
        return out


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("slots", C.c_int), ("bypass", C.c_int)]


REQ_SHOTS, REQ_PROBS = 1, 2


class Server:
    """Request loop with continuous batching (qs_server_*)."""

    def __init__(self, budget_bytes=None, slots=None, bypass=None):
        o = ServerOpts()
        check(lib().qs_server_default_opts(C.byref(o)))
        if budget_bytes is not None:
            o.hbm_budget_bytes = int(budget_bytes)
        if slots is not None:
            o.slots = int(slots)
        if bypass is not None:
            o.bypass = int(bypass)
        h = C.c_void_p()
        check(lib().qs_server_create(C.byref(o), C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, n, gates, kind="shots", uniforms=None):
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        rid = C.c_uint64()
        if kind == "shots":
            u = np.ascontiguousarray(uniforms, dtype=np.float64)
            shots = u.size // n
            out = np.zeros(shots, dtype=np.uint64)
            check(lib().qs_server_submit(self._h, int(n), g.ctypes.data, g.size, REQ_SHOTS, _dptr(u), shots,
                                         out.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(rid)))
            self._keep[rid.value] = (u, out, n)
        else:
            check(lib().qs_server_submit(self._h, int(n), g.ctypes.data, g.size, REQ_PROBS, None, 0, None,
                                         C.byref(rid)))
            self._keep[rid.value] = (None, None, n)
        return rid.value

    def wait(self, rid):
        lat, svc = C.c_double(), C.c_double()
        check(lib().qs_server_wait(self._h, C.c_uint64(rid), C.byref(lat), C.byref(svc)))
        return lat.value, svc.value

    def shots(self, rid):
        return self._keep[rid][1]

    def fetch_probs(self, rid):
        out = np.empty(1 << self._keep[rid][2])
        check(lib().qs_server_fetch_probs(self._h, C.c_uint64(rid), _dptr(out)))
        return out

    def release(self, rid):
        check(lib().qs_server_release(self._h, C.c_uint64(rid)))
        self._keep.pop(rid, None)

    def stats(self):
        a, b, c = C.c_size_t(), C.c_size_t(), C.c_size_t()
        check(lib().qs_server_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"served": a.value, "max_concurrent": b.value, "hbm_in_use": c.value}

    def close(self):
        if self._h:
            lib().qs_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
