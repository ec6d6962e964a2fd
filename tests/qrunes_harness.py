"""ctypes access to tests/qrunes/_build/libqrunes_runner.so (see
tests/qrunes/Makefile): QRunes programs through the reference's own parser and
dispatcher with either backend.  TEST INFRASTRUCTURE."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
RUNNER_SO = os.path.join(HERE, "qrunes", "_build", "libqrunes_runner.so")
CPU, B200_C128, B200_C64, GPU_UNIT = 0, 1, 2, 3
EMU_SO = os.path.join(os.path.dirname(HERE), "qpanda_b200", "_lib", "libGPUEmulator.so")


def available():
    return os.path.exists(RUNNER_SO)


_lib = None


def runner():
    global _lib
    if _lib is None:
        import qpanda_b200
        qpanda_b200.lib()                      # the product library first (same process)
        # the GPU compute unit dlopens "libGPUEmulator.so" by name: load ours first
        C.CDLL(EMU_SO, mode=C.RTLD_GLOBAL)
        _lib = C.CDLL(RUNNER_SO)
        _lib.qr_run.restype = C.c_int
        _lib.qr_run.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_size_t]
        _lib.qr_run_ex.restype = C.c_int
        _lib.qr_run_ex.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_size_t,
                                   C.POINTER(C.c_int)]
        _lib.qr_qstate.restype = C.c_long
        _lib.qr_qstate.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_size_t]
    return _lib


def run(path, backend, seed=12345, repeat=1, sample=False, runs_out=None):
    """Returns (kind, {bitstring: value}, n_qubits).  sample: a B200 backend
    runs a program whose measurements are all terminal once and samples the
    shots (B200QuantumGates deferred measurement); runs_out (a list) receives
    the number of simulations."""
    buf = C.create_string_buffer(1 << 20)
    runs = C.c_int(0)
    n = runner().qr_run_ex(path.encode(), backend, seed, repeat, int(sample), buf, len(buf), C.byref(runs))
    if n < 0:
        raise RuntimeError(f"qr_run({path}, backend={backend}) failed: {n}")
    if runs_out is not None:
        runs_out.append(runs.value)
    text = buf.value.decode()
    kind, _, rest = text.partition(" ")
    res = {}
    for item in filter(None, rest.split(",")):
        k, v = item.split(":")
        res[k] = float(v)
    return kind, res, n


def qstate_text(path, backend, seed=12345):
    """The backend's getQState text after one run of the program."""
    need = 1 << 16
    while True:
        buf = C.create_string_buffer(need)
        r = runner().qr_qstate(path.encode(), backend, seed, buf, len(buf))
        if r >= 0:
            return buf.value.decode()
        if r < -5 and -r > need:
            need = -r
            continue
        raise RuntimeError(f"qr_qstate({path}, backend={backend}) failed: {r}")
