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
    return _lib


def run(path, backend, seed=12345, repeat=1):
    """Returns (kind, {bitstring: value}, n_qubits)."""
    buf = C.create_string_buffer(1 << 20)
    n = runner().qr_run(path.encode(), backend, seed, repeat, buf, len(buf))
    if n < 0:
        raise RuntimeError(f"qr_run({path}, backend={backend}) failed: {n}")
    text = buf.value.decode()
    kind, _, rest = text.partition(" ")
    res = {}
    for item in filter(None, rest.split(",")):
        k, v = item.split(":")
        res[k] = float(v)
    return kind, res, n
