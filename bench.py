"""Benchmark: 32-qubit random circuit on one B200 (and N replicas on N GPUs).

Workload: 32 qubits, complex64 state (32 GiB, far larger than L2, so no flush
between steps), depth 16; each layer an RX/RY/RZ on every qubit (axis and
angle seeded) then a two-qubit gate on every pair of a seeded random perfect
matching: CNOT, or iSWAP on 10% of the pairs.  768 gates.

A step = reset to |0...0> and run the whole circuit: on the fused path
(default) the gate list fused into dense 5-qubit blocks applied on the tensor
cores, on the plain path one kernel per gate.  The other path runs one step in
the same process for the comparison, and a 30-qubit run of the same circuit
structure checks the fused complex64 result against the complex128 per-gate
path (fidelity, max amplitude error).  `value` is circuits per second over
all ranks (each rank runs its own replica: the state does not shard at 32
qubits); `e2e` is the same metric through the C ABI with the gate list and
the shot uniforms copied from pinned host memory each step and 1024 sampled
bitstrings copied back.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--path plain|fused]
  python bench.py --impl reference      # the reference CPU backend on the host
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "32q random-circuit time & HBM GB/s: fused-TC vs plain per-gate, 1 B200, fid≥1-1e-6"
N_QUBITS, DEPTH, ISWAP_FRAC, SEED = 32, 16, 0.1, 20240601
SHOTS = 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--path", default="fused", choices=["plain", "fused"])
    ap.add_argument("--kernel", default="tiled", choices=["tiled", "single"],
                    help="fused path: tiled passes (up to 3 blocks per pass) or one block per pass")
    ap.add_argument("--max-sub", type=int, default=2, choices=[1, 2, 3],
                    help="tiled passes: fused blocks per pass")
    ap.add_argument("--low", type=int, default=3, choices=[1, 2, 3, 4, 5],
                    help="tiled passes: qubits 0..low-1 in every tile (contiguous runs of 2^low amplitudes)")
    ap.add_argument("--remap", type=int, default=1, choices=[0, 1],
                    help="tiled passes: 1 = contiguous tile writes through a second state-size buffer")
    ap.add_argument("--tile-in-tmem", type=int, default=1, choices=[0, 1],
                    help="tiled passes: 1 = the tile in tensor memory where a pass fits (k_tile_tmem), "
                         "0 = always in shared memory (k_fused_tile)")
    ap.add_argument("--tune", type=int, default=1, choices=[0, 1],
                    help="fused tiled path: 1 = pick tile_in_tmem, max_sub and low by timing the candidates on "
                         "the state first (qs_plan_autotune, untimed); 0 = use the flags as given")
    ap.add_argument("--tpr", type=int, default=1, choices=[1, 2],
                    help="tiled passes: threads per tile row (1: 128 per lane, 2: 256, 16 columns each)")
    ap.add_argument("--qubits", type=int, default=N_QUBITS)
    ap.add_argument("--depth", type=int, default=DEPTH)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="default workload: skip the short runs of the other workloads")
    ap.add_argument("--workload", default="circuit32",
                    choices=["circuit32", "circuit20", "vqe-sweep", "requests", "qft28", "passes", "kernels"],
                    help="circuit32: the 32-qubit random circuit (default); circuit20: the 20-qubit complex128 "
                         "random circuit on the per-gate path, CPU reference timed directly; vqe-sweep: 4096 "
                         "hardware-efficient-ansatz circuits of 10-22 qubits in one persistent launch; "
                         "requests: Poisson request trace against the server; qft28: 28-qubit QFT on the "
                         "plain per-gate path in complex64 and complex128; passes: the random circuit "
                         "(--qubits) applied once per tiled layout (in place, remap 1, remap 2) with its "
                         "pass structure, for per-launch profiling")
    ap.add_argument("--circuits", type=int, default=4096)
    ap.add_argument("--no-autotune", action="store_true",
                    help="vqe-sweep: run with the default batch options instead of the autotuned ones")
    ap.add_argument("--requests", type=int, default=20000, help="requests workload: trace length")
    ap.add_argument("--every", type=int, default=10, help="requests workload: serve every k-th request")
    return ap.parse_args()


# ----------------------------------------------------------------- distributed
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws, backend):
    import datetime

    import torch.distributed as dist
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws, device=None):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(gpu_id)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- workload
def workload(n, depth):
    from qpanda_b200 import circuits
    return circuits.random_layers(n, depth, SEED, iswap_frac=ISWAP_FRAC)


def kernel_kind(g):
    from qpanda_b200.capi import OP
    op = int(g["op"])
    if op in (OP["H"], OP["X"], OP["RX"], OP["RY"], OP["RZ"]) and int(g["nctrl"]) == 0:
        return "k_pair (1-qubit, dense 2x2)"
    if op in (OP["CNOT"], OP["ISWAP"], OP["SQISWAP"], OP["SWAP"], OP["TOFFOLI"], OP["CSWAP"]):
        return "k_pair (controlled / exchange)"
    if op == OP["CR"]:
        return "k_phase"
    return "other"


def load_traffic():
    """Per-launch DRAM traffic of the bench kernels from the committed ncu
    summary (profiles/traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------- reference arm
REF_QUBITS = 30          # the largest state the reference takes (QPandaAPI.cpp:87), complex128: 16 GiB
REF_GATES_PER_STEP = 8


def circuit_gate_count(n, depth):
    """Gates of random_layers(n, depth): a rotation per qubit and a pair gate
    per matched pair, per layer."""
    return depth * (n + n // 2)


class RefSampler:
    """The reference CPU backend (CPUQuantumGates.cpp compiled from its
    sources, oracle/_ref) on the benchmark circuit's structure at
    min(n, 30) qubits in complex128 (its only precision): each step applies
    the next `REF_GATES_PER_STEP` gates of that circuit (cycling) and is timed
    on its own.  A circuit of n qubits is then  seconds per gate x its gate
    count x 2^(n - sample qubits)  (every gate of the reference loops over the
    whole state).  omp: the -fopenmp build on every host core, else the
    shipped single-threaded build."""

    def __init__(self, n, depth, omp):
        from oracle.pyoracle import RefState, ref_available
        if not ref_available(omp):
            raise FileNotFoundError("oracle/_ref not built")
        self.n, self.depth, self.omp = n, depth, omp
        self.ns = min(n, REF_QUBITS)
        self.gates = workload(self.ns, depth)
        self.state = RefState(self.ns, omp=omp)
        self.pos = 0
        self.secs = 0.0
        self.count = 0

    def step(self, k=REF_GATES_PER_STEP, record=True):
        idx = [(self.pos + i) % len(self.gates) for i in range(k)]
        self.pos = (self.pos + k) % len(self.gates)
        g = self.gates[idx]
        t0 = time.perf_counter()
        self.state.apply(g)
        dt = time.perf_counter() - t0
        if record:
            self.secs += dt
            self.count += k
        return dt

    def circuit_seconds(self):
        return self.secs / self.count * circuit_gate_count(self.n, self.depth) * 2 ** (self.n - self.ns)

    def describe(self):
        cores = os.cpu_count() or 1
        build = f"-O3 -fopenmp, {cores} threads" if self.omp else "-O3, 1 thread (as shipped)"
        return (f"reference CPUQuantumGates.cpp ({build}, complex128) on the {self.n}-qubit depth-{self.depth} "
                f"circuit's structure at {self.ns} qubits: {self.count} gates in {self.secs:.2f} s, "
                f"{1e3 * self.secs / self.count:.0f} ms per gate; x{circuit_gate_count(self.n, self.depth)} gates"
                + (f" x{2 ** (self.n - self.ns)} (state size)" if self.n > self.ns else "")
                + f" = {self.circuit_seconds():.0f} s per circuit"
                + (f" (extrapolated: a {self.n}-qubit complex128 state is {16 << self.n >> 30} GiB and the reference "
                   f"caps programs at {REF_QUBITS} qubits)" if self.n > self.ns else ""))

    def close(self):
        self.state = None


def cpu_baseline_entry(n, depth):
    """The cpu_baseline of the B200 line: a bounded sample on both builds."""
    cores = os.cpu_count() or 1
    omp = RefSampler(n, depth, omp=True)
    omp.step(record=False)                     # first touch of the 16 GiB state
    for _ in range(3):
        omp.step()
    out = {"value": 1.0 / omp.circuit_seconds(), "unit": "circuits/s", "cores": cores, "kind": "reference",
           "sample": omp.describe()}
    omp.close()
    one = RefSampler(n, depth, omp=False)
    one.step(k=4)
    out["single_core"] = {"value": 1.0 / one.circuit_seconds(), "unit": "circuits/s", "cores": 1,
                          "sample": one.describe()}
    one.close()
    out["host"] = host_cpu()
    return out


def host_cpu():
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "model": model}


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    n, depth = args.qubits, args.depth
    if args.workload == "circuit20":
        return run_reference_circuit20(args)
    cores = os.cpu_count() or 1
    smp = RefSampler(n, depth, omp=True)
    smp.step(record=False)                     # first touch of the state
    steps = []
    for i in range(args.warmup + args.steps):
        dt = smp.step(record=i >= args.warmup)
        if i >= args.warmup:
            steps.append(dt)
    circuit_s = smp.circuit_seconds()
    value = 1.0 / circuit_s
    sample = smp.describe() + f"; each step = {REF_GATES_PER_STEP} consecutive gates of that circuit"
    smp.close()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "circuits/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(steps) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"random-circuit-{n}q-depth{depth}", "qubits": n, "depth": depth,
                   "iswap_frac": ISWAP_FRAC, "seed": SEED, "sample_qubits": smp.ns,
                   "gates_per_step": REF_GATES_PER_STEP},
        "cpu_baseline": {"value": value, "unit": "circuits/s", "cores": cores, "kind": "reference",
                         "sample": sample, "host": host_cpu()},
        "e2e": {"value": value, "unit": "circuits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ----------------------------------------------------------------- B200 arm
def timed_steps(L, h, gates, plan, steps, stream, torch, kinds, path):
    """Run `steps` circuits on the device with an event after every launch.
    Returns per-step device seconds; appends per-launch durations to kinds."""
    import ctypes as C
    from qpanda_b200.capi import check
    ng = len(gates)
    nb = plan.num_launches() if plan is not None else 0
    nl = nb if path == "fused" else ng
    fused_name = (("k_tile_tmem (tiled pass, tile in tensor memory)" if getattr(plan, "tile_in_tmem", 0)
                   else "k_fused_tile (tiled pass)") if getattr(plan, "kernel", "tiled") == "tiled"
                  else "k_fused_tc (5-qubit block)")
    gptr = [gates[i:i + 1].ctypes.data for i in range(ng)]
    whole = path == "fused" and getattr(plan, "remap", False)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(nl + 1)] for _ in range(steps)]
    for k in range(steps):
        check(L.qs_reset_zero(h))
        ev[k][0].record(stream)
        if whole:
            # a remapping plan's passes hand their layouts on to each other:
            # one application, timed as a whole
            check(L.qs_plan_apply(h, plan.handle))
            ev[k][nl].record(stream)
            continue
        for i in range(nl):
            if path == "fused":
                check(L.qs_plan_apply_range(h, plan.handle, i, 1))
            else:
                check(L.qs_gate_apply(h, C.c_void_p(gptr[i])))
            ev[k][i + 1].record(stream)
    torch.cuda.synchronize()
    out = []
    for k in range(steps):
        out.append(ev[k][0].elapsed_time(ev[k][nl]) / 1e3)
        if whole:
            kinds.setdefault(fused_name, []).extend([out[-1] / nl] * nl)
            continue
        for i in range(nl):
            kind = fused_name if path == "fused" else kernel_kind(gates[i])
            kinds.setdefault(kind, []).append(ev[k][i].elapsed_time(ev[k][i + 1]) / 1e3)
    return out


def kernel_table(kinds):
    tot = sum(sum(v) for v in kinds.values())
    return {k: {"launches": len(v), "mean_ms": statistics.mean(v) * 1e3, "share": sum(v) / tot}
            for k, v in kinds.items()}


def run_b200(args):
    import ctypes as C

    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist_init(ws, "nccl")
    from qpanda_b200 import FusionPlan, StateVector, circuits, lib
    from qpanda_b200.capi import check

    n, depth = args.qubits, args.depth
    gates = workload(n, depth)
    ng = len(gates)
    amp_b = 8
    L = lib()
    stream = torch.cuda.current_stream()
    sv = StateVector(n, "c64")
    h = sv.handle
    remap = args.kernel == "tiled" and args.remap == 1
    tuned = None
    if args.tune and args.kernel == "tiled" and args.path == "fused" and args.tpr == 1:
        from qpanda_b200 import autotune_plan
        best, tms = autotune_plan(sv, gates, remap=remap, reps=1)
        choice = torch.tensor([best.tile_in_tmem, best.max_sub, best.low_qubits], dtype=torch.int64,
                              device=f"cuda:{local}")
        if ws > 1:                                   # every rank runs rank 0's choice
            import torch.distributed as dist
            dist.broadcast(choice, 0)
        args.tile_in_tmem, args.max_sub, args.low = (int(x) for x in choice.tolist())
        tuned = {"by": "qs_plan_autotune (12 candidates with remap, 8 without; one timed application each, "
                       "before warm-up)",
                 "tile_in_tmem": args.tile_in_tmem, "max_sub": args.max_sub, "low_qubits": args.low,
                 "tuning_ms_per_application": tms}
        sv.reset()
    plan = FusionPlan(n, gates, kernel=args.kernel, remap=remap, low_qubits=args.low, max_sub=args.max_sub,
                      tile_in_tmem=args.tile_in_tmem,
                      threads_per_row=args.tpr)
    plan.remap = remap
    plan.tile_in_tmem = args.tile_in_tmem
    nb = plan.num_launches()
    nblocks = plan.num_blocks()
    path = args.path

    # warm-up (untimed)
    wk = {}
    timed_steps(L, h, gates, plan, args.warmup, stream, torch, wk, path)

    # timed region: barrier + sync on both sides, events on the launching stream
    props = torch.cuda.get_device_properties(local)
    gpu_id = "GPU-" + str(props.uuid) if getattr(props, "uuid", None) else str(local)
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(gpu_id)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    kinds = {}
    timed_steps(L, h, gates, plan, args.steps, stream, torch, kinds, path)
    end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(ws)
    elapsed = max_over_ranks(start.elapsed_time(end) / 1e3, ws, device=f"cuda:{local}")
    # fused: reset, the passes, and the plan's closing norm check (k_norm_fix)
    launches = args.steps * (1 + (nb + 1 if path == "fused" else ng))
    circuit_s = elapsed / args.steps

    peak, peak_kind = peaks()
    dom = max(kinds, key=lambda k: sum(kinds[k]))
    dom_t = statistics.mean(kinds[dom])
    dom_bytes = 2 * amp_b * (1 << n)          # algorithmic: read + write every amplitude once
    achieved = dom_bytes / dom_t / 1e9
    traffic = None
    tr = load_traffic()
    if tr and dom in tr.get("kernels", {}):
        traffic = tr["kernels"][dom].get("bytes_per_launch")
    pass_bytes = (nb * dom_bytes) if path == "fused" else circuits.gate_bytes(gates, n, amp_b)

    # the other path, one step, for the fused-vs-plain comparison
    other = "plain" if path == "fused" else "fused"
    okinds = {}
    ot = timed_steps(L, h, gates, plan, 1, stream, torch, okinds, other)[0]
    odom = max(okinds, key=lambda k: sum(okinds[k]))
    o_ach = dom_bytes / statistics.mean(okinds[odom]) / 1e9
    other_line = {"circuit_s": ot, "launches": (nb + 1 if other == "fused" else ng) + 1,
                  "hbm_gbs_effective": ((nb * dom_bytes) if other == "fused"
                                        else circuits.gate_bytes(gates, n, amp_b)) / ot / 1e9,
                  "dominant_kernel": odom, "dominant_gbs": o_ach, "dominant_frac": o_ach / peak,
                  "kernels": kernel_table(okinds)}
    # the plain path as a caller gets it: qs_gates_apply, whose runs of gates
    # on one tile's qubits go through shared memory in one pass each
    staged_s = None
    if other == "plain" or path == "plain":
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        check(L.qs_reset_zero(h))
        e0.record(stream)
        check(L.qs_gates_apply(h, C.c_void_p(gates.ctypes.data), ng))
        e1.record(stream)
        torch.cuda.synchronize()
        staged_s = e0.elapsed_time(e1) / 1e3
        if other == "plain":
            other_line["circuit_s_per_gate_launches"] = ot
            other_line["circuit_s"] = ot = staged_s
            other_line["hbm_gbs_effective"] = circuits.gate_bytes(gates, n, amp_b) / ot / 1e9
            other_line["note"] = ("circuit_s: qs_gates_apply (runs of consecutive gates whose targets share "
                                  "one tile's 10 qubits staged in shared memory and registers, one pass each); "
                                  "kernels: the same gates one launch each")

    # fidelity of the fused complex64 run against the complex128 per-gate path
    # (the FP64 oracle on the GPU) at 30 qubits on the same circuit structure
    fid = None
    if rank == 0 and n >= 30:
        nf = 30
        gf = workload(nf, depth)
        pf = FusionPlan(nf, gf, kernel=args.kernel, remap=remap, low_qubits=args.low, max_sub=args.max_sub,
                        tile_in_tmem=args.tile_in_tmem,
                        threads_per_row=args.tpr)
        a = StateVector(nf, "c64")
        pf.apply(a)
        pf.status(a)
        d = StateVector(nf, "c128")
        d.apply(gf)
        ip = a.inner(d)
        fidelity = abs(ip) ** 2 / (a.norm2() * d.norm2())
        mx, ss = a.diff(d)
        fid = {"qubits": nf, "fidelity": fidelity, "infidelity": 1 - fidelity, "max_abs_err": mx,
               "l2_err": math.sqrt(ss), "blocks": pf.num_blocks(), "passes": pf.num_launches(),
               "oracle": "complex128 per-gate path"}
        a.close()
        d.close()
        pf.close()

    # e2e through the C ABI: host gate list + host uniforms in, host shots out
    pin_g = torch.empty(gates.nbytes, dtype=torch.uint8).pin_memory()
    pin_g.numpy()[:] = np.frombuffer(gates.tobytes(), dtype=np.uint8)
    qs = np.arange(n, dtype=np.int32)
    rng = np.random.default_rng(SEED)
    pin_u = torch.empty(SHOTS * n, dtype=torch.float64).pin_memory()
    pin_u.numpy()[:] = rng.uniform(size=SHOTS * n)
    pin_o = torch.empty(SHOTS, dtype=torch.int64).pin_memory()
    e2e_steps = max(1, min(args.steps, 2))

    phase_s = {"reset": 0.0, "plan_build": 0.0, "circuit": 0.0, "sample": 0.0}

    def e2e_step():
        c0 = time.perf_counter()
        check(L.qs_reset_zero(h))
        c1 = time.perf_counter()
        if path == "fused":
            from qpanda_b200.capi import PlanOpts
            ph, o = C.c_void_p(), PlanOpts()
            check(L.qs_plan_default_opts(C.byref(o)))
            if args.kernel == "single":
                o.kernel, o.max_sub = 1, 1
            o.remap = 1 if remap else 0
            o.low_qubits = args.low
            if args.kernel == "tiled":
                o.max_sub = args.max_sub
                o.threads_per_row = args.tpr
                o.tile_in_tmem = args.tile_in_tmem
            check(L.qs_plan_create_ex(n, C.c_void_p(pin_g.data_ptr()), ng, C.byref(o), C.byref(ph)))
            c2 = time.perf_counter()
            check(L.qs_plan_apply(h, ph))
        else:
            c2 = time.perf_counter()
            check(L.qs_gates_apply(h, C.c_void_p(pin_g.data_ptr()), ng))
        check(L.qs_synchronize(h))
        c3 = time.perf_counter()
        check(L.qs_sample(h, qs.ctypes.data_as(C.POINTER(C.c_int)), n,
                          C.cast(C.c_void_p(pin_u.data_ptr()), C.POINTER(C.c_double)), SHOTS,
                          C.cast(C.c_void_p(pin_o.data_ptr()), C.POINTER(C.c_uint64))))
        if path == "fused":
            L.qs_plan_destroy(ph)
        c4 = time.perf_counter()
        for k, v in (("reset", c1 - c0), ("plan_build", c2 - c1), ("circuit", c3 - c2), ("sample", c4 - c3)):
            phase_s[k] += v

    # one untimed step first: the sampler's scratch and first kernel loads
    e2e_step()
    for k in phase_s:
        phase_s[k] = 0.0
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, ws, device=f"cuda:{local}")

    sv.close()
    plan.close()

    # the other benchmark workloads, summarised, on one GPU
    secondary = None
    if rank == 0 and ws == 1 and not args.no_secondary:
        secondary = secondary_summaries(args, gpu_id)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_entry(n, depth)
        except Exception as ex:   # the reference build is absent
            cpu = {"value": None, "unit": "circuits/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": ws / circuit_s, "unit": "circuits/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": circuit_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3->f32 (complex64 state)" if path == "fused" else "f32 (complex64 state)",
            "data": "synthetic",
            "config": {"workload": f"random-circuit-{n}q-depth{depth}-c64", "qubits": n, "depth": depth,
                       "gates": ng, "fused_blocks": nblocks, "fused_passes": nb, "kernel": args.kernel,
                       "remap": remap, "low_qubits": args.low, "max_sub": args.max_sub,
                       "threads_per_row": args.tpr, "tile_in_tmem": args.tile_in_tmem, "tuned": tuned,
                       "device_bytes": (amp_b << n) * (2 if remap and path == "fused" else 1),
                       "iswap_frac": ISWAP_FRAC, "seed": SEED, "path": path,
                       "state_bytes": amp_b << n, "l2": "inputs larger than L2 (32 GiB state), no flush",
                       "parallelism": f"replicas x{ws}"},
            "circuit_s": circuit_s,
            "hbm_gbs_effective": pass_bytes / circuit_s / 1e9,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": dom_bytes, "launch_s": dom_t},
            "kernels": kernel_table(kinds),
            other: other_line,
            "speedup_fused_vs_plain": (ot / circuit_s) if path == "fused" else (circuit_s / ot),
            "fidelity_check": fid,
            "cpu_baseline": cpu,
            "e2e": {"value": ws / e2e_s, "unit": "circuits/s",
                    "h2d_bytes_per_step": int(gates.nbytes + SHOTS * n * 8),
                    "d2h_bytes_per_step": SHOTS * 8, "shots": SHOTS,
                    "includes": "plan build on the host, circuit, 1024-shot sampling",
                    "phase_ms": {k: 1e3 * v / e2e_steps for k, v in phase_s.items()}},
            "gpu_launches": launches,
            "clocks": clk,
            "secondary": secondary,
        }
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ----------------------------------------------------------------- 20-qubit circuit
C20_QUBITS, C20_LAYERS = 20, 20
C20_METRIC = "20q random-circuit time, complex128 per-gate path (the drop-in), L2-resident state"


def c20_gates():
    """20 qubits, 20 layers of a rotation on every qubit and CNOTs on a seeded
    perfect matching: 600 gates."""
    from qpanda_b200 import circuits
    return circuits.random_layers(C20_QUBITS, C20_LAYERS, SEED)


def circuit20_line(args, steps=None, warmup=None, gpu_id=None):
    """The 20-qubit circuit on the per-gate kernels in complex128 (the
    reference's precision): device time per circuit (reset + 600 gates), end
    to end through the C ABI (gate list from pinned host memory, the full 2^20
    probability vector and 1024 shots back), and the reference CPU backend
    timed on the whole circuit (no extrapolation) with one thread and with
    every host core.  The 16 MiB state stays in L2, so `roofline` is reported
    against L2-resident traffic, not HBM."""
    import ctypes as C

    import torch
    from qpanda_b200 import StateVector, circuits, lib
    from qpanda_b200.capi import check
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    n = C20_QUBITS
    g = c20_gates()
    L = lib()
    stream = torch.cuda.current_stream()
    sv = StateVector(n, "c128")
    h = sv.handle
    gp = g.ctypes.data

    def circuit():
        check(L.qs_reset_zero(h))
        check(L.qs_gates_apply(h, C.c_void_p(gp), len(g)))

    for _ in range(max(3, warmup)):
        circuit()
    torch.cuda.synchronize()
    clocks = ClockSampler(gpu_id) if gpu_id is not None else None
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    ev[0].record(stream)
    for k in range(steps):
        circuit()
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    per = [ev[k].elapsed_time(ev[k + 1]) / 1e3 for k in range(steps)]
    circuit_s = statistics.mean(per)
    # end to end through the C ABI
    pin_g = torch.empty(g.nbytes, dtype=torch.uint8).pin_memory()
    pin_g.numpy()[:] = np.frombuffer(g.tobytes(), dtype=np.uint8)
    qs = np.arange(n, dtype=np.int32)
    pin_u = torch.empty(SHOTS * n, dtype=torch.float64).pin_memory()
    pin_u.numpy()[:] = np.random.default_rng(SEED).uniform(size=SHOTS * n)
    pin_p = torch.empty(1 << n, dtype=torch.float64).pin_memory()
    pin_o = torch.empty(SHOTS, dtype=torch.int64).pin_memory()

    def e2e_step():
        check(L.qs_reset_zero(h))
        check(L.qs_gates_apply(h, C.c_void_p(pin_g.data_ptr()), len(g)))
        check(L.qs_probs(h, qs.ctypes.data_as(C.POINTER(C.c_int)), n,
                         C.cast(C.c_void_p(pin_p.data_ptr()), C.POINTER(C.c_double))))
        check(L.qs_sample(h, qs.ctypes.data_as(C.POINTER(C.c_int)), n,
                          C.cast(C.c_void_p(pin_u.data_ptr()), C.POINTER(C.c_double)), SHOTS,
                          C.cast(C.c_void_p(pin_o.data_ptr()), C.POINTER(C.c_uint64))))

    e2e_step()
    torch.cuda.synchronize()
    e2e_n = max(3, min(steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_n):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / e2e_n
    sv.close()
    alg = circuits.gate_bytes(g, n, 16)
    cpu = None
    if not args.no_cpu_baseline:
        try:
            cpu = c20_cpu()
        except Exception as ex:   # the reference build is absent
            cpu = {"value": None, "unit": "circuits/s", "kind": "reference", "sample": f"unavailable: {ex}"}
    return {
        "metric": C20_METRIC, "value": 1.0 / circuit_s, "unit": "circuits/s", "n_gpus": 1, "steps": steps,
        "warmup": max(3, warmup), "ms_per_step": circuit_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (complex128 state)", "data": "synthetic",
        "config": {"workload": "random-circuit-20q-depth20-c128", "qubits": n, "layers": C20_LAYERS,
                   "gates": len(g), "seed": SEED, "path": "per-gate",
                   "l2": "16 MiB state, L2-resident by design (the configuration's size); no flush"},
        "roofline": {"bound": "l2", "kernel": "k_pair / k_phase (per gate)", "achieved": alg / circuit_s / 1e9,
                     "peak": None, "unit": "GB/s", "frac": None, "traffic": None,
                     "note": "algorithmic bytes of the 600 gates per second; the state never leaves L2"},
        "cpu_baseline": cpu,
        "e2e": {"value": 1.0 / e2e_s, "unit": "circuits/s", "h2d_bytes_per_step": int(g.nbytes + SHOTS * n * 8),
                "d2h_bytes_per_step": int(8 << n) + SHOTS * 8,
                "includes": "gate list from pinned host memory, the circuit, the full probability vector and "
                            "1024 shots to the host"},
        "gpu_launches": steps * (1 + len(g)),
        "clocks": clk,
    }


def c20_cpu():
    """The reference CPU backend on the whole 20-qubit circuit (600 gates)
    plus its pMeasure over all qubits, timed directly: one thread (the
    shipped build) and every host core (-fopenmp)."""
    from oracle.pyoracle import RefState, ref_available
    g = c20_gates()
    qs = list(range(C20_QUBITS))
    out = {}
    for omp in (True, False):
        if not ref_available(omp):
            raise FileNotFoundError("oracle/_ref not built")
        times = []
        for _ in range(2 if omp else 1):
            r = RefState(C20_QUBITS, omp=omp)
            t0 = time.perf_counter()
            r.apply(g)
            r.pmeasure(qs)
            times.append(time.perf_counter() - t0)
        out[omp] = min(times)
    cores = os.cpu_count() or 1
    return {"value": 1.0 / out[True], "unit": "circuits/s", "cores": cores, "kind": "reference",
            "sample": (f"reference CPUQuantumGates.cpp, the whole circuit (600 gates) and pMeasure over the 20 "
                       f"qubits, complex128: {out[True]:.3f} s with -fopenmp on {cores} threads (value), "
                       f"{out[False]:.3f} s as shipped on 1 thread; measured, not extrapolated"),
            "single_core": {"value": 1.0 / out[False], "unit": "circuits/s", "cores": 1},
            "host": host_cpu()}


def run_circuit20(args):
    ws, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    dist_init(ws, "nccl")
    props = torch.cuda.get_device_properties(local)
    gpu_id = "GPU-" + str(props.uuid) if getattr(props, "uuid", None) else str(local)
    barrier(ws)
    if rank != 0 or ws > 1:
        args.no_cpu_baseline = True
    line = circuit20_line(args, gpu_id=gpu_id)
    barrier(ws)
    elapsed = max_over_ranks(line["ms_per_step"] / 1e3, ws, device=f"cuda:{local}")
    line["value"] = ws / elapsed
    line["n_gpus"] = ws
    line["config"]["parallelism"] = f"replicas x{ws}"
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference_circuit20(args):
    from oracle.pyoracle import RefState
    g = c20_gates()
    qs = list(range(C20_QUBITS))
    times = []
    for i in range(args.warmup + args.steps):
        r = RefState(C20_QUBITS, omp=True)
        t0 = time.perf_counter()
        r.apply(g)
        r.pmeasure(qs)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = 1.0 / statistics.median(times)
    cores = os.cpu_count() or 1
    print(json.dumps({
        "impl": "reference", "metric": C20_METRIC, "value": value, "unit": "circuits/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(times) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "random-circuit-20q-depth20-c128", "qubits": C20_QUBITS, "layers": C20_LAYERS,
                   "seed": SEED},
        "cpu_baseline": {"value": value, "unit": "circuits/s", "cores": cores, "kind": "reference",
                         "sample": (f"reference CPUQuantumGates.cpp (-fopenmp, {cores} threads, complex128): "
                                    "each step = the whole circuit and pMeasure over all qubits"),
                         "host": host_cpu()},
        "e2e": {"value": value, "unit": "circuits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ----------------------------------------------------------------- secondary workloads
def secondary_summaries(args, gpu_id):
    """Short runs of the other benchmark workloads for the default line, each
    timed with CUDA events and its clocks sampled: the 20-qubit complex128
    circuit (with the reference CPU backend timed on it directly), the 28-qubit
    QFT on the per-gate kernels, the 4096-circuit batched sweep (autotuned on
    every 64th circuit) and a slice of the request trace."""
    import copy
    quiet = copy.copy(args)
    quiet.no_cpu_baseline = True
    out = {}

    def keep(name, f):
        t0 = time.perf_counter()
        try:
            out[name] = f()
        except Exception as ex:
            out[name] = {"error": f"{type(ex).__name__}: {ex}"}
        out[name]["wall_s"] = round(time.perf_counter() - t0, 1)

    def c20():
        ln = circuit20_line(args, steps=10, warmup=3, gpu_id=gpu_id)
        cpu = ln["cpu_baseline"] or {}
        return {"workload": ln["config"]["workload"], "circuits_per_s": ln["value"], "ms_per_circuit": ln["ms_per_step"],
                "e2e_circuits_per_s": ln["e2e"]["value"], "e2e_includes": ln["e2e"]["includes"],
                "l2_resident_gbs": ln["roofline"]["achieved"],
                "cpu_reference_circuits_per_s": cpu.get("value"), "cpu_cores": cpu.get("cores"),
                "cpu_reference_1core_circuits_per_s": (cpu.get("single_core") or {}).get("value"),
                "cpu_sample": cpu.get("sample"), "clocks": ln["clocks"]}

    def qft():
        ln = qft_line(quiet, 28, steps=2, warmup=1, gpu_id=gpu_id)
        res = {"workload": ln["config"]["workload"], "peak_gbs": ln["roofline"]["peak"],
               "peak_source": ln["roofline"]["peak_source"], "error_c64": ln["error_c64"],
               "fused_c64": ln["fused_c64"], "clocks": ln["clocks"]}
        for dt in ("complex64", "complex128"):
            res[dt] = {"circuit_ms": 1e3 * ln[dt]["circuit_s"], "hbm_gbs_effective": ln[dt]["hbm_gbs_effective"],
                       "staged_circuit_ms": 1e3 * ln[dt]["staged_circuit_s"],
                       "kernels": {k: {"gbs": v["gbs"], "frac": v["frac"], "mean_ms": v["mean_ms"]}
                                   for k, v in ln[dt]["kernels"].items()}}
        return res

    def vqe():
        ln = vqe_line(quiet, steps=3, warmup=3, tune_stride=64, gpu_id=gpu_id)
        return {"workload": "vqe-sweep-4096", "circuits_per_s": ln["value"], "ms_per_sweep": ln["ms_per_step"],
                "hbm_gbs": ln["roofline"]["achieved"], "frac": ln["roofline"]["frac"],
                "e2e_circuits_per_s": ln["e2e"]["value"], "autotuned": ln["config"]["autotuned"],
                "build_s": ln["config"]["build_s"], "clocks": ln["clocks"]}

    def req():
        ln = requests_line(args, 2000, 20, gpu_id=gpu_id, budget_gb=100)
        return {"workload": "requests", "served": ln["config"]["served"], "failed": ln["failed"],
                "circuits_per_s": ln["value"], "latency_s": ln["latency_s"], "service_s": ln["service_s"],
                "subsample": "every 20th of the first 2000 requests of the trace (0.1 of its rate), real time",
                "cpu_reference_circuits_per_s": (ln.get("cpu_baseline") or {}).get("value"),
                "cpu_sample": (ln.get("cpu_baseline") or {}).get("sample"),
                "clocks": ln["clocks"]}

    keep("circuit20_c128", c20)
    keep("qft28", qft)
    keep("vqe_sweep", vqe)
    keep("requests", req)
    return out


# ----------------------------------------------------------------- batched sweep
SWEEP_SEED = 777


def sweep_bytes(sweep):
    """Algorithmic HBM bytes of one batched run: 2 x 8 B x 2^max(q,12) per
    fused pass (a read and a write of the state), minus the read of the first
    pass, which starts from |0> without one."""
    from qpanda_b200 import FusionPlan
    tot, cache = 0, {}
    for q, g in sweep:
        key = (q, len(g))
        if key not in cache:
            cache[key] = FusionPlan(max(q, 12), g).num_launches()
        tot += (2 * cache[key] - 1) * 8 * (1 << max(q, 12))
    return tot


def vqe_line(args, steps, warmup, tune_stride=16, gpu_id=None, rank=0):
    """The batched sweep on one GPU: autotune (every tune_stride-th circuit),
    build, `warmup` + `steps` graph replays timed with CUDA events, then end
    to end through the C ABI.  Returns the result line."""
    import ctypes as C

    import torch
    from qpanda_b200 import Batch, autotune_batch, circuits
    from qpanda_b200.capi import _concat, _iptr, BatchOpts, check, lib

    sweep = circuits.vqe_sweep(args.circuits, SWEEP_SEED + rank)
    t0 = time.perf_counter()
    cache = os.environ.get("QS_TUNE_CACHE", os.path.join(tempfile.gettempdir(), "qpanda_b200_tune.txt"))
    hit = None
    if args.no_autotune:
        opts, tune_ms = BatchOpts(), None
        check(lib().qs_batch_default_opts(C.byref(opts)))
    else:
        opts, tune_ms, hit = autotune_batch(sweep, stride=tune_stride, cache=cache)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b = Batch(sweep, opts=opts)
    build_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    for _ in range(max(3, warmup)):
        b.run(C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    clocks = ClockSampler(gpu_id) if gpu_id is not None else None
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    ev[0].record(stream)
    for k in range(steps):
        b.run(C.c_void_p(stream.cuda_stream))
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    per = [ev[k].elapsed_time(ev[k + 1]) / 1e3 for k in range(steps)]
    step_s = statistics.mean(per)
    zz = b.zz()
    alg = sweep_bytes(sweep)
    peak, peak_kind = peaks()
    # e2e: build from host gate records, run, read every <ZZ> back
    nq, gates, offs = _concat(sweep)
    e2e_steps = max(1, min(steps, 2))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        h = C.c_void_p()
        check(lib().qs_batch_create(len(nq), _iptr(nq), gates.ctypes.data,
                                    offs.ctypes.data_as(C.POINTER(C.c_size_t)), C.byref(opts), C.byref(h)))
        check(lib().qs_batch_run(h, None))
        cnt = C.c_size_t()
        check(lib().qs_batch_zz(h, None, C.byref(cnt)))
        out = np.empty(cnt.value)
        check(lib().qs_batch_zz(h, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cnt)))
        lib().qs_batch_destroy(h)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    b.close()
    cpu = None
    if not args.no_cpu_baseline:
        try:
            from oracle.pyoracle import RefState
            sample = sweep[:: max(1, len(sweep) // 48)]
            t0 = time.perf_counter()
            work_s = 0
            for q, g in sample:
                r = RefState(q, omp=True)
                r.apply(g)
                work_s += len(g) << q
            secs = time.perf_counter() - t0
            work_all = sum(len(g) << q for q, g in sweep)
            cpu = {"value": len(sweep) / (secs * work_all / work_s), "unit": "circuits/s",
                   "cores": os.cpu_count(), "kind": "reference",
                   "sample": (f"reference CPUQuantumGates.cpp (-fopenmp, {os.cpu_count()} threads, complex128) "
                              f"on {len(sample)} of the {len(sweep)} circuits: {secs:.2f} s, extrapolated by "
                              f"gate x amplitude work ({work_all / work_s:.1f}x)")}
        except Exception as ex:
            cpu = {"value": None, "unit": "circuits/s", "kind": "reference", "sample": f"unavailable: {ex}"}
    return {
        "metric": "batched VQE sweep throughput (circuits/s)", "value": len(sweep) / step_s,
        "unit": "circuits/s", "n_gpus": 1, "steps": steps, "warmup": max(3, warmup),
        "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16x3->f32 (complex64 states)", "data": "synthetic",
        "config": {"workload": "vqe-sweep", "circuits": len(sweep), "qubits": "U{10..22}",
                   "layers": "U{4..12}", "seed": SWEEP_SEED, "outputs": "all <Z_i Z_{i+1}>",
                   "launch": "one persistent kernel, CUDA graph replay",
                   "autotuned": {"block_qubits": opts.block_qubits, "max_sub": opts.max_sub,
                                 "low_qubits": opts.low_qubits, "order": opts.order,
                                 "tile_in_tmem": opts.tile_in_tmem, "sample_ms": tune_ms,
                                 "tune_s": tune_s, "stride": None if args.no_autotune else tune_stride,
                                 "cache": None if args.no_autotune else cache, "from_cache": hit},
                   "build_s": build_s, "l2": "21 GB of states >> L2"},
        "roofline": {"bound": "hbm",
                     "kernel": "k_batch_tmem" if (opts.tile_in_tmem and opts.max_sub <= 2) else "k_batch",
                     "achieved": alg / step_s / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg / step_s / 1e9 / peak, "peak_source": peak_kind,
                     "traffic": None, "algorithmic_bytes_per_launch": alg, "launch_s": step_s},
        "zz_checksum": float(sum(float(np.sum(z)) for z in zz)),
        "cpu_baseline": cpu,
        "e2e": {"value": len(sweep) / e2e_s, "unit": "circuits/s",
                "h2d_bytes_per_step": int(gates.nbytes), "d2h_bytes_per_step": int(8 * sum(len(z) for z in zz)),
                "includes": "planning and upload of every circuit, the run, all <ZZ> to the host"},
        "gpu_launches": steps, "clocks": clk,
    }


def run_vqe_sweep(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist_init(ws, "nccl")
    props = torch.cuda.get_device_properties(local)
    gpu_id = "GPU-" + str(props.uuid) if getattr(props, "uuid", None) else str(local)
    if rank != 0 or ws > 1:
        args.no_cpu_baseline = True
    barrier(ws)
    line = vqe_line(args, args.steps, args.warmup, gpu_id=gpu_id, rank=rank)
    barrier(ws)
    step_s = max_over_ranks(line["ms_per_step"] / 1e3, ws, device=f"cuda:{local}")
    line["value"] = ws * args.circuits / step_s
    line["n_gpus"] = ws
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ----------------------------------------------------------------- request loop
TRACE_SEED = 4242


def requests_line(args, n_requests, every, gpu_id=None, rank=0, budget_gb=120):
    """Replay requests 0, every, 2 every, ... of the first n_requests of the
    seeded Poisson trace against the continuous-batching server, each at its
    original arrival time; returns the line (circuits/s, latency
    percentiles)."""
    import threading

    from qpanda_b200 import Server, circuits

    trace = circuits.request_trace(n_requests, TRACE_SEED + rank)
    sample = trace[:: every]
    srv = Server(budget_bytes=budget_gb << 30, slots=8)
    # warm-up: one small request of each kind (module loading, pools)
    for kind in ("shots", "probs"):
        g = circuits.random_layers(14, 2, 1)
        rid = srv.submit(14, g, kind, np.random.default_rng(0).uniform(size=(1024, 14)))
        srv.wait(rid)
        srv.release(rid)
    results, lock = {}, threading.Lock()
    ids = []

    def waiter():
        k = 0
        while True:
            with lock:
                if k >= len(ids):
                    if done_submitting.is_set():
                        break
                    item = None
                else:
                    item = ids[k]
            if item is None:
                time.sleep(0.001)
                continue
            rid, req, t_sub = item
            try:
                lat, svc = srv.wait(rid)
                ok = True
            except Exception:
                lat, svc, ok = float("nan"), float("nan"), False
            results[rid] = (req, t_sub, lat, svc, ok)
            srv.release(rid)
            k += 1

    done_submitting = threading.Event()
    th = threading.Thread(target=waiter)
    th.start()
    clocks = ClockSampler(gpu_id) if gpu_id is not None else None
    t0 = time.perf_counter()
    alg_bytes = 0
    for req in sample:
        now = time.perf_counter() - t0
        if req["arrival"] > now:
            time.sleep(req["arrival"] - now)
        q = req["qubits"]
        g = circuits.random_layers(q, req["depth"], req["seed"])
        u = np.random.default_rng(req["seed"]).uniform(size=(SHOTS, q)) if req["kind"] == "shots" else None
        t_sub = time.perf_counter() - t0
        rid = srv.submit(q, g, req["kind"], u)
        with lock:
            ids.append((rid, req, t_sub))
    done_submitting.set()
    th.join()
    clk = clocks.stop() if clocks else None
    ends = [t + lat for (_, t, lat, _, ok) in results.values() if ok]
    makespan = max(ends) - min(t for (_, t, _, _, _) in results.values())
    lats = np.array([lat for (_, _, lat, _, ok) in results.values() if ok])
    svcs = np.array([svc for (_, _, _, svc, ok) in results.values() if ok])
    n_ok = int(len(lats))
    stats = srv.stats()
    srv.close()
    from qpanda_b200 import FusionPlan
    for req in sample:
        q = req["qubits"]
        if q >= 12:
            nl = FusionPlan(q, circuits.random_layers(q, req["depth"], req["seed"])).num_launches()
            alg_bytes += 2 * 8 * (1 << q) * nl
    peak, peak_kind = peaks()
    cpu = None
    if not getattr(args, "no_cpu_baseline", False):
        cpu = requests_cpu_baseline(sample)
    return {
            "metric": "request loop: circuits/s with p50/p99 latency", "value": n_ok / makespan,
            "unit": "circuits/s", "n_gpus": 1, "steps": 1, "warmup": 2, "ms_per_step": makespan * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3->f32 (complex64 states)", "data": "synthetic",
            "config": {"workload": "requests", "trace": n_requests, "served": len(sample), "every": every,
                       "rate_per_s": 2000.0 / every, "qubits": "U{8..30}", "depth": "U{4..32}",
                       "kinds": "1024 shots or full probability vector", "seed": TRACE_SEED,
                       "server": {"slots": 8, "hbm_budget_gb": budget_gb, "max_concurrent": stats["max_concurrent"]},
                       "subsample": (f"every {every}th request of the first {n_requests} of the trace, at its "
                                     "original arrival time (the full trace is about 1.3 PB of state traffic)")},
            "latency_s": {"p50": float(np.percentile(lats, 50)), "p99": float(np.percentile(lats, 99)),
                          "mean": float(lats.mean())},
            "service_s": {"p50": float(np.percentile(svcs, 50)), "p99": float(np.percentile(svcs, 99))},
            "failed": len(sample) - n_ok,
            "roofline": {"bound": "hbm", "kernel": "fused tiled passes (all requests)",
                         "achieved": alg_bytes / makespan / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": alg_bytes / makespan / 1e9 / peak,
                         "peak_source": peak_kind, "traffic": None, "algorithmic_bytes_per_launch": alg_bytes,
                         "launch_s": makespan},
            "e2e": {"value": n_ok / makespan, "unit": "circuits/s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "includes": "host circuit generation, submission in real time, shots to the host"},
            "cpu_baseline": cpu,
            "clocks": clk,
    }


def requests_cpu_baseline(sample, max_q=22, max_n=6):
    """The reference CPU backend (oracle/_ref, -fopenmp, complex128) on the
    largest served requests of at most max_q qubits (max_n of them, states
    beyond the host caches), each circuit simulated once; extrapolated to the
    whole served sample by gate x amplitude work.  A lower bound on the
    reference's own cost: its shot loop re-simulates the circuit per shot."""
    from qpanda_b200 import circuits
    try:
        from oracle.pyoracle import RefState
        small = sorted((r for r in sample if r["qubits"] <= max_q), key=lambda r: -r["qubits"])[:max_n]
        t0 = time.perf_counter()
        work_s = 0
        for r in small:
            g = circuits.random_layers(r["qubits"], r["depth"], r["seed"])
            st = RefState(r["qubits"], omp=True)
            st.apply(g)
            work_s += len(g) << r["qubits"]
        secs = time.perf_counter() - t0
        work_all = sum((len(circuits.random_layers(r["qubits"], r["depth"], r["seed"])) << r["qubits"])
                       for r in sample)
        return {"value": len(sample) / (secs * work_all / max(work_s, 1)), "unit": "circuits/s",
                "cores": os.cpu_count(), "kind": "reference",
                "sample": (f"reference CPUQuantumGates.cpp (-fopenmp, {os.cpu_count()} threads, complex128) on "
                           f"the {len(small)} largest of the {len(sample)} served requests of <= {max_q} qubits, each "
                           f"circuit once: {secs:.2f} s, extrapolated by gate x amplitude "
                           f"work ({work_all / max(work_s, 1):.0f}x; the reference re-simulates per shot, so its "
                           "shots requests cost more)")}
    except Exception as ex:
        return {"value": None, "unit": "circuits/s", "kind": "reference", "sample": f"unavailable: {ex}"}


def run_requests(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist_init(ws, "nccl")
    props = torch.cuda.get_device_properties(local)
    gpu_id = "GPU-" + str(props.uuid) if getattr(props, "uuid", None) else str(local)
    line = requests_line(args, args.requests, args.every, gpu_id=gpu_id, rank=rank)
    makespan = max_over_ranks(line["ms_per_step"] / 1e3, ws, device=f"cuda:{local}")
    served = line["config"]["served"] - line["failed"]
    line["value"] = line["e2e"]["value"] = ws * served / makespan
    line["n_gpus"] = ws
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ----------------------------------------------------------------- 28-qubit QFT
QFT_SEED = 28028


def qft_line(args, n, steps, warmup, gpu_id=None):
    """n-qubit QFT (H and CR(pi/2^k) on all pairs, then the reversal swaps) on a
    seeded normalised complex Gaussian state, on the plain per-gate path in
    complex64 and complex128: per-kernel HBM GB/s from CUDA events after every
    gate, and the complex64 error against the complex128 run.  Returns the line."""
    import ctypes as C

    import torch
    from qpanda_b200 import FusionPlan, StateVector, circuits, lib
    from qpanda_b200.capi import OP, check

    gates = circuits.qft(n)
    rng = np.random.default_rng(QFT_SEED)
    init = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    init /= np.linalg.norm(init)
    L = lib()
    stream = torch.cuda.current_stream()
    kind_of = {OP["H"]: "k_pair (H, dense 2x2)", OP["CR"]: "k_phase (CR, N/4 amplitudes)",
               OP["SWAP"]: "k_pair (SWAP exchange, N/2 amplitudes)"}
    frac_of = {OP["H"]: 1.0, OP["CR"]: 0.25, OP["SWAP"]: 0.5}
    gptr = [gates[i:i + 1].ctypes.data for i in range(len(gates))]
    peak, peak_kind = peaks()
    out, states = {}, {}
    clocks = ClockSampler(gpu_id) if gpu_id is not None else None
    for dt, amp_b, npdt in (("c64", 8, np.complex64), ("c128", 16, np.complex128)):
        sv = StateVector(n, dt)
        host = init.astype(npdt)
        kinds, circ = {}, []
        for k in range(warmup + steps):
            sv.set_state(host)
            torch.cuda.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(gates) + 1)]
            ev[0].record(stream)
            for i in range(len(gates)):
                check(L.qs_gate_apply(sv.handle, C.c_void_p(gptr[i])))
                ev[i + 1].record(stream)
            torch.cuda.synchronize()
            if k < warmup:
                continue
            circ.append(ev[0].elapsed_time(ev[-1]) / 1e3)
            for i in range(len(gates)):
                op = int(gates[i]["op"])
                kinds.setdefault(op, []).append(ev[i].elapsed_time(ev[i + 1]) / 1e3)
        table = {}
        for op, ts in kinds.items():
            t = statistics.mean(ts)
            gbs = 2 * amp_b * frac_of[op] * (1 << n) / t / 1e9
            table[kind_of[op]] = {"launches_per_circuit": len(ts) // steps, "mean_ms": t * 1e3,
                                  "gbs": gbs, "frac": gbs / peak}
        cs = statistics.mean(circ)
        # the same gates through qs_gates_apply: runs of gates that share one
        # tile's qubits staged, one pass each (the state it leaves is the one above)
        staged = []
        for k in range(warmup + steps):
            sv.set_state(host)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            check(L.qs_gates_apply(sv.handle, C.c_void_p(gates.ctypes.data), len(gates)))
            e1.record(stream)
            torch.cuda.synchronize()
            if k >= warmup:
                staged.append(e0.elapsed_time(e1) / 1e3)
        ss = statistics.mean(staged)
        out[dt] = {"circuit_s": cs, "hbm_gbs_effective": circuits.gate_bytes(gates, n, amp_b) / cs / 1e9,
                   "kernels": table, "staged_circuit_s": ss,
                   "staged_note": "qs_gates_apply: runs of consecutive gates whose targets share one tile's 10 qubits, one staged pass each"}
        states[dt] = sv
    clk = clocks.stop() if clocks else None
    a, d = states["c64"], states["c128"]
    ip = a.inner(d)
    mx, ss = a.diff(d)
    err = {"max_abs_err": mx, "l2_err": math.sqrt(ss), "fidelity": abs(ip) ** 2 / (a.norm2() * d.norm2()),
           "oracle": "complex128 per-gate path (pinned to the CPU oracle by the GPU tests)"}
    # the fused path on the same input, for comparison
    a.set_state(init.astype(np.complex64))
    p = FusionPlan(n, gates, remap=1)
    p.apply(a)
    torch.cuda.synchronize()
    a.set_state(init.astype(np.complex64))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    p.apply(a)
    e1.record(stream)
    torch.cuda.synchronize()
    fmx, _ = a.diff(d)
    fused = {"circuit_s": e0.elapsed_time(e1) / 1e3, "passes": p.num_launches(), "max_abs_err_vs_c128": fmx}
    p.close()
    # e2e through the C ABI: host state in, gates, host state out (complex64)
    pin_in = torch.empty((1 << n) * 8, dtype=torch.uint8).pin_memory()
    pin_in.numpy().view(np.complex64)[:] = init.astype(np.complex64)
    pin_out = torch.empty((1 << n) * 8, dtype=torch.uint8).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    check(L.qs_set_state(a.handle, C.c_void_p(pin_in.data_ptr()), 0))
    check(L.qs_gates_apply(a.handle, gates.ctypes.data, len(gates)))
    check(L.qs_get_state(a.handle, C.c_void_p(pin_out.data_ptr()), 0))
    e2e_s = time.perf_counter() - t0
    cpu = None
    if not args.no_cpu_baseline:
        try:
            from oracle.pyoracle import RefState
            ns = 22
            r = RefState(ns, omp=True)
            t0 = time.perf_counter()
            r.apply(circuits.qft(ns))
            secs = time.perf_counter() - t0
            scale = (1 << (n - ns)) * len(gates) / len(circuits.qft(ns))
            cpu = {"value": circuits.gate_bytes(gates, n, 16) / (secs * scale) / 1e9, "unit": "GB/s",
                   "cores": os.cpu_count(), "kind": "reference",
                   "sample": (f"reference CPUQuantumGates.cpp (-fopenmp, {os.cpu_count()} threads, complex128) "
                              f"on the {ns}-qubit QFT: {secs:.2f} s, extrapolated x{scale:.0f} to {n} qubits "
                              f"({secs * scale:.0f} s); value = the same algorithmic bytes per second")}
        except Exception as ex:
            cpu = {"value": None, "unit": "GB/s", "kind": "reference", "sample": f"unavailable: {ex}"}
    dom = max(out["c64"]["kernels"], key=lambda k: out["c64"]["kernels"][k]["mean_ms"] *
              out["c64"]["kernels"][k]["launches_per_circuit"])
    dk = out["c64"]["kernels"][dom]
    a.close()
    d.close()
    if True:
        return ({
            "metric": "28q QFT HBM GB/s, plain per-gate path", "value": out["c64"]["hbm_gbs_effective"],
            "unit": "GB/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": out["c64"]["circuit_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (complex64 state); f64 line under complex128", "data": "synthetic",
            "config": {"workload": f"qft-{n}q", "qubits": n, "gates": len(gates), "seed": QFT_SEED,
                       "input": "normalised i.i.d. complex Gaussian", "l2": "2-4 GiB states > L2, no flush"},
            "complex64": out["c64"], "complex128": out["c128"], "error_c64": err, "fused_c64": fused,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": dk["gbs"], "peak": peak, "unit": "GB/s",
                         "frac": dk["gbs"] / peak, "peak_source": peak_kind, "traffic": None,
                         "algorithmic_bytes_per_launch": None, "launch_s": dk["mean_ms"] / 1e3},
            "cpu_baseline": cpu,
            "e2e": {"value": circuits.gate_bytes(gates, n, 8) / e2e_s / 1e9, "unit": "GB/s",
                    "h2d_bytes_per_step": 8 << n, "d2h_bytes_per_step": 8 << n,
                    "includes": "host state in, the QFT per gate, host state out (complex64)"},
            "gpu_launches": len(gates) * (warmup + steps) * 2, "clocks": clk,
        })


def run_qft(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist_init(ws, "nccl")
    props = torch.cuda.get_device_properties(local)
    gpu_id = "GPU-" + str(props.uuid) if getattr(props, "uuid", None) else str(local)
    if rank != 0 or ws > 1:
        args.no_cpu_baseline = True
    n = 28 if args.qubits == N_QUBITS else args.qubits
    line = qft_line(args, n, args.steps, args.warmup, gpu_id=gpu_id)
    line["n_gpus"] = ws
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ----------------------------------------------------------------- every kernel
def run_kernels(args):
    """Each kernel of the library on one complex64 state of --qubits (28 when
    left at 32: 2 GiB, far above L2), a few launches each after one untimed
    one, timed with CUDA events: mean time, algorithmic bytes (reads plus
    writes the operation needs, per the per-gate byte rule) and GB/s against
    the HBM peak.  The command the per-kernel ncu captures run."""
    import ctypes as C

    import torch
    from qpanda_b200 import Batch, FusionPlan, StateVector, circuits, lib
    from qpanda_b200.capi import check
    torch.cuda.set_device(0)
    n = 28 if args.qubits == N_QUBITS else args.qubits
    N, S = 1 << n, 8
    L = lib()
    stream = torch.cuda.current_stream()
    peak, peak_kind = peaks()
    sv = StateVector(n, "c64")
    h = sv.handle
    init = circuits.make_gates([("H", (q,)) for q in range(n)] + [("RY", (q,), 0.3 + 0.1 * q) for q in range(n)])
    sv.apply(init)
    reps = max(2, args.steps)
    out = {}

    def timed(name, fn, bytes_per_call, calls=reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(calls):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / calls
        out[name] = {"ms": t * 1e3, "algorithmic_bytes": bytes_per_call, "gbs": bytes_per_call / t / 1e9,
                     "frac": bytes_per_call / t / 1e9 / peak}

    def gate(spec):
        g = circuits.make_gates(spec)
        return lambda: check(L.qs_gate_apply(h, C.c_void_p(g.ctypes.data)))

    timed("k_pair: dense 2x2 on qubit 0", gate([("RX", (0,), 0.7)]), 2 * S * N)
    timed("k_pair: dense 2x2 on qubit 13", gate([("RX", (13,), 0.7)]), 2 * S * N)
    timed("k_pair: dense 2x2 on qubit 27", gate([("RX", (n - 1,), 0.7)]), 2 * S * N)
    timed("k_pair: CNOT (2, 20)", gate([("CNOT", (2, 20))]), 2 * S * N // 2)
    timed("k_pair: SWAP (1, 24)", gate([("SWAP", (1, 24))]), 2 * S * N // 2)
    timed("k_phase: CR (0, 1)", gate([("CR", (0, 1), 0.4)]), 2 * S * N // 4)
    timed("k_phase: CR (12, 25)", gate([("CR", (12, 25), 0.4)]), 2 * S * N // 4)
    m2 = np.eye(4, dtype=np.complex128).reshape(-1).view(np.float64).copy()
    timed("k_quad: 4x4 on (3, 17)", lambda: check(L.qs_apply_2q(h, 3, 17, m2.ctypes.data_as(C.POINTER(C.c_double)),
                                                                 0)), 2 * S * N)
    run = circuits.make_gates([("RY", (q,), 0.2 * q) for q in range(10)])
    timed("k_lowstage: 10 rotations on qubits 0..9 (one pass)",
          lambda: check(L.qs_gates_apply(h, C.c_void_p(run.ctypes.data), len(run))), 2 * S * N)
    run_hi = circuits.make_gates([("RY", (q,), 0.2 * q) for q in range(n - 7, n)])
    timed(f"k_lowstage: 7 rotations on qubits {n - 7}..{n - 1} (one pass; tile qubits 0..2 and {n - 7}..{n - 1})",
          lambda: check(L.qs_gates_apply(h, C.c_void_p(run_hi.ctypes.data), len(run_hi))), 2 * S * N)
    qs20 = np.arange(20, dtype=np.int32)
    dev = torch.empty(1 << 20, dtype=torch.float64, device="cuda")
    timed("k_marginal_direct: qubits 0..19 (the sampler's first levels)",
          lambda: check(L.qs_probs_device(h, qs20.ctypes.data_as(C.POINTER(C.c_int)), 20, C.c_void_p(dev.data_ptr()))),
          S * N + (8 << 20))
    q3 = np.array([3, 17, n - 2], dtype=np.int32)
    dev3 = torch.empty(8, dtype=torch.float64, device="cuda")
    timed("k_marginal: qubits (3, 17, 26)",
          lambda: check(L.qs_probs_device(h, q3.ctypes.data_as(C.POINTER(C.c_int)), 3, C.c_void_p(dev3.data_ptr()))),
          S * N)
    qs = np.arange(n, dtype=np.int32)
    u = np.random.default_rng(1).uniform(size=(SHOTS, n))
    timed("qs_sample: marginal + fold + k_shots, 1024 shots of all qubits", lambda: sv.sample(qs, u), S * N, calls=2)
    timed("qs_prob_zero: k_half_sum + k_finalize (qubit 5)", lambda: sv.prob_zero(5), S * N // 2)
    timed("qs_measure: k_half_sum + k_finalize + k_collapse (qubit 6)", lambda: sv.measure(6, 0.5),
          S * N // 2 + S * N + S * N // 2, calls=2)
    amp = C.c_void_p()
    check(L.qs_device_ptr(h, C.byref(amp)))
    ow = torch.zeros(2, dtype=torch.float64, device="cuda")
    timed("qs_measure_noalloc: k_na_chunk_sum + k_na_decide + k_na_collapse (qubit 7)",
          lambda: check(L.qs_measure_noalloc(amp, n, 0, 7, 0.5, C.c_void_p(ow.data_ptr()),
                                             C.c_void_p(ow.data_ptr() + 8), None)),
          S * N // 2 + S * N + S * N // 2, calls=2)
    other = StateVector(n, "c64")
    timed("k_inner: <a|b>", lambda: sv.inner(other), 2 * S * N)
    g = circuits.random_layers(n, 4, SEED, iswap_frac=0.1)
    for name, kw in (("k_tile_tmem: tiled pass, tile in tensor memory", {}),
                     ("k_fused_tile: tiled pass, tile in shared memory", {"tile_in_tmem": 0})):
        plan = FusionPlan(n, g, **kw)
        npass = plan.num_launches()
        timed(name + f" (mean of the {npass} passes of a 4-layer circuit)",
              lambda: (plan.apply(sv), None)[1], 2 * S * N * npass)
        out[name + f" (mean of the {npass} passes of a 4-layer circuit)"]["ms"] /= npass
        plan.close()
    sweep = circuits.vqe_sweep(512, SWEEP_SEED)
    b = Batch(sweep)
    timed("k_batch: 512 circuits of 10-22 qubits", lambda: b.run(), sweep_bytes(sweep))
    b.close()
    # the plan of a circuit and then of its inverse: the state returns to |0..0>
    # and the inverse plan's closing rescale (k_norm_fix) restores the norm its
    # last pass drifted
    fwd = circuits.random_layers(n, 16, SEED + 1, iswap_frac=0.1)
    inv = np.array(fwd[::-1], copy=True)
    inv["dagger"] ^= 1
    pf, pi = FusionPlan(n, fwd), FusionPlan(n, inv)
    npass = pf.num_launches() + pi.num_launches()
    timed(f"round trip: a 16-layer circuit's plan and its inverse's ({npass} passes, then k_norm_fix)",
          lambda: (pf.apply(sv), pi.apply(sv), None)[2], 2 * S * N * npass)
    pf.close()
    pi.close()
    # a sharded state: two local shards of n - 1 qubits; a gate on the qubit at
    # the global position first swaps it in (k_swap_halves: each shard trades
    # half of its slice in place), then runs on both shards
    ranks = np.arange(2, dtype=np.int32)
    hs = C.c_void_p()
    check(L.qs_sharded_create(n, 1, 0, ranks.ctypes.data_as(C.POINTER(C.c_int)), 2, None, None, C.byref(hs)))
    spos = np.empty(n, dtype=np.int32)

    def global_gate():
        check(L.qs_sharded_positions(hs, spos.ctypes.data_as(C.POINTER(C.c_int))))
        q = int(np.nonzero(spos == n - 1)[0][0])
        gg = circuits.make_gates([("RY", (q,), 0.3)])
        check(L.qs_sharded_apply(hs, C.c_void_p(gg.ctypes.data), 1))

    timed(f"k_swap_halves + k_pair: a gate on the global qubit of {n} qubits over 2 local shards "
          f"(one in-place swap of half of each shard, then the gate)", global_gate, 2 * S * N // 2 + 2 * S * N)
    L.qs_sharded_destroy(hs)
    other.close()
    sv.close()
    print(json.dumps({"workload": f"kernels-{n}q-c64", "peak_gbs": peak, "peak_source": peak_kind,
                      "l2": f"{S * N >> 30} GiB state > L2", "kernels": out}))


# ----------------------------------------------------------------- pass profile
def run_passes(args):
    """The random circuit at --qubits applied once in each tiled layout (in
    place, remap 1, remap 2) after one warm-up each; prints the pass structure
    and each application's time.  Meant to run under a per-launch profiler."""
    import ctypes as C

    import torch
    torch.cuda.set_device(0)
    from qpanda_b200 import FusionPlan, StateVector, lib

    n = args.qubits
    gates = workload(n, args.depth)
    sv = StateVector(n, "c64")
    stream = torch.cuda.current_stream()
    res = {}
    for remap in (0, 1, 2):
        p = FusionPlan(n, gates, remap=remap, low_qubits=args.low, max_sub=args.max_sub, threads_per_row=args.tpr)
        p.apply(sv)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        p.apply(sv)
        e1.record(stream)
        torch.cuda.synchronize()
        res[f"remap{remap}"] = {"passes": p.num_launches(), "circuit_ms": e0.elapsed_time(e1)}
        if remap == 0:
            L = lib()
            struct = []
            for i in range(p.num_launches()):
                nb, T, Q = C.c_int(), (C.c_int * 12)(), (C.c_int * 15)()
                L.qs_plan_pass(p.handle, i, C.byref(nb), T, Q)
                struct.append({"tile": list(T), "blocks": [list(Q[5 * b:5 * b + 5]) for b in range(nb.value)]})
            res["structure"] = struct
        p.close()
    sv.close()
    print(json.dumps({"workload": f"passes-{n}q-depth{args.depth}", "low_qubits": args.low, **res}))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "vqe-sweep":
        run_vqe_sweep(args)
    elif args.workload == "requests":
        run_requests(args)
    elif args.workload == "qft28":
        run_qft(args)
    elif args.workload == "passes":
        run_passes(args)
    elif args.workload == "circuit20":
        run_circuit20(args)
    elif args.workload == "kernels":
        run_kernels(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
