"""A state vector sharded over 2^g ranks (one GPU each), for states larger than
one GPU's memory (33 qubits and up in complex64).

Layout: physical position p of the n-bit amplitude index is a local bit for
p < L = n - g (each rank holds the 2^L amplitudes of its slice) and rank bit
p - L above.  Logical qubit q lives at physical position pos[q]; gates are
applied in physical positions.  The reference has no counterpart (it caps
programs at 30 qubits on one machine, QuantumInstructionHandleAPI.cpp);
each shard runs the same single-GPU kernels as an unsharded state.

A gate on qubits that are all local runs on every shard with no
communication.  A gate that touches a global qubit first swaps it with a
local position outside the gate: the two ranks that differ in that rank bit
exchange half of their shards - rank with rank bit b sends its half with local
bit p = 1 - b and receives the partner's half with local bit p = b into the
same place - after which the qubit is local.  The swap target is the highest
local position the gate does not use, preferring the local qubit whose next
use lies furthest ahead; the top position p = L - 1 makes the half one
contiguous block, so the exchange is a single send/receive of 2^(L-1)
amplitudes over NVLink.

`schedule()` is pure host logic; `ShardedState` runs a schedule with a local
engine per shard (the C ABI on the GPU) and an exchanger: `NcclExchanger`
(one process per GPU, torch.distributed point-to-point, NCCL on GPUs or gloo
on CPU tensors) or `LocalExchanger` (all shards in one process, device
copies).
"""
import numpy as np

from .capi import GATE_DTYPE, OP


def gate_qubits(g):
    """Every qubit a gate record reads or writes (operands and controls)."""
    op = int(g["op"])
    k = 1 if op in (OP["H"], OP["X"], OP["RX"], OP["RY"], OP["RZ"]) else \
        3 if op in (OP["TOFFOLI"], OP["CSWAP"]) else 2
    return [int(x) for x in g["q"][:k]] + [int(x) for x in g["ctrl"][:int(g["nctrl"])]]


def _relabel(g, pos):
    """A copy of gate record g with its qubits at physical positions pos[q]."""
    h = np.array(g, dtype=GATE_DTYPE)
    k = len(gate_qubits(g)) - int(h["nctrl"])
    for j in range(k):
        h["q"][j] = pos[int(g["q"][j])]
    for j in range(int(h["nctrl"])):
        h["ctrl"][j] = pos[int(g["ctrl"][j])]
    return h


def schedule(n, n_global, gates):
    """Steps for applying `gates` (logical qubits) to an n-qubit state whose
    top n_global physical positions are rank bits, starting from pos[q] = q:
      ("local", records)  - gate records in physical positions, all local;
      ("swap", j, p)      - exchange rank bit j with local position p.
    Returns (steps, final_pos)."""
    L = n - n_global
    if L < 1 or n_global < 0:
        raise ValueError("need at least one local qubit")
    gates = np.atleast_1d(np.asarray(gates, dtype=GATE_DTYPE))
    if any(len(gate_qubits(g)) > L for g in gates):
        raise ValueError("a gate has more qubits than a shard has local positions")
    pos = list(range(n))
    at = list(range(n))                       # at[p] = logical qubit at position p
    uses = [gate_qubits(g) for g in gates]
    steps, seg = [], []
    for i, g in enumerate(gates):
        qs = uses[i]
        for q in qs:
            if pos[q] < L:
                continue
            busy = {pos[x] for x in qs if pos[x] < L}

            def next_use(p):
                lq = at[p]
                for k in range(i, len(gates)):
                    if lq in uses[k]:
                        return k
                return len(gates)
            cands = [p for p in range(L - 1, -1, -1) if p not in busy]
            far = max(next_use(p) for p in cands)
            p = next(p for p in cands if next_use(p) == far)   # highest position among the furthest-used
            if seg:
                steps.append(("local", np.array(seg, dtype=GATE_DTYPE)))
                seg = []
            gp = pos[q]
            steps.append(("swap", gp - L, p))
            lq = at[p]
            pos[q], pos[lq] = p, gp
            at[p], at[gp] = q, lq
        seg.append(_relabel(g, pos))
    if seg:
        steps.append(("local", np.array(seg, dtype=GATE_DTYPE)))
    return steps, pos


def half_view(t, L, p, value):
    """View of the amplitudes of a local shard tensor t (2^L complex entries)
    whose local bit p equals value: shape (2^(L-1-p), 2^p), contiguous when
    p = L - 1."""
    return t.view(1 << (L - 1 - p), 2, 1 << p)[:, value, :]


class NcclExchanger:
    """One shard per process: rank r holds rank bits r.  The half exchange of
    a swap is a series of torch.distributed send/receive pairs with the
    partner rank (NCCL between GPUs, gloo for CPU tensors), chunk by chunk:
    each chunk of the outgoing half is sent from where it lies while the
    partner's matching chunk lands in a staging buffer, which is then copied
    into the chunk just sent.  The staging buffer (at most `chunk_amps`
    amplitudes) is allocated once and reused by every swap."""

    def __init__(self, group=None, chunk_amps=1 << 26):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.chunk_amps = int(chunk_amps)
        self.stage = None

    def shards(self):
        return [self.rank]

    def _staging(self, like, amps):
        import torch
        if (self.stage is None or self.stage.device != like.device or self.stage.dtype != like.dtype
                or self.stage.numel() < amps):
            self.stage = torch.empty(amps, dtype=like.dtype, device=like.device)
        return self.stage[:amps]

    def swap(self, tensors, L, j, p):
        import torch
        (t,) = tensors
        partner = self.rank ^ (1 << j)
        b = (self.rank >> j) & 1
        out = half_view(t, L, p, 1 - b)                   # (2^(L-1-p), 2^p)
        rows, cols = out.shape
        # chunks of whole rows (contiguous runs of 2^p amplitudes), or of one row
        per = max(1, min(rows, self.chunk_amps // cols)) if cols <= self.chunk_amps else 1
        width = cols if cols <= self.chunk_amps else self.chunk_amps
        for r0 in range(0, rows, per):
            r1 = min(rows, r0 + per)
            for c0 in range(0, cols, width):
                blk = out[r0:r1, c0:c0 + width]
                send = blk if blk.is_contiguous() else blk.contiguous()
                recv = self._staging(send, send.numel()).view(send.shape)
                ops = [self.dist.P2POp(self.dist.isend, torch.view_as_real(send), partner, self.group),
                       self.dist.P2POp(self.dist.irecv, torch.view_as_real(recv), partner, self.group)]
                for req in self.dist.batch_isend_irecv(ops):
                    req.wait()
                blk.copy_(recv)


class LocalExchanger:
    """All 2^g shards in one process (one GPU or the host): a swap exchanges
    the two halves with device copies through one staging buffer."""

    def __init__(self, n_shards):
        self.n = n_shards

    def shards(self):
        return list(range(self.n))

    def swap(self, tensors, L, j, p):
        for r in range(self.n):
            if (r >> j) & 1:
                continue
            a = half_view(tensors[r], L, p, 1)                 # rank bit 0 sends local bit 1
            b = half_view(tensors[r | (1 << j)], L, p, 0)      # rank bit 1 sends local bit 0
            tmp = a.clone()
            a.copy_(b)
            b.copy_(tmp)


class ShardedState:
    """An n-qubit state over 2^n_global shards.  `engines[i]` runs gate records
    on the shard's 2^L amplitudes and exposes them as a torch tensor
    (`.tensor()`); `exchanger` moves halves between shards.  Starts in
    |0...0> (the shard with rank bits 0 holds amplitude 1)."""

    def __init__(self, n, n_global, engines, exchanger):
        self.n, self.g, self.L = n, n_global, n - n_global
        self.engines = engines
        self.x = exchanger
        self.pos = list(range(n))
        self.swaps = 0

    def run(self, gates):
        steps, self.pos = schedule_from(self.n, self.g, gates, self.pos)
        for st in steps:
            if st[0] == "local":
                for e in self.engines:
                    e.apply(st[1])
            else:
                _, j, p = st
                for e in self.engines:
                    e.synchronize()
                self.x.swap([e.tensor() for e in self.engines], self.L, j, p)
                self.swaps += 1
        return steps


class GpuShard:
    """Local engine of one shard: a 2^L-amplitude state in this process's
    GPU, driven through the C ABI; `tensor()` is a torch view of its device
    amplitudes (no copy) for the exchange.  Shards other than rank bits 0
    start all zero, so that the whole starts in |0...0>.  Several shards of
    one process (LocalExchanger) share the device and its default stream,
    so their kernels and copies run in order, none waiting on another."""

    def __init__(self, L, dtype="c64", rank_bits=0, fused=False):
        from .capi import StateVector
        self.sv = StateVector(L, dtype)
        self.L = L
        self.dtype = dtype
        self.fused = fused
        if rank_bits:
            self.tensor().zero_()

    def apply(self, records):
        """The segment's gates: one kernel per gate, or (fused) as dense
        5-qubit blocks on the tensor cores."""
        if self.fused and len(records) > 1:
            from .capi import FusionPlan
            plan = FusionPlan(self.L, records)
            plan.apply(self.sv)
            plan.close()
        else:
            self.sv.apply(records)

    def synchronize(self):
        self.sv.synchronize()

    def tensor(self):
        import ctypes as C

        import torch

        from .capi import check, lib
        p = C.c_void_p()
        check(lib().qs_device_ptr(self.sv.handle, C.byref(p)))

        class _Dev:
            pass
        d = _Dev()
        d.__cuda_array_interface__ = {"shape": (2 << self.L,), "typestr": "<f4" if self.dtype == "c64" else "<f8",
                                      "data": (p.value, False), "version": 3, "strides": None}
        return torch.view_as_complex(torch.as_tensor(d, device="cuda").view(-1, 2))

    def host(self):
        return self.sv.get_state()

    def close(self):
        self.sv.close()


def schedule_from(n, n_global, gates, pos):
    """schedule() starting from the layout pos (logical -> physical)."""
    L = n - n_global
    # relabel the gate list through pos, schedule from the identity, and map back
    gates = np.atleast_1d(np.asarray(gates, dtype=GATE_DTYPE))
    inv = [0] * n
    for q, p in enumerate(pos):
        inv[p] = q
    moved = np.array([_relabel(g, pos) for g in gates], dtype=GATE_DTYPE) if len(gates) else gates
    steps, p2 = schedule(n, n_global, moved)
    final = [p2[pos[q]] for q in range(n)]
    assert sorted(final) == list(range(n)) and L >= 1
    return steps, final


def gather_logical(shard_states, n, n_global, pos):
    """Full 2^n state in logical qubit order from the host copies of the shards
    (shard r holds rank bits r), for tests and small states."""
    L = n - n_global
    full = np.concatenate([np.asarray(s) for s in shard_states])   # physical index = r * 2^L + local
    t = full.reshape([2] * n)                                        # axis k = physical bit n-1-k
    # logical bit q is physical bit pos[q]: axis order for logical bits n-1..0
    axes = [n - 1 - pos[q] for q in range(n - 1, -1, -1)]
    return np.ascontiguousarray(t.transpose(axes)).reshape(-1)


