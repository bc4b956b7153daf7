"""Batches of excitons built and solved together on one GPU (xatu_batch_* of the C ABI).

    batch = ExcitonBatch()
    for ex in excitons:              # configured ExcitonTB objects (mesh set)
        batch.add(ex)
    batch.run(nstates=8)
    eigval, eigvec = batch.result(0)

Every member goes through what initializeHamiltonian + BShamiltonian("mixed") +
diagonalize("davidson") do for one system; the batch records the work in CUDA
graphs on its first run (after tuning the assembly tiles) and replays them.
"""
from __future__ import annotations

import ctypes
import json

import numpy as np

from . import _lib as L


def member_cost(nk: int, nv: int, nc: int) -> int:
    """Work of one member, in units of matrix elements: the assembly writes and every K.X product reads
    the N x N kernel, N = nk * nv * nc."""
    n = nk * nv * nc
    return n * n


def shard_members(costs, world: int):
    """Partition of batch members over `world` ranks with balanced total cost: members in decreasing cost
    (ties by index), each to the rank with the least cost so far (ties to the lowest rank).  Deterministic,
    so every rank computes the same partition from the same list without communicating.  Returns one
    sorted list of member indices per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


class ExcitonBatch:
    def __init__(self, device: int = 0):
        self.device = device
        b = ctypes.c_void_p()
        L.check(L.lib().xatu_batch_create(ctypes.byref(b), device))
        self._b = b
        self.size = 0
        self.nstates = None

    def _call(self, name: str, *args):
        st = getattr(L.lib(), name)(self._b, *args)
        if st != L.XATU_OK:
            msg = L.lib().xatu_batch_last_error(self._b)
            raise L.XatuError(st, msg.decode() if msg else "")

    def set_stream(self, stream_ptr: int):
        self._call("xatu_batch_set_stream", ctypes.c_void_p(stream_ptr))

    def add(self, exciton) -> int:
        sd, ed, keep = exciton.descriptors()
        idx = ctypes.c_int()
        self._call("xatu_batch_add", ctypes.byref(sd), ctypes.byref(ed), ctypes.byref(idx))
        self.size += 1
        return idx.value

    def run(self, nstates: int = 8, tol: float = 0.0, max_iter: int = 0):
        self._call("xatu_batch_run", int(nstates), float(tol), int(max_iter))
        self.nstates = int(nstates)

    def dim(self, index: int) -> int:
        n = ctypes.c_int64()
        self._call("xatu_batch_dim", int(index), ctypes.byref(n))
        return n.value

    def result(self, index: int, vectors: bool = True):
        ev = np.zeros(self.nstates)
        vec = np.zeros((self.dim(index), self.nstates), dtype=np.complex128, order="F") if vectors else None
        self._call("xatu_batch_result", int(index), L.ptr(ev), L.ptr(vec))
        return ev, vec

    def stats(self) -> dict:
        b, s, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        per = (ctypes.c_int * max(1, self.size))()
        buf = ctypes.create_string_buffer(8192)
        self._call("xatu_batch_stats", ctypes.byref(b), ctypes.byref(s), ctypes.byref(it), per, buf, 8192)
        return {"build_ms": b.value, "solve_ms": s.value, "iterations": it.value,
                "member_iterations": list(per)[: self.size], "tuning": json.loads(buf.value.decode() or "{}")}

    def close(self):
        if self._b is not None:
            L.lib().xatu_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
