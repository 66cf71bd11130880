"""Task tables: many independent GEMVERs or incompressible NS residuals, anywhere in device memory, in one launch
(cspb_gemver_tasks, cspb_ns_incomp_tasks). A table is a numpy structured array with the C layout of
cspb_gemver_task / cspb_ns_incomp_task, uploaded to the device before the launch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from . import _capi
from ._capi import BF16, F32, lib

GEMVER_TASK = np.dtype([("n", "<i8"), ("lda", "<i8"), ("ldb", "<i8"), ("A", "<u8"), ("B", "<u8"), ("u1", "<u8"),
                        ("v1", "<u8"), ("u2", "<u8"), ("v2", "<u8"), ("y", "<u8"), ("z", "<u8"), ("x", "<u8"),
                        ("w", "<u8"), ("alpha", "<f4"), ("beta", "<f4")])
NS_TASK = np.dtype([("nx", "<i4"), ("ny", "<i4"), ("h", "<f8"), ("nu", "<f8"), ("u", "<u8"), ("v", "<u8"),
                    ("p", "<u8"), ("ru", "<u8"), ("rv", "<u8"), ("rc", "<u8"), ("norms", "<u8")])
assert GEMVER_TASK.itemsize == C.sizeof(_capi.GemverTask) and NS_TASK.itemsize == C.sizeof(_capi.NsIncompTask)


def _torch():
    import torch
    return torch


class TaskRunner:
    """Uploads task tables and launches them; owns a growable table buffer and workspace per runner (one runner per
    stream)."""

    def __init__(self, device=None):
        torch = _torch()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._table = None
        self._ws = None

    def _buf(self, name, nbytes):
        torch = _torch()
        cur = getattr(self, name)
        if cur is None or cur.numel() < nbytes + 256:
            cur = torch.empty(int(nbytes) + 4096, dtype=torch.uint8, device=self.device)
            setattr(self, name, cur)
        p = int(cur.data_ptr())
        return (p + 255) // 256 * 256, cur.numel() - ((p + 255) // 256 * 256 - p)

    def upload(self, table: np.ndarray, stream=None, host_staging=None) -> int:
        """Copies the table to the device on `stream` and returns its device address."""
        torch = _torch()
        raw = np.ascontiguousarray(table).view(np.uint8)
        addr, _ = self._buf("_table", raw.nbytes)
        src = torch.from_numpy(raw) if host_staging is None else host_staging[:raw.nbytes]
        if host_staging is not None:
            host_staging[:raw.nbytes].copy_(torch.from_numpy(raw))
        dst = self._table.narrow(0, addr - int(self._table.data_ptr()), raw.nbytes)
        s = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(s):
            dst.copy_(src, non_blocking=host_staging is not None)
        return addr

    def gemver(self, table: np.ndarray, *, bf16: bool, tune: int = 0, lowrank: bool | None = None, stream=None,
               host_staging=None, no_b: bool | None = None):
        """Runs a GEMVER task table. lowrank: the low-rank form (the rank-2 update as dot products) for tasks without
        B, and for w of bf16 tasks with B; None (the default) follows cb.gemver's 'auto' schedule, so that every task
        gets the single call's form: low-rank for bf16, not for f32. no_b: pass CSPB_BATCH_NO_B (the kernel variant
        without the Â paths, for a bf16 low-rank table in which no task has B); None (the default) passes it exactly
        when no task has B. Returns the workspace pointer, whose status word cspb_read_status reads."""
        import cospanmdao_b200 as cb
        torch = _torch()
        count = int(table.size)
        if count == 0:
            return
        n = table["n"].astype(np.int64)
        max_elems = int((n * n).sum())
        max_vec = int(n.sum())
        s = stream if stream is not None else torch.cuda.current_stream()
        taddr = self.upload(table, s, host_staging)
        need = int(lib().cspb_gemver_batched_workspace_bytes(count, max_elems, max_vec))
        wp, wb = self._buf("_ws", need)
        if lowrank is None:
            lowrank = bf16
        word = int(tune) | (_capi.BATCH_LOWRANK if lowrank else 0)
        if no_b is None:
            no_b = bool(lowrank and bf16 and not table["B"].any())
        if no_b:
            word |= _capi.BATCH_NO_B  # no task stores Â: the variant without those paths
        st = lib().cspb_gemver_tasks(C.c_void_p(taddr), count, max_elems, max_vec, BF16 if bf16 else F32, word,
                                     C.c_void_p(wp), wb, C.c_void_p(int(s.cuda_stream)))
        cb._raise(st, "gemver tasks")
        return wp

    def ns(self, table: np.ndarray, *, bf16: bool, stream=None, host_staging=None):
        import cospanmdao_b200 as cb
        torch = _torch()
        count = int(table.size)
        if count == 0:
            return
        max_cells = int((table["nx"].astype(np.int64) * table["ny"].astype(np.int64)).sum())
        s = stream if stream is not None else torch.cuda.current_stream()
        taddr = self.upload(table, s, host_staging)
        need = int(lib().cspb_ns_incomp_tasks_workspace_bytes(count, max_cells))
        wp, wb = self._buf("_ws", need)
        st = lib().cspb_ns_incomp_tasks(C.c_void_p(taddr), count, max_cells, BF16 if bf16 else F32, C.c_void_p(wp),
                                        wb, C.c_void_p(int(s.cuda_stream)))
        cb._raise(st, "ns tasks")
        return wp


def gemver_task(A, u1, v1, u2, v2, y, z, x, w, *, alpha: float, beta: float, B=None) -> np.ndarray:
    t = np.zeros(1, dtype=GEMVER_TASK)
    n = A.shape[0]
    t["n"], t["lda"] = n, A.stride(0)
    t["ldb"] = B.stride(0) if B is not None else n
    t["A"] = A.data_ptr()
    t["B"] = B.data_ptr() if B is not None else 0
    for k, v in (("u1", u1), ("v1", v1), ("u2", u2), ("v2", v2), ("y", y), ("x", x), ("w", w)):
        t[k] = v.data_ptr()
    t["z"] = z.data_ptr() if z is not None else 0
    t["alpha"], t["beta"] = alpha, beta
    return t


def ns_task(u, v, p, ru, rv, rc, norms, *, h: float, nu: float) -> np.ndarray:
    t = np.zeros(1, dtype=NS_TASK)
    t["ny"], t["nx"] = u.shape
    t["h"], t["nu"] = h, nu
    for k, a in (("u", u), ("v", v), ("p", p), ("ru", ru), ("rv", rv), ("rc", rc)):
        t[k] = a.data_ptr()
    t["norms"] = norms.data_ptr() if norms is not None else 0
    return t
