"""Continuous-batching serving of GEMVER and NS-residual evaluations on one GPU.

Requests arrive over time (a Poisson process, or all at once for saturation). Each names a MODEL — a GEMVER matrix A
of size n, or an NS state (u, v, p) on an N×N grid — and brings its own small inputs (a GEMVER's six vectors; an NS
evaluation needs none). Models stay resident on the device under an HBM budget: a model is loaded (generated on the
device) on first use and evicted least-recently-used when the budget needs room and no in-flight batch uses it.

Storage precision per kind: GEMVER matrices in BF16 (x and w stay within 2e-4 of f64: the row and column sums average
the rounding out), NS fields in FP32. BF16 fields cannot carry a finite-difference residual: neighbouring cells
differ by about h·|∂f| ≈ 1e-3·|f| on these grids, below BF16's resolution (2^-8 relative), and the measured residual
error against f64 is of order 1 (0.6 to 1.4 on the 4096² fields).

The loop admits requests as they arrive: whenever one of `depth` launch slots (a stream each) is free and requests are
waiting, it takes up to `max_batch` of them in arrival order — requests that arrived while earlier batches are still
on the GPU included — uploads their inputs in ONE host→device copy, launches every GEMVER of the batch in one
persistent launch (cspb_gemver_tasks) and every NS residual in another (cspb_ns_incomp_tasks), copies the results
back in one device→host copy per kind, and records an event. Batches on different slots overlap on the device.
Completion times come from CUDA events on a common origin, so latency = device completion − arrival.

`plain()` serves the same requests the way a caller without batching would: one request at a time, FP32 storage,
the fused single-request kernels (Â written, as the reference's gemver does), one stream. Its dtype / want_B options
give it the server's storage and bytes (BF16 or FP32 without Â), so that a throughput ratio at equal precision and
equal bytes shows what the batching alone buys.

Per-request results do not depend on the batch a request lands in (task tables compute each task exactly as the
single call does); `check_mix()` verifies it.
"""
from __future__ import annotations

import collections
import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from ._capi import lib
from .tasks import GEMVER_TASK, NS_TASK, TaskRunner
from .workloads import hash_unit01

KIND_GEMVER, KIND_NS = 0, 1


def _torch():
    import torch
    return torch


# ---- the workload ---------------------------------------------------------------------------------------------
@dataclass
class Workload:
    kind: np.ndarray          # per request: 0 GEMVER, 1 NS
    model: np.ndarray         # per request: model id
    size: np.ndarray          # per request: n (GEMVER) or N (NS)
    arrival: np.ndarray       # seconds from the start
    in_off: np.ndarray        # per request: offset (floats) of its inputs in `inputs` (count + 1)
    out_off: np.ndarray       # per request: offset (floats) of its x, w in the output buffer (count + 1)
    inputs: object            # pinned host float32: GEMVER u1 v1 u2 v2 y z back to back, per request
    model_size: dict          # model id -> (kind, size)
    alpha: float = 1.5
    beta: float = 1.2
    nu: float = 1e-3

    @property
    def count(self) -> int:
        return int(self.kind.size)


def make_workload(n_req: int = 20000, *, rate: float | None = None, seed: int = 0, frac_gemver: float = 0.7,
                  gemver_models: int = 512, ns_models: int = 64, n_lo: int = 128, n_hi: int = 8192,
                  grids=(256, 512, 1024, 2048)) -> Workload:
    """The serving stream: `n_req` requests, 70% GEMVER on models of n ~ log-U[n_lo, n_hi], 30% NS residual on
    grids drawn from `grids`; Poisson arrivals at `rate` per second (None: all at t = 0)."""
    torch = _torch()
    r = np.arange(n_req, dtype=np.uint64)
    s = 16 * seed
    is_g = hash_unit01(s + 12, r) < frac_gemver
    kind = np.where(is_g, KIND_GEMVER, KIND_NS).astype(np.int32)
    gm = np.minimum((hash_unit01(s + 13, r) * gemver_models).astype(np.int64), gemver_models - 1)
    nm = np.minimum((hash_unit01(s + 14, r) * ns_models).astype(np.int64), ns_models - 1)
    model = np.where(is_g, gm, gemver_models + nm)
    u = hash_unit01(s + 15, np.arange(gemver_models, dtype=np.uint64)).astype(np.float64)
    gsize = np.clip(np.rint(n_lo * (n_hi / n_lo) ** u), n_lo, n_hi).astype(np.int64)
    gi = np.minimum((hash_unit01(s + 16, np.arange(ns_models, dtype=np.uint64)) * len(grids)).astype(np.int64),
                    len(grids) - 1)
    nsize = np.array(grids, dtype=np.int64)[gi]
    model_size = {int(m): (KIND_GEMVER, int(gsize[m])) for m in range(gemver_models)}
    model_size.update({gemver_models + int(m): (KIND_NS, int(nsize[m])) for m in range(ns_models)})
    size = np.array([model_size[int(m)][1] for m in model], dtype=np.int64)
    if rate is None or math.isinf(rate):
        arrival = np.zeros(n_req)
    else:
        e = -np.log1p(-hash_unit01(s + 17, r).astype(np.float64) * (1 - 2 ** -24)) / rate
        arrival = np.cumsum(e)
    nin = np.where(kind == KIND_GEMVER, 6 * size, 0)
    nout = np.where(kind == KIND_GEMVER, 2 * size, 0)
    in_off = np.concatenate([[0], np.cumsum(nin)]).astype(np.int64)
    out_off = np.concatenate([[0], np.cumsum(nout)]).astype(np.int64)
    inputs = torch.empty(int(in_off[-1]), dtype=torch.float32, pin_memory=True)
    # each request's vectors: the hash generator U[0, 1) over the packed index (generated on the device, in chunks)
    import cospanmdao_b200 as cb
    chunk = 1 << 26
    tmp = torch.empty(min(chunk, max(int(in_off[-1]), 1)), dtype=torch.float32, device="cuda")
    for a in range(0, int(in_off[-1]), chunk):
        b = min(int(in_off[-1]), a + chunk)
        cb.fill_hash(tmp[:b - a], s + 18, 1, base=a)
        inputs[a:b].copy_(tmp[:b - a])
    del tmp
    return Workload(kind, model, size, arrival, in_off, out_off, inputs, model_size)


# ---- resident models --------------------------------------------------------------------------------------------
def model_matrix(n: int, dtype, seed: int, device):
    """A GEMVER model's matrix: the seeded generator's n×n values (element (i, j) from index i·n + j), stored with its
    rows padded to a multiple of 8 elements so that every row starts on 16 bytes (the kernels' vector loads need it;
    an unpadded odd n would leave most rows misaligned). Returns the (n, n) view; its stride(0) is the padded pitch."""
    import cospanmdao_b200 as cb
    torch = _torch()
    ld = (n + 7) // 8 * 8
    buf = torch.empty((n, ld), dtype=dtype, device=device)
    if ld == n:
        cb.fill_hash(buf, seed, 0)
    else:
        tmp = torch.empty((n, n), dtype=dtype, device=device)
        cb.fill_hash(tmp, seed, 0)
        buf[:, :n].copy_(tmp)
        del tmp
    return buf[:, :n]



@dataclass
class Model:
    id: int
    kind: int
    size: int
    tensors: dict
    nbytes: int
    in_use: int = 0
    last_used: int = 0


class ModelStore:
    """Device-resident models under a byte budget, loaded on first use, evicted least-recently-used."""

    def __init__(self, wl: Workload, *, dtype, budget_bytes: float, device, ns_dtype=None,
                 h_of=lambda N: 2 * math.pi / N):
        self.wl = wl
        self.dtype = dtype
        self.ns_dtype = ns_dtype or _torch().float32
        self.budget = float(budget_bytes)
        self.device = device
        self.models: dict[int, Model] = {}
        self.used = 0
        self.clock = 0
        self.loads = 0
        self.evictions = 0
        self.h_of = h_of

    def bytes_of(self, mid: int) -> int:
        kind, size = self.wl.model_size[mid]
        dt = self.dtype if kind == KIND_GEMVER else self.ns_dtype
        es = 2 if dt == _torch().bfloat16 else 4
        if kind == KIND_GEMVER:
            return size * ((size + 7) // 8 * 8) * es  # rows padded to 8 elements (model_matrix)
        return size * size * es * 3

    def _load(self, mid: int) -> Model:
        import cospanmdao_b200 as cb
        from . import workloads
        torch = _torch()
        kind, size = self.wl.model_size[mid]
        if kind == KIND_GEMVER:
            t = {"A": model_matrix(size, self.dtype, 16 * (1000 + mid) + 1, self.device)}
        else:
            u, v, p, h = workloads.ns_fields(size, seed=1000 + mid, dtype=self.ns_dtype, device=self.device)
            t = {"u": u, "v": v, "p": p, "h": h}
        self.loads += 1
        return Model(mid, kind, size, t, self.bytes_of(mid))

    def acquire(self, mids) -> bool:
        """Makes every model in `mids` resident and marks it in use; False if the budget cannot hold them now."""
        want = list(dict.fromkeys(int(x) for x in mids))
        wanted = set(want)
        need = [m for m in want if m not in self.models]
        extra = sum(self.bytes_of(m) for m in need)
        if self.used + extra > self.budget:
            for m in sorted(self.models.values(), key=lambda q: q.last_used):
                if self.used + extra <= self.budget:
                    break
                if m.in_use == 0 and m.id not in wanted:
                    del self.models[m.id]
                    self.used -= m.nbytes
                    self.evictions += 1
            if self.used + extra > self.budget:
                return False
        for m in need:
            self.models[m] = self._load(m)
            self.used += self.models[m].nbytes
        self.clock += 1
        for m in want:
            self.models[m].in_use += 1
            self.models[m].last_used = self.clock
        return True

    def release(self, mids):
        for m in dict.fromkeys(int(x) for x in mids):
            self.models[m].in_use -= 1


# ---- the batching server ----------------------------------------------------------------------------------------
@dataclass
class Slot:
    stream: object
    runner_g: TaskRunner
    runner_n: TaskRunner
    dev_in: object = None
    dev_out: object = None
    dev_norm: object = None
    dev_ns: object = None
    end: object = None
    lo: int = 0
    hi: int = 0
    mids: tuple = ()
    stage_g: object = None
    stage_n: object = None


def _grow(t, n, dtype, device):
    torch = _torch()
    if t is None or t.numel() < n:
        return torch.empty(max(int(n), 1) + (int(n) >> 2), dtype=dtype, device=device)
    return t


class Server:
    def __init__(self, wl: Workload, *, budget_bytes: float = 120e9, dtype=None, max_batch: int = 512,
                 depth: int = 4, device=None, preload: bool = True):
        torch = _torch()
        self.wl = wl
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.dtype = dtype or torch.bfloat16
        self.max_batch = int(max_batch)
        self.store = ModelStore(wl, dtype=self.dtype, budget_bytes=budget_bytes, device=self.device)
        self.slots = [Slot(torch.cuda.Stream(self.device), TaskRunner(self.device), TaskRunner(self.device))
                      for _ in range(depth)]
        for s in self.slots:
            s.stage_g = torch.empty(self.max_batch * GEMVER_TASK.itemsize, dtype=torch.uint8, pin_memory=True)
            s.stage_n = torch.empty(self.max_batch * NS_TASK.itemsize, dtype=torch.uint8, pin_memory=True)
        self.out = torch.empty(int(wl.out_off[-1]) + 1, dtype=torch.float32, pin_memory=True)
        self.norms = torch.empty((wl.count, 3), dtype=torch.float64, pin_memory=True)
        if preload:
            mids = sorted(wl.model_size)
            fits = []
            tot = 0
            for m in mids:
                if tot + self.store.bytes_of(m) <= budget_bytes:
                    fits.append(m)
                    tot += self.store.bytes_of(m)
            self.store.acquire(fits)
            self.store.release(fits)
            torch.cuda.synchronize()

    def _launch(self, slot: Slot, lo: int, hi: int):
        torch = _torch()
        wl = self.wl
        kinds = wl.kind[lo:hi]
        mids = wl.model[lo:hi]
        gi = np.nonzero(kinds == KIND_GEMVER)[0] + lo
        ni = np.nonzero(kinds == KIND_NS)[0] + lo
        in0, in1 = int(wl.in_off[lo]), int(wl.in_off[hi])
        o0, o1 = int(wl.out_off[lo]), int(wl.out_off[hi])
        dev = self.device
        s = slot.stream
        ns_cells = int((wl.size[ni] ** 2).sum()) if ni.size else 0
        with torch.cuda.stream(s):
            # scratch of the slot, allocated on the slot's stream (stream-ordered reuse)
            slot.dev_in = _grow(slot.dev_in, in1 - in0, torch.float32, dev)
            slot.dev_out = _grow(slot.dev_out, o1 - o0, torch.float32, dev)
            slot.dev_norm = _grow(slot.dev_norm, 3 * (hi - lo), torch.float64, dev)
            slot.dev_ns = _grow(slot.dev_ns, 3 * ns_cells, torch.float32, dev)
            if in1 > in0:
                slot.dev_in[:in1 - in0].copy_(wl.inputs[in0:in1], non_blocking=True)
            if gi.size:
                t = np.zeros(gi.size, dtype=GEMVER_TASK)
                n = wl.size[gi]
                base_in = int(slot.dev_in.data_ptr()) + 4 * (wl.in_off[gi] - in0)
                base_out = int(slot.dev_out.data_ptr()) + 4 * (wl.out_off[gi] - o0)
                mats = [self.store.models[int(m)].tensors["A"] for m in wl.model[gi]]
                t["n"] = n
                t["lda"] = [a.stride(0) for a in mats]
                t["ldb"] = n
                t["A"] = [a.data_ptr() for a in mats]
                for k, name in enumerate(("u1", "v1", "u2", "v2", "y", "z")):
                    t[name] = base_in + 4 * k * n
                t["x"] = base_out
                t["w"] = base_out + 4 * n
                t["alpha"] = wl.alpha
                t["beta"] = wl.beta
                slot.runner_g.gemver(t, bf16=self.dtype == torch.bfloat16, stream=s, host_staging=slot.stage_g)
            if ni.size:
                t = np.zeros(ni.size, dtype=NS_TASK)
                N = wl.size[ni]
                cells = N * N
                coff = np.concatenate([[0], np.cumsum(cells)])[:-1]
                base = int(slot.dev_ns.data_ptr())
                t["nx"] = N
                t["ny"] = N
                t["h"] = 2 * math.pi / N
                t["nu"] = wl.nu
                ms = [self.store.models[int(m)].tensors for m in wl.model[ni]]
                t["u"] = [m["u"].data_ptr() for m in ms]
                t["v"] = [m["v"].data_ptr() for m in ms]
                t["p"] = [m["p"].data_ptr() for m in ms]
                t["ru"] = base + 4 * coff
                t["rv"] = base + 4 * (ns_cells + coff)
                t["rc"] = base + 4 * (2 * ns_cells + coff)
                t["norms"] = int(slot.dev_norm.data_ptr()) + 8 * 3 * (ni - lo)
                slot.runner_n.ns(t, bf16=self.store.ns_dtype == torch.bfloat16, stream=s, host_staging=slot.stage_n)
            if o1 > o0:
                self.out[o0:o1].copy_(slot.dev_out[:o1 - o0], non_blocking=True)
            self.norms[lo:hi].view(-1).copy_(slot.dev_norm[:3 * (hi - lo)], non_blocking=True)
            slot.end = torch.cuda.Event(enable_timing=True)
            slot.end.record(s)
        slot.lo, slot.hi, slot.mids = lo, hi, tuple(mids)

    def run(self) -> dict:
        """Serves the whole workload; returns throughput and latency statistics."""
        torch = _torch()
        wl = self.wl
        N = wl.count
        done_t = np.full(N, np.nan)
        torch.cuda.synchronize()
        origin = torch.cuda.Event(enable_timing=True)
        origin.record(torch.cuda.current_stream())
        origin.synchronize()
        t0 = time.perf_counter()
        free = collections.deque(self.slots)
        busy = []
        i = 0
        batches = 0
        sizes = []
        while i < N or busy:
            # retire finished batches
            still = []
            for sl in busy:
                if sl.end.query():
                    done_t[sl.lo:sl.hi] = origin.elapsed_time(sl.end) * 1e-3
                    self.store.release(sl.mids)
                    free.append(sl)
                else:
                    still.append(sl)
            busy = still
            now = time.perf_counter() - t0
            if free and i < N and wl.arrival[i] <= now:
                j = i
                lim = min(N, i + self.max_batch)
                while j < lim and wl.arrival[j] <= now:
                    j += 1
                while not self.store.acquire(wl.model[i:j]):
                    if busy:
                        j = i  # wait for in-flight batches to release models
                        break
                    if j - i == 1:
                        raise RuntimeError("the HBM budget cannot hold the model of one request")
                    j = i + (j - i) // 2  # admit fewer requests whose models fit
                if j == i:
                    continue
                sl = free.popleft()
                self._launch(sl, i, j)
                busy.append(sl)
                batches += 1
                sizes.append(j - i)
                i = j
            elif not (free and i < N):
                time.sleep(0)
        torch.cuda.synchronize()
        lat = done_t - wl.arrival
        span = float(np.nanmax(done_t) - wl.arrival.min())
        return {"requests": N, "req_per_s": N / span, "makespan_s": span,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3), "batches": batches, "mean_batch": float(np.mean(sizes)),
                "loads": self.store.loads, "evictions": self.store.evictions,
                "resident_gb": self.store.used / 1e9}


# ---- the per-request FP32 path ---------------------------------------------------------------------------------
def plain(wl: Workload, *, device=None, stream=None, dtype=None, want_B: bool = True) -> dict:
    """Each request on its own: the single-request kernels, one stream, no batching. By default FP32 models with Â
    written (what a caller of the reference's gemver gets); dtype=bfloat16 and/or want_B=False give the per-request
    path the same storage and the same bytes as the batched server, so that the two differ by the batching alone."""
    import cospanmdao_b200 as cb
    from . import workloads
    torch = _torch()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    gdt = dtype or torch.float32
    models = {}
    for m, (kind, size) in wl.model_size.items():
        if kind == KIND_GEMVER:
            models[m] = {"A": model_matrix(size, gdt, 16 * (1000 + m) + 1, dev)}
        else:
            u, v, p, h = workloads.ns_fields(size, seed=1000 + m, dtype=torch.float32, device=dev)
            models[m] = {"u": u, "v": v, "p": p, "h": h}
    nmax = max(s for k, s in wl.model_size.values() if k == KIND_GEMVER)
    gmax = max(s for k, s in wl.model_size.values() if k == KIND_NS)
    B = torch.empty(nmax * nmax if want_B else 1, dtype=torch.float32, device=dev)
    vin = torch.empty(6 * nmax, dtype=torch.float32, device=dev)
    xw = torch.empty(2 * nmax, dtype=torch.float32, device=dev)
    rns = [torch.empty(gmax * gmax, dtype=torch.float32, device=dev) for _ in range(3)]
    nrm = torch.empty(3, dtype=torch.float64, device=dev)
    out = torch.empty(int(wl.out_off[-1]) + 1, dtype=torch.float32, pin_memory=True)
    norms = torch.empty((wl.count, 3), dtype=torch.float64, pin_memory=True)
    ws = cb.Workspace(dev)
    s = stream or torch.cuda.current_stream()
    N = wl.count
    ends = [None] * N
    torch.cuda.synchronize()
    origin = torch.cuda.Event(enable_timing=True)
    origin.record(s)
    origin.synchronize()
    t0 = time.perf_counter()
    for r in range(N):
        while wl.arrival[r] > time.perf_counter() - t0:
            time.sleep(0)
        md = models[int(wl.model[r])]
        n = int(wl.size[r])
        with torch.cuda.stream(s):
            if wl.kind[r] == KIND_GEMVER:
                a, b = int(wl.in_off[r]), int(wl.in_off[r + 1])
                vin[:b - a].copy_(wl.inputs[a:b], non_blocking=True)
                v = [vin[k * n:(k + 1) * n] for k in range(6)]
                cb.gemver(md["A"], *v, alpha=wl.alpha, beta=wl.beta, want_B=want_B,
                          B=B[:n * n].view(n, n) if want_B else None, x=xw[:n], w=xw[n:2 * n], workspace=ws, stream=s)
                o = int(wl.out_off[r])
                out[o:o + 2 * n].copy_(xw[:2 * n], non_blocking=True)
            else:
                cells = n * n
                cb.ns_incompressible(md["u"], md["v"], md["p"], h=md["h"], nu=wl.nu,
                                     out=tuple(t[:cells].view(n, n) for t in rns), norms=nrm, workspace=ws, stream=s)
                norms[r].copy_(nrm, non_blocking=True)
            e = torch.cuda.Event(enable_timing=True)
            e.record(s)
            ends[r] = e
    torch.cuda.synchronize()
    done_t = np.array([origin.elapsed_time(e) * 1e-3 for e in ends])
    lat = done_t - wl.arrival
    span = float(done_t.max() - wl.arrival.min())
    return {"requests": N, "req_per_s": N / span, "makespan_s": span,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "out": out, "norms": norms}


# ---- checks: the same alone and in the mix; error against f64 --------------------------------------------------------
def result_of(server: Server, r: int):
    """Request r's result as served in the mix: (x, w) for a GEMVER, the 3 norms for an NS residual (host arrays)."""
    wl = server.wl
    if wl.kind[r] == KIND_GEMVER:
        n = int(wl.size[r])
        o = int(wl.out_off[r])
        return server.out[o:o + n].numpy().copy(), server.out[o + n:o + 2 * n].numpy().copy()
    return server.norms[r].numpy().copy()


def serve_alone(server: Server, r: int):
    """Request r served by itself (a batch of one) on the same server."""
    torch = _torch()
    sl = server.slots[0]
    if not server.store.acquire(server.wl.model[r:r + 1]):
        raise RuntimeError("the HBM budget cannot hold the model")
    server._launch(sl, r, r + 1)
    sl.end.synchronize()
    server.store.release(sl.mids)
    torch.cuda.synchronize()
    return result_of(server, r)


def check_mix(server: Server, sample) -> bool:
    """Every sampled request's served result equals, bit for bit, the same request served alone."""
    ok = True
    mixed = {r: result_of(server, r) for r in sample}
    for r in sample:
        alone = serve_alone(server, r)
        if isinstance(alone, tuple):
            ok = ok and all(np.array_equal(a, b) for a, b in zip(alone, mixed[r]))
        else:
            ok = ok and np.array_equal(alone, mixed[r])
    return ok


def errors_vs_f64(server: Server, sample) -> dict:
    """Relative L2 error of sampled requests' results against f64 (torch on the GPU) computed from the model in f32
    — the BF16 storage error included. Returns the maxima per output."""
    import cospanmdao_b200 as cb
    from . import workloads
    torch = _torch()
    wl = server.wl
    worst = {"x": 0.0, "w": 0.0, "norms": 0.0}
    dev = server.device
    for r in sample:
        m = int(wl.model[r])
        n = int(wl.size[r])
        got = result_of(server, r)
        if wl.kind[r] == KIND_GEMVER:
            A = torch.empty((n, n), dtype=torch.float32, device=dev)
            cb.fill_hash(A, 16 * (1000 + m) + 1, 0)
            a = int(wl.in_off[r])
            v = [wl.inputs[a + k * n:a + (k + 1) * n].to(dev).double() for k in range(6)]
            B = A.double() + torch.outer(v[0], v[1]) + torch.outer(v[2], v[3])
            x = wl.beta * (B.t() @ v[4]) + v[5]
            w = wl.alpha * (B @ x)
            for key, want, have in (("x", x, got[0]), ("w", w, got[1])):
                e = float(torch.linalg.vector_norm(torch.from_numpy(have).to(dev).double() - want)
                          / torch.linalg.vector_norm(want))
                worst[key] = max(worst[key], e)
        else:
            u, v, p, h = workloads.ns_fields(n, seed=1000 + m, dtype=torch.float32, device=dev)
            U, V, P = u.double(), v.double(), p.double()

            def dx(f):
                return (torch.roll(f, -1, 1) - torch.roll(f, 1, 1)) / (2 * h)

            def dy(f):
                return (torch.roll(f, -1, 0) - torch.roll(f, 1, 0)) / (2 * h)

            def lap(f):
                return ((torch.roll(f, -1, 1) - f) + (torch.roll(f, 1, 1) - f) + (torch.roll(f, -1, 0) - f)
                        + (torch.roll(f, 1, 0) - f)) / (h * h)
            ru = U * dx(U) + V * dy(U) + dx(P) - wl.nu * lap(U)
            rv = U * dx(V) + V * dy(V) + dy(P) - wl.nu * lap(V)
            rc = dx(U) + dy(V)
            want = torch.stack([torch.linalg.vector_norm(t) for t in (ru, rv, rc)]).cpu().numpy()
            worst["norms"] = max(worst["norms"], float(np.max(np.abs(got - want) / want)))
    return worst
