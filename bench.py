#!/usr/bin/env python
"""bench.py — the fused-chain hot path on B200, measured against HBM roofline, with the reference's CPU path beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--quick]

Headline (`value`): the fused GEMVER at n = 16384 in f32 (A is 1 GiB: inputs larger than L2), as achieved HBM GB/s of
algorithmic traffic (read A, write Â, read Â again, the vectors: 12n² + 32n bytes per step), device-timed with CUDA
events over K steps on the launching stream, max over ranks. Beside it in the same line: the roofline of the
kernel, the CPU baseline (the reference's unfused component loops, f32, OpenMP on all host threads), the end-to-end
number through the C ABI from pinned host buffers, SM clocks sampled during the measurement, and secondary
workloads (BF16-storage GEMVER, both NS residuals at 4096², the gemver chain) with their errors against f64.

With --impl reference, the same metric and configuration measured on the reference's CPU implementation of the path
(the oracle's port of the unfused component loops; AdaptiveCpp is not available to build the reference itself).
Under torchrun, each rank runs its own replica of the workload (independent units: no collective on the data path).
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GEMVER/NS-residual HBM GB/s & %roofline; batched req/s + p50/p99 vs plain, ≤1e-3 rel err"
N_HEAD = 16384
FALLBACK_HBM = 6650.0


def gemver_bytes(n: int, a_bytes: int = 4, store_B: bool = True, second_read_bytes: int | None = None) -> float:
    """Algorithmic bytes of one GEMVER: A once, Â written (if stored), the matrix read once more, vectors."""
    rb = a_bytes if second_read_bytes is None else second_read_bytes
    return float(n) * n * (a_bytes + (4 if store_B else 0) + rb) + 32.0 * n


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": FALLBACK_HBM, "source": "fallback"}


def profile_traffic(name: str):
    """Per-launch DRAM bytes recorded from an ncu capture (a line `traffic_bytes_per_launch = N` in profiles/<name>)."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch"):
            try:
                return float(line.split("=")[1].split()[0])
            except (IndexError, ValueError):
                return None
    return None


# ---- distributed plumbing ----------------------------------------------------------------------------------------
class Dist:
    """One rank per GPU (cospanmdao_b200.replicas.Ranks): each rank runs its own replica of the workload, the step
    time is the max over ranks, and no collective touches the data path."""

    def __init__(self):
        from cospanmdao_b200.replicas import Ranks
        self.r = Ranks()
        self.world, self.rank, self.local = self.r.world, self.r.rank, self.r.local

    def init(self, torch):
        self.r.init("nccl", timeout_s=120)

    def barrier(self, torch):
        self.r.barrier()

    def max(self, torch, x: float) -> float:
        return self.r.max(x)

    def close(self):
        self.r.close()


# ---- clocks -----------------------------------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampled every 200 ms while the measurement runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                rows.append({"sm": float(f[1]), "max": float(f[2]), "util": float(f[4]), "hw": f[6], "hwt": f[7],
                             "swt": f[8], "pcap": f[9]})
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [r for r in rows if r["util"] > 0] or rows
        reasons = []
        for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                          ("pcap", "sw_power_cap")):
            if any(r[key].lower().startswith("active") for r in load):
                reasons.append(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in load), "sm_max_mhz": load[0]["max"],
                "reasons": reasons, "samples": len(rows), "samples_under_load": len(load)}


# ---- timing -----------------------------------------------------------------------------------------------------
def timed(torch, dist: Dist, step, K: int, W: int, soak_s: float = 0.0) -> float:
    """W untimed steps (plus an untimed soak), then K steps between two CUDA events on the current stream, with a
    barrier and a synchronize on both sides. Returns ms per step, max over ranks."""
    for _ in range(W):
        step()
    if soak_s > 0:
        t0 = time.time()
        while time.time() - t0 < soak_s:
            for _ in range(10):
                step()
            torch.cuda.synchronize()
    dist.barrier(torch)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(K):
        step()
    e1.record(s)
    e1.synchronize()
    dist.barrier(torch)
    return dist.max(torch, e0.elapsed_time(e1) / K)


def relerr(torch, got, want) -> float:
    got = got.double()
    want = want.double()
    den = float(torch.linalg.vector_norm(want))
    num = float(torch.linalg.vector_norm(got - want))
    return num / den if den else (0.0 if num == 0 else float("inf"))


# ---- workloads --------------------------------------------------------------------------------------------------
def gemver_f64_reference(torch, d, alpha, beta, A=None):
    """x, w of the GEMVER in f64 on the GPU (torch), from the f32 / bf16 operands: the error yardstick."""
    A = (d["A"] if A is None else A).double()
    B = A + torch.outer(d["u1"].double(), d["v1"].double()) + torch.outer(d["u2"].double(), d["v2"].double())
    x = beta * (B.t() @ d["y"].double()) + d["z"].double()
    w = alpha * (B @ x)
    return B, x, w


def bench_gemver(torch, cb, dist, args, peak):
    from cospanmdao_b200 import workloads
    n = args.n
    dev = torch.device("cuda", torch.cuda.current_device())
    d = workloads.gemver_inputs(n, 0, device=dev)
    B = torch.empty((n, n), dtype=torch.float32, device=dev)
    x = torch.empty(n, dtype=torch.float32, device=dev)
    w = torch.empty(n, dtype=torch.float32, device=dev)
    ws = cb.Workspace(dev)
    alpha, beta = 1.5, 1.2

    def step():
        cb.gemver(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=alpha, beta=beta, B=B, x=x, w=w,
                  schedule=args.schedule, lag=args.lag, workspace=ws)

    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    ms = timed(torch, dist, step, args.steps, args.warmup, soak_s=args.soak)
    clk = clocks.stop()
    nbytes = gemver_bytes(n)
    gbs = nbytes / (ms * 1e-3) / 1e9
    # errors per output against f64 (computed once, outside the timed region)
    B64, x64, w64 = gemver_f64_reference(torch, d, alpha, beta)
    err = {"B": relerr(torch, B, B64), "x": relerr(torch, x, x64), "w": relerr(torch, w, w64)}
    del B64, x64, w64
    torch.cuda.empty_cache()

    # end to end through the C ABI: inputs from pinned host memory, x and w back to the host, every step
    hA = torch.empty((n, n), dtype=torch.float32, pin_memory=True)
    hA.copy_(d["A"])
    hv = {k: d[k].cpu().pin_memory() for k in workloads.VECTORS}
    hx = torch.empty(n, dtype=torch.float32, pin_memory=True)
    hw = torch.empty(n, dtype=torch.float32, pin_memory=True)
    dA = torch.empty_like(d["A"])
    dv = {k: torch.empty_like(d[k]) for k in workloads.VECTORS}

    def e2e_step():
        dA.copy_(hA, non_blocking=True)
        for k in workloads.VECTORS:
            dv[k].copy_(hv[k], non_blocking=True)
        cb.gemver(dA, dv["u1"], dv["v1"], dv["u2"], dv["v2"], dv["y"], dv["z"], alpha=alpha, beta=beta, B=B, x=x,
                  w=w, workspace=ws)
        hx.copy_(x, non_blocking=True)
        hw.copy_(w, non_blocking=True)

    if args.no_e2e:
        return {"ms": ms, "gbs": gbs, "bytes": nbytes, "err": err, "clocks": clk, "e2e": None}
    ke = max(3, min(args.steps, 10))
    ms_e2e = timed(torch, dist, e2e_step, ke, 2)
    h2d = n * n * 4 + 6 * n * 4
    d2h = 2 * n * 4
    del hA, dA
    out = {
        "ms": ms, "gbs": gbs, "bytes": nbytes, "err": err, "clocks": clk,
        "e2e": {"value": dist.world * nbytes / (ms_e2e * 1e-3) / 1e9, "unit": "GB/s", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
    }
    del d, B
    torch.cuda.empty_cache()
    return out


def bench_gemver_bf16(torch, cb, dist, args):
    from cospanmdao_b200 import workloads
    n = args.n
    dev = torch.device("cuda", torch.cuda.current_device())
    d = workloads.gemver_inputs(n, 0, device=dev)
    A16 = d["A"].to(torch.bfloat16)
    x = torch.empty(n, dtype=torch.float32, device=dev)
    w = torch.empty(n, dtype=torch.float32, device=dev)
    B = torch.empty((n, n), dtype=torch.float32, device=dev)
    ws = cb.Workspace(dev)
    res = {}
    for store in (True, False):
        def step():
            cb.gemver(A16, d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2,
                      B=B if store else None, want_B=store, x=x, w=w, workspace=ws)
        ms = timed(torch, dist, step, args.steps, args.warmup)
        nbytes = gemver_bytes(n, a_bytes=2, store_B=store, second_read_bytes=2)
        res["store_B" if store else "no_B"] = {"ms": ms, "gbs": nbytes / (ms * 1e-3) / 1e9, "bytes": nbytes}
    # without Â the default schedule is the low-rank form (the rank-2 update as dot products): its own error check
    xl = torch.empty_like(x)
    wl = torch.empty_like(w)
    cb.gemver(A16, d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2, want_B=False, x=xl, w=wl,
              workspace=ws)
    cb.gemver(A16, d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2, B=B, x=x, w=w,
              workspace=ws)
    B64, x64, w64 = gemver_f64_reference(torch, d, 1.5, 1.2)  # the f32 matrix: storage error included
    res["err_vs_f64_of_f32_A"] = {"B": relerr(torch, B, B64), "x": relerr(torch, x, x64), "w": relerr(torch, w, w64),
                                  "x_no_B": relerr(torch, xl, x64), "w_no_B": relerr(torch, wl, w64)}
    res["no_B"]["schedule"] = "lowrank"
    del B64, x64, w64, B, A16, d
    torch.cuda.empty_cache()
    return res


def bench_sharded(torch, cb, dist, args):
    """ONE GEMVER of size n split by rows over the job's ranks (cospanmdao_b200.sharded): strong scaling, the rank's
    rows per GPU plus one exchange of the n f64 column-sum shares (all-gather over NCCL, summed in rank order). ms is
    the max over ranks; GB/s is the whole GEMVER's algorithmic bytes over it."""
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.sharded import gemver_sharded, shard_rows
    n = args.n
    dev = torch.device("cuda", torch.cuda.current_device())
    d = workloads.gemver_inputs(n, 0, device=dev)  # every rank builds the same GEMVER and takes its rows
    r0, r1 = shard_rows(n, dist.world)[dist.rank]
    A = d["A"][r0:r1].contiguous()
    rows = {k: d[k][r0:r1].contiguous() for k in ("u1", "u2", "y")}
    del d["A"]
    ws = cb.Workspace(dev)
    ranks = dist.r if dist.world > 1 else None

    def step():
        gemver_sharded(A, rows["u1"], d["v1"], rows["u2"], d["v2"], rows["y"], d["z"], alpha=1.5, beta=1.2,
                       ranks=ranks, workspace=ws)

    ms = timed(torch, dist, step, args.steps, args.warmup)
    nbytes = gemver_bytes(n)
    del A, rows, d
    torch.cuda.empty_cache()
    return {"ms": ms, "gbs_whole_gemver": nbytes / (ms * 1e-3) / 1e9, "ranks": dist.world, "rows_per_rank": r1 - r0,
            "scaling": "strong", "exchange_bytes_per_rank": 8 * n}


def bench_ns_sharded(torch, cb, dist, args):
    """ONE incompressible NS residual on the --grid² periodic grid split into y-slabs over the job's ranks
    (cospanmdao_b200.sharded): strong scaling, one all-gather of the slabs' boundary rows and one of their squared
    sums per step. ms is the max over ranks; GB/s is the whole grid's 24 B per cell over it."""
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.sharded import ns_incompressible_sharded, shard_rows
    N = args.grid
    dev = torch.device("cuda", torch.cuda.current_device())
    u, v, p, h = workloads.ns_fields(N, seed=0, device=dev)  # every rank builds the same grid and takes its rows
    r0, r1 = shard_rows(N, dist.world, 32)[dist.rank]
    mine = [f[r0:r1].contiguous() for f in (u, v, p)]
    del u, v, p
    ws = cb.Workspace(dev)
    ranks = dist.r if dist.world > 1 else None

    def step():
        ns_incompressible_sharded(*mine, h=h, nu=1e-3, ranks=ranks, workspace=ws)

    ms = timed(torch, dist, step, args.steps, args.warmup)
    del mine
    torch.cuda.empty_cache()
    return {"ms": ms, "gbs_whole_grid": 24.0 * N * N / (ms * 1e-3) / 1e9, "ranks": dist.world, "rows_per_rank": r1 - r0,
            "scaling": "strong", "halo_bytes_per_rank": 2 * 3 * 4 * N}


def bench_chain(torch, cb, dist, args):
    from cospanmdao_b200 import workloads
    n = args.n
    dev = torch.device("cuda", torch.cuda.current_device())
    d = workloads.gemver_inputs(n, 0, device=dev, dist="reference")
    a = {k: d[k] for k in workloads.VECTORS}
    b = {k: d[k] for k in ("u1", "v1", "u2", "v2")}
    out = {k: torch.empty((n, n) if k.startswith("B") else (n,), dtype=torch.float32, device=dev)
           for k in ("B1", "x1", "w1", "q", "s", "B2", "x2", "w2")}
    ws = cb.Workspace(dev)
    ab = 1.0 / math.sqrt(n)

    def step():
        cb.gemver_chain(d["A"], a, b, alpha=ab, beta=ab, out=out, workspace=ws)

    ms = timed(torch, dist, step, max(3, args.steps // 2), args.warmup)
    alg = 24.0 * n * n + 80.0 * n
    nominal = 8.0 * n * n * 4  # the reference's quoted traffic (examples/gemver-chain/README.md:136)
    del out, d
    torch.cuda.empty_cache()
    return {"ms": ms, "gbs_algorithmic": alg / (ms * 1e-3) / 1e9, "gbs_nominal_reference_formula": nominal / (ms * 1e-3) / 1e9,
            "reference_rtx4090_crafted_ms": 8.359}


def bench_ns(torch, cb, dist, args):
    from cospanmdao_b200 import workloads
    N = args.grid
    dev = torch.device("cuda", torch.cuda.current_device())
    res = {}
    u, v, p, h = workloads.ns_fields(N, seed=0, device=dev)
    out = tuple(torch.empty((N, N), dtype=torch.float32, device=dev) for _ in range(3))
    norms = torch.empty(3, dtype=torch.float64, device=dev)
    ws = cb.Workspace(dev)

    def step():
        cb.ns_incompressible(u, v, p, h=h, nu=1e-3, out=out, norms=norms, workspace=ws)

    ms = timed(torch, dist, step, args.steps, args.warmup)
    nbytes = 24.0 * N * N
    # f64 yardstick of the formula (torch on the GPU)
    U, V, P = u.double(), v.double(), p.double()

    def ddx(f):
        return (torch.roll(f, -1, 1) - torch.roll(f, 1, 1)) / (2 * h)

    def ddy(f):
        return (torch.roll(f, -1, 0) - torch.roll(f, 1, 0)) / (2 * h)

    def lap(f):
        return ((torch.roll(f, -1, 1) - f) + (torch.roll(f, 1, 1) - f) + (torch.roll(f, -1, 0) - f)
                + (torch.roll(f, 1, 0) - f)) / (h * h)
    ru64 = U * ddx(U) + V * ddy(U) + ddx(P) - 1e-3 * lap(U)
    rv64 = U * ddx(V) + V * ddy(V) + ddy(P) - 1e-3 * lap(V)
    rc64 = ddx(U) + ddy(V)
    n64 = torch.stack([torch.linalg.vector_norm(t) for t in (ru64, rv64, rc64)])
    res["incompressible_f32"] = {
        "grid": N, "ms": ms, "gbs": nbytes / (ms * 1e-3) / 1e9, "bytes": nbytes,
        "err": {"r_u": relerr(torch, out[0], ru64), "r_v": relerr(torch, out[1], rv64), "r_c": relerr(torch, out[2], rc64),
                "norms": float(((norms - n64).abs() / n64).max())}}
    ub, vb, pb = (t.to(torch.bfloat16) for t in (u, v, p))

    def step16():
        cb.ns_incompressible(ub, vb, pb, h=h, nu=1e-3, out=out, norms=norms, workspace=ws)

    ms16 = timed(torch, dist, step16, args.steps, args.warmup)
    b16 = 18.0 * N * N
    res["incompressible_bf16"] = {"ms": ms16, "gbs": b16 / (ms16 * 1e-3) / 1e9, "bytes": b16,
                                  "err_vs_f64_of_f32_fields": {"r_u": relerr(torch, out[0], ru64),
                                                               "r_v": relerr(torch, out[1], rv64),
                                                               "r_c": relerr(torch, out[2], rc64)}}
    del U, V, P, ru64, rv64, rc64, u, v, p, ub, vb, pb, out
    torch.cuda.empty_cache()

    Uc = cb.ns_init_cons(N, N, 1.0, device=dev)
    R = torch.empty_like(Uc)
    diag = torch.empty(18, dtype=torch.float32, device=dev)
    sq = torch.empty(4, dtype=torch.float64, device=dev)
    for bc, lim, exact in (("walls", "minmod", False), ("periodic", "minmod", False), ("walls", "vanleer", False),
                           ("walls", "minmod", True), ("walls", "vanleer", True)):
        def stepc():
            cb.ns_compressible(Uc, limiter=lim, bc=bc, R=R, diag=diag, det_sq64=sq, workspace=ws,
                               reference_rounding=exact)
        msc = timed(torch, dist, stepc, args.steps, args.warmup)
        key = f"compressible_{bc}_{lim}" + ("_reference_rounding" if exact else "")
        res[key] = {"grid": N, "ms": msc, "gbs_nominal": 32.0 * N * N / (msc * 1e-3) / 1e9,
                    "reference_rtx4090_handwritten_ms": 3.550 if (bc == "walls" and lim == "minmod") else None}
    del Uc, R
    torch.cuda.empty_cache()
    return res


def bench_scan(torch, cb, dist, args, peak):
    """The single-pass decoupled-lookback scan (cspb_exclusive_scan_u32 / _u64) and the fused ragged-column builder
    (cspb_build_column, counts mode from i32) at 2^28 items (--scan-log2): algorithmic bytes 8 B/item (u32 in, u32 out),
    16 B/item (u64) and 12 B/item (i32 counts in, u32 extents and u32 offsets out). Inputs are 1..2 GiB at 2^28, larger
    than L2 from 2^25 on."""
    import ctypes
    from cospanmdao_b200 import _capi
    n = 1 << args.scan_log2
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = cb.lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ws = cb.Workspace(dev)
    wp, wb = ws.ptr(lib.cspb_scan_workspace_bytes(n))
    res = {}
    g = torch.Generator(device=dev).manual_seed(0)
    for name, dt, fn, bpi in (("scan_u32", torch.int32, lib.cspb_exclusive_scan_u32, 8.0),
                              ("scan_u64", torch.int64, lib.cspb_exclusive_scan_u64, 16.0)):
        vals = torch.randint(0, 1000, (n,), dtype=dt, device=dev, generator=g)
        out = torch.empty(n + 1, dtype=dt, device=dev)

        def step():
            rc = fn(ctypes.c_void_p(vals.data_ptr()), ctypes.c_void_p(out.data_ptr()), n, wp, wb, st)
            if rc != 0:
                raise RuntimeError(f"{name}: {rc}")

        ms = timed(torch, dist, step, args.steps, args.warmup)
        # bit-exact check of the last step against torch's cumsum (int64: exact for these values)
        mask = 0xffffffff if dt == torch.int32 else -1
        want = torch.cumsum(vals.to(torch.int64), 0)
        ok = bool(torch.equal(out[1:].to(torch.int64) & mask, want & mask)) and int(out[0]) == 0
        gbs = bpi * n / (ms * 1e-3) / 1e9
        res[name] = {"items": n, "ms": ms, "gbs": gbs, "frac_of_measured_hbm": gbs / peak["hbm_gbs"],
                     "bytes_per_item": bpi, "bit_exact_vs_cumsum": ok}
        del vals, out, want
        torch.cuda.empty_cache()
    counts = torch.randint(0, 16, (n,), dtype=torch.int32, device=dev, generator=g)
    ext = torch.empty(n, dtype=torch.int32, device=dev)
    offs = torch.empty(n + 1, dtype=torch.int32, device=dev)
    tf = torch.empty(2, dtype=torch.int32, device=dev)

    def stepc():
        rc = lib.cspb_build_column(ctypes.c_void_p(counts.data_ptr()), _capi.I32, n, 1, 0,
                                   ctypes.c_void_p(ext.data_ptr()), ctypes.c_void_p(offs.data_ptr()),
                                   ctypes.c_void_p(tf.data_ptr()), wp, wb, st)
        if rc != 0:
            raise RuntimeError(f"build_column: {rc}")

    ms = timed(torch, dist, stepc, args.steps, args.warmup)
    want = torch.cumsum(counts.to(torch.int64), 0)
    ok = bool(torch.equal(offs[1:].to(torch.int64) & 0xffffffff, want & 0xffffffff)) and \
        int(tf[0]) & 0xffffffff == int(want[-1]) & 0xffffffff and int(tf[1]) == 0
    gbs = 12.0 * n / (ms * 1e-3) / 1e9
    res["build_column_i32"] = {"items": n, "ms": ms, "gbs": gbs, "frac_of_measured_hbm": gbs / peak["hbm_gbs"],
                               "bytes_per_item": 12.0, "bit_exact_vs_cumsum": ok}
    del counts, ext, offs, want
    torch.cuda.empty_cache()
    return res


def bench_ragged(torch, cb, dist, args, peak):
    """4096 independent GEMVERs, n ~ log-U[64, 4096], f32, packed, in one persistent launch with device-scanned u64
    offsets, replayed as a CUDA graph; the tile geometry per size bucket, the work items per grab and the blocks
    per SM picked by the autotuner."""
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.batched import RaggedBatch, autotune
    sizes = workloads.ragged_sizes(args.ragged)
    b = RaggedBatch(sizes).fill(seed=0)
    b.run(check=True)
    torch.cuda.synchronize()
    offsets_ok = b.offsets_match()
    tuned = autotune(b, reps=4)  # the candidates differ by 1-2 %: four runs a trial keep the pick stable
    tune = tuned["tune"]
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b.run(tune=tune)  # warm the allocations outside the capture
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        b.run(tune=tune)
    ms = timed(torch, dist, graph.replay, max(3, args.steps // 5), args.warmup)
    nbytes = b.algorithmic_bytes()
    gbs = nbytes / (ms * 1e-3) / 1e9
    del graph, b
    torch.cuda.empty_cache()
    return {"instances": int(sizes.size), "sum_n2": float((sizes.astype(np.float64) ** 2).sum()),
            "ms": ms, "gbs": gbs, "frac": gbs / peak["hbm_gbs"], "offsets_bit_exact": bool(offsets_ok),
            "tune": tune, "tune_codes": tuned["codes"], "tune_group": tuned["group"], "tune_blocks": tuned["blocks"],
            "tune_trials": len(tuned["trials"]), "cuda_graph": True}


def bench_serving(torch, dist, args):
    """The serving stream: 20k requests, 70% GEMVER n ~ log-U[128, 8192], 30% NS residual grids {256², .., 2048²};
    batched BF16 storage vs the per-request FP32 path; saturation throughput and latency at a Poisson rate."""
    from cospanmdao_b200 import serving
    res = {}
    wl = serving.make_workload(args.requests, rate=None, seed=0)
    srv = serving.Server(wl, budget_bytes=120e9, max_batch=args.max_batch, depth=4)
    srv.run()  # warm-up pass (allocations, first launches)
    # the server is driven from the host: a host stall longer than the queued work (4 batches, ~24 ms) idles the GPU,
    # so each figure is the median run of three, with every run's value listed
    runs = sorted((srv.run() for _ in range(3)), key=lambda r: r["req_per_s"])
    sat = dict(runs[1], runs_req_per_s=[r["req_per_s"] for r in runs])
    sample = [int(i) for i in np.linspace(0, wl.count - 1, 24).astype(int)]
    res["batched_bf16_saturation"] = {k: v for k, v in sat.items()}
    res["same_alone_and_in_mix"] = bool(serving.check_mix(srv, sample))
    res["max_rel_err_vs_f64"] = serving.errors_vs_f64(srv, sample)
    del srv
    torch.cuda.empty_cache()
    pl = serving.plain(wl)
    res["plain_f32_saturation"] = {k: v for k, v in pl.items() if k not in ("out", "norms")}
    res["throughput_ratio_batched_over_plain"] = sat["req_per_s"] / pl["req_per_s"]
    # like for like: the per-request path with the server's storage and bytes (no Â), and a batched FP32 server, so
    # that each ratio below is the batching alone at equal precision and equal bytes
    pl_b16 = serving.plain(wl, dtype=torch.bfloat16, want_B=False)
    pl_f32 = serving.plain(wl, want_B=False)
    srv32 = serving.Server(wl, budget_bytes=120e9, max_batch=args.max_batch, depth=4, dtype=torch.float32)
    srv32.run()  # warm-up pass
    runs32 = sorted((srv32.run() for _ in range(3)), key=lambda r: r["req_per_s"])
    sat32 = dict(runs32[1], runs_req_per_s=[r["req_per_s"] for r in runs32])
    del srv32
    torch.cuda.empty_cache()
    strip = lambda d: {k: v for k, v in d.items() if k not in ("out", "norms")}  # noqa: E731
    res["plain_bf16_noB_saturation"] = strip(pl_b16)
    res["plain_f32_noB_saturation"] = strip(pl_f32)
    res["batched_f32_noB_saturation"] = sat32
    res["like_for_like_ratio"] = {
        "bf16_noB_batched_over_plain": sat["req_per_s"] / pl_b16["req_per_s"],
        "f32_noB_batched_over_plain": sat32["req_per_s"] / pl_f32["req_per_s"],
        "bytes_only_plain_bf16_noB_over_plain_f32_withB": pl_b16["req_per_s"] / pl["req_per_s"]}
    rate = 0.5 * sat["req_per_s"]
    wl2 = serving.make_workload(args.requests, rate=rate, seed=1)
    srv2 = serving.Server(wl2, budget_bytes=120e9, max_batch=args.max_batch, depth=4)
    srv2.run()  # warm-up pass
    runs = sorted((srv2.run() for _ in range(3)), key=lambda r: r["p99_ms"])
    res["batched_bf16_at_rate"] = dict(runs[1], rate_req_per_s=rate, runs_p99_ms=[r["p99_ms"] for r in runs])
    del srv2
    torch.cuda.empty_cache()
    pl2 = serving.plain(wl2)
    res["plain_f32_at_rate"] = dict({k: v for k, v in pl2.items() if k not in ("out", "norms")}, rate_req_per_s=rate)
    return res


def bench_reference_programs(args):
    """The reference's own example programs, unchanged, compiled against this package's cs:: runtime (its fast paths
    run the GEMVER, BiCGK and NS stages as cspb kernels): ms per chain / evaluation at the reference's published sizes,
    beside the reference's own numbers on an RTX 4090 (examples/gemver-chain/README.md:140-174,
    examples/ns-residual/README.md:85-101)."""
    ex = ROOT / "cospanmdao_b200" / "_examples"
    res = {}
    eager = {"NAGA_COSPAN_NO_GRAPH": "1"}  # no CUDA-graph replay of steady forwards
    runs = [("gemver_chain_fused_n16384", ["gemver-chain", "--n", "16384", "--iters", "20", "--warmup", "3",
                                           "--variant", "fused"], "fused", 9.150, {}),
            ("gemver_chain_crafted_n16384", ["gemver-chain", "--n", "16384", "--iters", "20", "--warmup", "3",
                                             "--variant", "crafted"], "crafted", 8.359, {}),
            ("ns_residual_fused_4096", ["ns-residual", "--nx", "4096", "--ny", "4096", "--iters", "20", "--warmup", "3",
                                        "--variant", "fused", "--range-split", "flatten"], "fused-flatten", 5.810, {}),
            ("ns_residual_unfused_4096", ["ns-residual", "--nx", "4096", "--ny", "4096", "--iters", "20", "--warmup",
                                          "3", "--variant", "unfused"], "unfused", 9.685, {})]
    # small sizes, where the reference's per-forward host work dominates: replayed forwards, and eager ones
    for tag, env in (("", {}), ("_eager", eager)):
        runs += [(f"gemver_chain_fused_n2048{tag}", ["gemver-chain", "--n", "2048", "--iters", "200", "--warmup", "3",
                                                    "--variant", "fused"], "fused", 1.582, env),
                 (f"gemver_chain_unfused_n2048{tag}", ["gemver-chain", "--n", "2048", "--iters", "200", "--warmup", "3",
                                                      "--variant", "unfused"], "unfused", 1.925, env),
                 (f"ns_residual_fused_1024{tag}", ["ns-residual", "--nx", "1024", "--ny", "1024", "--iters", "200",
                                                  "--warmup", "3", "--variant", "fused", "--range-split", "flatten"],
                  "fused-flatten", 1.532, env),
                 (f"ns_residual_unfused_1024{tag}", ["ns-residual", "--nx", "1024", "--ny", "1024", "--iters", "200",
                                                    "--warmup", "3", "--variant", "unfused"], "unfused", 3.260, env)]
    for key, cmd, row, ref_ms, env in runs:
        exe = ex / cmd[0]
        if not exe.exists():
            res[key] = {"skipped": f"{exe.name} not built (python -m cospanmdao_b200.examples)"}
            continue
        r = subprocess.run([str(exe), *cmd[1:]], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                           timeout=600, env=dict(os.environ, **env))
        ms = None
        for line in r.stdout.splitlines():
            f = line.split()
            if f and f[0] == row and len(f) > 1:
                try:
                    ms = float(f[1])
                except ValueError:
                    pass
        res[key] = {"ms": ms, "rc": r.returncode, "reference_rtx4090_ms": ref_ms}
    return res


# ---- the CPU path ---------------------------------------------------------------------------------------------
def cpu_gemver(n: int, target_s: float = 2.0, reps: int = 5, warmup: int = 2) -> dict:
    """The reference's unfused GEMVER component loops in f32 (oracle port, OpenMP, every host thread, threads bound to
    cores) on a bounded sample of the n = 16384 workload: a band of rows sized to ~target_s per run, up to the whole
    matrix. The reference's own protocol (examples/run_benchmarks.nu:9-22): warm-up runs, then `reps` timed runs,
    median with min and max. Returns GB/s of the same algorithmic traffic per row."""
    import os
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    import numpy as np
    import oracle
    lib = oracle.restatement()
    A = np.empty(n * n, dtype=np.float32)
    lib.orc_fill_hash(A.ctypes.data_as(__import__("ctypes").c_void_p), n * n, 0, 1, 0)
    vecs = [oracle.hash_fill(n, s, 1) for s in range(2, 8)]
    B = np.zeros(n * n, dtype=np.float32)  # touched here, not inside a timed run
    x = np.empty(n, dtype=np.float32)
    w = np.empty(n, dtype=np.float32)
    P = lambda a: a.ctypes.data_as(__import__("ctypes").c_void_p)  # noqa: E731

    def run(rows):
        t0 = time.perf_counter()
        lib.orc_gemver_f32_unfused(n, 64, P(A), *[P(v) for v in vecs], 1.5, 1.2, P(B), P(x), P(w), 0, rows)
        return time.perf_counter() - t0

    rows = 256
    t = run(rows)
    while t < target_s / 4 and rows < n:
        rows = min(n, rows * 4)
        t = run(rows)
    if t < target_s and rows < n:
        rows = min(n, int(rows * target_s / max(t, 1e-3)) // 64 * 64 or 64)
    for _ in range(max(0, warmup)):
        run(rows)
    times = [run(rows) for _ in range(max(1, reps))]
    tmed = statistics.median(times)
    bytes_ = 12.0 * rows * n + 32.0 * n
    return {"value": bytes_ / tmed / 1e9, "unit": "GB/s", "cores": oracle.threads(), "kind": "port",
            "sample": f"rows 0..{rows} of the n={n} f32 GEMVER (A, Â, Â re-read of those rows); {warmup} warm-up "
                      f"runs, median of {len(times)} timed runs",
            "seconds_per_sample": tmed, "runs": len(times),
            "min_max_gbs": [bytes_ / max(times) / 1e9, bytes_ / min(times) / 1e9],
            "omp": {"OMP_PROC_BIND": os.environ.get("OMP_PROC_BIND"), "OMP_PLACES": os.environ.get("OMP_PLACES")}}


# ---- main -------------------------------------------------------------------------------------------------------
def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_HEAD)
    ap.add_argument("--grid", type=int, default=4096)
    ap.add_argument("--soak", type=float, default=1.0, help="seconds of untimed steps before the timed region")
    ap.add_argument("--quick", action="store_true", help="headline only (no secondary workloads, no CPU baseline)")
    ap.add_argument("--schedule", default="barrier", choices=["panel", "barrier", "bulk"], help="GEMVER schedule")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--lag", type=int, default=0, help="panel-schedule lag (0: automatic)")
    ap.add_argument("--ragged", type=int, default=4096, help="instances of the ragged batch")
    ap.add_argument("--requests", type=int, default=20000, help="requests of the serving stream")
    ap.add_argument("--max-batch", type=int, default=512, help="serving: requests per batch at most")
    ap.add_argument("--scan-log2", type=int, default=28, help="scan: log2 of the items per launch")
    ap.add_argument("--only", default="", help="comma list of secondary workloads to run (gemver_bf16_storage, "
                    "gemver_chain, ns_residual, ragged_batch, scan, serving, reference_programs); default all, none with "
                    "--quick")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)
    dist = Dist()

    config = {"workload": f"fused GEMVER n={args.n} f32 (A {args.n * args.n * 4 / 2**30:.2f} GiB), one launch",
              "n": args.n, "alpha": 1.5, "beta": 1.2, "seed": 0,
              "l2": "inputs larger than L2 (A and Â are 1 GiB each vs 126 MB)",
              "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU"}

    if args.impl == "reference":
        if dist.rank != 0:
            return 0
        # K timed samples of ~1 s each after W warm-up samples (W capped at 3): the run stays within a few minutes
        cpu = cpu_gemver(args.n, target_s=1.0, reps=args.steps, warmup=min(args.warmup, 3))
        line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": "GB/s", "n_gpus": dist.world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": cpu["seconds_per_sample"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded hash generator of the reference example)", "config": config,
                "cpu_baseline": cpu,
                "e2e": {"value": cpu["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference's unfused GEMVER component loops (examples/gemver-chain/components.hpp:85-265) "
                        "restated in C++ with OpenMP; AdaptiveCpp is not available to build the reference itself"}
        print(json.dumps(line))
        return 0

    import torch
    import cospanmdao_b200 as cb
    dist.init(torch)
    cb.lib()
    pk = peaks()
    g = bench_gemver(torch, cb, dist, args, pk)
    total_bytes = g["bytes"] * dist.world
    value = total_bytes / (g["ms"] * 1e-3) / 1e9
    kernel_gbs = g["bytes"] / (g["ms"] * 1e-3) / 1e9  # per launch on one GPU
    traffic = profile_traffic("gemver_f32_n16384.md")
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": g["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded hash generator: A ~ U[-1,1), vectors ~ U[0,1), seed 0)",
        "config": config,
        "roofline": {"bound": "hbm", "achieved": kernel_gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": kernel_gbs / pk["hbm_gbs"], "peak_source": pk["source"],
                     "traffic": traffic, "algorithmic_bytes_per_launch": g["bytes"],
                     "kernel": {"panel": "cspb::k_gemver_panel<float, true>",
                                "bulk": "cspb::k_gemver_bulk<float, true, 6>"}.get(args.schedule,
                                                                                  "cspb::k_gemver<float, true>")},
        "e2e": g["e2e"],
        "gpu_launches": args.steps,
        "clocks": g["clocks"],
        "err_vs_f64": g["err"],
    }
    secondaries = {
        "gemver_bf16_storage": lambda: bench_gemver_bf16(torch, cb, dist, args),
        "gemver_chain": lambda: bench_chain(torch, cb, dist, args),
        "gemver_sharded": lambda: bench_sharded(torch, cb, dist, args),
        "ns_sharded": lambda: bench_ns_sharded(torch, cb, dist, args),
        "ns_residual": lambda: bench_ns(torch, cb, dist, args),
        "ragged_batch": lambda: bench_ragged(torch, cb, dist, args, pk),
        "scan": lambda: bench_scan(torch, cb, dist, args, pk),
        "serving": lambda: bench_serving(torch, dist, args),
        "reference_programs": lambda: bench_reference_programs(args),
    }
    wanted = [w for w in args.only.split(",") if w] or ([] if args.quick else list(secondaries))
    unknown = [w for w in wanted if w not in secondaries]
    if unknown:
        raise SystemExit(f"bench.py: unknown workload(s) {unknown}; choose from {list(secondaries)}")
    if wanted:
        line["secondary"] = {w: secondaries[w]() for w in wanted}
    if dist.rank == 0 and not args.quick:
        line["cpu_baseline"] = cpu_gemver(args.n)
    if dist.rank == 0:
        print(json.dumps(line))
    dist.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
