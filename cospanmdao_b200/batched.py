"""Ragged batches of independent GEMVERs in one launch (cspb_gemver_batched), and the autotuner of their tiles.

A RaggedBatch owns the packed device arrays of a batch: instance k's matrix at element a_off[k] with row stride
ld_k = n_k rounded up to 8, its vectors at v_off[k]. The offsets are computed by the kernel call itself (device
decoupled-lookback scans); the host computes the same offsets with numpy only to size the arrays and to slice
instance views, and `offsets_match()` checks the two bit for bit.

The tile geometry of an instance is chosen per size bucket (n < 512, < 1024, < 2048, >= 2048) by a 2-bit code in the
tuning word; `autotune()` picks the codes by coordinate descent over the buckets on the actual batch, device-timed,
and caches them per (device name, dtype) in a JSON file (CSPB_TUNE_CACHE, default ~/.cache/cospanmdao_b200/tune.json).
Because the geometry is a function of (n, dtype, tuning) only, an instance's result never depends on the rest of
the batch.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import threading
from pathlib import Path

import numpy as np

from . import _capi
from ._capi import BF16, F32, lib

BUCKETS = (512, 1024, 2048)
CODES = (0, 1, 2)  # 8 warps as 2×4, 1×8, 4×2


def _torch():
    import torch
    return torch


def layout(sizes: np.ndarray):
    """Host copy of the packed layout: (ld, a_off, v_off) as numpy uint64 (count + 1 offsets)."""
    n = np.asarray(sizes, dtype=np.uint64)
    ld = (n + np.uint64(7)) // np.uint64(8) * np.uint64(8)
    a_off = np.concatenate([[0], np.cumsum(n * ld, dtype=np.uint64)]).astype(np.uint64)
    v_off = np.concatenate([[0], np.cumsum(n, dtype=np.uint64)]).astype(np.uint64)
    return ld, a_off, v_off


class RaggedBatch:
    """Packed device storage of a batch of GEMVERs of sizes `sizes`."""

    def __init__(self, sizes, *, dtype=None, want_B: bool = True, device=None):
        torch = _torch()
        self.sizes = np.asarray(sizes, dtype=np.uint32)
        if self.sizes.ndim != 1 or self.sizes.size == 0:
            raise ValueError("a ragged batch needs at least one instance")
        if self.sizes.min() < 1 or self.sizes.max() > 65536:
            raise ValueError("every instance size must be in [1, 65536]")
        self.dtype = dtype or torch.float32
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.count = int(self.sizes.size)
        self.ld, self.a_off_h, self.v_off_h = layout(self.sizes)
        self.max_elems = int(self.a_off_h[-1])
        self.max_vec = int(self.v_off_h[-1])
        dev = self.device
        self.n = torch.from_numpy(self.sizes.view(np.int32).copy()).to(dev)
        self.A = torch.empty(self.max_elems, dtype=self.dtype, device=dev)
        self.B = torch.empty(self.max_elems, dtype=torch.float32, device=dev) if want_B else None
        self.vec = {k: torch.empty(self.max_vec, dtype=torch.float32, device=dev)
                    for k in ("u1", "v1", "u2", "v2", "y", "z")}
        self.x = torch.empty(self.max_vec, dtype=torch.float32, device=dev)
        self.w = torch.empty(self.max_vec, dtype=torch.float32, device=dev)
        self.alpha = torch.empty(self.count, dtype=torch.float32, device=dev)
        self.beta = torch.empty(self.count, dtype=torch.float32, device=dev)
        self.a_off = torch.zeros(self.count + 1, dtype=torch.int64, device=dev)
        self.v_off = torch.zeros(self.count + 1, dtype=torch.int64, device=dev)
        self.ws_bytes = int(lib().cspb_gemver_batched_workspace_bytes(self.count, self.max_elems, self.max_vec))
        self.ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=dev)

    # ---- data ----------------------------------------------------------------------------------------------------
    def fill(self, seed: int = 0, alpha: float = 1.5, beta: float = 1.2):
        """Seeded inputs: A ~ U[-1, 1) and vectors ~ U[0, 1) from the hash generator over the packed index."""
        import cospanmdao_b200 as cb
        cb.fill_hash(self.A, 16 * seed + 1, 0)
        for sid, k in enumerate(("u1", "v1", "u2", "v2", "y", "z"), start=2):
            cb.fill_hash(self.vec[k], 16 * seed + sid, 1)
        self.alpha.fill_(alpha)
        self.beta.fill_(beta)
        return self

    def instance(self, k: int) -> dict:
        """Views of instance k: A and B as (n, n) with row stride ld, and its vectors."""
        n, ld = int(self.sizes[k]), int(self.ld[k])
        ao, vo = int(self.a_off_h[k]), int(self.v_off_h[k])
        out = {"n": n, "A": self.A[ao:ao + n * ld].view(n, ld)[:, :n]}
        if self.B is not None:
            out["B"] = self.B[ao:ao + n * ld].view(n, ld)[:, :n]
        for key, t in self.vec.items():
            out[key] = t[vo:vo + n]
        out["x"] = self.x[vo:vo + n]
        out["w"] = self.w[vo:vo + n]
        out["alpha"] = float(self.alpha[k])
        out["beta"] = float(self.beta[k])
        return out

    # ---- the launch ------------------------------------------------------------------------------------------------
    def run(self, tune: int = 0, stream=None, check: bool = False, lowrank: bool | None = None):
        """One launch over the batch. lowrank: instances without B take the low-rank form (the rank-2 update as dot
        products; with B only w of a bf16 batch); None follows cb.gemver's 'auto' schedule (bf16)."""
        import cospanmdao_b200 as cb
        torch = _torch()
        if lowrank is None:
            lowrank = self.dtype == torch.bfloat16
        tune = int(tune) | (_capi.BATCH_LOWRANK if lowrank else 0)
        p = int(self.ws.data_ptr())
        wp = (p + 255) // 256 * 256
        d = _capi.BatchedDesc(self.count, self.max_elems, self.max_vec, BF16 if self.dtype == torch.bfloat16 else F32,
                              int(tune), int(self.n.data_ptr()), int(self.A.data_ptr()),
                              *[int(self.vec[k].data_ptr()) for k in ("u1", "v1", "u2", "v2", "y", "z")],
                              int(self.alpha.data_ptr()), int(self.beta.data_ptr()),
                              int(self.B.data_ptr()) if self.B is not None else None, int(self.x.data_ptr()),
                              int(self.w.data_ptr()), int(self.a_off.data_ptr()), int(self.v_off.data_ptr()), wp,
                              self.ws_bytes)
        s = stream if stream is not None else torch.cuda.current_stream()
        cb._raise(lib().cspb_gemver_batched(C.byref(d), C.c_void_p(int(s.cuda_stream))), "gemver-batched")
        if check:
            raw = _capi.u32(0)
            st = lib().cspb_read_status(C.c_void_p(wp), C.byref(raw), C.c_void_p(int(s.cuda_stream)))
            cb._raise(st, "gemver-batched (device)")
        return self

    def offsets_match(self) -> bool:
        """The device-scanned offsets equal the host's, bit for bit."""
        return (np.array_equal(self.a_off.cpu().numpy().view(np.uint64), self.a_off_h)
                and np.array_equal(self.v_off.cpu().numpy().view(np.uint64), self.v_off_h))

    def algorithmic_bytes(self) -> float:
        """Matrix read, Â written (when kept), matrix read again, vectors: per batch step."""
        a = 2 if self.dtype == _torch().bfloat16 else 4
        n2 = float((self.sizes.astype(np.float64) ** 2).sum())
        second = a if (self.B is None or a == 2) else 4
        return n2 * (a + (4 if self.B is not None else 0) + second) + 32.0 * float(self.sizes.astype(np.float64).sum())


def gemver_batched(sizes, *, seed: int = 0, dtype=None, want_B: bool = True, tune: int | None = None):
    """Convenience: build, fill and run one batch. Returns the RaggedBatch."""
    b = RaggedBatch(sizes, dtype=dtype, want_B=want_B).fill(seed)
    return b.run(tune=choose_tune(b) if tune is None else tune)


# ---- the autotuner --------------------------------------------------------------------------------------------------
GROUPS = (0, 1, 2, 3)  # work items per grab: 4, 1, 2, 8
BLOCKS = (0, 1, 2, 3)  # blocks per SM: as many as fit, one fewer, two, one


def tune_word(codes, group: int = 0, blocks: int = 0) -> int:
    """The tuning word: 2 bits of tile geometry per size bucket, then the grab-group and blocks-per-SM codes."""
    w = int(sum((int(c) & 3) << (2 * b) for b, c in enumerate(codes)))
    return w | ((int(group) & 3) << 8) | ((int(blocks) & 3) << 10)


def _cache_path() -> Path:
    p = os.environ.get("CSPB_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "cospanmdao_b200" / "tune.json"


_cache_lock = threading.Lock()


def _cache_key(batch: RaggedBatch) -> str:
    torch = _torch()
    name = torch.cuda.get_device_name(batch.device).replace(" ", "_")
    return f"{name}:{'bf16' if batch.dtype == torch.bfloat16 else 'f32'}:{'B' if batch.B is not None else 'noB'}"


def choose_tune(batch: RaggedBatch) -> int:
    """The cached tuning word for this batch's (device, dtype), 0 when none is cached."""
    with _cache_lock:
        p = _cache_path()
        if p.exists():
            try:
                return int(json.loads(p.read_text()).get(_cache_key(batch), {}).get("tune", 0))
            except (ValueError, OSError):
                return 0
    return 0


def _time_ms(batch: RaggedBatch, tune: int, reps: int) -> float:
    torch = _torch()
    batch.run(tune=tune)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        batch.run(tune=tune)
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(batch: RaggedBatch, reps: int = 3, save: bool = True) -> dict:
    """Coordinate descent, device-timed on `batch`, over the four size buckets' geometry codes, then the work items a
    block takes per grab, then the blocks per SM. Returns {'tune': word, 'codes': [...], 'group': g, 'blocks': b,
    'ms': best, 'trials': [...]} and caches it."""
    codes = [0, 0, 0, 0]
    group = blocks = 0
    present = set(int(np.searchsorted(BUCKETS, n, side="right")) for n in batch.sizes)
    best = _time_ms(batch, tune_word(codes), reps)
    trials = [(tune_word(codes), best)]
    for b in range(4):
        if b not in present:
            continue
        for c in CODES:
            if c == codes[b]:
                continue
            trial = list(codes)
            trial[b] = c
            ms = _time_ms(batch, tune_word(trial), reps)
            trials.append((tune_word(trial), ms))
            if ms < best:
                best, codes = ms, trial
    for g in GROUPS:
        if g == group:
            continue
        ms = _time_ms(batch, tune_word(codes, g, blocks), reps)
        trials.append((tune_word(codes, g, blocks), ms))
        if ms < best:
            best, group = ms, g
    for k in BLOCKS:
        if k == blocks:
            continue
        ms = _time_ms(batch, tune_word(codes, group, k), reps)
        trials.append((tune_word(codes, group, k), ms))
        if ms < best:
            best, blocks = ms, k
    res = {"tune": tune_word(codes, group, blocks), "codes": codes, "group": group, "blocks": blocks, "ms": best,
           "trials": trials}
    if save:
        with _cache_lock:
            p = _cache_path()
            p.parent.mkdir(parents=True, exist_ok=True)
            data = {}
            if p.exists():
                try:
                    data = json.loads(p.read_text())
                except ValueError:
                    data = {}
            data[_cache_key(batch)] = {"tune": res["tune"], "codes": codes, "group": group, "blocks": blocks,
                                       "ms": best}
            p.write_text(json.dumps(data, indent=1))
    return res
