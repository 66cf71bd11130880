"""Seeded synthetic inputs of the benchmark configurations, generated on the device.

GEMVER (matrix A ~ U[-1, 1), vectors ~ U[0, 1), seed s): every array is the reference's hash generator
(examples/gemver-chain/common/chain_data.hpp:34-49) on its own stream, seed 16·s + id with id A=1, u1=2, v1=3, u2=4,
v2=5, y=6, z=7 (the reference's own seeds when s = 0). dist 'reference' reproduces the reference example's inputs
(every array hash_unit in [-1, 1), seeds 1..7).

Incompressible NS fields (u, v, p on an N×N periodic grid, h = 2π/N): per field the sum of 16 Fourier modes
a·cos(kx·x + ky·y + φ) with integer (kx, ky), 1 <= |k| <= 8, a ~ N(0, 1)/|k|², φ ~ U[0, 2π) — drawn with numpy's PCG64
from the seed, so the mode table is reproducible anywhere — evaluated in f64, plus 1e-3·U[-1, 1) noise from the hash
generator (seed 16·s + 8/9/10), rounded once to the storage dtype.

Ragged batch sizes: n_k = round(64 · 64^U_k), U_k = the hash generator in [0, 1) on seed 16·s + 11, so n is
log-uniform in [64, 4096].
"""
from __future__ import annotations

import math

import numpy as np

GEMVER_SEEDS = {"A": 1, "u1": 2, "v1": 3, "u2": 4, "v2": 5, "y": 6, "z": 7}
VECTORS = ("u1", "v1", "u2", "v2", "y", "z")


def _torch():
    import torch
    return torch


def gemver_inputs(n: int, seed: int = 0, *, dtype=None, dist: str = "config", device="cuda") -> dict:
    """A (n×n, dtype float32 or bfloat16) and the six f32 vectors, generated on the device."""
    import cospanmdao_b200 as cb
    torch = _torch()
    dtype = dtype or torch.float32
    out = {}
    for k, sid in GEMVER_SEEDS.items():
        shape = (n, n) if k == "A" else (n,)
        t = torch.empty(shape, dtype=dtype if k == "A" else torch.float32, device=device)
        s = sid if dist == "reference" else 16 * seed + sid
        d = 0 if (dist == "reference" or k == "A") else 1
        cb.fill_hash(t, s, d)
        out[k] = t
    return out


def ns_modes(seed: int = 0, modes: int = 16, kmax: int = 8):
    """The mode table {field: (kx, ky, amp, phase)} of the incompressible NS inputs."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cand = [(kx, ky) for kx in range(-kmax, kmax + 1) for ky in range(-kmax, kmax + 1)
            if 1 <= math.hypot(kx, ky) <= kmax]
    table = {}
    for f in ("u", "v", "p"):
        pick = rng.integers(0, len(cand), size=modes)
        k = np.array([cand[i] for i in pick], dtype=np.float64)
        kk = np.hypot(k[:, 0], k[:, 1])
        amp = rng.standard_normal(modes) / kk ** 2
        phase = rng.uniform(0.0, 2.0 * math.pi, size=modes)
        table[f] = (k[:, 0], k[:, 1], amp, phase)
    return table


def ns_fields(N: int, seed: int = 0, *, dtype=None, device="cuda", noise: float = 1e-3):
    """u, v, p (N×N) on the device, evaluated in f64 and rounded once. Returns (u, v, p, h)."""
    import cospanmdao_b200 as cb
    torch = _torch()
    dtype = dtype or torch.float32
    h = 2.0 * math.pi / N
    table = ns_modes(seed)
    x = torch.arange(N, dtype=torch.float64, device=device) * h
    out = []
    for idx, f in enumerate(("u", "v", "p")):
        kx, ky, amp, ph = table[f]
        acc = torch.zeros((N, N), dtype=torch.float64, device=device)
        for m in range(len(amp)):
            # row j is y = j·h, column i is x = i·h
            acc += float(amp[m]) * torch.cos(float(kx[m]) * x[None, :] + float(ky[m]) * x[:, None] + float(ph[m]))
        nz = torch.empty((N, N), dtype=torch.float32, device=device)
        cb.fill_hash(nz, 16 * seed + 8 + idx, 0)
        acc += noise * nz.double()
        out.append(acc.to(dtype))
        del acc
    return out[0], out[1], out[2], h


def _mix32(x: np.ndarray) -> np.ndarray:
    x = x ^ (x >> np.uint32(16))
    x = x * np.uint32(0x7FEB352D)
    x = x ^ (x >> np.uint32(15))
    x = x * np.uint32(0x846CA68B)
    return x ^ (x >> np.uint32(16))


def hash_unit01(seed: int, index: np.ndarray) -> np.ndarray:
    """The hash generator's [0, 1) value h·2^-24 on the host (numpy, bit-identical to the device generator)."""
    idx = np.asarray(index, dtype=np.uint64)
    lo = (idx & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    hi = (idx >> np.uint64(32)).astype(np.uint32)
    s = np.uint32(seed & 0xFFFFFFFF)
    with np.errstate(over="ignore"):
        a = _mix32(np.full(idx.shape, s * np.uint32(0x9E3779B9) + np.uint32(0x85EBCA6B), dtype=np.uint32))
        b = _mix32(lo + _mix32(hi + s))
        h = _mix32(a ^ b) >> np.uint32(8)
    return h.astype(np.float32) * np.float32(1.0 / 16777216.0)


def ragged_sizes(count: int, seed: int = 0, lo: int = 64, hi: int = 4096) -> np.ndarray:
    """n_k = round(lo · (hi/lo)^U_k), U_k ~ U[0, 1) from the hash generator: log-uniform sizes (u32)."""
    u = hash_unit01(16 * seed + 11, np.arange(count, dtype=np.uint64)).astype(np.float64)
    n = np.rint(lo * (hi / lo) ** u).astype(np.int64)
    return np.clip(n, lo, hi).astype(np.uint32)
