"""TEST INFRASTRUCTURE ONLY — the CPU oracle of the cspb kernels.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this package, as a checker or a timed
baseline; the product (cospanmdao_b200) never does.

  restatement()  liboracle.so   — cspb_oracle.cpp, this repository's restatement of the reference's algorithms
  reference()    _ref/libref.so — the reference's own plain-C++ oracles (gemver_chain::reference_chain,
                                   nsr::reference_residual) compiled in place from the reference tree; None when it was
                                   never built (the reference tree is only present where the library is built)
Both are built by `make -C oracle` (build() below).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libref.so"

_P = C.c_void_p
_I64 = C.c_int64
_I = C.c_int
_D = C.c_double
_F = C.c_float


def build(reference_dir: str | None = None) -> None:
    env = dict(os.environ)
    if reference_dir:
        env["REFERENCE_DIR"] = reference_dir
    r = subprocess.run(["make", "-s", "-C", str(HERE)], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout)


_orc = None
_ref = None


def restatement() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            build()
        h = C.CDLL(str(ORACLE_SO))
        h.orc_fill_hash.argtypes = [_P, _I64, C.c_uint64, C.c_uint32, _I]
        h.orc_gemver_f64.argtypes = [_I64, _I64, _P, _P, _P, _P, _P, _P, _P, _D, _D, _P, _P, _P]
        h.orc_bicgk_f64.argtypes = [_I64, _I64, _P, _P, _P, _P, _P]
        h.orc_chain_f64.argtypes = [_I64] + [_P] * 11 + [_D, _D] + [_P] * 7
        h.orc_gemver_f32_unfused.argtypes = [_I64, _I64] + [_P] * 7 + [_F, _F, _P, _P, _P, _I64, _I64]
        h.orc_ns_comp_f64.argtypes = [_I, _I, _I, _I, _P, _P, _P]
        h.orc_ns_comp_f32.argtypes = [_I, _I, _I, _I, _P, _P, _P]
        h.orc_ns_init_cons.argtypes = [_I, _I, _F, _P]
        h.orc_ns_incomp_f64.argtypes = [_I, _I, _D, _D, _P, _P, _P, _P, _P, _P, _P]
        h.orc_exclusive_scan_u32.argtypes = [_P, _P, _I64]
        h.orc_exclusive_scan_u64.argtypes = [_P, _P, _I64]
        h.orc_build_column.argtypes = [_P, _I, _I64, _I64, _I, _P, _P, _P]
        h.orc_threads.restype = _I
        _orc = h
    return _orc


def reference() -> C.CDLL | None:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        h = C.CDLL(str(REF_SO))
        h.ref_hash_unit.restype = _F
        h.ref_hash_unit.argtypes = [C.c_uint32, C.c_uint64]
        h.ref_make_matrix_A0.argtypes = [_I64, _P]
        h.ref_make_vectors.argtypes = [_I64, _P]
        h.ref_reference_chain.argtypes = [_I64, _P, _P]
        h.ref_relative_l2.restype = _D
        h.ref_relative_l2.argtypes = [_P, _P, _I64]
        h.ref_init_cons.argtypes = [_I, _I, _F, _P]
        h.ref_reference_residual.argtypes = [_I, _I, _I, _I, _P, _P, _P]
        _ref = h
    return _ref


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---- numpy conveniences ------------------------------------------------------------------------------------------
def hash_fill(count: int, seed: int, dist: int = 0, base: int = 0) -> np.ndarray:
    out = np.empty(count, dtype=np.float32)
    restatement().orc_fill_hash(_p(out), count, base, seed, dist)
    return out


def gemver_inputs(n: int, seed: int = 0, dist: str = "config") -> dict:
    """Seeded GEMVER inputs. dist 'config': A ~ U[-1,1), vectors ~ U[0,1) from stream seeds 16·seed + id;
    dist 'reference': the reference example's own inputs (every array hash_unit in [-1,1), seeds 1..7)."""
    ids = {"A": 1, "u1": 2, "v1": 3, "u2": 4, "v2": 5, "y": 6, "z": 7}
    out = {}
    for k, i in ids.items():
        if dist == "reference":
            out[k] = hash_fill(n * n if k == "A" else n, i, 0)
        else:
            out[k] = hash_fill(n * n if k == "A" else n, 16 * seed + i, 0 if k == "A" else 1)
    out["A"] = out["A"].reshape(n, n)
    return out


def gemver_f64(n, A, u1, v1, u2, v2, y, z, alpha, beta, want_B=False):
    A = np.ascontiguousarray(A, dtype=np.float32)
    x = np.empty(n)
    w = np.empty(n)
    B = np.empty((n, n)) if want_B else None
    restatement().orc_gemver_f64(n, A.shape[1], _p(A), _p(u1), _p(v1), _p(u2), _p(v2), _p(y), _p(z), alpha, beta,
                                 _p(x), _p(w), _p(B))
    return x, w, B


def bicgk_f64(B, p, r):
    B = np.ascontiguousarray(B, dtype=np.float32)
    n = B.shape[0]
    q = np.empty(n)
    s = np.empty(n)
    restatement().orc_bicgk_f64(n, B.shape[1], _p(B), _p(p), _p(r), _p(q), _p(s))
    return q, s


def chain_f64(A0, a: dict, b: dict, alpha, beta, want_B2=False):
    n = A0.shape[0]
    outs = {k: np.empty(n) for k in ("x1", "w1", "q", "s", "x2", "w2")}
    B2 = np.empty((n, n)) if want_B2 else None
    restatement().orc_chain_f64(n, _p(A0), _p(a["u1"]), _p(a["v1"]), _p(a["u2"]), _p(a["v2"]), _p(a["y"]),
                                _p(a.get("z")), _p(b["u1"]), _p(b["v1"]), _p(b["u2"]), _p(b["v2"]), alpha, beta,
                                *[_p(outs[k]) for k in ("x1", "w1", "q", "s", "x2", "w2")], _p(B2))
    if want_B2:
        outs["B2"] = B2
    return outs


def ns_comp_f64(U: np.ndarray, walls: bool, limiter: int):
    _, ny, nx = U.shape
    R = np.empty((4, ny, nx))
    d = np.empty(6)
    restatement().orc_ns_comp_f64(nx, ny, int(walls), limiter, _p(np.ascontiguousarray(U, np.float32)), _p(R), _p(d))
    return R, d


def ns_comp_f32(U: np.ndarray, walls: bool, limiter: int):
    _, ny, nx = U.shape
    R = np.empty((4, ny, nx), dtype=np.float32)
    d = np.empty(6)
    restatement().orc_ns_comp_f32(nx, ny, int(walls), limiter, _p(np.ascontiguousarray(U, np.float32)), _p(R), _p(d))
    return R, d


def ns_init(nx: int, ny: int, amp: float) -> np.ndarray:
    U = np.empty((4, ny, nx), dtype=np.float32)
    restatement().orc_ns_init_cons(nx, ny, amp, _p(U))
    return U


def ns_incomp_f64(u, v, p, h, nu, want_fields=True):
    ny, nx = u.shape
    outs = [np.empty((ny, nx)) for _ in range(3)] if want_fields else [None] * 3
    norms = np.empty(3)
    restatement().orc_ns_incomp_f64(nx, ny, h, nu, *[_p(np.ascontiguousarray(a, np.float32)) for a in (u, v, p)],
                                    *[_p(o) for o in outs], _p(norms))
    return outs[0], outs[1], outs[2], norms


def exclusive_scan(values: np.ndarray) -> np.ndarray:
    n = values.shape[0]
    if values.dtype == np.uint32:
        out = np.empty(n + 1, dtype=np.uint32)
        restatement().orc_exclusive_scan_u32(_p(values), _p(out), n)
    else:
        values = values.astype(np.uint64)
        out = np.empty(n + 1, dtype=np.uint64)
        restatement().orc_exclusive_scan_u64(_p(values), _p(out), n)
    return out


_DT = {np.dtype(np.int32): 0, np.dtype(np.uint32): 1, np.dtype(np.int64): 2, np.dtype(np.uint64): 3}


def build_column(src: np.ndarray, offsets_mode: bool = False):
    src = np.ascontiguousarray(src)
    count = src.shape[0]
    k = src.shape[1] if src.ndim == 2 else 1
    n = count - 1 if offsets_mode else count
    ext = np.zeros(max(n, 0), dtype=np.uint32)
    offs = np.zeros(n + 1, dtype=np.uint32)
    tf = np.zeros(2, dtype=np.uint32)
    restatement().orc_build_column(_p(src), _DT[src.dtype], count, k, int(offsets_mode), _p(ext), _p(offs), _p(tf))
    return ext, offs, int(tf[0]), int(tf[1])


def threads() -> int:
    return int(restatement().orc_threads())


# ---- the reference's own oracles ---------------------------------------------------------------------------------
def ref_chain(n: int, want_B2: bool = False):
    r = reference()
    if r is None:
        return None
    out = np.empty(6 * n)
    B2 = np.empty(n * n) if want_B2 else None
    r.ref_reference_chain(n, _p(out), _p(B2))
    d = dict(zip(("x1", "w1", "q", "s", "x2", "w2"), out.reshape(6, n)))
    if want_B2:
        d["B2"] = B2.reshape(n, n)
    return d


def ref_inputs(n: int):
    r = reference()
    if r is None:
        return None
    A = np.empty(n * n, dtype=np.float32)
    v = np.empty(6 * n, dtype=np.float32)
    r.ref_make_matrix_A0(n, _p(A))
    r.ref_make_vectors(n, _p(v))
    d = dict(zip(("u1", "v1", "u2", "v2", "y", "z"), v.reshape(6, n)))
    d["A"] = A.reshape(n, n)
    return d


def ref_residual(U: np.ndarray, walls: bool, limiter: int):
    r = reference()
    if r is None:
        return None
    _, ny, nx = U.shape
    R = np.empty((4, ny, nx))
    d = np.empty(6)
    r.ref_reference_residual(nx, ny, int(walls), limiter, _p(np.ascontiguousarray(U, np.float32)), _p(R), _p(d))
    return R, d


def ref_init(nx: int, ny: int, amp: float):
    r = reference()
    if r is None:
        return None
    U = np.empty((4, ny, nx), dtype=np.float32)
    r.ref_init_cons(nx, ny, amp, _p(U))
    return U


def rel_l2(got, want) -> float:
    got = np.asarray(got, dtype=np.float64).ravel()
    want = np.asarray(want, dtype=np.float64).ravel()
    num = float(np.sum((got - want) ** 2))
    den = float(np.sum(want ** 2))
    if np.isnan(num):
        return float("inf")
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return (num / den) ** 0.5
