"""cospanmdao_b200 — the B200 (sm_100a) backend of CoSpan's fused component chains.

The kernels live in libcspb.so behind the C ABI of include/cspb.h. This module is the Python view of that ABI for
tests, the benchmark and the serving loop: each function takes torch tensors that are already on the GPU, checks them
the way the reference's components check their ports, and launches on torch's current stream. Nothing here computes
on the CPU: when the library is missing every call raises (``LibraryMissing``).

Errors follow the reference: an argument the reference would reject with std::invalid_argument raises ValueError with
the offending port named; a device-side failure (a bounded wait that gave up) raises RuntimeError.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
from typing import Optional, Sequence

from . import _capi
from ._capi import BF16, F32, LibraryMissing, lib

__all__ = [
    "LibraryMissing", "lib", "version", "Workspace", "gemver", "bicgk", "gemver_chain", "gemver_batched",
    "ns_incompressible", "ns_compressible", "ns_init_cons", "exclusive_scan", "build_column", "fill_hash",
    "read_status", "CspbError", "DeviceTimeout",
]


class CspbError(RuntimeError):
    """A CUDA-side failure reported by libcspb."""


class DeviceTimeout(CspbError):
    """A bounded device-side wait gave up (outputs of that call are not valid)."""


def _torch():
    import torch  # deferred: importing the package must not need a GPU
    return torch


def version() -> str:
    return lib().cspb_version().decode()


def _raise(status: int, what: str) -> None:
    if status == _capi.OK:
        return
    msg = f"{what}: {lib().cspb_status_string(status).decode()}"
    if status in (_capi.ERR_ARGUMENT, _capi.ERR_UNSUPPORTED, _capi.ERR_WORKSPACE, _capi.ERR_NEGATIVE,
                  _capi.ERR_EXCEEDS32, _capi.ERR_CAPACITY, _capi.ERR_TOO_LARGE):
        raise ValueError(msg)
    if status == _capi.ERR_TIMEOUT:
        raise DeviceTimeout(msg)
    raise CspbError(msg)


def _stream(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _ptr(t) -> Optional[int]:
    return None if t is None else int(t.data_ptr())


class Workspace:
    """A growable device workspace (uint8), reused across calls on one stream. Calls that share one must be ordered
    on one stream; the default workspaces are per (device, stream)."""

    def __init__(self, device=None):
        self.device = device
        self.buf = None

    def get(self, nbytes: int):
        torch = _torch()
        need = max(int(nbytes), 256)
        if self.buf is None or self.buf.numel() < need:
            self.buf = torch.empty(need + 255, dtype=torch.uint8, device=self.device)
        return self.buf

    def ptr(self, nbytes: int) -> tuple[int, int]:
        b = self.get(nbytes)
        p = int(b.data_ptr())
        aligned = (p + 255) // 256 * 256
        return aligned, b.numel() - (aligned - p)


_ws_lock = threading.Lock()
_default_ws: dict = {}


def default_workspace(device=None, stream=None) -> Workspace:
    torch = _torch()
    dev = torch.device(device) if device is not None else torch.device("cuda")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    key = (dev.index, _stream(stream))
    with _ws_lock:
        ws = _default_ws.get(key)
        if ws is None:
            ws = _default_ws[key] = Workspace(dev)
        return ws


def read_status(ws: Workspace, stream=None) -> int:
    """Synchronizes the stream and returns the CSPB_ERR_* code held in the workspace's device status word."""
    raw = _capi.u32(0)
    p, _ = ws.ptr(256)
    return lib().cspb_read_status(C.c_void_p(p), C.byref(raw), C.c_void_p(_stream(stream)))


# ---- port checks, in the reference's words ---------------------------------------------------------------------
def _need(t, name: str, shape: Sequence[int] | None = None, dtypes=None, contiguous=True):
    torch = _torch()
    if t is None:
        raise ValueError(f"'{name}' is not set")
    if not t.is_cuda:
        raise ValueError(f"'{name}' must be a CUDA tensor")
    if dtypes is not None and t.dtype not in dtypes:
        raise ValueError(f"'{name}' has dtype {t.dtype}, expected one of {list(dtypes)}")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"'{name}' has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if contiguous and not t.is_contiguous():
        raise ValueError(f"'{name}' must be contiguous")
    return t


def _f32(t, name, n):
    torch = _torch()
    return _need(t, name, (n,), (torch.float32,))


def _mat_dtype(t):
    torch = _torch()
    if t.dtype == torch.float32:
        return F32
    if t.dtype == torch.bfloat16:
        return BF16
    raise ValueError(f"matrix dtype {t.dtype} is not float32 or bfloat16")


# ---- GEMVER family ------------------------------------------------------------------------------------------------
def gemver(A, u1, v1, u2, v2, y, z=None, *, alpha: float, beta: float, want_B: bool = True, B=None, x=None, w=None,
           schedule: str = "auto", lag: int = 0, workspace: Workspace | None = None, stream=None):
    """Â = A + u1·v1ᵀ + u2·v2ᵀ, x = β·Âᵀy + z, w = α·Â·x in one launch. A: (n, n) float32 or bfloat16 (a row
    stride from A.stride(0) is honoured). schedule 'barrier' (three streaming passes), 'bulk' (the same passes fed
    through a shared-memory ring by bulk copies; used when n is a multiple of 4 (f32) / 8 (bf16) and the operands are
    16-byte aligned, else 'barrier') or 'panel' (column panels pipelined through L2) all give the same bits.
    'lowrank' applies the rank-2 update as four dot products: without Â both passes over A are plain GEMVs; with Â
    and a bfloat16 matrix only w does (pass 2 re-reads A); with Â and a float32 matrix it is 'barrier'. Other rounding,
    within the f64 tolerance. 'auto' (the default) is 'lowrank' for a bfloat16 matrix and 'barrier' otherwise.
    Returns (B or None, x, w)."""
    if schedule not in ("auto", "panel", "barrier", "bulk", "lowrank"):
        raise ValueError("schedule must be 'auto', 'barrier', 'bulk', 'panel' or 'lowrank'")
    torch = _torch()
    if A is None or A.dim() != 2 or A.shape[0] != A.shape[1]:
        raise ValueError("'A' must be a square matrix")
    n = A.shape[0]
    if A.stride(1) != 1:
        raise ValueError("'A' rows must be contiguous")
    _need(A, "A", None, (torch.float32, torch.bfloat16), contiguous=False)
    for t, nm in ((u1, "u1"), (v1, "v1"), (u2, "u2"), (v2, "v2"), (y, "y")):
        _f32(t, nm, n)
    if z is not None:
        _f32(z, "z", n)
    dev = A.device
    if want_B and B is None:
        B = torch.empty((n, n), dtype=torch.float32, device=dev)
    if B is not None:
        _need(B, "B", None, (torch.float32,), contiguous=False)
        if tuple(B.shape) != (n, n) or B.stride(1) != 1:
            raise ValueError("'B' must be (n, n) with contiguous rows")
    x = torch.empty(n, dtype=torch.float32, device=dev) if x is None else _f32(x, "x", n)
    w = torch.empty(n, dtype=torch.float32, device=dev) if w is None else _f32(w, "w", n)
    ws = workspace or default_workspace(dev, stream)
    need = lib().cspb_gemver_workspace_bytes(n)
    wp, wb = ws.ptr(need)
    if not 0 <= int(lag) <= 255:
        raise ValueError("lag must be in [0, 255]")
    if schedule == "auto":
        schedule = "lowrank" if A.dtype == torch.bfloat16 else "barrier"
    flags = {"panel": _capi.GEMVER_PANEL, "bulk": _capi.GEMVER_BULK,
             "lowrank": _capi.GEMVER_LOWRANK}.get(schedule, 0) | (int(lag) << 8)
    d = _capi.GemverDesc(n, A.stride(0), B.stride(0) if B is not None else n, _mat_dtype(A), flags, _ptr(A), _ptr(u1),
                         _ptr(v1), _ptr(u2), _ptr(v2), _ptr(y), _ptr(z), float(alpha), float(beta), _ptr(B), _ptr(x),
                         _ptr(w), wp, wb)
    _raise(lib().cspb_gemver_fused(C.byref(d), C.c_void_p(_stream(stream))), "gemver")
    return B, x, w


def bicgk(B, p, r, *, q=None, s=None, workspace: Workspace | None = None, stream=None):
    """q = B·p, s = Bᵀ·r in one pass over B. Returns (q, s)."""
    torch = _torch()
    if B is None or B.dim() != 2 or B.shape[0] != B.shape[1] or B.stride(1) != 1:
        raise ValueError("'B' must be a square matrix with contiguous rows")
    n = B.shape[0]
    _f32(p, "p", n)
    _f32(r, "r", n)
    q = torch.empty(n, dtype=torch.float32, device=B.device) if q is None else _f32(q, "q", n)
    s = torch.empty(n, dtype=torch.float32, device=B.device) if s is None else _f32(s, "s", n)
    ws = workspace or default_workspace(B.device, stream)
    wp, wb = ws.ptr(lib().cspb_bicgk_workspace_bytes(n))
    d = _capi.BicgkDesc(n, B.stride(0), _mat_dtype(B), 0, _ptr(B), _ptr(p), _ptr(r), _ptr(q), _ptr(s), wp, wb)
    _raise(lib().cspb_bicgk_fused(C.byref(d), C.c_void_p(_stream(stream))), "bicgk")
    return q, s


CHAIN_OUTPUTS = ("B1", "x1", "w1", "q", "s", "B2", "x2", "w2")


def gemver_chain(A0, a: dict, b: dict, *, alpha: float, beta: float, out: dict | None = None,
                 workspace: Workspace | None = None, stream=None) -> dict:
    """The gemver chain G1 -> BiCGK -> G2 in one launch. a: u1 v1 u2 v2 y z (G1), b: u1 v1 u2 v2 (G2).
    Returns the eight outputs by the reference's promoted names."""
    torch = _torch()
    if A0 is None or A0.dim() != 2 or A0.shape[0] != A0.shape[1] or not A0.is_contiguous():
        raise ValueError("'A' must be a contiguous square matrix")
    _need(A0, "A", None, (torch.float32,))
    n = A0.shape[0]
    for k in ("u1", "v1", "u2", "v2", "y", "z"):
        _f32(a.get(k), k + "a", n)
    for k in ("u1", "v1", "u2", "v2"):
        _f32(b.get(k), k + "b", n)
    out = dict(out or {})
    for k in CHAIN_OUTPUTS:
        if k not in out:
            shape = (n, n) if k.startswith("B") else (n,)
            out[k] = torch.empty(shape, dtype=torch.float32, device=A0.device)
    ws = workspace or default_workspace(A0.device, stream)
    wp, wb = ws.ptr(lib().cspb_chain_workspace_bytes(n))
    d = _capi.ChainDesc(n, _ptr(A0), _ptr(a["u1"]), _ptr(a["v1"]), _ptr(a["u2"]), _ptr(a["v2"]), _ptr(a["y"]),
                        _ptr(a["z"]), _ptr(b["u1"]), _ptr(b["v1"]), _ptr(b["u2"]), _ptr(b["v2"]), float(alpha),
                        float(beta), *[_ptr(out[k]) for k in CHAIN_OUTPUTS], wp, wb)
    _raise(lib().cspb_gemver_chain(C.byref(d), C.c_void_p(_stream(stream))), "gemver-chain")
    return out


def gemver_batched(*args, **kwargs):
    from .batched import gemver_batched as impl
    return impl(*args, **kwargs)


# ---- NS residuals -------------------------------------------------------------------------------------------------
def ns_incompressible(u, v, p, *, h: float, nu: float, out=None, norms=None, workspace: Workspace | None = None,
                      stream=None):
    """r_u, r_v, r_c of the incompressible residual on a periodic (ny, nx) grid; u, v, p float32 or bfloat16.
    Returns (ru, rv, rc, norms) with norms a float64 tensor of 3 on the device."""
    torch = _torch()
    if u is None or u.dim() != 2:
        raise ValueError("'u' must be (ny, nx)")
    ny, nx = u.shape
    for t, nm in ((u, "u"), (v, "v"), (p, "p")):
        _need(t, nm, (ny, nx), (torch.float32, torch.bfloat16))
    if not (u.dtype == v.dtype == p.dtype):
        raise ValueError("'u', 'v', 'p' must share one dtype")
    dev = u.device
    if out is None:
        out = tuple(torch.empty((ny, nx), dtype=torch.float32, device=dev) for _ in range(3))
    ru, rv, rc = out
    if norms is None:
        norms = torch.empty(3, dtype=torch.float64, device=dev)
    ws = workspace or default_workspace(dev, stream)
    wp, wb = ws.ptr(lib().cspb_ns_incomp_workspace_bytes(nx, ny))
    d = _capi.NsIncompDesc(nx, ny, _mat_dtype(u), 0, float(h), float(nu), _ptr(u), _ptr(v), _ptr(p), _ptr(ru),
                           _ptr(rv), _ptr(rc), _ptr(norms), wp, wb)
    _raise(lib().cspb_ns_incompressible(C.byref(d), C.c_void_p(_stream(stream))), "ns-incompressible")
    return ru, rv, rc, norms


NS_DIAG = ("Dt", "Ws", "Sq0", "Sq1", "Sq2", "Sq3", "detn0", "detn1", "detn2", "detn3", "detd", "detw",
           "err_dt", "err_ws", "err_sq0", "err_sq1", "err_sq2", "err_sq3")


def ns_compressible(U, *, limiter: str = "minmod", bc: str = "walls", R=None, diag=None, det_sq64=None,
                    reference_rounding: bool = False, workspace: Workspace | None = None, stream=None):
    """The reference's compressible residual and diagnostics. U: (4, ny, nx) float32. Returns (R, diag, det_sq64)
    with diag the 18 floats of include/cspb.h (NS_DIAG names them). reference_rounding=True selects the kernel that
    rounds every operation as a sequential f32 evaluation of the reference's physics.hpp does (the same bits)."""
    torch = _torch()
    if limiter not in ("minmod", "vanleer"):
        raise ValueError("--limiter must be minmod|vanleer")
    if bc not in ("walls", "periodic"):
        raise ValueError("--bc must be walls|periodic")
    if U is None or U.dim() != 3 or U.shape[0] != 4:
        raise ValueError("'U' must be (4, ny, nx)")
    _need(U, "U", None, (torch.float32,))
    ny, nx = U.shape[1], U.shape[2]
    dev = U.device
    R = torch.empty_like(U) if R is None else _need(R, "R", tuple(U.shape), (torch.float32,))
    diag = torch.empty(18, dtype=torch.float32, device=dev) if diag is None else diag
    det_sq64 = torch.empty(4, dtype=torch.float64, device=dev) if det_sq64 is None else det_sq64
    ws = workspace or default_workspace(dev, stream)
    wp, wb = ws.ptr(lib().cspb_ns_comp_workspace_bytes(nx, ny))
    d = _capi.NsCompDesc(nx, ny, 0 if limiter == "minmod" else 1, 1 if bc == "walls" else 0,
                         _capi.NS_REFERENCE_ROUNDING if reference_rounding else 0, 0, _ptr(U), _ptr(R),
                         _ptr(diag), _ptr(det_sq64), wp, wb)
    _raise(lib().cspb_ns_compressible(C.byref(d), C.c_void_p(_stream(stream))), "ns-residual")
    return R, diag, det_sq64


def ns_init_cons(nx: int, ny: int, amp: float, *, U=None, device=None, stream=None):
    torch = _torch()
    U = torch.empty((4, ny, nx), dtype=torch.float32, device=device or "cuda") if U is None else U
    _raise(lib().cspb_ns_init_cons(_ptr(U), nx, ny, float(amp), C.c_void_p(_stream(stream))), "ns init")
    return U


# ---- scans and ragged columns -----------------------------------------------------------------------------------
def exclusive_scan(values, *, out=None, workspace: Workspace | None = None, stream=None):
    """n + 1 outputs: the exclusive scan of `values` (int32 storage = u32, int64 storage = u64; wrapping), then the
    total."""
    torch = _torch()
    if values is None or values.dim() != 1:
        raise ValueError("'values' must be a vector")
    _need(values, "values", None, (torch.int32, torch.int64, torch.uint32, torch.uint64))
    n = values.shape[0]
    wide = values.element_size() == 8
    out = torch.empty(n + 1, dtype=values.dtype, device=values.device) if out is None else out
    ws = workspace or default_workspace(values.device, stream)
    wp, wb = ws.ptr(lib().cspb_scan_workspace_bytes(n))
    f = lib().cspb_exclusive_scan_u64 if wide else lib().cspb_exclusive_scan_u32
    _raise(f(_ptr(values), _ptr(out), n, wp, wb, C.c_void_p(_stream(stream))), "device scan")
    return out


_COL_DTYPES = None


def build_column(src, *, offsets_mode: bool = False, workspace: Workspace | None = None, stream=None,
                 path: str = "counts"):
    """cs::ragged::counts_from / offsets_from on the device: returns (extents u32, offs u32 (N+1), total, flag) and
    raises ValueError with the reference's messages when the flag is set."""
    torch = _torch()
    dts = {torch.int32: _capi.I32, torch.uint32: _capi.U32, torch.int64: _capi.I64, torch.uint64: _capi.U64}
    if src is None or src.dtype not in dts:
        raise ValueError(f"naga::cospan: shape hook: '{path}' drives per-index extents by value and must have an "
                         f"integer dtype")
    if not src.is_contiguous():
        raise ValueError(f"'{path}' must be contiguous")
    if offsets_mode:
        if src.dim() != 1:
            raise ValueError(f"naga::cospan: shape hook: '{path}' drives per-index extents by value and must be rank 1 "
                             "(N + 1 offsets)")
        count, k = src.shape[0], 1
        if count == 0:
            raise ValueError(f"naga::cospan: shape hook: '{path}' holds no offsets (it needs N + 1 >= 1 entries)")
        n = count - 1
    else:
        if src.dim() not in (1, 2):
            raise ValueError(f"naga::cospan: shape hook: '{path}' drives per-index extents by value and must be rank 1 "
                             "[N] or rank 2 [N, k]")
        count = src.shape[0]
        k = src.shape[1] if src.dim() == 2 else 1
        if src.dim() == 2 and k == 0:
            raise ValueError(f"naga::cospan: shape hook: '{path}' has no column 0")
        n = count
    dev = src.device
    extents = torch.empty(max(n, 0), dtype=torch.int32, device=dev)
    offs = torch.empty(n + 1, dtype=torch.int32, device=dev)
    tf = torch.empty(2, dtype=torch.int32, device=dev)
    ws = workspace or default_workspace(dev, stream)
    wp, wb = ws.ptr(lib().cspb_scan_workspace_bytes(n))
    st = lib().cspb_build_column(_ptr(src), dts[src.dtype], count, k, 1 if offsets_mode else 0, _ptr(extents),
                                 _ptr(offs), _ptr(tf), wp, wb, C.c_void_p(_stream(stream)))
    if st != _capi.OK:
        _raise(st, f"shape hook '{path}'")
    total, flag = (int(v) & 0xffffffff for v in tf.cpu().tolist())
    if flag & _capi.COLUMN_TIMEOUT:
        raise RuntimeError(f"shape hook '{path}': the device scan's bounded wait gave up; the offsets are not valid")
    if flag & 1:
        raise ValueError(f"naga::cospan: shape hook: '{path}' holds a negative or invalid count or offset")
    if flag & 2:
        raise ValueError(f"naga::cospan: shape hook: '{path}' has a value or a total past 2^32 - 1 (ragged totals "
                         "are limited to 2^32 - 1 elements)")
    return extents, offs, total, flag


def fill_hash(out, seed: int, dist: int = 0, base: int = 0, stream=None):
    """The reference's seeded generator on the device (float32 or bfloat16 output)."""
    _raise(lib().cspb_fill_hash(_ptr(out), _mat_dtype(out), out.numel(), int(base), int(seed) & 0xffffffff,
                                int(dist), C.c_void_p(_stream(stream))), "fill_hash")
    return out
