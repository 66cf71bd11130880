"""One large GEMVER split by rows, and one NS residual split into y-slabs, across the GPUs of a node (one process per
GPU), each with its one exchange step.

GEMVER
Rank r holds rows [r0, r1) of A (and of B, u1, u2, y, w) and all of v1, v2, z (shard_rows gives the split). Every row
is independent except for the column sums Âᵀy, which need every row. So a forward is:

  1. cspb_gemver_rows_partial: the rank's Â rows and its share of the column sums, n values in f64;
  2. the exchange: an all-gather of the shares (n · 8 bytes per rank; NCCL over NVLink on GPUs, gloo on the CPU) and
     their sum in rank order, so that every rank holds the same total and forms the same x;
  3. cspb_gemver_rows_finish: x over all n columns, then w over the rank's rows.

The all-gather plus a fixed-order sum (instead of an all-reduce) keeps x independent of the collective's reduction
order. Scaling is strong (the GEMVER's size is fixed); the exchange is n · 8 · world bytes against a shard's 12 · n²
/ world bytes of matrix traffic.
"""
from __future__ import annotations

import ctypes as C

from . import _capi
from ._capi import BF16, F32, lib


def shard_rows(n: int, world: int, align: int = 128) -> list[tuple[int, int]]:
    """Contiguous row ranges [r0, r1) for `world` ranks, near-equal and (but the last) multiples of `align` rows, so
    that shards cut at the kernels' 128-row strips. A rank may get an empty range when n is small."""
    if n < 0 or world < 1 or align < 1:
        raise ValueError("shard_rows needs n >= 0, world >= 1 and align >= 1")
    blocks = (n + align - 1) // align
    cuts = [min(n, (blocks * r // world) * align) for r in range(world)] + [n]
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def combine_column_sums(share, ranks):
    """The sum of every rank's share of the column sums, added in rank order (the same bits on every rank)."""
    parts = ranks.all_gather_tensor(share) if ranks is not None else [share]
    total = parts[0].clone()
    for p in parts[1:]:
        total += p
    return total


def _desc(A, u1, v1, u2, v2, y, z, alpha, beta, B, x, w, wp, wb):
    import torch
    n = A.shape[1]
    return _capi.GemverRowsDesc(n, A.shape[0], A.stride(0), B.stride(0) if B is not None else n,
                                BF16 if A.dtype == torch.bfloat16 else F32, 0, _ptr(A), _ptr(u1), _ptr(v1), _ptr(u2),
                                _ptr(v2), _ptr(y), _ptr(z), float(alpha), float(beta), _ptr(B), _ptr(x), _ptr(w), wp,
                                wb)


def _ptr(t):
    return None if t is None else int(t.data_ptr())


def gemver_rows_partial(A, u1, v1, u2, v2, y, *, B=None, colsum=None, workspace=None, stream=None):
    """The rank's Â rows (into B when given) and its share of the column sums (f64, n). A: (rows, n) f32 or bf16
    with contiguous rows; u1, u2, y: rows; v1, v2: n."""
    import torch
    import cospanmdao_b200 as cb
    rows, n = A.shape
    colsum = torch.empty(n, dtype=torch.float64, device=A.device) if colsum is None else colsum
    ws = workspace or cb.default_workspace(A.device, stream)
    wp, wb = ws.ptr(int(lib().cspb_gemver_rows_workspace_bytes(n, rows)))
    d = _desc(A, u1, v1, u2, v2, y, None, 0.0, 0.0, B, None, None, wp, wb)
    cb._raise(lib().cspb_gemver_rows_partial(C.byref(d), C.c_void_p(_ptr(colsum)), C.c_void_p(cb._stream(stream))),
              "gemver rows partial")
    return colsum


def gemver_rows_finish(A, u1, v1, u2, v2, y, z, total, *, alpha, beta, B=None, x=None, w=None, workspace=None,
                       stream=None):
    """x over all n columns from the summed column sums, then w over the rank's rows. Returns (x, w)."""
    import torch
    import cospanmdao_b200 as cb
    rows, n = A.shape
    x = torch.empty(n, dtype=torch.float32, device=A.device) if x is None else x
    w = torch.empty(rows, dtype=torch.float32, device=A.device) if w is None else w
    ws = workspace or cb.default_workspace(A.device, stream)
    wp, wb = ws.ptr(int(lib().cspb_gemver_rows_workspace_bytes(n, rows)))
    d = _desc(A, u1, v1, u2, v2, y, z, alpha, beta, B, x, w, wp, wb)
    cb._raise(lib().cspb_gemver_rows_finish(C.byref(d), C.c_void_p(_ptr(total)), C.c_void_p(cb._stream(stream))),
              "gemver rows finish")
    return x, w


def gemver_sharded(A, u1, v1, u2, v2, y, z=None, *, alpha, beta, ranks=None, want_B=True, workspace=None,
                   stream=None):
    """This rank's part of one row-sharded GEMVER: (B rows or None, x (all n), w rows). `ranks` is a
    replicas.Ranks joined to the job's process group (None: a single rank)."""
    import torch
    rows, n = A.shape
    B = torch.empty((rows, n), dtype=torch.float32, device=A.device) if want_B else None
    share = gemver_rows_partial(A, u1, v1, u2, v2, y, B=B, workspace=workspace, stream=stream)
    total = combine_column_sums(share, ranks)
    x, w = gemver_rows_finish(A, u1, v1, u2, v2, y, z, total, alpha=alpha, beta=beta, B=B, workspace=workspace,
                              stream=stream)
    return B, x, w


# ---- the incompressible NS residual in y-slabs ------------------------------------------------------------------------
# Rank r holds rows [r0, r1) of u, v, p (shard_rows(ny, world, 32): tile-aligned). The stencil needs one row above and
# one below each slab (periodic over the whole grid): every rank contributes its first and last rows to ONE
# all-gather (2 · 3 · nx floats per rank) and takes the last row of the previous rank and the first row of the next.
# Each rank then runs cspb_ns_incomp_slab; its residual rows are bit-identical to the whole grid's. The norms are
# the square roots of the slabs' squared sums, added in rank order (a second all-gather of 3 doubles per rank).

def exchange_halos(first, last, ranks):
    """first, last: this rank's first and last rows of u, v, p (three (nx,) tensors each). Returns (up, dn): the rows
    above this rank's slab (the previous rank's last rows, periodic) and below it (the next rank's first rows), three
    tensors each. One slab: the grid wraps onto itself, and the rows are returned as they are (no copy)."""
    import torch
    if ranks is None or ranks.world == 1:
        return list(last), list(first)
    parts = ranks.all_gather_tensor(torch.stack([torch.stack(list(first)), torch.stack(list(last))]))
    up = parts[(ranks.rank - 1) % ranks.world][1]
    dn = parts[(ranks.rank + 1) % ranks.world][0]
    return [up[f] for f in range(3)], [dn[f] for f in range(3)]


def combine_sums(sums, ranks):
    """The squared sums of every rank's slab, added in rank order, then their roots: the whole grid's norms."""
    if ranks is None or ranks.world == 1:
        return sums.sqrt()
    parts = ranks.all_gather_tensor(sums)
    total = parts[0].clone()
    for q in parts[1:]:
        total += q
    return total.sqrt()


def ns_incompressible_slab(u, v, p, up, dn, *, h, nu, out=None, sums=None, workspace=None, stream=None):
    """The residual of one slab: u, v, p (rows, nx) f32; up, dn the rows above and below it (three (nx,) rows of u,
    v, p each, or a (3, nx) tensor). Returns (ru, rv, rc, sums), sums being the slab's 3 squared sums (f64)."""
    import torch
    import cospanmdao_b200 as cb
    rows, nx = u.shape
    dev = u.device
    ru, rv, rc = out if out is not None else tuple(torch.empty((rows, nx), dtype=torch.float32, device=dev)
                                                  for _ in range(3))
    sums = torch.empty(3, dtype=torch.float64, device=dev) if sums is None else sums
    up = [up[f].contiguous() for f in range(3)]
    dn = [dn[f].contiguous() for f in range(3)]
    ws = workspace or cb.default_workspace(dev, stream)
    wp, wb = ws.ptr(int(lib().cspb_ns_incomp_slab_workspace_bytes(nx, rows)))
    d = _capi.NsIncompSlabDesc(nx, rows, F32, 0, float(h), float(nu), _ptr(u), _ptr(v), _ptr(p),
                               (C.c_void_p * 3)(*[_ptr(up[f]) for f in range(3)]),
                               (C.c_void_p * 3)(*[_ptr(dn[f]) for f in range(3)]), _ptr(ru), _ptr(rv), _ptr(rc),
                               _ptr(sums), wp, wb)
    cb._raise(lib().cspb_ns_incomp_slab(C.byref(d), C.c_void_p(cb._stream(stream))), "ns incompressible slab")
    return ru, rv, rc, sums


def ns_incompressible_sharded(u, v, p, *, h, nu, ranks=None, workspace=None, stream=None):
    """This rank's slab of one NS residual: (ru, rv, rc) of its rows and the whole grid's norms (3, f64)."""
    import torch
    up, dn = exchange_halos((u[0], v[0], p[0]), (u[-1], v[-1], p[-1]), ranks)
    ru, rv, rc, sums = ns_incompressible_slab(u, v, p, up, dn, h=h, nu=nu, workspace=workspace, stream=stream)
    return ru, rv, rc, combine_sums(sums, ranks)


# ---- the compressible NS residual in y-slabs ----------------------------------------------------------------------
# Rank r holds rows [r0, r1) of U (4, rows, nx), rows >= 2. The reference's tiles read a 2-cell halo
# (examples/ns-residual/tile.hpp:39-49), so every rank contributes its first two and its last two rows of the four
# fields to ONE all-gather (2 · 4 · 2 · nx floats per rank) and takes the previous rank's last two rows (halo_lo) and
# the next rank's first two (halo_hi). In a periodic grid every edge between ranks is interior, the ranks wrapping
# around; with walls the first rank's lower edge and the last rank's upper edge take the mirror instead. Each rank runs
# cspb_ns_comp_slab, whose residual rows are bit-identical to the whole grid's. The diagnostics combine in rank order:
# min dt and max wave speed exactly, the squared sums added in rank order (an all-gather of each slab's 18
# diagnostics and 4 f64 sums).

def comp_slab_edges(rank: int, world: int, walls: bool) -> int:
    """The interior edges of rank `rank`'s slab (bit 1 below, bit 2 above): none for a single slab (the whole grid
    takes its own boundary rule); with walls, not the grid's first and last edges."""
    if world == 1:
        return 0
    lo = 1 if (not walls or rank > 0) else 0
    hi = 2 if (not walls or rank < world - 1) else 0
    return lo | hi


def exchange_comp_halos(U, ranks, walls: bool):
    """U: this rank's slab (4, rows, nx). Returns (halo_lo, halo_hi, edges): the neighbours' two rows of each field
    ((4, 2, nx) tensors, None where the edge is not interior) and the edge bits for cspb_ns_comp_slab."""
    import torch
    if ranks is None or ranks.world == 1:
        return None, None, 0
    if U.shape[1] < 2:
        raise ValueError("a compressible slab needs at least 2 rows")
    mine = torch.stack([U[:, :2, :], U[:, -2:, :]]).contiguous()  # (2, 4, 2, nx): first rows, last rows
    parts = ranks.all_gather_tensor(mine)
    edges = comp_slab_edges(ranks.rank, ranks.world, walls)
    lo = parts[(ranks.rank - 1) % ranks.world][1].contiguous() if edges & 1 else None
    hi = parts[(ranks.rank + 1) % ranks.world][0].contiguous() if edges & 2 else None
    return lo, hi, edges


def ns_compressible_slab(U, halo_lo=None, halo_hi=None, edges: int = 0, *, limiter: str = "minmod",
                         bc: str = "walls", reference_rounding: bool = False, R=None, diag=None, det_sq64=None,
                         workspace=None, stream=None):
    """The residual of one slab (cspb_ns_comp_slab): returns (R, diag, det_sq64) over the slab's cells."""
    import torch
    import cospanmdao_b200 as cb
    if limiter not in ("minmod", "vanleer") or bc not in ("walls", "periodic"):
        raise ValueError("limiter must be minmod|vanleer and bc walls|periodic")
    if U.dim() != 3 or U.shape[0] != 4 or U.dtype != torch.float32 or not U.is_contiguous():
        raise ValueError("'U' must be a contiguous (4, rows, nx) float32 tensor")
    _, rows, nx = U.shape
    dev = U.device
    for name, h, bit in (("halo_lo", halo_lo, 1), ("halo_hi", halo_hi, 2)):
        if edges & bit and (h is None or tuple(h.shape) != (4, 2, nx) or not h.is_contiguous()):
            raise ValueError(f"'{name}' must be a contiguous (4, 2, {nx}) tensor for an interior edge")
    R = torch.empty_like(U) if R is None else R
    diag = torch.empty(18, dtype=torch.float32, device=dev) if diag is None else diag
    det_sq64 = torch.empty(4, dtype=torch.float64, device=dev) if det_sq64 is None else det_sq64
    ws = workspace or cb.default_workspace(dev, stream)
    wp, wb = ws.ptr(int(lib().cspb_ns_comp_slab_workspace_bytes(nx, rows)))
    d = _capi.NsCompSlabDesc(nx, rows, 0 if limiter == "minmod" else 1, 1 if bc == "walls" else 0,
                             _capi.NS_REFERENCE_ROUNDING if reference_rounding else 0, int(edges), _ptr(U),
                             _ptr(halo_lo) if edges & 1 else None, _ptr(halo_hi) if edges & 2 else None, _ptr(R),
                             _ptr(diag), _ptr(det_sq64), wp, wb)
    cb._raise(lib().cspb_ns_comp_slab(C.byref(d), C.c_void_p(cb._stream(stream))), "ns compressible slab")
    return R, diag, det_sq64


def combine_comp_diag(diags, sums):
    """The whole grid's 18 diagnostics from every slab's (diags: per-slab (18,) float32 tensors in rank order, sums:
    their (4,) f64 squared sums): the atomic and deterministic min dt / max wave speed exactly, the atomic sums in f32
    and the deterministic ones in f64, each added in rank order; the error stage atomic - deterministic."""
    import torch
    D = torch.stack([d.float().cpu() for d in diags])
    S = torch.stack([s.double().cpu() for s in sums])
    out = torch.empty(18, dtype=torch.float32)
    out[0] = D[:, 0].min()
    out[1] = D[:, 1].max()
    sq = D[0, 2:6].clone()
    det = S[0].clone()
    for q in range(1, D.shape[0]):
        sq += D[q, 2:6]
        det += S[q]
    out[2:6] = sq
    out[6:10] = det.float()
    out[10] = D[:, 10].min()
    out[11] = D[:, 11].max()
    out[12] = out[0] - out[10]
    out[13] = out[1] - out[11]
    out[14:18] = out[2:6] - out[6:10]
    return out, det


def ns_compressible_sharded(U, *, limiter: str = "minmod", bc: str = "walls", ranks=None,
                            reference_rounding: bool = False, workspace=None, stream=None):
    """This rank's slab of one compressible residual: (R of its rows, the whole grid's 18 diagnostics, the whole
    grid's 4 f64 squared sums)."""
    lo, hi, edges = exchange_comp_halos(U, ranks, bc == "walls")
    R, diag, sq = ns_compressible_slab(U, lo, hi, edges, limiter=limiter, bc=bc,
                                       reference_rounding=reference_rounding, workspace=workspace, stream=stream)
    if ranks is None or ranks.world == 1:
        return R, diag, sq
    d_all = ranks.all_gather_tensor(diag)
    s_all = ranks.all_gather_tensor(sq)
    out, det = combine_comp_diag(d_all, s_all)
    return R, out.to(diag.device), det.to(sq.device)
