"""One GEMVER split by rows (cospanmdao_b200.sharded, cspb_gemver_rows_partial / _finish), on one GPU.

The ranks run one after another on the same GPU: each partial is a complete launch, the exchange is the rank-order sum
of the shares on the host side, and no kernel waits on another rank. Â rows must equal the fused GEMVER's bit for
bit (the same per-element formula), x must be the same on every rank, and x and w must match the fused GEMVER and the
f64 oracle within the f32 tolerance (the column sums are grouped by shard)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _np(t):
    return t.detach().float().cpu().numpy()


@pytest.mark.parametrize("n,world,dtype_name,want_B", [(1000, 1, "float32", True), (1000, 2, "float32", True),
                                                       (3000, 3, "float32", False), (2048, 4, "bfloat16", True),
                                                       (777, 2, "bfloat16", False), (300, 3, "float32", True)])
def test_row_shards_match_the_fused_gemver(cuda, n, world, dtype_name, want_B):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.sharded import gemver_rows_finish, gemver_rows_partial, shard_rows
    dt = getattr(torch, dtype_name)
    d = workloads.gemver_inputs(n, 13, dtype=dt, device=cuda)
    alpha, beta = 1.5, -0.7
    Bf, xf, wf = cb.gemver(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=alpha, beta=beta,
                           want_B=want_B, schedule="barrier")
    shards = shard_rows(n, world)
    assert shards[0][0] == 0 and shards[-1][1] == n
    Bs, shares = [], []
    for r0, r1 in shards:
        B = torch.empty((r1 - r0, n), dtype=torch.float32, device=cuda) if want_B else None
        shares.append(gemver_rows_partial(d["A"][r0:r1], d["u1"][r0:r1], d["v1"], d["u2"][r0:r1], d["v2"],
                                          d["y"][r0:r1], B=B, workspace=cb.Workspace(cuda)))
        Bs.append(B)
    total = shares[0].clone()
    for s in shares[1:]:
        total += s
    xs, ws = [], []
    for (r0, r1), B in zip(shards, Bs):
        x, w = gemver_rows_finish(d["A"][r0:r1], d["u1"][r0:r1], d["v1"], d["u2"][r0:r1], d["v2"], d["y"][r0:r1],
                                  d["z"], total, alpha=alpha, beta=beta, B=B, workspace=cb.Workspace(cuda))
        xs.append(x)
        ws.append(w)
    torch.cuda.synchronize()
    for x in xs[1:]:
        assert torch.equal(x, xs[0])  # every rank forms the same x from the same total
    w = torch.cat(ws)
    if want_B:
        assert torch.equal(torch.cat(Bs), Bf)
    assert oracle.rel_l2(_np(xs[0]), _np(xf)) < TOL and oracle.rel_l2(_np(w), _np(wf)) < TOL
    h = {k: _np(v) for k, v in d.items()}
    xo, wo, _ = oracle.gemver_f64(n, h["A"], h["u1"], h["v1"], h["u2"], h["v2"], h["y"], h["z"], alpha, beta)
    assert oracle.rel_l2(_np(xs[0]), xo) < TOL and oracle.rel_l2(_np(w), wo) < TOL


def test_one_shard_equals_the_rank_loop_helper(cuda):
    """gemver_sharded with no process group is the one-shard case."""
    import torch
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.sharded import gemver_sharded
    n = 512
    d = workloads.gemver_inputs(n, 2, device=cuda)
    B, x, w = gemver_sharded(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.0, beta=2.0)
    B2, x2, w2 = gemver_sharded(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.0, beta=2.0)
    torch.cuda.synchronize()
    assert torch.equal(B, B2) and torch.equal(x, x2) and torch.equal(w, w2)
    h = {k: _np(v) for k, v in d.items()}
    xo, wo, _ = oracle.gemver_f64(n, h["A"], h["u1"], h["v1"], h["u2"], h["v2"], h["y"], h["z"], 1.0, 2.0)
    assert oracle.rel_l2(_np(x), xo) < TOL and oracle.rel_l2(_np(w), wo) < TOL


def test_row_shard_argument_errors(cuda):
    import ctypes as C
    from cospanmdao_b200 import _capi
    lib = _capi.lib()
    d = _capi.GemverRowsDesc()
    d.n, d.rows = 100, 101  # more rows than columns
    assert lib.cspb_gemver_rows_partial(C.byref(d), None, None) == _capi.ERR_ARGUMENT
    assert lib.cspb_gemver_rows_workspace_bytes(100, 101) == 0


@pytest.mark.parametrize("nx,ny,world", [(512, 512, 1), (512, 512, 2), (260, 150, 3), (1024, 700, 5)])
def test_ns_slabs_match_the_whole_grid(cuda, nx, ny, world):
    """cspb_ns_incomp_slab on y-slabs with the neighbouring rows passed as halos: the residual rows equal the whole
    grid's bit for bit (the same per-cell formula), and the roots of the rank-order sums of the slabs' squared sums
    equal the whole grid's norms to f64 rounding."""
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200.sharded import ns_incompressible_slab, shard_rows
    g = torch.Generator(device="cpu").manual_seed(nx + ny + world)
    u, v, p = ((torch.rand((ny, nx), generator=g) - 0.5).to(cuda) for _ in range(3))
    h, nu = 0.05, 1e-3
    ru, rv, rc, norms = cb.ns_incompressible(u, v, p, h=h, nu=nu)
    outs, sums = [], []
    for r0, r1 in shard_rows(ny, world, 32):
        assert r1 > r0
        up = torch.stack([f[(r0 - 1) % ny] for f in (u, v, p)])
        dn = torch.stack([f[r1 % ny] for f in (u, v, p)])
        a, b, c, s = ns_incompressible_slab(u[r0:r1], v[r0:r1], p[r0:r1], up, dn, h=h, nu=nu,
                                            workspace=cb.Workspace(cuda))
        outs.append((a, b, c))
        sums.append(s)
    torch.cuda.synchronize()
    for k, whole in enumerate((ru, rv, rc)):
        assert torch.equal(torch.cat([o[k] for o in outs]), whole)
    total = sums[0].clone()
    for s in sums[1:]:
        total += s
    assert torch.allclose(total.sqrt(), norms, rtol=1e-12, atol=0)


@pytest.mark.parametrize("walls", [True, False])
@pytest.mark.parametrize("lim,exact", [("minmod", False), ("vanleer", False), ("minmod", True)])
def test_compressible_slabs_bit_identical_to_whole_grid(cuda, walls, lim, exact):
    # three slabs of one grid, run one after the other on one GPU with the halos each would receive: R bit-identical
    # to the whole grid's, min dt / max wave speed exactly, the f64 squared sums to rounding of their grouping
    import torch
    import numpy as np
    import cospanmdao_b200 as cb
    from cospanmdao_b200.sharded import combine_comp_diag, comp_slab_edges, ns_compressible_slab, shard_rows
    nx, ny, world = 256, 301, 3
    bc = "walls" if walls else "periodic"
    U = cb.ns_init_cons(nx, ny, 1.0, device=cuda)
    R, diag, sq = cb.ns_compressible(U, limiter=lim, bc=bc, reference_rounding=exact)
    Rs, ds, ss = [], [], []
    for q, (r0, r1) in enumerate(shard_rows(ny, world, 16)):
        edges = comp_slab_edges(q, world, walls)
        lo = U[:, [(r0 - 2) % ny, (r0 - 1) % ny], :].contiguous()
        hi = U[:, [r1 % ny, (r1 + 1) % ny], :].contiguous()
        Rq, dq, sq_q = ns_compressible_slab(U[:, r0:r1].contiguous(), lo, hi, edges, limiter=lim, bc=bc,
                                            reference_rounding=exact)
        Rs.append(Rq)
        ds.append(dq.clone())
        ss.append(sq_q.clone())
    torch.cuda.synchronize()
    assert torch.equal(torch.cat(Rs, dim=1), R)
    out, det = combine_comp_diag(ds, ss)
    d = diag.cpu()
    assert out[10] == d[10] and out[11] == d[11] and out[0] == d[0] and out[1] == d[1]
    assert np.allclose(det.numpy(), sq.cpu().numpy(), rtol=1e-12, atol=0)


def test_compressible_single_slab_equals_whole_grid(cuda):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200.sharded import ns_compressible_slab
    U = cb.ns_init_cons(128, 64, 1.0, device=cuda)
    for bc in ("walls", "periodic"):
        R, diag, sq = cb.ns_compressible(U, bc=bc)
        R1, d1, s1 = ns_compressible_slab(U, None, None, 0, bc=bc)
        assert torch.equal(R, R1) and torch.equal(diag[6:12], d1[6:12]) and torch.equal(sq, s1)
