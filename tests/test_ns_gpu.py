"""The NS residuals on the GPU: the reference's compressible residual against its own f64 oracle (reference_residual,
pinned by the golden fixture) and the incompressible residual against the f64 restatement of its formula."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().float().cpu().numpy()


@pytest.mark.parametrize("tag,walls,lim", [("walls_minmod", True, 0), ("periodic_vanleer", False, 1)])
def test_ns_compressible_matches_reference_golden(cuda, golden, tag, walls, lim):
    import torch
    import cospanmdao_b200 as cb
    g = golden("ns_comp_ref_32.npz")
    U = torch.from_numpy(oracle.ns_init(32, 32, 1.0)).to(cuda)
    R, diag, sq64 = cb.ns_compressible(U, limiter=["minmod", "vanleer"][lim], bc="walls" if walls else "periodic")
    Rr, dr = g[f"R_{tag}"], g[f"diag_{tag}"]
    assert oracle.rel_l2(_np(R), Rr) < 1e-4  # the reference's --check bound (examples/ns-residual/main.cpp:317)
    dg = diag.cpu().numpy()
    assert abs(dg[10] - dr[0]) / dr[0] < 1e-4 and abs(dg[11] - dr[1]) / dr[1] < 1e-4
    assert np.allclose(sq64.cpu().numpy(), dr[2:], rtol=1e-4)
    # atomic min / max equal to the deterministic ones (main.cpp:318)
    assert dg[0] == dg[10] and dg[1] == dg[11]
    assert dg[12] == 0.0 and dg[13] == 0.0


# tiles of 32 x 15 cells, the deterministic diagnostics combined in groups of 256 tiles: 512 x 240 is exactly one group,
# 32 x 3855 is 257 tiles (a last group of one), 512 x 512 is 560 tiles (a partial third group)
@pytest.mark.parametrize("nx,ny", [(64, 48), (96, 80), (250, 130), (512, 512), (512, 240), (32, 3855)])
@pytest.mark.parametrize("walls,lim", [(True, 0), (False, 1), (True, 1), (False, 0)])
def test_ns_compressible_vs_oracle(cuda, nx, ny, walls, lim):
    import torch
    import cospanmdao_b200 as cb
    Uh = oracle.ns_init(nx, ny, 1.0)
    U = torch.from_numpy(Uh).to(cuda)
    R, diag, sq64 = cb.ns_compressible(U, limiter=["minmod", "vanleer"][lim], bc="walls" if walls else "periodic")
    Ro, do = oracle.ns_comp_f64(Uh, walls, lim)
    err = oracle.rel_l2(_np(R), Ro)
    assert err < 1e-4, err
    dg = diag.cpu().numpy()
    assert dg[0] == dg[10] and dg[1] == dg[11]
    assert abs(dg[10] - do[0]) / do[0] < 1e-6 and abs(dg[11] - do[1]) / do[1] < 1e-6
    assert np.allclose(sq64.cpu().numpy(), do[2:], rtol=1e-4)


def test_ns_uniform_periodic_flow_gives_exactly_zero(cuda):
    import torch
    import cospanmdao_b200 as cb
    U = cb.ns_init_cons(160, 96, 0.0, device=cuda)
    R, diag, _ = cb.ns_compressible(U, limiter="vanleer", bc="periodic")
    assert float(R.abs().max()) == 0.0


def test_ns_device_init_matches_host_init(cuda):
    import torch
    import cospanmdao_b200 as cb
    U = cb.ns_init_cons(128, 64, 1.0, device=cuda)
    Uh = oracle.ns_init(128, 64, 1.0)
    # CUDA's sinf / cosf and the host's may differ in the last bit
    assert np.max(np.abs(_np(U) - Uh)) < 1e-5


def test_ns_compressible_deterministic(cuda):
    import torch
    import cospanmdao_b200 as cb
    U = cb.ns_init_cons(1024, 512, 1.0, device=cuda)
    R0, d0, s0 = cb.ns_compressible(U)
    R1, d1, s1 = cb.ns_compressible(U)
    assert torch.equal(R0, R1) and torch.equal(s0, s1)
    assert torch.equal(d0[6:12], d1[6:12])


# ---- incompressible ---------------------------------------------------------------------------------------------
TOL_I = 1e-5


@pytest.mark.parametrize("N", [32, 130, 256, 1024])
def test_ns_incompressible_vs_oracle(cuda, N):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    u, v, p, h = workloads.ns_fields(N, seed=0, device=cuda)
    ru, rv, rc, norms = cb.ns_incompressible(u, v, p, h=h, nu=1e-3)
    o = oracle.ns_incomp_f64(_np(u), _np(v), _np(p), h, 1e-3)
    for got, want in ((ru, o[0]), (rv, o[1]), (rc, o[2])):
        assert oracle.rel_l2(_np(got), want) < TOL_I
    assert np.allclose(norms.cpu().numpy(), o[3], rtol=1e-5)


@pytest.mark.parametrize("nx,ny", [(37, 19), (130, 66), (3, 3)])
def test_ns_incompressible_ragged_sizes(cuda, nx, ny):
    import torch
    import cospanmdao_b200 as cb
    g = torch.Generator(device="cpu").manual_seed(nx * ny)
    u, v, p = (torch.rand((ny, nx), generator=g) + 0.5 for _ in range(3))
    u, v, p = u.to(cuda), v.to(cuda), p.to(cuda)
    ru, rv, rc, norms = cb.ns_incompressible(u, v, p, h=0.1, nu=1e-3)
    o = oracle.ns_incomp_f64(_np(u), _np(v), _np(p), 0.1, 1e-3)
    for got, want in ((ru, o[0]), (rv, o[1]), (rc, o[2])):
        assert oracle.rel_l2(_np(got), want) < TOL_I


def test_ns_incompressible_bf16_storage(cuda):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    N = 512
    u, v, p, h = workloads.ns_fields(N, seed=0, device=cuda)
    ub, vb, pb = (t.to(torch.bfloat16) for t in (u, v, p))
    ru, rv, rc, norms = cb.ns_incompressible(ub, vb, pb, h=h, nu=1e-3)
    # exact semantics on the bf16 fields
    o = oracle.ns_incomp_f64(_np(ub), _np(vb), _np(pb), h, 1e-3)
    for got, want in ((ru, o[0]), (rv, o[1]), (rc, o[2])):
        assert oracle.rel_l2(_np(got), want) < TOL_I
    # the storage error against the f32 fields is reported by the benchmark; the residual amplifies it (1/h)


@pytest.mark.parametrize("nx,ny", [(8, 3), (8, 40), (520, 17), (1032, 33), (512, 16), (36, 20)])
def test_ns_incompressible_bf16_shapes(cuda, nx, ny):
    # bf16 fields take tiles of 512 x 16 cells when nx % 8 == 0: a grid one tile wide, a last tile column of 8 cells
    # (520), three columns (1032), one exact tile (512 x 16), rows short of a tile; the halo cells come in as aligned
    # pairs of cells. 36 % 8 != 0 takes the register path.
    import torch
    import cospanmdao_b200 as cb
    g = torch.Generator(device="cpu").manual_seed(nx * 1000 + ny)
    u, v, p = ((torch.rand((ny, nx), generator=g) + 0.5).to(torch.bfloat16).to(cuda) for _ in range(3))
    ru, rv, rc, norms = cb.ns_incompressible(u, v, p, h=0.1, nu=1e-3)
    o = oracle.ns_incomp_f64(_np(u), _np(v), _np(p), 0.1, 1e-3)
    for got, want in ((ru, o[0]), (rv, o[1]), (rc, o[2])):
        assert oracle.rel_l2(_np(got), want) < TOL_I
    assert np.allclose(norms.cpu().numpy(), o[3], rtol=1e-5)


def test_ns_incompressible_after_other_calls_on_one_workspace(cuda):
    # The tile path clears the workspace's control block with a kernel that lets the tiles start before it ends (they
    # wait for it only at their completion count). Calls of other entry points in between leave that block dirty.
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    ws = cb.Workspace(cuda)
    u, v, p, h = workloads.ns_fields(512, seed=3, device=cuda)
    ub, vb, pb = (t.to(torch.bfloat16) for t in (u, v, p))
    first = [t.clone() for t in cb.ns_incompressible(u, v, p, h=h, nu=1e-3, workspace=ws)]
    first16 = [t.clone() for t in cb.ns_incompressible(ub, vb, pb, h=h, nu=1e-3, workspace=ws)]
    d = workloads.gemver_inputs(640, seed=1, device=cuda)
    for _ in range(2):
        cb.gemver(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2, workspace=ws)
        cb.exclusive_scan(torch.arange(5000, dtype=torch.int32, device=cuda), workspace=ws)
        again = cb.ns_incompressible(u, v, p, h=h, nu=1e-3, workspace=ws)
        again16 = cb.ns_incompressible(ub, vb, pb, h=h, nu=1e-3, workspace=ws)
        assert all(torch.equal(x, y) for x, y in zip(first, again))
        assert all(torch.equal(x, y) for x, y in zip(first16, again16))


def test_ns_incompressible_deterministic(cuda):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    u, v, p, h = workloads.ns_fields(768, seed=2, device=cuda)
    a = cb.ns_incompressible(u, v, p, h=h, nu=1e-3)
    b = cb.ns_incompressible(u, v, p, h=h, nu=1e-3)
    assert all(torch.equal(x, y) for x, y in zip(a, b))
