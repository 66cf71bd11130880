"""The oracle (CPU) against the golden fixtures generated from the reference's own code, and against the reference's
oracles themselves where they were built here; plus the analytic properties of the incompressible residual, which no
reference code computes."""
import math

import numpy as np
import pytest

import oracle
from cospanmdao_b200 import workloads


def test_hash_generator_matches_reference(golden):
    g = golden("hash_ref.npz")
    for si, seed in enumerate(g["seeds"]):
        for k, idx in enumerate(g["index"]):
            got = oracle.hash_fill(1, int(seed), 0, int(idx))[0]
            assert got == g["value"][si, k], (seed, idx)
    # the product's host copy of the generator (ragged sizes) is the same stream
    u = workloads.hash_unit01(3, g["index"])
    assert np.array_equal(u, (g["value"][2] + np.float32(1.0)) / np.float32(2.0))


def test_chain_restatement_matches_reference_chain(golden):
    g = golden("chain_ref_n256.npz")
    n = int(g["n"])
    inp = oracle.gemver_inputs(n, dist="reference")
    a = {k: inp[k] for k in ("u1", "v1", "u2", "v2", "y", "z")}
    b = {k: inp[k] for k in ("u1", "v1", "u2", "v2")}
    ab = 1.0 / math.sqrt(n)
    mine = oracle.chain_f64(inp["A"], a, b, ab, ab, want_B2=True)
    for k in ("x1", "w1", "q", "s", "x2", "w2"):
        assert oracle.rel_l2(mine[k], g[k]) < 1e-13, k
    assert mine["B2"].sum() == pytest.approx(float(g["B2_sum"]), rel=1e-13)
    assert (mine["B2"] ** 2).sum() == pytest.approx(float(g["B2_sumsq"]), rel=1e-13)
    assert np.allclose(mine["B2"][:8, :8], g["B2_corner"], rtol=0, atol=1e-15)


def test_single_gemver_is_the_first_stage_of_the_chain(golden):
    g = golden("chain_ref_n256.npz")
    n = int(g["n"])
    inp = oracle.gemver_inputs(n, dist="reference")
    ab = 1.0 / math.sqrt(n)
    x, w, _ = oracle.gemver_f64(n, inp["A"], inp["u1"], inp["v1"], inp["u2"], inp["v2"], inp["y"], inp["z"], ab, ab)
    assert oracle.rel_l2(x, g["x1"]) < 1e-13
    assert oracle.rel_l2(w, g["w1"]) < 1e-13


@pytest.mark.parametrize("tag,walls,lim", [("walls_minmod", True, 0), ("periodic_vanleer", False, 1)])
def test_ns_compressible_restatement_matches_reference_residual(golden, tag, walls, lim):
    g = golden("ns_comp_ref_32.npz")
    U = oracle.ns_init(32, 32, 1.0)
    R, d = oracle.ns_comp_f64(U, walls, lim)
    assert np.max(np.abs(R - g[f"R_{tag}"])) <= 1e-15 * np.max(np.abs(g[f"R_{tag}"]))
    assert np.allclose(d, g[f"diag_{tag}"], rtol=1e-13, atol=0)


def test_ns_uniform_periodic_flow_is_exactly_zero(golden):
    assert float(golden("ns_comp_ref_32.npz")["uniform_periodic_max"]) == 0.0
    R, _ = oracle.ns_comp_f64(oracle.ns_init(48, 32, 0.0), False, 0)
    assert np.max(np.abs(R)) == 0.0
    R32, _ = oracle.ns_comp_f32(oracle.ns_init(48, 32, 0.0), False, 1)
    assert np.max(np.abs(R32)) == 0.0


def test_ns_f32_restatement_within_reference_tolerance():
    U = oracle.ns_init(64, 64, 1.0)
    for walls, lim in ((True, 0), (False, 1)):
        R64, d64 = oracle.ns_comp_f64(U, walls, lim)
        R32, d32 = oracle.ns_comp_f32(U, walls, lim)
        assert oracle.rel_l2(R32, R64) < 1e-4  # the reference's own --check bound (main.cpp:317)


@pytest.mark.skipif(oracle.reference() is None, reason="the reference's oracle library was not built here")
def test_restatement_against_reference_live():
    for n in (256, 512):
        ref = oracle.ref_chain(n)
        inp = oracle.ref_inputs(n)
        a = {k: inp[k] for k in ("u1", "v1", "u2", "v2", "y", "z")}
        b = {k: inp[k] for k in ("u1", "v1", "u2", "v2")}
        ab = 1.0 / math.sqrt(n)
        mine = oracle.chain_f64(inp["A"], a, b, ab, ab)
        for k in ref:
            assert oracle.rel_l2(mine[k], ref[k]) < 1e-13
    for nx, ny in ((48, 32), (80, 16)):
        U = oracle.ref_init(nx, ny, 1.0)
        assert np.array_equal(U, oracle.ns_init(nx, ny, 1.0))
        for walls in (True, False):
            for lim in (0, 1):
                Rr, dr = oracle.ref_residual(U, walls, lim)
                R, d = oracle.ns_comp_f64(U, walls, lim)
                assert np.max(np.abs(R - Rr)) <= 1e-15 * np.max(np.abs(Rr))


def test_scan_oracle_known_answers(golden):
    g = golden("scan_known.npz")
    names = [k[3:] for k in g if k.startswith("in_")]
    assert len(names) == 12
    for nm in names:
        assert np.array_equal(oracle.exclusive_scan(g["in_" + nm]), g["out_" + nm]), nm


def test_scan_u64_wraps():
    v = np.array([2 ** 63, 2 ** 63, 5], dtype=np.uint64)
    assert oracle.exclusive_scan(v).tolist() == [0, 2 ** 63, 0, 5]


def test_build_column_oracle_semantics():
    ext, offs, total, flag = oracle.build_column(np.array([3, 0, 5], dtype=np.int32))
    assert ext.tolist() == [3, 0, 5] and offs.tolist() == [0, 3, 3, 8] and total == 8 and flag == 0
    _, _, _, flag = oracle.build_column(np.array([3, -1, 5], dtype=np.int64))
    assert flag & 1
    _, _, _, flag = oracle.build_column(np.array([2 ** 33], dtype=np.int64))
    assert flag & 2
    _, offs, total, flag = oracle.build_column(np.array([2 ** 31, 2 ** 31, 1], dtype=np.uint32))
    assert flag & 2 and total == 1  # the u32 total wrapped
    # rank 2 [N, k]: column 0
    src = np.array([[4, 9], [1, 9], [2, 9]], dtype=np.int32)
    ext, offs, total, flag = oracle.build_column(src)
    assert ext.tolist() == [4, 1, 2] and total == 7
    # offsets mode
    ext, offs, total, flag = oracle.build_column(np.array([0, 2, 2, 7], dtype=np.int32), offsets_mode=True)
    assert ext.tolist() == [2, 0, 5] and total == 7 and flag == 0
    _, _, _, flag = oracle.build_column(np.array([1, 2], dtype=np.int32), offsets_mode=True)
    assert flag & 1
    _, _, _, flag = oracle.build_column(np.array([0, 5, 3], dtype=np.int32), offsets_mode=True)
    assert flag & 1
    ext, offs, total, flag = oracle.build_column(np.zeros(0, dtype=np.int32))
    assert offs.tolist() == [0] and total == 0 and flag == 0


def _incomp(u, v, p, h, nu=1e-3):
    return oracle.ns_incomp_f64(u, v, p, h, nu)


def test_ns_incompressible_constant_field_is_zero():
    N = 32
    c = np.full((N, N), 0.75, dtype=np.float32)
    ru, rv, rc, norms = _incomp(c, c * 0.5, c * 2, 2 * math.pi / N)
    assert np.all(ru == 0) and np.all(rv == 0) and np.all(rc == 0) and np.all(norms == 0)


def test_ns_incompressible_divergence_free_field():
    # u = sin(y), v = sin(x): du/dx = 0 and dv/dy = 0 exactly on the grid, so r_c is exactly 0
    N = 64
    h = 2 * math.pi / N
    x = np.arange(N) * h
    u = np.broadcast_to(np.sin(x)[:, None], (N, N)).astype(np.float32)
    v = np.broadcast_to(np.sin(x)[None, :], (N, N)).astype(np.float32)
    p = np.zeros((N, N), np.float32)
    _, _, rc, norms = _incomp(u, v, p, h)
    assert np.max(np.abs(rc)) == 0.0 and norms[2] == 0.0


def test_ns_incompressible_second_order_convergence():
    # u = cos(x + 2y), v = 0, p = 0: r_u = u·u_x − ν∇²u, r_c = u_x; the error vs the closed form falls by ~4 per
    # halving of h
    errs = []
    for N in (32, 64, 128):
        h = 2 * math.pi / N
        x = np.arange(N) * h
        X, Y = np.meshgrid(x, x)  # column i -> x, row j -> y
        u = np.cos(X + 2 * Y)
        ux = -np.sin(X + 2 * Y)
        lap = -5 * np.cos(X + 2 * Y)
        nu = 1e-3
        exact = u * ux - nu * lap
        z = np.zeros((N, N), np.float32)
        ru, _, rc, _ = oracle.ns_incomp_f64(u.astype(np.float32), z, z, h, nu)
        # compare against the same f32-rounded u
        errs.append(np.max(np.abs(rc - ux)))
    rates = [errs[i] / errs[i + 1] for i in range(2)]
    assert all(3.5 < r < 4.5 for r in rates), rates


def test_ragged_sizes_are_log_uniform():
    n = workloads.ragged_sizes(4096)
    assert n.min() >= 64 and n.max() <= 4096
    lg = np.log(n.astype(np.float64) / 64) / np.log(64)
    assert abs(lg.mean() - 0.5) < 0.02
    assert 7.5e9 < float((n.astype(np.float64) ** 2).sum()) < 9.5e9
