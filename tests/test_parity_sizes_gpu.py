"""Parity at the benchmark configurations' own sizes, against the reference's FP32 arithmetic and against f64.

The reference's checks (examples/ns-residual/main.cpp:304-329, examples/gemver-chain/main.cpp:192-234) compare each
variant with an f64 evaluation at 1e-4. These tests go further, at the sizes the benchmarks run:

* compressible NS residual, 4096² (walls and periodic, minmod) and 1024² (van Leer):
  - the reference-rounding kernel (CSPB_NS_REFERENCE_ROUNDING) is BIT-IDENTICAL to the oracle's sequential f32
    evaluation of physics.hpp (ns_comp_f32), R and the per-cell min dt / max wave speed alike;
  - the fast kernel is held to the accuracy of that f32 arithmetic: per conserved variable its relative L2 error
    against f64 stays within 1.25x of the f32 arithmetic's own error (which is 1.1e-5 .. 1.8e-5 at 4096²: the residual
    is a difference of O(1) face fluxes, so the last bit of any flux shows at that level). Two f32 evaluations that
    round differently therefore differ by about that much from each other; the test bounds that distance too.
* GEMVER n = 16384 f32: x and w within 1e-5 of the oracle's f32 evaluation of the reference's unfused component loops
  (orc_gemver_f32_unfused) and of f64, Â bit-exact against the f32 formula.
* the ragged batch at its configuration (4096 log-uniform sizes in [64, 4096]): sampled instances against f64.
* the seeded generator (cspb_fill_hash): bit-exact against the reference's own hash_unit values
  (tests/golden/hash_ref.npz, indices past 2^32 included) and against the host restatement over a 2^20 range that
  crosses 2^32.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().float().cpu().numpy()


NS_CASES = [(4096, True, 0), (4096, False, 0), (1024, True, 1), (1024, False, 1), (250, True, 1), (130, False, 0)]


def _ns_ids(c):
    return f"{c[0]}-{'walls' if c[1] else 'periodic'}-{'vanleer' if c[2] else 'minmod'}"


@pytest.mark.parametrize("case", NS_CASES, ids=_ns_ids)
def test_ns_compressible_reference_rounding_bit_exact(cuda, case):
    import torch
    import cospanmdao_b200 as cb
    N, walls, lim = case
    ny = N if N >= 1024 else N // 2 + 3
    Uh = oracle.ns_init(N, ny, 1.0)
    U = torch.from_numpy(Uh).to(cuda)
    R, diag, sq64 = cb.ns_compressible(U, limiter=["minmod", "vanleer"][lim], bc="walls" if walls else "periodic",
                                       reference_rounding=True)
    R32, d32 = oracle.ns_comp_f32(Uh, walls, lim)
    got = R.cpu().numpy()
    diff = int(np.count_nonzero(got.view(np.uint32) != R32.view(np.uint32)))
    assert diff == 0, f"{diff} of {got.size} residual values differ from the f32 evaluation of physics.hpp"
    dg = diag.cpu().numpy()
    assert dg[10] == np.float32(d32[0]) and dg[11] == np.float32(d32[1])  # min dt, max wave speed: the same bits
    assert dg[0] == dg[10] and dg[1] == dg[11]
    # the f64 sums of R² over the same f32 residuals, added in another order (16.7M terms: about 1e-12 apart)
    assert np.allclose(sq64.cpu().numpy(), d32[2:], rtol=1e-9, atol=0)


@pytest.mark.parametrize("case", NS_CASES[:4], ids=_ns_ids)
def test_ns_compressible_fast_as_accurate_as_f32_arithmetic(cuda, case):
    import torch
    import cospanmdao_b200 as cb
    N, walls, lim = case
    Uh = oracle.ns_init(N, N, 1.0)
    U = torch.from_numpy(Uh).to(cuda)
    R, diag, sq64 = cb.ns_compressible(U, limiter=["minmod", "vanleer"][lim], bc="walls" if walls else "periodic")
    got = R.cpu().numpy()
    R32, _ = oracle.ns_comp_f32(Uh, walls, lim)
    R64, d64 = oracle.ns_comp_f64(Uh, walls, lim)
    ref = oracle.ref_residual(Uh, walls, lim)  # the reference's own f64 reference_residual, where it was built
    for v in range(4):
        e_fast = oracle.rel_l2(got[v], R64[v])
        e_f32 = oracle.rel_l2(R32[v], R64[v])
        assert e_fast <= 1.25 * e_f32, (v, e_fast, e_f32)
        assert e_fast < 1e-4  # the reference's own --check bound
        assert oracle.rel_l2(got[v], R32[v]) <= 2.0 * e_f32, v
        if ref is not None:
            assert oracle.rel_l2(got[v], ref[0][v]) <= 1.25 * e_f32, v
    dg = diag.cpu().numpy()
    assert abs(dg[10] - d64[0]) / d64[0] < 1e-6 and abs(dg[11] - d64[1]) / d64[1] < 1e-6
    assert np.allclose(sq64.cpu().numpy(), d64[2:], rtol=1e-4)


def test_gemver_n16384_against_f32_component_loops_and_f64(cuda):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    n = 16384
    d = workloads.gemver_inputs(n, 0, device=cuda)
    B, x, w = cb.gemver(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2)
    h = {k: v.cpu().numpy() for k, v in d.items()}
    # Â: the f32 formula (a + u1·v1) + u2·v2 with each operation rounded, row block by row block
    Bh = B.cpu().numpy()
    for r0 in range(0, n, 2048):
        sl = slice(r0, r0 + 2048)
        want = (h["A"][sl] + np.outer(h["u1"][sl], h["v1"]).astype(np.float32)) + \
            np.outer(h["u2"][sl], h["v2"]).astype(np.float32)
        assert np.array_equal(Bh[sl], want), r0
    del Bh, B, d
    torch.cuda.empty_cache()
    x32 = np.empty(n, np.float32)
    w32 = np.empty(n, np.float32)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    oracle.restatement().orc_gemver_f32_unfused(n, 64, P(h["A"]), *[P(h[k]) for k in ("u1", "v1", "u2", "v2", "y", "z")],
                                                1.5, 1.2, None, P(x32), P(w32), 0, n)
    xo, wo, _ = oracle.gemver_f64(n, h["A"], h["u1"], h["v1"], h["u2"], h["v2"], h["y"], h["z"], 1.5, 1.2)
    xg, wg = _np(x), _np(w)
    assert oracle.rel_l2(xg, x32) < 1e-5 and oracle.rel_l2(wg, w32) < 1e-5
    assert oracle.rel_l2(xg, xo) < 1e-5 and oracle.rel_l2(wg, wo) < 1e-5


def test_gemver_bf16_storage_n16384_per_output_error(cuda):
    # BF16 storage of A, f32 arithmetic, f64 column sums: error against f64 of the SAME bf16 matrix, per output
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    n = 16384
    d = workloads.gemver_inputs(n, 0, dtype=torch.bfloat16, device=cuda)
    B, x, w = cb.gemver(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2,
                        want_B=False)
    h = {k: _np(v) for k, v in d.items()}
    xo, wo, _ = oracle.gemver_f64(n, h["A"], h["u1"], h["v1"], h["u2"], h["v2"], h["y"], h["z"], 1.5, 1.2)
    assert oracle.rel_l2(_np(x), xo) < 1e-5 and oracle.rel_l2(_np(w), wo) < 1e-5


def test_ragged_batch_config_sampled_instances(cuda):
    import torch
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.batched import RaggedBatch
    torch.cuda.empty_cache()
    sizes = workloads.ragged_sizes(4096)
    b = RaggedBatch(sizes, want_B=False).fill(seed=0).run(check=True)
    torch.cuda.synchronize()
    assert b.offsets_match()
    rng = np.random.default_rng(3)
    picks = sorted(set(rng.choice(b.count, 12, replace=False).tolist()) | {int(np.argmax(sizes)), int(np.argmin(sizes))})
    for k in picks:
        dk = b.instance(k)
        n = dk["n"]
        hk = {key: _np(dk[key]) for key in ("A", "u1", "v1", "u2", "v2", "y", "z")}
        xo, wo, _ = oracle.gemver_f64(n, hk["A"], hk["u1"], hk["v1"], hk["u2"], hk["v2"], hk["y"], hk["z"],
                                      dk["alpha"], dk["beta"])
        assert oracle.rel_l2(_np(dk["x"]), xo) < 1e-5, (k, n)
        assert oracle.rel_l2(_np(dk["w"]), wo) < 1e-5, (k, n)
    del b
    torch.cuda.empty_cache()


def test_fill_hash_bit_exact_against_reference_values(cuda, golden):
    import torch
    import cospanmdao_b200 as cb
    g = golden("hash_ref.npz")
    idx, seeds, want = g["index"], g["seeds"], g["value"]
    out = torch.empty(1, dtype=torch.float32, device=cuda)
    for si, seed in enumerate(seeds):
        for ii, i in enumerate(idx):
            cb.fill_hash(out, int(seed), 0, base=int(i))
            got = out.cpu().numpy()
            assert got.view(np.uint32)[0] == want[si, ii:ii + 1].view(np.uint32)[0], (int(seed), int(i))
    # a 2^20 range that crosses 2^32, both distributions, against the host restatement
    base = 2 ** 32 - 2 ** 19
    big = torch.empty(2 ** 20, dtype=torch.float32, device=cuda)
    for dist in (0, 1):
        cb.fill_hash(big, 5, dist, base=base)
        host = oracle.hash_fill(2 ** 20, 5, dist, base)
        assert np.array_equal(big.cpu().numpy().view(np.uint32), host.view(np.uint32)), dist
    # bf16 output: round to nearest even of the same f32 values
    bb = torch.empty(2 ** 16, dtype=torch.bfloat16, device=cuda)
    cb.fill_hash(bb, 7, 0, base=base)
    want16 = torch.from_numpy(oracle.hash_fill(2 ** 16, 7, 0, base)).to(torch.bfloat16)
    assert torch.equal(bb.cpu(), want16)
