"""The ragged batch of GEMVERs in one launch: device-scanned offsets bit-exact, every instance against the f64
oracle, and every instance's result the same alone and in the mix."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _np(t):
    return t.detach().float().cpu().numpy()


def _rank2_f32(A, u1, v1, u2, v2):
    A = A.astype(np.float32)
    return (A + np.outer(u1, v1).astype(np.float32)) + np.outer(u2, v2).astype(np.float32)


SIZES = np.array([64, 1, 3, 100, 257, 511, 512, 700, 1023, 1024, 1500, 2048, 2100, 127, 8, 4096, 65, 333],
                 dtype=np.uint32)


@pytest.mark.parametrize("dtype_name,want_B", [("float32", True), ("float32", False), ("bfloat16", True)])
def test_batched_against_oracle(cuda, dtype_name, want_B):
    import torch
    from cospanmdao_b200.batched import RaggedBatch
    b = RaggedBatch(SIZES, dtype=getattr(torch, dtype_name), want_B=want_B).fill(seed=4).run(check=True)
    torch.cuda.synchronize()
    assert b.offsets_match()
    for k in range(b.count):
        d = b.instance(k)
        n = d["n"]
        h = {key: _np(d[key]) for key in ("A", "u1", "v1", "u2", "v2", "y", "z")}
        xo, wo, _ = oracle.gemver_f64(n, h["A"], h["u1"], h["v1"], h["u2"], h["v2"], h["y"], h["z"], d["alpha"],
                                      d["beta"])
        assert oracle.rel_l2(_np(d["x"]), xo) < TOL, (k, n)
        assert oracle.rel_l2(_np(d["w"]), wo) < TOL, (k, n)
        if want_B:
            assert np.array_equal(_np(d["B"]), _rank2_f32(h["A"], h["u1"], h["v1"], h["u2"], h["v2"])), (k, n)


def test_batched_same_alone_and_in_the_mix(cuda):
    import torch
    from cospanmdao_b200.batched import RaggedBatch
    mix = RaggedBatch(SIZES).fill(seed=9).run()
    torch.cuda.synchronize()
    for k in (0, 4, 11, 15):
        d = mix.instance(k)
        alone = RaggedBatch(SIZES[k:k + 1])
        a = alone.instance(0)
        a["A"].copy_(d["A"])
        for key in ("u1", "v1", "u2", "v2", "y", "z"):
            a[key].copy_(d[key])
        alone.alpha.fill_(d["alpha"])
        alone.beta.fill_(d["beta"])
        alone.run()
        torch.cuda.synchronize()
        a = alone.instance(0)
        assert torch.equal(a["x"], d["x"]) and torch.equal(a["w"], d["w"]) and torch.equal(a["B"], d["B"]), k


def test_batched_every_tuning_within_tolerance(cuda):
    import torch
    from cospanmdao_b200.batched import RaggedBatch, tune_word
    b = RaggedBatch(SIZES).fill(seed=1)
    ref = None
    for codes in ([0, 0, 0, 0], [1, 1, 1, 1], [2, 2, 2, 2], [1, 2, 0, 1]):
        b.run(tune=tune_word(codes))
        torch.cuda.synchronize()
        w = _np(b.w).copy()
        if ref is None:
            ref = w
        else:
            assert oracle.rel_l2(w, ref) < 2 * TOL


def test_batched_group_and_blocks_do_not_change_bits(cuda):
    """The work items a block takes per grab and the blocks per SM (tuning bits 8..11) move work between blocks only:
    x, w and Â are bit-identical for every value."""
    import torch
    from cospanmdao_b200.batched import RaggedBatch, tune_word, GROUPS, BLOCKS
    b = RaggedBatch(SIZES).fill(seed=2)
    b.run(tune=tune_word([1, 2, 0, 1]))
    torch.cuda.synchronize()
    ref = (b.x.clone(), b.w.clone(), b.B.clone())
    for g in GROUPS:
        for k in BLOCKS:
            b.x.fill_(float("nan"))
            b.run(tune=tune_word([1, 2, 0, 1], g, k))
            torch.cuda.synchronize()
            assert torch.equal(b.x, ref[0]) and torch.equal(b.w, ref[1]) and torch.equal(b.B, ref[2]), (g, k)


def test_batched_config_sizes_offsets_bit_exact(cuda):
    # the configuration's 4096 log-uniform sizes: the u64 offsets pass 2^32 and match the host's exactly
    import torch
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.batched import layout
    import cospanmdao_b200 as cb
    sizes = workloads.ragged_sizes(4096)
    _, a_off, v_off = layout(sizes)
    assert a_off[-1] > 2 ** 32
    n = sizes.astype(np.uint64)
    ld = (n + 7) // 8 * 8
    sz = torch.from_numpy((n * ld).view(np.int64)).cuda()
    out = cb.exclusive_scan(sz)
    assert np.array_equal(out.cpu().numpy().view(np.uint64), a_off)


def test_batched_rejects_invalid_sizes(cuda):
    import torch
    from cospanmdao_b200.batched import RaggedBatch
    b = RaggedBatch(np.array([16, 32], dtype=np.uint32)).fill()
    b.n[1] = 0  # an invalid size written on the device after the host sized the batch
    with pytest.raises(ValueError):
        b.run(check=True)
    b = RaggedBatch(np.array([16, 32], dtype=np.uint32)).fill()
    b.n[1] = 64  # the device total no longer fits the capacity the host declared
    with pytest.raises(ValueError):
        b.run(check=True)
