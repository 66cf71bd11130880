"""The single-pass device scan and the ragged column against tests/test_device_scan.cpp's cases (bit-exact)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _u32(t):
    return t.cpu().numpy().view(np.uint32)


def test_scan_known_answers(cuda, golden):
    import torch
    import cospanmdao_b200 as cb
    g = golden("scan_known.npz")
    for k in g:
        if not k.startswith("in_"):
            continue
        v = g[k]
        t = torch.from_numpy(v.view(np.int32)).to(cuda)
        out = cb.exclusive_scan(t)
        assert np.array_equal(_u32(out), g["out_" + k[3:]]), k


@pytest.mark.parametrize("n", [4095, 4096, 4097, 1 << 20, (1 << 24) + 5])
def test_scan_u32_large_wrapping(cuda, n):
    import torch
    import cospanmdao_b200 as cb
    rng = np.random.default_rng(n)
    v = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    out = cb.exclusive_scan(torch.from_numpy(v.view(np.int32)).to(cuda))
    assert np.array_equal(_u32(out), oracle.exclusive_scan(v))


@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 300001])
def test_scan_u64(cuda, n):
    import torch
    import cospanmdao_b200 as cb
    rng = np.random.default_rng(7 + n)
    v = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64) * np.uint64(3)  # wraps mod 2^64
    out = cb.exclusive_scan(torch.from_numpy(v.view(np.int64)).to(cuda))
    assert np.array_equal(out.cpu().numpy().view(np.uint64), oracle.exclusive_scan(v))


@pytest.mark.parametrize("misaligned", [False, True], ids=["l2-tiles", "register-tiles"])
@pytest.mark.parametrize("wide", [False, True], ids=["u32", "u64"])
@pytest.mark.parametrize("n", [1, 5, 2047, 2048, 2049, 4095, 4096, 4097, 8191, 8192, 8193, 16385, (1 << 22) + 3])
def test_scan_l2_and_register_tiles(cuda, n, wide, misaligned):
    """16-byte aligned input and output take the L2 re-read tiles (8192 u32 / 4096 u64 items); an array that starts
    one element off a 16-byte boundary takes the register-loaded tiles (4096 u32 / 2048 u64). Both are bit-exact, at
    and around the tile sizes."""
    import torch
    import cospanmdao_b200 as cb
    rng = np.random.default_rng(n * 2 + wide)
    npdt, tdt = (np.uint64, torch.int64) if wide else (np.uint32, torch.int32)
    v = rng.integers(0, np.iinfo(npdt).max, size=n + 1, dtype=np.uint64).astype(npdt)
    src = torch.from_numpy(v.view(np.int64 if wide else np.int32)).to(cuda)
    vals = src[1:] if misaligned else src[:n]
    store = torch.full((n + 2,), -1, dtype=tdt, device=cuda)
    out = store[1:] if misaligned else store[:n + 1]
    assert (vals.data_ptr() % 16 == 0) != misaligned and (out.data_ptr() % 16 == 0) != misaligned
    cb.exclusive_scan(vals, out=out)
    want = oracle.exclusive_scan(v[1:] if misaligned else v[:n])
    assert np.array_equal(out.cpu().numpy().view(npdt), want)
    if not misaligned:
        assert int(store[n + 1]) == -1  # nothing past out[n]


def test_scan_repeat_is_identical(cuda):
    import torch
    import cospanmdao_b200 as cb
    v = torch.randint(0, 1000, (3_000_000,), dtype=torch.int32, device=cuda)
    a = cb.exclusive_scan(v)
    b = cb.exclusive_scan(v)
    assert torch.equal(a, b)


@pytest.mark.parametrize("dtype", ["int32", "uint32", "int64", "uint64"])
def test_build_column_counts(cuda, dtype):
    import torch
    import cospanmdao_b200 as cb
    rng = np.random.default_rng(3)
    src = rng.integers(0, 5000, size=10007).astype(dtype)
    t = torch.from_numpy(src).to(cuda)
    ext, offs, total, flag = cb.build_column(t)
    e2, o2, tot2, f2 = oracle.build_column(src)
    assert np.array_equal(_u32(ext), e2) and np.array_equal(_u32(offs), o2) and total == tot2 and flag == 0


def test_build_column_rank2_and_offsets_mode(cuda):
    import torch
    import cospanmdao_b200 as cb
    src = np.array([[4, 9], [1, 9], [2, 9], [0, 1]], dtype=np.int32)
    ext, offs, total, _ = cb.build_column(torch.from_numpy(src).to(cuda))
    assert _u32(ext).tolist() == [4, 1, 2, 0] and _u32(offs).tolist() == [0, 4, 5, 7, 7] and total == 7
    o = np.array([0, 2, 2, 7, 11], dtype=np.int64)
    ext, offs, total, _ = cb.build_column(torch.from_numpy(o).to(cuda), offsets_mode=True)
    assert _u32(ext).tolist() == [2, 0, 5, 4] and total == 11
    ext, offs, total, _ = cb.build_column(torch.zeros(0, dtype=torch.int32, device=cuda))
    assert _u32(offs).tolist() == [0] and total == 0


def test_build_column_flags_raise_like_the_reference(cuda):
    import torch
    import cospanmdao_b200 as cb
    with pytest.raises(ValueError, match="negative"):
        cb.build_column(torch.tensor([3, -1, 5], dtype=torch.int64, device=cuda))
    with pytest.raises(ValueError, match="2\\^32"):
        cb.build_column(torch.tensor([2 ** 33], dtype=torch.int64, device=cuda))
    with pytest.raises(ValueError, match="2\\^32"):
        cb.build_column(torch.tensor([2 ** 31, 2 ** 31, 1], dtype=torch.int64, device=cuda))
    with pytest.raises(ValueError, match="negative"):
        cb.build_column(torch.tensor([1, 2], dtype=torch.int32, device=cuda), offsets_mode=True)
    with pytest.raises(ValueError, match="negative"):
        cb.build_column(torch.tensor([0, 5, 3], dtype=torch.int32, device=cuda), offsets_mode=True)


def test_build_column64_total_past_2_32(cuda):
    """cspb_build_column64: u64 offsets for a column whose total passes 2^32 - 1 (the u32 builder flags it as too large);
    each extent stays a u32, so a single count or offset difference past 2^32 - 1 is still flag 2."""
    import ctypes as C
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import _capi
    lib = cb.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def build(src_np, dtype_code, offsets_mode):
        src = torch.from_numpy(src_np).to(cuda)
        count = src_np.shape[0]
        n = count - 1 if offsets_mode else count
        ext = torch.zeros(max(n, 1), dtype=torch.int32, device=cuda)
        offs = torch.zeros(n + 1, dtype=torch.int64, device=cuda)
        tf = torch.full((2,), -1, dtype=torch.int64, device=cuda)
        wb = lib.cspb_scan_workspace_bytes(n)
        ws = torch.empty(wb + 256, dtype=torch.uint8, device=cuda)
        wp = (ws.data_ptr() + 255) // 256 * 256
        rc = lib.cspb_build_column64(C.c_void_p(src.data_ptr()), dtype_code, count, 1, int(offsets_mode),
                                     C.c_void_p(ext.data_ptr()), C.c_void_p(offs.data_ptr()), C.c_void_p(tf.data_ptr()),
                                     C.c_void_p(wp), wb, st)
        assert rc == 0, rc
        torch.cuda.synchronize()
        return (ext[:n].cpu().numpy().view(np.uint32), offs.cpu().numpy().view(np.uint64),
                tf.cpu().numpy().view(np.uint64))

    rng = np.random.default_rng(11)
    counts = np.concatenate([[2 ** 31 + 3, 2 ** 31 + 1], rng.integers(0, 1000, 20001)]).astype(np.int64)
    want = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    ext, offs, tf = build(counts, _capi.I64, False)
    assert np.array_equal(offs, want) and int(tf[0]) == int(want[-1]) > 2 ** 32 and int(tf[1]) == 0
    assert np.array_equal(ext.astype(np.int64), counts)
    # the u32 builder refuses the same counts (flag 2: the total passes 2^32 - 1)
    with pytest.raises(ValueError, match="2\\^32"):
        cb.build_column(torch.from_numpy(counts).to(cuda))
    # offsets mode: the N + 1 offsets themselves, past 2^32
    ext2, offs2, tf2 = build(want.astype(np.int64), _capi.I64, True)
    assert np.array_equal(offs2, want) and np.array_equal(ext2.astype(np.int64), counts) and int(tf2[1]) == 0
    assert int(tf2[0]) == int(want[-1])
    # a single count past 2^32 - 1, and an offset difference past it, are flag 2; a decrease is flag 1
    _, _, tf3 = build(np.array([5, 2 ** 32 + 1, 3], dtype=np.int64), _capi.I64, False)
    assert int(tf3[1]) & 0xffffffff == 2
    _, _, tf4 = build(np.array([0, 2 ** 32 + 1, 2 ** 32 + 4], dtype=np.int64), _capi.I64, True)
    assert int(tf4[1]) & 0xffffffff == 2
    _, _, tf5 = build(np.array([0, 9, 4], dtype=np.int64), _capi.I64, True)
    assert int(tf5[1]) & 0xffffffff == 1


@pytest.mark.parametrize("misaligned", [False, True], ids=["bulk-tiles", "register-tiles"])
@pytest.mark.parametrize("wide", [False, True], ids=["u32-offsets", "u64-offsets"])
@pytest.mark.parametrize("dtype", ["int32", "uint32"])
@pytest.mark.parametrize("n", [1, 6143, 6144, 6145, (1 << 20) + 7])
def test_build_column_bulk_and_register_tiles(cuda, n, dtype, wide, misaligned):
    """Counts from a 16-byte aligned 32-bit source take the bulk-copy tiles, a source one element off the boundary the
    register-loaded tiles; extents, offsets, total and flag agree with the oracle either way, for u32 offsets
    (cspb_build_column) and u64 offsets (cspb_build_column64), with and without negative counts (flag 1)."""
    import ctypes as C
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import _capi
    lib = cb.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(n + 3 * wide + 5 * misaligned)
    for negative in (False, True):
        v = rng.integers(0, 3000, size=n + 1).astype(np.int64)
        if negative and dtype == "int32":
            v[rng.integers(0, n + 1, size=3)] = -7
        src_np = v.astype(dtype)
        big = torch.from_numpy(src_np).to(cuda)
        src = big[1:] if misaligned else big[:n]
        assert (src.data_ptr() % 16 == 0) != misaligned
        host = src_np[1:] if misaligned else src_np[:n]
        ext = torch.zeros(n, dtype=torch.int32, device=cuda)
        offs = torch.zeros(n + 1, dtype=torch.int64 if wide else torch.int32, device=cuda)
        tf = torch.zeros(2, dtype=torch.int64 if wide else torch.int32, device=cuda)
        wb = lib.cspb_scan_workspace_bytes(n)
        ws = torch.empty(wb + 256, dtype=torch.uint8, device=cuda)
        wp = C.c_void_p((ws.data_ptr() + 255) // 256 * 256)
        code = _capi.I32 if dtype == "int32" else _capi.U32
        f = lib.cspb_build_column64 if wide else lib.cspb_build_column
        rc = f(C.c_void_p(src.data_ptr()), code, n, 1, 0, C.c_void_p(ext.data_ptr()), C.c_void_p(offs.data_ptr()),
               C.c_void_p(tf.data_ptr()), wp, wb, st)
        assert rc == 0, rc
        torch.cuda.synchronize()
        counts = np.where(host.astype(np.int64) < 0, 0, host.astype(np.int64))
        want_offs = np.concatenate([[0], np.cumsum(counts)])
        flag = 1 if (host.astype(np.int64) < 0).any() else 0
        assert np.array_equal(ext.cpu().numpy().view(np.uint32).astype(np.int64), counts)
        got = offs.cpu().numpy().view(np.uint64 if wide else np.uint32).astype(np.int64)
        assert np.array_equal(got, want_offs)
        tfh = tf.cpu().numpy().view(np.uint64 if wide else np.uint32)
        assert int(tfh[0]) == int(want_offs[-1]) and int(tfh[1]) == flag
        if not wide:
            e2, o2, tot2, f2 = oracle.build_column(host)
            assert np.array_equal(ext.cpu().numpy().view(np.uint32), e2) and tot2 == int(tfh[0]) and f2 == flag
