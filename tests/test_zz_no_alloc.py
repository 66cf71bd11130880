"""cspb_build_column_static (the build_column that allocates nothing) against cspb_build_column, through the C ABI.

Three calls in a row on different inputs (counts mode, offsets mode, counts mode on a rank-2 source's column), so that
each call on the fixed scratch sees what the one before left there. The results are integers: compared exactly.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOO_LARGE = 10
STATIC_MAX = 1 << 24


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _run_both(lib, src, dtype_code, count, k, offsets_mode):
    import torch
    dev = src.device
    n = count - 1 if offsets_mode else count
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    outs = []
    for static in (False, True):
        ext = torch.full((max(n, 1),), 0xDEAD, dtype=torch.int32, device=dev)
        offs = torch.full((n + 1,), 0xBEEF, dtype=torch.int32, device=dev)
        tf = torch.full((2,), 7, dtype=torch.int32, device=dev)
        if static:
            rc = lib.cspb_build_column_static(_ptr(src), dtype_code, count, k, int(offsets_mode), _ptr(ext), _ptr(offs),
                                              _ptr(tf), stream)
        else:
            wb = lib.cspb_scan_workspace_bytes(n)
            ws = torch.empty(wb, dtype=torch.uint8, device=dev)
            rc = lib.cspb_build_column(_ptr(src), dtype_code, count, k, int(offsets_mode), _ptr(ext), _ptr(offs),
                                       _ptr(tf), _ptr(ws), wb, stream)
        assert rc == 0, (static, rc, lib.cspb_status_string(rc))
        torch.cuda.synchronize(dev)
        outs.append((ext[:n].cpu().numpy(), offs.cpu().numpy(), tf.cpu().numpy()))
    return outs


def test_static_build_column_matches_two_calls_in_a_row(cuda):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import _capi
    lib = cb.lib()
    rng = np.random.default_rng(20261203)

    # call 1: counts mode, i32 counts, 3 000 017 extents (1 465 tiles of the u64 scan)
    counts = rng.integers(0, 97, size=3_000_017, dtype=np.int32)
    src = torch.from_numpy(counts).to(cuda)
    (e0, o0, t0), (e1, o1, t1) = _run_both(lib, src, _capi.I32, counts.size, 1, False)
    assert np.array_equal(e0, e1) and np.array_equal(o0, o1) and np.array_equal(t0, t1)
    assert int(t1[0]) == int(counts.astype(np.int64).sum()) and int(t1[1]) == 0

    # call 2: offsets mode, i64 offsets of 777 777 other extents
    ext2 = rng.integers(0, 1000, size=777_777).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum(ext2)]).astype(np.int64)
    src2 = torch.from_numpy(offsets).to(cuda)
    (e0, o0, t0), (e1, o1, t1) = _run_both(lib, src2, _capi.I64, offsets.size, 1, True)
    assert np.array_equal(e0, e1) and np.array_equal(o0, o1) and np.array_equal(t0, t1)
    assert np.array_equal(e1.view(np.uint32).astype(np.int64), ext2) and int(t1[1]) == 0

    # call 3: counts mode again, a rank-2 [N, 3] u64 source (column 0 read with stride k = 3)
    rk2 = rng.integers(0, 50, size=(123_457, 3), dtype=np.uint64)
    src3 = torch.from_numpy(rk2.view(np.int64)).to(cuda)
    (e0, o0, t0), (e1, o1, t1) = _run_both(lib, src3, _capi.U64, rk2.shape[0], 3, False)
    assert np.array_equal(e0, e1) and np.array_equal(o0, o1) and np.array_equal(t0, t1)
    assert int(t1[0]) == int(rk2[:, 0].sum())


def test_static_build_column_rejects_inputs_past_its_scratch(cuda):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import _capi
    lib = cb.lib()
    n = STATIC_MAX + 1
    src = torch.zeros(n, dtype=torch.int32, device=cuda)  # real buffers of the stated size: the call never reads them
    ext = torch.zeros(n, dtype=torch.int32, device=cuda)
    offs = torch.zeros(n + 1, dtype=torch.int32, device=cuda)
    tf = torch.full((2,), 5, dtype=torch.int32, device=cuda)
    stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    rc = lib.cspb_build_column_static(_ptr(src), _capi.I32, n, 1, 0, _ptr(ext), _ptr(offs), _ptr(tf), stream)
    assert rc == TOO_LARGE
    assert b"scratch" in lib.cspb_status_string(rc)
    torch.cuda.synchronize(cuda)
    assert tf.cpu().tolist() == [5, 5]  # nothing ran
    # the largest accepted size still works and agrees
    src_ok = torch.ones(STATIC_MAX, dtype=torch.int32, device=cuda)
    (e0, o0, t0), (e1, o1, t1) = _run_both(lib, src_ok, _capi.I32, STATIC_MAX, 1, False)
    assert np.array_equal(o0, o1) and np.array_equal(t0, t1) and int(t1[0]) == STATIC_MAX
