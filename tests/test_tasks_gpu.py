"""Task tables: GEMVERs and NS residuals scattered in device memory, many per launch. Every task's result must be
bit-identical to the single call on the same data (the same decomposition, the same reduction order): the same
alone and in the mix."""
import numpy as np
import pytest

import oracle
from cospanmdao_b200 import _capi

pytestmark = pytest.mark.gpu


def _gemver_case(torch, cb, n, seed, dtype, with_B, dev):
    from cospanmdao_b200 import workloads
    d = workloads.gemver_inputs(n, seed, dtype=dtype, device=dev)
    out = {"x": torch.empty(n, device=dev), "w": torch.empty(n, device=dev),
           "B": torch.empty((n, n), device=dev) if with_B else None}
    return d, out


@pytest.mark.parametrize("dtype_name", ["float32", "bfloat16"])
def test_gemver_tasks_match_single_calls(cuda, dtype_name):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200.tasks import TaskRunner, gemver_task
    dtype = getattr(torch, dtype_name)
    sizes = [128, 300, 1000, 2048, 4100, 77, 8192, 513]
    cases = [_gemver_case(torch, cb, n, 20 + i, dtype, i % 2 == 0, cuda) for i, n in enumerate(sizes)]
    table = np.concatenate([gemver_task(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], o["x"], o["w"],
                                        alpha=1.5, beta=1.2, B=o["B"]) for d, o in cases])
    TaskRunner(cuda).gemver(table, bf16=dtype == torch.bfloat16)
    torch.cuda.synchronize()
    for (d, o), n in zip(cases, sizes):
        B, x, w = cb.gemver(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2,
                            want_B=o["B"] is not None)
        torch.cuda.synchronize()
        assert torch.equal(x, o["x"]) and torch.equal(w, o["w"]), n
        if o["B"] is not None:
            assert torch.equal(B, o["B"]), n


def _status(cb, torch, wp):
    """the CSPB_ERR_* code in the status word of a task call's workspace (synchronizes the current stream)"""
    return cb.lib().cspb_read_status(cb.C.c_void_p(wp), None, cb.C.c_void_p(torch.cuda.current_stream().cuda_stream))


def _bf16_tasks_without_B(torch, cuda, sizes, seed0):
    from cospanmdao_b200.tasks import gemver_task
    cases = [_gemver_case(torch, None, n, seed0 + i, torch.bfloat16, False, cuda) for i, n in enumerate(sizes)]
    table = np.concatenate([gemver_task(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], o["x"], o["w"],
                                        alpha=1.5, beta=1.2, B=None) for d, o in cases])
    return cases, table


def test_gemver_tasks_lean_variant_matches(cuda):
    """A bf16 table with no B runs the kernel variant without the Â paths (CSPB_BATCH_NO_B, 3 blocks per SM): its x
    and w equal the full variant's and the single calls', bit for bit."""
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200.tasks import TaskRunner
    sizes = [128, 300, 1000, 2048, 4100, 77, 8192, 513, 64, 3000]
    cases, table = _bf16_tasks_without_B(torch, cuda, sizes, 40)
    runner = TaskRunner(cuda)
    wp = runner.gemver(table, bf16=True, no_b=False)
    assert _status(cb, torch, wp) == _capi.OK
    full = [(o["x"].clone(), o["w"].clone()) for _, o in cases]
    for _, o in cases:
        o["x"].fill_(float("nan"))
        o["w"].fill_(float("nan"))
    wp = runner.gemver(table, bf16=True)  # no task has B: the lean variant
    assert _status(cb, torch, wp) == _capi.OK
    for (d, o), (fx, fw), n in zip(cases, full, sizes):
        assert torch.equal(o["x"], fx) and torch.equal(o["w"], fw), n
        _, x, w = cb.gemver(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2,
                            want_B=False)
        torch.cuda.synchronize()
        assert torch.equal(x, o["x"]) and torch.equal(w, o["w"]), n


def test_gemver_tasks_no_b_flag_with_a_B_task(cuda):
    """CSPB_BATCH_NO_B on a table where a task has B: the call ends (no wait runs out) with CSPB_ERR_ARGUMENT in its
    status word, and no B is written. Its x and w are not valid, as after any device-reported error."""
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200.tasks import TaskRunner
    sizes = [256, 1000, 513]
    cases, table = _bf16_tasks_without_B(torch, cuda, sizes, 60)
    B = torch.full((sizes[1], sizes[1]), 7.0, device=cuda)
    table[1]["B"] = B.data_ptr()
    table[1]["ldb"] = sizes[1]
    wp = TaskRunner(cuda).gemver(table, bf16=True, no_b=True)
    raw = cb.C.c_uint32(0)
    st = cb.lib().cspb_read_status(cb.C.c_void_p(wp), cb.C.byref(raw),
                                   cb.C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _capi.ERR_ARGUMENT and raw.value == _capi.DEV_ARGUMENT, (st, raw.value)
    assert bool((B == 7.0).all())
    # the same table without the flag: the full variant, every task valid
    o = cases[0][1]
    wp = TaskRunner(cuda).gemver(table, bf16=True)
    assert _status(cb, torch, wp) == _capi.OK
    d = cases[0][0]
    _, x, w = cb.gemver(d["A"], d["u1"], d["v1"], d["u2"], d["v2"], d["y"], d["z"], alpha=1.5, beta=1.2, want_B=False)
    torch.cuda.synchronize()
    assert torch.equal(x, o["x"]) and torch.equal(w, o["w"])


@pytest.mark.parametrize("dtype_name", ["float32", "bfloat16"])
def test_ns_tasks_match_single_calls(cuda, dtype_name):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.tasks import TaskRunner, ns_task
    dtype = getattr(torch, dtype_name)
    grids = [256, 512, 64, 1024, 130, 200, 24]  # 200, 24: partial tiles at the grid's east and south edges
    cases = []
    for i, N in enumerate(grids):
        u, v, p, h = workloads.ns_fields(N, seed=i, dtype=dtype, device=cuda)
        outs = [torch.empty((N, N), device=cuda) for _ in range(3)]
        norms = torch.empty(3, dtype=torch.float64, device=cuda)
        cases.append((u, v, p, h, outs, norms))
    table = np.concatenate([ns_task(u, v, p, *outs, norms, h=h, nu=1e-3) for u, v, p, h, outs, norms in cases])
    TaskRunner(cuda).ns(table, bf16=dtype == torch.bfloat16)
    torch.cuda.synchronize()
    for u, v, p, h, outs, norms in cases:
        ru, rv, rc, nn = cb.ns_incompressible(u, v, p, h=h, nu=1e-3)
        torch.cuda.synchronize()
        assert torch.equal(ru, outs[0]) and torch.equal(rv, outs[1]) and torch.equal(rc, outs[2])
        assert torch.equal(nn, norms)
