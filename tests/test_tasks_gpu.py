"""Task tables: GEMVERs and NS residuals scattered in device memory, many per launch. Every task's result must be
bit-identical to the single call on the same data (the same decomposition, the same reduction order): the same
alone and in the mix."""
import numpy as np
import pytest

import oracle

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


@pytest.mark.parametrize("dtype_name", ["float32", "bfloat16"])
def test_ns_tasks_match_single_calls(cuda, dtype_name):
    import torch
    import cospanmdao_b200 as cb
    from cospanmdao_b200 import workloads
    from cospanmdao_b200.tasks import TaskRunner, ns_task
    dtype = getattr(torch, dtype_name)
    grids = [256, 512, 64, 1024, 130]
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
