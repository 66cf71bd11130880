"""The continuous-batching server on the GPU: every request served, each result bit-identical alone and in the mix,
BF16-storage results within 1e-3 of f64, the budget honoured with evictions, and the per-request FP32 path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_workload(rate=None, n=400):
    from cospanmdao_b200 import serving
    return serving.make_workload(n, rate=rate, seed=3, gemver_models=24, ns_models=6, n_lo=128, n_hi=1536,
                                 grids=(64, 128, 256))


def test_server_serves_mix_and_matches_alone(cuda):
    import torch
    from cospanmdao_b200 import serving
    wl = _small_workload()
    srv = serving.Server(wl, max_batch=64, depth=3, dtype=torch.bfloat16)
    st = srv.run()
    assert st["requests"] == wl.count and st["batches"] >= wl.count // 64
    sample = [int(i) for i in np.linspace(0, wl.count - 1, 12).astype(int)]
    assert serving.check_mix(srv, sample)
    err = serving.errors_vs_f64(srv, sample)
    assert err["x"] < 1e-3 and err["w"] < 1e-3 and err["norms"] < 1e-3, err


def test_server_honours_budget_with_evictions(cuda):
    import torch
    from cospanmdao_b200 import serving
    wl = _small_workload(n=300)
    # room for a few models only: the store must evict and reload, results unchanged
    big = max(serving.ModelStore(wl, dtype=torch.bfloat16, budget_bytes=1, device=cuda).bytes_of(m)
              for m in wl.model_size)
    srv = serving.Server(wl, max_batch=16, depth=2, dtype=torch.bfloat16, budget_bytes=3 * big, preload=False)
    st = srv.run()
    assert st["evictions"] > 0 and srv.store.used <= 3 * big
    ref = serving.Server(wl, max_batch=64, depth=2, dtype=torch.bfloat16)
    ref.run()
    for r in range(0, wl.count, 7):
        a, b = serving.result_of(srv, r), serving.result_of(ref, r)
        if isinstance(a, tuple):
            assert all(np.array_equal(p, q) for p, q in zip(a, b)), r
        else:
            assert np.array_equal(a, b), r


def test_server_with_poisson_arrivals_and_plain_path(cuda):
    import torch
    from cospanmdao_b200 import serving
    wl = _small_workload(rate=20000.0, n=300)
    srv = serving.Server(wl, max_batch=64, depth=3, dtype=torch.bfloat16)
    st = srv.run()
    assert st["p99_ms"] >= st["p50_ms"] > 0
    pl = serving.plain(wl)
    assert pl["requests"] == wl.count and pl["p99_ms"] >= pl["p50_ms"] > 0
