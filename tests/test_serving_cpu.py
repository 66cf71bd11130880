"""Host logic of the serving loop without a GPU: the workload generator and the model store's budget and LRU rules."""
import numpy as np
import pytest

from cospanmdao_b200 import serving


class FakeStore(serving.ModelStore):
    def _load(self, mid):
        kind, size = self.wl.model_size[mid]
        self.loads += 1
        return serving.Model(mid, kind, size, {}, self.bytes_of(mid))


class FakeWl:
    def __init__(self, sizes):
        self.model_size = {i: (serving.KIND_GEMVER, s) for i, s in enumerate(sizes)}


def test_store_budget_and_lru():
    import torch
    wl = FakeWl([96, 96, 96, 96])  # 96*96*2 = 18432 bytes each in bf16 (rows already a multiple of 8)
    st = FakeStore(wl, dtype=torch.bfloat16, budget_bytes=50000, device="cpu")
    assert st.acquire([0, 1])
    st.release([0, 1])
    assert st.used == 36864 and st.loads == 2
    assert st.acquire([2])          # evicts the least recently used (0)
    assert 0 not in st.models and {1, 2} <= set(st.models) and st.evictions == 1
    assert not st.acquire([0, 3])   # 2 is in use and 1 + two new ones do not fit
    st.release([2])
    assert st.acquire([0, 3]) and st.used <= 50000
    assert st.models[0].in_use == 1 and st.models[3].in_use == 1
    # a model in use is never evicted
    assert not st.acquire([1, 2])
    st.release([0, 3])


def test_store_counts_padded_rows():
    import torch
    st = FakeStore(FakeWl([100]), dtype=torch.bfloat16, budget_bytes=1e9, device="cpu")
    assert st.bytes_of(0) == 100 * 104 * 2  # rows padded to 8 elements


def test_store_repeated_model_counts_once():
    import torch
    st = FakeStore(FakeWl([10, 10]), dtype=torch.float32, budget_bytes=1e9, device="cpu")
    assert st.acquire(np.array([1, 1, 1, 0]))
    assert st.models[1].in_use == 1 and st.loads == 2
    st.release(np.array([1, 1, 1, 0]))
    assert st.models[1].in_use == 0
