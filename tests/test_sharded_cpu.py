"""The host side of the row-sharded GEMVER (cospanmdao_b200.sharded) on the CPU: the row split, and the exchange of
the column-sum shares between two gloo ranks. Each rank's share is computed here in numpy f64 from the oracle's
formula (standing in for cspb_gemver_rows_partial); the exchange must give both ranks the same total, bit for bit
the rank-order sum, and the x formed from it must match the f64 oracle's."""
import json
import os
import socket
from pathlib import Path

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(n):
    rng = np.random.default_rng(5)
    A = rng.uniform(-1, 1, (n, n)).astype(np.float32)
    vec = {k: rng.uniform(0, 1, n).astype(np.float32) for k in ("u1", "v1", "u2", "v2", "y", "z")}
    return A, vec


def _share(A, vec, r0, r1):
    # Σ_{i in [r0, r1)} Â[i][j]·y[i] in f64, Â in f32 as the kernels form it
    Ah = (A[r0:r1] + np.outer(vec["u1"][r0:r1], vec["v1"]).astype(np.float32)) + \
        np.outer(vec["u2"][r0:r1], vec["v2"]).astype(np.float32)
    return (Ah.astype(np.float64) * vec["y"][r0:r1, None].astype(np.float64)).sum(axis=0)


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch
    from cospanmdao_b200.replicas import Ranks
    from cospanmdao_b200.sharded import combine_column_sums, shard_rows
    r = Ranks().init("gloo", timeout_s=60)
    n = 600
    A, vec = _problem(n)
    r0, r1 = shard_rows(n, world)[rank]
    share = torch.from_numpy(_share(A, vec, r0, r1))
    total = combine_column_sums(share, r)
    np.save(Path(out_dir) / f"total{rank}.npy", total.numpy())
    Path(out_dir, f"r{rank}.json").write_text(json.dumps({"r0": r0, "r1": r1}))
    r.barrier()
    r.close()


def test_two_ranks_exchange_the_column_sums(tmp_path):
    import torch.multiprocessing as mp
    import oracle
    world, n = 2, 600
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    totals = [np.load(tmp_path / f"total{r}.npy") for r in range(world)]
    assert np.array_equal(totals[0], totals[1])
    A, vec = _problem(n)
    spans = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    assert spans[0]["r0"] == 0 and spans[0]["r1"] == spans[1]["r0"] and spans[1]["r1"] == n
    want = _share(A, vec, spans[0]["r0"], spans[0]["r1"]) + _share(A, vec, spans[1]["r0"], spans[1]["r1"])
    assert np.array_equal(totals[0], want)  # the rank-order sum, bit for bit
    x = (vec["z"].astype(np.float64) + 1.2 * totals[0]).astype(np.float32)
    xo, _, _ = oracle.gemver_f64(n, A, vec["u1"], vec["v1"], vec["u2"], vec["v2"], vec["y"], vec["z"], 1.0, 1.2)
    assert oracle.rel_l2(x, xo) < 1e-5


def test_shard_rows():
    from cospanmdao_b200.sharded import shard_rows
    for n in (0, 1, 127, 128, 129, 1000, 16384):
        for world in (1, 2, 3, 8):
            s = shard_rows(n, world)
            assert len(s) == world and s[0][0] == 0 and s[-1][1] == n
            assert all(a <= b for a, b in s) and all(s[i][1] == s[i + 1][0] for i in range(world - 1))
            assert all(a % 128 == 0 for a, _ in s)
    assert shard_rows(16384, 8) == [(2048 * r, 2048 * (r + 1)) for r in range(8)]
    with pytest.raises(ValueError):
        shard_rows(10, 0)


def _halo_rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch
    from cospanmdao_b200.replicas import Ranks
    from cospanmdao_b200.sharded import combine_sums, exchange_halos
    r = Ranks().init("gloo", timeout_s=60)
    nx = 12
    # rank q's first row of field f holds 100·q + 10·f + 0, its last row 100·q + 10·f + 1 (every column)
    first = [torch.full((nx,), 100.0 * rank + 10 * f) for f in range(3)]
    last = [t + 1 for t in first]
    up, dn = exchange_halos(first, last, r)
    up, dn = torch.stack(up), torch.stack(dn)
    norms = combine_sums(torch.tensor([1.0 + rank, 2.0, 3.0 * rank], dtype=torch.float64), r)
    np.save(Path(out_dir) / f"halo{rank}.npy", np.stack([up.numpy(), dn.numpy()]))
    np.save(Path(out_dir) / f"norms{rank}.npy", norms.numpy())
    r.barrier()
    r.close()


def test_three_ranks_exchange_halo_rows(tmp_path):
    import torch.multiprocessing as mp
    world = 3
    mp.start_processes(_halo_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for q in range(world):
        up, dn = np.load(tmp_path / f"halo{q}.npy")
        prev, nxt = (q - 1) % world, (q + 1) % world
        for f in range(3):
            assert np.all(up[f] == 100.0 * prev + 10 * f + 1)  # the previous rank's last row
            assert np.all(dn[f] == 100.0 * nxt + 10 * f)       # the next rank's first row
    want = np.sqrt(np.array([1.0 + 2.0 + 3.0, 2.0 * 3, 3.0 * (0 + 1 + 2)]))
    for q in range(world):
        assert np.array_equal(np.load(tmp_path / f"norms{q}.npy"), want)


# ---- the compressible residual's slabs --------------------------------------------------------------------------
NXC, NYC = 20, 23


def _comp_rank(rank, world, port, out_dir, walls):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch
    import oracle
    from cospanmdao_b200.replicas import Ranks
    from cospanmdao_b200.sharded import combine_comp_diag, exchange_comp_halos, shard_rows
    r = Ranks().init("gloo", timeout_s=60)
    U = torch.from_numpy(oracle.ns_init(NXC, NYC, 1.0))
    r0, r1 = shard_rows(NYC, world, 2)[rank]
    lo, hi, edges = exchange_comp_halos(U[:, r0:r1].contiguous(), r, walls)
    blank = torch.full((4, 2, NXC), float("nan"))
    np.save(Path(out_dir) / f"c{rank}.npy", np.stack([(lo if lo is not None else blank).numpy(),
                                                      (hi if hi is not None else blank).numpy()]))
    # stand-in slab diagnostics: [dt, ws, sq0..3, detn0..3, detd, detw, err..] and f64 sums, distinct per rank
    diag = torch.arange(18, dtype=torch.float32) + 100 * rank
    diag[0] = diag[10] = 5.0 - rank
    diag[1] = diag[11] = 1.0 + rank
    sums = torch.tensor([1.0, 2.0, 3.0, 4.0], dtype=torch.float64) * (rank + 1) + 0.1
    out, det = combine_comp_diag(r.all_gather_tensor(diag), r.all_gather_tensor(sums))
    np.save(Path(out_dir) / f"d{rank}.npy", np.concatenate([out.numpy().astype(np.float64), det.numpy()]))
    Path(out_dir, f"e{rank}.json").write_text(json.dumps({"edges": edges, "r0": r0, "r1": r1}))
    r.barrier()
    r.close()


@pytest.mark.parametrize("world,walls", [(2, True), (3, True), (3, False)])
def test_ranks_exchange_compressible_halos(tmp_path, world, walls):
    import torch.multiprocessing as mp
    import oracle
    mp.start_processes(_comp_rank, args=(world, _free_port(), str(tmp_path), walls), nprocs=world, join=True,
                       start_method="spawn")
    U = oracle.ns_init(NXC, NYC, 1.0)
    outs = []
    for q in range(world):
        lo, hi = np.load(tmp_path / f"c{q}.npy")
        e = json.loads((tmp_path / f"e{q}.json").read_text())
        r0, r1 = e["r0"], e["r1"]
        want_lo = not walls or q > 0
        want_hi = not walls or q < world - 1
        assert e["edges"] == (1 if want_lo else 0) | (2 if want_hi else 0)
        if want_lo:  # global rows r0 - 2, r0 - 1, wrapped
            assert np.array_equal(lo, U[:, [(r0 - 2) % NYC, (r0 - 1) % NYC], :])
        else:
            assert np.isnan(lo).all()
        if want_hi:
            assert np.array_equal(hi, U[:, [r1 % NYC, (r1 + 1) % NYC], :])
        else:
            assert np.isnan(hi).all()
        outs.append(np.load(tmp_path / f"d{q}.npy"))
    for q in range(1, world):
        assert np.array_equal(outs[q], outs[0])  # every rank combines to the same bits
    d = outs[0]
    assert d[0] == 5.0 - (world - 1) and d[10] == d[0]  # min dt
    assert d[1] == 1.0 + (world - 1) and d[11] == d[1]  # max wave speed
    det = sum(np.array([1.0, 2.0, 3.0, 4.0]) * (q + 1) + 0.1 for q in range(world))
    assert np.allclose(d[18:], det, rtol=0, atol=1e-12)
