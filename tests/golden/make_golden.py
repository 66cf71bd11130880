"""Generates the golden fixtures of tests/golden from the reference's OWN code.

    python tests/golden/make_golden.py        (needs oracle/_ref/libref.so, built by `make -C oracle` where the
                                               reference tree is present)

Fixtures (all small, numpy .npz):
  chain_ref_n256.npz      gemver_chain::reference_chain(256) on the reference's own hash inputs
                          (examples/gemver-chain/common/chain_data.hpp:93-144): x1 w1 q s x2 w2 (f64) and B2 checksums
  ns_comp_ref_32.npz      nsr::reference_residual on nsr::init_cons(amp 1) 32x32, for walls/minmod and
                          periodic/vanleer (examples/ns-residual/reference.hpp:30-130): R (f64) and [dt, ws, sq0..3];
                          plus max|R| of uniform periodic flow (must be exactly 0, main.cpp:183-188)
  hash_ref.npz            gemver_chain::hash_unit at seeds 1..7 (chain_data.hpp:43-48) on a spread of indices,
                          including indices past 2^32
  scan_known.npz          the sizes and input pattern of tests/test_device_scan.cpp:24-87 with their expected outputs
                          (std::exclusive_scan + total, computed here with numpy's cumsum in uint64 then wrapped)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent


def main() -> int:
    if oracle.reference() is None:
        print("oracle/_ref/libref.so is not built: run `make -C oracle` where the reference tree exists",
              file=sys.stderr)
        return 1

    n = 256
    ref = oracle.ref_chain(n, want_B2=True)
    B2 = ref.pop("B2")
    np.savez_compressed(OUT / "chain_ref_n256.npz", n=n, **ref, B2_sum=B2.sum(), B2_sumsq=(B2 ** 2).sum(),
                        B2_corner=B2[:8, :8])

    res = {}
    for tag, walls, lim in (("walls_minmod", True, 0), ("periodic_vanleer", False, 1)):
        U = oracle.ref_init(32, 32, 1.0)
        R, d = oracle.ref_residual(U, walls, lim)
        res[f"R_{tag}"] = R
        res[f"diag_{tag}"] = d
    U0 = oracle.ref_init(32, 32, 0.0)
    R0, _ = oracle.ref_residual(U0, False, 0)
    res["uniform_periodic_max"] = np.abs(R0).max()
    np.savez_compressed(OUT / "ns_comp_ref_32.npz", **res)

    r = oracle.reference()
    idx = np.array([0, 1, 2, 3, 255, 256, 65535, 65536, 2 ** 31 - 1, 2 ** 31, 2 ** 32 - 1, 2 ** 32, 2 ** 32 + 7,
                    2 ** 40 + 3], dtype=np.uint64)
    table = np.array([[r.ref_hash_unit(seed, int(i)) for i in idx] for seed in range(1, 8)], dtype=np.float32)
    np.savez_compressed(OUT / "hash_ref.npz", index=idx, seeds=np.arange(1, 8), value=table)

    def pattern(k: int) -> np.ndarray:
        i = np.arange(k, dtype=np.uint64)
        return ((i * np.uint64(2654435761) + np.uint64(7)) % np.uint64(11)).astype(np.uint32)

    cases = {}
    for k in (0, 1, 2, 37, 255, 256, 257, 1000, 4096 + 3, 256 * 256 + 17):
        cases[f"pattern_{k}"] = pattern(k)
    cases["zeros_700"] = np.zeros(700, dtype=np.uint32)
    big = np.zeros(700, dtype=np.uint32)
    big[699] = 1 << 30
    cases["big_700"] = big
    out = {}
    for name, v in cases.items():
        c = np.concatenate([[0], np.cumsum(v.astype(np.uint64))]).astype(np.uint64)
        out["in_" + name] = v
        out["out_" + name] = (c & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    np.savez_compressed(OUT / "scan_known.npz", **out)
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
