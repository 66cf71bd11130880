"""Builds the reference's example programs, unchanged, against the cs:: runtime of this package.

    python -m cospanmdao_b200.examples [--reference /path/to/CospanMDAO]

The sources are read from the reference tree (gemver-chain, ns-residual, getting-started), passed through the
annotation step (annotate.py: nvcc needs __host__ __device__ on what kernels call), and compiled with nvcc for sm_100a
against cospanmdao_b200/include. Binaries go to cospanmdao_b200/_examples/ (built here, next to the library, so they
travel with the tree); the annotated copies go to cospanmdao_b200/_examples/src/. Nothing of the reference is kept in
the repository.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

from .annotate import annotate_tree
from .build import ARCH, nvcc

PKG = Path(__file__).resolve().parent
# a host-only function called from device code (nvcc's diagnostic 20011) would run nothing on the GPU: make it an error
STRICT = ["--diag-error=20011,20014"]
# the runtime's fast paths call libcspb through include/cspb.h; the binaries find the library next to _examples/
LINK = ["-I", str(PKG.parent / "include"), "-L", str(PKG), "-lcspb", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/.."]
OUT = PKG / "_examples"
PROGRAMS = {
    "gemver-chain": ("examples/gemver-chain", "main.cpp"),
    "ns-residual": ("examples/ns-residual", "main.cpp"),
    "getting-started": ("getting-started", "main.cpp"),
}


def default_reference() -> Path:
    """The reference checkout when none is named: a sibling of this repository called `reference`."""
    return PKG.parent.parent / "reference"


def build_examples(reference: str | os.PathLike | None = None, verbose: bool = False) -> dict[str, Path]:
    ref = Path(reference or os.environ.get("CSPB_REFERENCE_DIR") or default_reference())
    if not (ref / "examples").is_dir():
        raise FileNotFoundError(f"no reference tree at {ref}")
    built = {}
    procs = []
    for name, (sub, main) in PROGRAMS.items():
        src = OUT / "src" / name
        annotate_tree(ref / sub, src)
        exe = OUT / name
        cmd = [nvcc(), "-std=c++20", "-O2", *ARCH, "-I", str(PKG / "include"), "--extended-lambda",
               "--expt-relaxed-constexpr", *STRICT, "-x", "cu", str(src / main), *LINK, "-o", str(exe)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((name, exe, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    errors = []
    for name, exe, cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errors.append(f"{name}: {' '.join(cmd)}\n{out}")
        else:
            built[name] = exe
    if errors:
        raise RuntimeError("building the examples failed:\n" + "\n".join(errors))
    return built


RUNTIME_TESTS = {"runtime-fused-groups": "fused_groups.cu", "runtime-ragged": "ragged.cu", "runtime-replay": "replay.cu",
                 "runtime-decoy": "decoy.cu", "runtime-ragged-wide": "ragged_wide.cu"}


def build_runtime_tests(verbose: bool = False) -> dict[str, Path]:
    """The runtime's own test programs (tests/runtime/*.cu, written against the cs:: API) -> cospanmdao_b200/_examples/."""
    src_dir = PKG.parent / "tests" / "runtime"
    OUT.mkdir(parents=True, exist_ok=True)
    built = {}
    for name, src in RUNTIME_TESTS.items():
        exe = OUT / name
        cmd = [nvcc(), "-std=c++20", "-O2", *ARCH, "-I", str(PKG / "include"), "--extended-lambda",
               "--expt-relaxed-constexpr", *STRICT, "-x", "cu", str(src_dir / src), *LINK, "-o", str(exe)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"building {name} failed: {' '.join(cmd)}\n{r.stdout}")
        built[name] = exe
    return built


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    for k, v in {**build_runtime_tests(a.verbose), **build_examples(a.reference, a.verbose)}.items():
        print(k, v)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
