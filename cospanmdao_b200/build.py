"""Builds libcspb.so (the sm_100a kernels behind include/cspb.h) in-tree with nvcc.

    python -m cospanmdao_b200.build            # build if any source is newer than the library
    python -m cospanmdao_b200.build --force    # rebuild

The library is written next to this file so that it travels with the source tree; nothing is installed.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libcspb.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["capi.cu", "gemver.cu", "scan.cu", "ns_incomp.cu", "ns_comp.cu", "batched.cu"]


def nvcc() -> str:
    cand = os.environ.get("CSPB_NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists() and shutil.which(cand) is None:
        raise RuntimeError("nvcc not found: set CSPB_NVCC or put CUDA's bin directory on PATH")
    return cand


def sources() -> list[Path]:
    return [CSRC / s for s in SOURCES if (CSRC / s).exists()]


def deps() -> list[Path]:
    return sources() + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "cspb.h"]


def stale(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps())


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compiles every source to an object (in parallel) and links libcspb.so. Returns its path."""
    if not force and not stale():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
                    "--expt-relaxed-constexpr"]
    cmds = []
    objs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        objs.append(obj)
        cmds.append([nvcc(), *flags, "-c", str(src), "-o", str(obj)])
    procs = []
    for c in cmds:
        if verbose:
            print(" ".join(c), file=sys.stderr)
        procs.append(subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    failed = []
    for c, p in zip(cmds, procs):
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((c, out))
        elif verbose and out:
            print(out, file=sys.stderr)
    if failed:
        msg = "\n".join(" ".join(c) + "\n" + out for c, out in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    tmp = LIB.with_suffix(".so.tmp")
    # cudart is linked statically: the library carries the runtime it was compiled against, and shares the device's
    # primary context (and so torch's allocations and streams) through the driver.
    link = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp)]
    r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + " ".join(link) + "\n" + r.stdout)
    os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
