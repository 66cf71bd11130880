"""Build-time annotation of CoSpan sources for nvcc.

A SYCL compiler compiles any function a kernel calls for the device. nvcc compiles for the device only what is
marked __device__ (and has no switch like clang's `#pragma clang force_cuda_host_device`). This pass marks, in a
COPY of a CoSpan program's sources, the functions its kernels call, so that the program compiles unchanged against
cospanmdao_b200/include with nvcc:

  - every component body `static void compute_forward(`                         -> __host__ __device__
  - namespace-scope `inline` functions and `template <...> inline` functions      -> __host__ __device__
    (numeric helpers: index arithmetic, physics, tile stages), except those returning std::vector / std::string
  - static member function templates `template <class T> static T name(`         -> __host__ __device__
  - lambdas handed to the device, `[=](sycl::id<..>` / `[=](sycl::nd_item<..>`     -> [=] __host__ __device__ (...)
  - a namespace-scope `auto f(` whose body returns `cs::init::custom<...>(...)`   -> naga::cospan::InitSpec f(
    (nvcc compiles no device lambda inside a function with a deduced return type; the type is spelled out)

Lambdas defined inside an annotated function take its execution space, so they need nothing. Files that are host-only
by design (the FP64 host references, the shared data generator) are copied as they are.
"""
from __future__ import annotations

import re
import shutil
from pathlib import Path

HD = "__host__ __device__ "

_RE_BODY = re.compile(r"(?<![\w])static\s+void\s+compute_forward\s*\(")
_RE_INLINE = re.compile(r"^(\s*(?:template\s*<[^>]*>\s*)?)inline\s+(?!namespace)(?P<ret>[\w:<>,\s\*&]+?)\s+(?P<name>\w+)\s*\(",
                        re.M)
_RE_STATIC_TMPL = re.compile(r"^(\s*template\s*<[^>]*>\s*)static\s+(?=[\w:<>]+\s+\w+\s*\()", re.M)
_RE_LAMBDA = re.compile(r"\[=\]\s*\((?=\s*sycl::(?:id|nd_item)\s*<)")
_RE_AUTO_INIT = re.compile(r"^auto\s+(\w+)\s*\(([^)]*)\)\s*\{\s*\n\s*return\s+(?:cs|naga::cospan)::init::custom<", re.M)


def annotate_text(text: str) -> str:
    text = _RE_BODY.sub(lambda m: HD + m.group(0), text)

    def inline_sub(m: re.Match) -> str:
        ret = m.group("ret")
        if "std::vector" in ret or "std::string" in ret or "__device__" in ret:
            return m.group(0)
        return m.group(1) + HD + "inline " + ret + " " + m.group("name") + "("
    text = _RE_INLINE.sub(inline_sub, text)
    text = _RE_STATIC_TMPL.sub(lambda m: m.group(1) + HD + "static ", text)
    text = _RE_LAMBDA.sub("[=] " + HD + "(", text)
    text = _RE_AUTO_INIT.sub(lambda m: m.group(0).replace("auto " + m.group(1), "naga::cospan::InitSpec " + m.group(1), 1),
                             text)
    # undo double marks, if a source already had them
    text = text.replace(HD + HD, HD)
    return text


def annotate_tree(src: Path, dst: Path, host_only=("reference.hpp", "chain_data.hpp")) -> list[Path]:
    """Copies every .hpp/.cpp under src to dst, annotating all but the host-only files. Returns the written files."""
    out = []
    for f in sorted(src.rglob("*")):
        if f.suffix not in (".hpp", ".cpp", ".h") or not f.is_file():
            continue
        rel = f.relative_to(src)
        target = dst / rel
        target.parent.mkdir(parents=True, exist_ok=True)
        if f.name in host_only:
            shutil.copyfile(f, target)
        else:
            target.write_text(annotate_text(f.read_text()))
        out.append(target)
    return out
