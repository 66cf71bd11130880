"""The C ABI without a GPU: the library loads, exports every function include/cspb.h declares, sizes workspaces
sanely, and rejects bad arguments before touching CUDA."""
import ctypes as C
import re
from pathlib import Path

import pytest

import cospanmdao_b200 as cb
from cospanmdao_b200 import _capi

HEADER = Path(__file__).resolve().parents[1] / "include" / "cspb.h"


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cspb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = cb.lib()
    names = declared()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python view knows every one of them
    assert set(names) <= set(_capi.PROTOTYPES), set(names) - set(_capi.PROTOTYPES)


def test_header_flags_match_the_python_view():
    """Every CSPB_ flag and device status bit the header defines has the same value in the Python view."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    defs = dict(re.findall(r"#define CSPB_([A-Z0-9_]+) \(?([0-9a-fx <u]+?)\)?\s*$", text, flags=re.M))
    want = {"DEV_TIMEOUT", "DEV_NEGATIVE", "DEV_EXCEEDS32", "DEV_CAPACITY", "DEV_ARGUMENT", "GEMVER_PANEL",
            "GEMVER_BULK", "GEMVER_LOWRANK", "BATCH_LOWRANK", "BATCH_NO_B", "COLUMN_NEGATIVE", "COLUMN_EXCEEDS32",
            "COLUMN_TIMEOUT"}
    assert want <= set(defs), want - set(defs)
    for name in want:
        assert eval(defs[name].replace("u", "")) == getattr(_capi, name), name


def test_version_and_status_strings():
    assert "sm_100a" in cb.version()
    lib = cb.lib()
    for code in range(9):
        assert lib.cspb_status_string(code)
    assert lib.cspb_status_string(99) == b"unknown status"


def test_workspace_sizes():
    lib = cb.lib()
    for f in (lib.cspb_gemver_workspace_bytes, lib.cspb_bicgk_workspace_bytes, lib.cspb_chain_workspace_bytes):
        assert f(0) == 0
        prev = 0
        for n in (1, 7, 256, 1000, 4096, 16384):
            b = f(n)
            assert b % 256 == 0 and b >= prev
            prev = b
    # GEMVER at n = 16384: the f64 column partials (n/128 strips) dominate, well under 1% of the matrix
    assert lib.cspb_gemver_workspace_bytes(16384) < 24 * 2 ** 20
    assert lib.cspb_scan_workspace_bytes(0) >= 256
    assert lib.cspb_ns_incomp_workspace_bytes(2, 2) == 0
    assert lib.cspb_ns_incomp_workspace_bytes(4096, 4096) > 256
    # one call's workspace serves either storage type: room for the control block and 3 f64 norm partials per tile
    # of the f32 tiles (128 x 32 cells) and of the bf16 tiles (512 x 16), whichever there are more of (a grid 8 wide
    # and 10000 tall has 313 f32 tiles and 625 bf16 ones)
    import math
    for nx, ny in ((8, 10000), (4096, 4096), (520, 17), (8, 3), (12000, 40)):
        tiles = max(math.ceil(nx / 128) * math.ceil(ny / 32), math.ceil(nx / 512) * math.ceil(ny / 16))
        assert lib.cspb_ns_incomp_workspace_bytes(nx, ny) >= 256 + 24 * tiles, (nx, ny)
    # the compressible residual: the control block, one u32 count per group of 256 tiles of 32 x 15 cells, and the
    # tile and group partials (4 B + 4 B + 32 B each)
    for nx, ny in ((4096, 4096), (32, 3855), (64, 48)):
        tiles = math.ceil(nx / 32) * math.ceil(ny / 15)
        groups = math.ceil(tiles / 256)
        assert lib.cspb_ns_comp_workspace_bytes(nx, ny) >= 256 + 4 * groups + 40 * tiles + 40 * groups, (nx, ny)


def test_arguments_are_rejected_before_cuda():
    lib = cb.lib()
    assert lib.cspb_gemver_fused(None, None) == _capi.ERR_ARGUMENT
    d = _capi.GemverDesc()
    d.n = 0
    assert lib.cspb_gemver_fused(C.byref(d), None) == _capi.ERR_ARGUMENT
    d.n, d.lda, d.ldb = 8, 8, 8
    fake = 0x1000
    for f in ("A", "u1", "v1", "u2", "v2", "y", "x", "w"):
        setattr(d, f, fake)
    d.a_dtype = 7
    assert lib.cspb_gemver_fused(C.byref(d), None) == _capi.ERR_UNSUPPORTED
    d.a_dtype = _capi.F32
    d.lda = 4
    assert lib.cspb_gemver_fused(C.byref(d), None) == _capi.ERR_ARGUMENT
    d.lda = 8
    d.workspace, d.workspace_bytes = 0x100, 16
    assert lib.cspb_gemver_fused(C.byref(d), None) == _capi.ERR_WORKSPACE
    d.workspace = 0x101  # misaligned
    d.workspace_bytes = 1 << 30
    assert lib.cspb_gemver_fused(C.byref(d), None) == _capi.ERR_WORKSPACE
    assert lib.cspb_bicgk_fused(None, None) == _capi.ERR_ARGUMENT
    assert lib.cspb_gemver_chain(None, None) == _capi.ERR_ARGUMENT
    assert lib.cspb_exclusive_scan_u32(None, None, -1, None, 0, None) == _capi.ERR_ARGUMENT
    assert lib.cspb_exclusive_scan_u64(fake, None, 4, None, 0, None) == _capi.ERR_ARGUMENT
    assert lib.cspb_build_column(fake, 9, 4, 1, 0, fake, fake, fake, None, 0, None) == _capi.ERR_UNSUPPORTED
    assert lib.cspb_build_column(fake, 0, 0, 1, 1, fake, fake, fake, None, 0, None) == _capi.ERR_ARGUMENT
    nd = _capi.NsIncompDesc()
    nd.nx, nd.ny = 2, 8
    assert lib.cspb_ns_incompressible(C.byref(nd), None) == _capi.ERR_ARGUMENT
    assert lib.cspb_fill_hash(fake, 0, 10, 0, 1, 5, None) == _capi.ERR_ARGUMENT


def test_python_view_raises_value_errors_like_the_reference():
    # port checks happen before any device work
    with pytest.raises(ValueError):
        cb.gemver(None, None, None, None, None, None, alpha=1.0, beta=1.0)
    with pytest.raises(ValueError, match="limiter"):
        cb.ns_compressible(None, limiter="superbee")
    with pytest.raises(ValueError, match="bc"):
        cb.ns_compressible(None, bc="open")
