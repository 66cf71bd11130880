"""The reference's own example programs — gemver-chain, ns-residual, getting-started — compiled unchanged against
this package's cs:: runtime (cospanmdao_b200.examples) and run with their own --check: every variant must report
ALL OK against the reference's host FP64 oracles (and, for gemver-chain, the variants must agree with each other the
way the reference requires: bitwise for unfused / parallel / fused)."""
import os
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

EX = Path(__file__).resolve().parents[1] / "cospanmdao_b200" / "_examples"


def _run(args, timeout=300, env=None):
    exe = EX / args[0]
    if not exe.exists():
        pytest.fail(f"{exe} was not built (python -m cospanmdao_b200.examples)")
    full_env = dict(os.environ, **(env or {}))
    r = subprocess.run([str(exe), *args[1:]], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=timeout, env=full_env)
    return r.returncode, r.stdout


# "fast": the runtime's registered fast paths (patterns.hpp) run the whole gemver chain as one cspb kernel;
# "generic": every component runs its own body (NAGA_COSPAN_GENERIC); "eager": the fast paths with no CUDA-graph
# replay of steady forwards (NAGA_COSPAN_NO_GRAPH)
MODES = {"fast": {}, "generic": {"NAGA_COSPAN_GENERIC": "1"}, "eager": {"NAGA_COSPAN_NO_GRAPH": "1"}}


def test_runtime_fused_groups(cuda):
    """The runtime's own fused-group cases (tests/runtime/fused_groups.cu): shared and partitioned local memory, a tie
    declared by the group, a stage without local memory in a launch that has some."""
    rc, out = _run(["runtime-fused-groups"])
    assert rc == 0 and "ALL OK" in out, out


def test_runtime_ragged(cuda):
    """Ragged ports and counts_from / offsets_from hooks (tests/runtime/ragged.cu): device-built columns over forwards
    with changing counts, declared counts at connects, dense rows read as blocks, the hook's error flags, host views,
    and ragged stages inside a fused group (the reference refuses those)."""
    rc, out = _run(["runtime-ragged"])
    assert rc == 0 and "ALL OK" in out, out


def test_runtime_replay(cuda):
    """CUDA-graph replay of steady forwards (tests/runtime/replay.cu): captured after one steady forward, replayed
    bit-identical to eager forwards, dropped by update_input, never used for a model whose hooks read the device."""
    rc, out = _run(["runtime-replay"])
    assert rc == 0 and "ALL OK" in out, out


def test_runtime_ragged_u64_offsets(cuda):
    """A ragged variable of 2^32 + 11 elements: counts_from<std::uint64_t> (and host counts past 2^32 - 1) place every
    block where its u64 offset says; the default u32 column refuses the total with an error naming the u64 form."""
    rc, out = _run(["runtime-ragged-wide"])
    assert rc == 0 and "ALL OK" in out, out[-3000:]


def test_runtime_decoy_component_not_replaced(cuda):
    """A component named Gemv with the reference's ports and wiring but other arithmetic is not replaced by the GEMVER
    kernel: the first forward compares kernel and bodies, and only the honest system keeps the kernel."""
    rc, out = _run(["runtime-decoy"], env={"NAGA_COSPAN_TRACE": "1"})
    assert rc == 0 and "ALL OK" in out, out[-3000:]
    assert "agrees with the components' own bodies" in out, out[-3000:]
    assert "not used: the kernel and the components' own bodies differ in" in out, out[-3000:]


def test_getting_started(cuda):
    rc, out = _run(["getting-started"])
    assert rc == 0, out
    assert out.split() == ["3", "5", "7", "9"], out


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("variant", ["unfused", "parallel", "fused", "onepass", "naive", "crafted"])
def test_gemver_chain_variant(cuda, variant, mode):
    rc, out = _run(["gemver-chain", "--n", "1024", "--R", "64", "--iters", "2", "--warmup", "1", "--variant", variant,
                    "--check"], env=MODES[mode])
    assert rc == 0 and "ALL OK" in out, out


@pytest.mark.parametrize("mode", sorted(MODES))
def test_gemver_chain_all_variants_agree(cuda, mode):
    rc, out = _run(["gemver-chain", "--n", "512", "--R", "64", "--iters", "1", "--warmup", "1", "--check"],
                   env=MODES[mode])
    assert rc == 0 and "ALL OK" in out, out
    assert out.count("bitwise equal") >= 2, out


def test_gemver_chain_fast_paths_engage(cuda):
    """Every style runs the whole chain as one cspb_gemver_chain call (six matrix passes): the unfused, parallel,
    fused, onepass and naive styles as a GEMVER run, a BiCGK run and a GEMVER run; the crafted style as its three
    groups (G1, BiCGK with G2's update from the same tile, G2's products)."""
    for variant in ("unfused", "parallel", "fused", "onepass", "naive", "crafted"):
        rc, out = _run(["gemver-chain", "--n", "512", "--R", "64", "--iters", "1", "--warmup", "1", "--variant",
                        variant], env={"NAGA_COSPAN_TRACE": "1"})
        assert rc == 0, out
        assert out.count("fast path cspb_gemver_chain") >= 1, (variant, out[-2000:])
        assert "fast path cspb_gemver_fused" not in out and "fast path cspb_bicgk_fused" not in out, variant


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("bc", ["walls", "periodic"])
@pytest.mark.parametrize("variant", ["unfused", "fused"])
def test_ns_residual_variant(cuda, variant, bc, mode):
    rc, out = _run(["ns-residual", "--nx", "128", "--ny", "96", "--iters", "2", "--warmup", "1", "--variant", variant,
                    "--bc", bc, "--check"], env=MODES[mode])
    assert rc == 0 and "ALL OK" in out, out


@pytest.mark.parametrize("mode", sorted(MODES))
def test_ns_residual_vanleer_fused(cuda, mode):
    rc, out = _run(["ns-residual", "--nx", "64", "--ny", "64", "--iters", "1", "--warmup", "1", "--variant", "fused",
                    "--limiter", "vanleer", "--range-split", "all", "--check"], env=MODES[mode])
    assert rc == 0 and "ALL OK" in out, out


def test_ns_residual_fast_path_engages(cuda):
    for variant in ("unfused", "fused"):
        rc, out = _run(["ns-residual", "--nx", "128", "--ny", "128", "--iters", "1", "--warmup", "1", "--variant",
                        variant], env={"NAGA_COSPAN_TRACE": "1"})
        assert rc == 0, out
        assert "fast path cspb_ns_compressible 128x128" in out, (variant, out[-2000:])
