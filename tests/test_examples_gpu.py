"""The reference's own example programs — gemver-chain, ns-residual, getting-started — compiled unchanged against
this package's cs:: runtime (cospanmdao_b200.examples) and run with their own --check: every variant must report
ALL OK against the reference's host FP64 oracles (and, for gemver-chain, the variants must agree with each other the
way the reference requires: bitwise for unfused / parallel / fused)."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

EX = Path(__file__).resolve().parents[1] / "cospanmdao_b200" / "_examples"


def _run(args, timeout=300):
    exe = EX / args[0]
    if not exe.exists():
        pytest.fail(f"{exe} was not built (python -m cospanmdao_b200.examples)")
    r = subprocess.run([str(exe), *args[1:]], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=timeout)
    return r.returncode, r.stdout


def test_runtime_fused_groups(cuda):
    """The runtime's own fused-group cases (tests/runtime/fused_groups.cu): shared and partitioned local memory, a tie
    declared by the group, a stage without local memory in a launch that has some."""
    rc, out = _run(["runtime-fused-groups"])
    assert rc == 0 and "ALL OK" in out, out


def test_getting_started(cuda):
    rc, out = _run(["getting-started"])
    assert rc == 0, out
    assert out.split() == ["3", "5", "7", "9"], out


@pytest.mark.parametrize("variant", ["unfused", "parallel", "fused", "onepass", "naive", "crafted"])
def test_gemver_chain_variant(cuda, variant):
    rc, out = _run(["gemver-chain", "--n", "1024", "--R", "64", "--iters", "2", "--warmup", "1", "--variant", variant,
                    "--check"])
    assert rc == 0 and "ALL OK" in out, out


def test_gemver_chain_all_variants_agree(cuda):
    rc, out = _run(["gemver-chain", "--n", "512", "--R", "64", "--iters", "1", "--warmup", "1", "--check"])
    assert rc == 0 and "ALL OK" in out, out
    assert out.count("bitwise equal") >= 2, out


@pytest.mark.parametrize("bc", ["walls", "periodic"])
@pytest.mark.parametrize("variant", ["unfused", "fused"])
def test_ns_residual_variant(cuda, variant, bc):
    rc, out = _run(["ns-residual", "--nx", "128", "--ny", "96", "--iters", "2", "--warmup", "1", "--variant", variant,
                    "--bc", bc, "--check"])
    assert rc == 0 and "ALL OK" in out, out


def test_ns_residual_vanleer_fused(cuda):
    rc, out = _run(["ns-residual", "--nx", "64", "--ny", "64", "--iters", "1", "--warmup", "1", "--variant", "fused",
                    "--limiter", "vanleer", "--range-split", "all", "--check"])
    assert rc == 0 and "ALL OK" in out, out
