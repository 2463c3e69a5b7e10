"""The built diagnostics behind the tensor-core gridders' design: probe_tcgen05_mma checks the
MN-major no-swizzle operand layouts (FP16, and unsigned x signed 8-bit as the integer gridder uses
them) exactly against a host product and measures tcgen05.mma issue rates; probe_shared_red
measures shared-memory reduction rates. Both print their figures (pytest -s shows them)."""
import os
import subprocess

import pytest

from svdimager_b200 import build

pytestmark = pytest.mark.gpu


def _run(name):
    exe = os.path.join(build.BIN_DIR, name)
    assert os.path.exists(exe), f"{exe} missing: run svdimager_b200/build.py"
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    return r


def test_tcgen05_operand_layouts_and_rates(cuda_device):
    r = _run("probe_tcgen05_mma")
    assert r.returncode == 0, r.stdout + r.stderr
    checks = [l for l in r.stdout.splitlines() if l.startswith("layout check")]
    assert len(checks) == 2
    for l in checks:
        assert "wait status 0, mismatched cells 0 of" in l, l
    assert any(l.startswith("rate u8s8 M 128 N  96") for l in r.stdout.splitlines())


def test_shared_reduction_rates(cuda_device):
    r = _run("probe_shared_red")
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("done")
