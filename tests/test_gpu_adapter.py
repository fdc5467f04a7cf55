"""The C++ adapter (CudaEngine : DecisionEngine, celv2_b200/host/cuda_engine.cpp) run through the
reference's own interface and RowGate against the reference's CpuEngine and rules.

The test program (tests/cpp/test_cuda_engine.cpp) links the reference's sources, so it is built
where they are present (oracle/Makefile, target adapter-test) and travels prebuilt."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_cuda_engine")


def test_adapter_matches_reference_cpu_engine():
    if not os.path.exists(BIN):
        pytest.skip("the adapter test program was not built (the reference's sources were absent)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all adapter cases passed" in r.stdout
