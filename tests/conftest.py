import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

GPU_LIB = os.path.join(ROOT, "sparselizard_b200", "_build", "libslz_gpu.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libslz_ref.so")
ENGINE_LIB = os.path.join(ROOT, "sparselizard_b200", "lib", "libslgpu.so")
ORACLE_LIB = os.path.join(ROOT, "oracle", "libslref.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def ref_lib():
    if not os.path.exists(REF_LIB):
        pytest.skip("reference build oracle/_ref/libslz_ref.so missing (run __graft_entry__.build())")
    return REF_LIB


@pytest.fixture(scope="session")
def gpu_lib():
    assert os.path.exists(GPU_LIB), "GPU drop-in not built (run __graft_entry__.build())"
    return GPU_LIB
