"""Shared test setup.

Markers: ``gpu`` for tests that need a CUDA device (run on a B200); everything
else runs on the CPU. The CPU checkers live under oracle/ (test infrastructure);
the product is libeu3d.so, reached through eu3d-gpu_b200/eu3d.py.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "eu3d-gpu_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# the reference checkout the oracle/_ref build compiles from (absent on GPU boxes)
REFERENCE = os.environ.get("EU3D_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _make(target_dir, *args):
    subprocess.run(["make", "-C", target_dir, *args], check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def port_lib():
    """The C restatement (built on demand; it needs only gcc)."""
    import oracle
    if not os.path.exists(oracle.PORT_LIB):
        _make(os.path.join(ROOT, "oracle"), "port")
    return oracle.PortOracle


@pytest.fixture(scope="session")
def ref_lib():
    """The reference's own CPU path (oracle/_ref). Built here when the reference
    checkout is present; it also travels prebuilt to GPU hosts."""
    import oracle
    if not os.path.exists(oracle.REF_LIB) and os.path.isdir(REFERENCE):
        _make(os.path.join(ROOT, "oracle"), "ref", f"REFERENCE={REFERENCE}")
    if not os.path.exists(oracle.REF_LIB):
        pytest.skip("oracle/_ref not built and the reference sources are not present")
    return oracle.RefOracle


@pytest.fixture(scope="session")
def eu3d_lib():
    import eu3d
    if not os.path.exists(eu3d.LIB_PATH):
        _make(os.path.join(ROOT, "eu3d-gpu_b200"), "-j4")
    return eu3d


def has_cuda_device():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu(eu3d_lib):
    if not has_cuda_device():
        pytest.fail("this test needs a CUDA device")
    return eu3d_lib
