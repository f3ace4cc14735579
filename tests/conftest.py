import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: long-running")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device on this host")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def _gpu_present() -> bool:
    """True if this host has an NVIDIA GPU by any of three independent signs: the driver's
    device nodes, the CUDA runtime's device count, torch. Torch is not required to answer."""
    import glob
    if os.path.exists("/dev/nvidiactl") or glob.glob("/dev/nvidia[0-9]*"):
        return True
    import ctypes
    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            rt = ctypes.CDLL(name)
        except OSError:
            continue
        n = ctypes.c_int(0)
        if rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0:
            return True
        break
    return _cuda_available()


@pytest.fixture
def host_only():
    """For tests that hand the library fake device addresses to see its host-side checks
    reject them: they run only where no GPU is present. A call that a check let through would
    reach a kernel launch, which fails harmlessly without a device but would touch those
    addresses on a GPU."""
    if _gpu_present():
        pytest.skip("fake device addresses are passed only on hosts without a GPU")


@pytest.fixture(scope="session")
def p2r():
    import p2r_tests_b200 as m
    m.lib()  # raises if the library is missing: there is no fallback path
    return m


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden_dir():
    return ROOT / "tests" / "golden"
