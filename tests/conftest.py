import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def _ensure_built():
    from bulbit_b200 import build
    build.build()
    # Where the reference sources are present, bring the oracle (and the
    # drop-in test program, which links the product library) up to date.
    ref = os.environ.get("BULBIT_REFERENCE", "/root/reference")
    if os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", f"REF={ref}"], check=True,
                       stdout=subprocess.DEVNULL)


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    from oracle import ref
    if not ref.available():
        pytest.fail("oracle library missing (oracle/_ref/libbulbit_ref.so); build it with make -C oracle")
    ref.init(0)
    return ref


@pytest.fixture(scope="session")
def has_gpu():
    import torch
    return torch.cuda.is_available()
