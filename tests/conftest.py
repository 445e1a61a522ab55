import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    if not O.ORACLE_SO.exists():
        O.build()
    return O


@pytest.fixture(scope="session")
def native():
    from tim_raytracing_b200 import _native as N
    if not N.LIB_PATH.exists():
        from tim_raytracing_b200 import build
        build.build()
    return N


@pytest.fixture(scope="session")
def ctx(native):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = native.Context(0)
    yield c
    c.close()


@pytest.fixture
def tmp_path(request):
    """Scratch folder inside the repository (tests/_tmp/<test>, git-ignored),
    replacing pytest's system-wide temporary directory."""
    import re
    import shutil
    d = ROOT / "tests" / "_tmp" / re.sub(r"[^\w.-]", "_", request.node.name)
    if d.exists():
        shutil.rmtree(d)
    d.mkdir(parents=True)
    return d
