import os
import sys

import pytest

# The oracle's mixture loops use schedule(runtime), as the reference does
# (int_ion_mix.f:159,223); with OMP_SCHEDULE unset, libgomp schedules them
# dynamically with chunks of one iteration, which makes a full-size call take
# a minute.  Set before the oracle's OpenMP runtime is loaded.
os.environ.setdefault("OMP_SCHEDULE", "static")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Build the engine library and the CPU oracle if they are missing."""
    from yukawamd_b200 import build as ybuild
    from oracle import oracle as orc
    ybuild.build()
    if not (os.path.exists(os.path.join(ROOT, "oracle", "liborc.so"))
            and os.path.exists(os.path.join(ROOT, "oracle", "liborc_ld.so"))):
        orc.build()
    return True


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA GPU")
    return torch.cuda.get_device_name(0)
