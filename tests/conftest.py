import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# the reference checkout: CUTS_REFERENCE_DIR, else "reference" beside the repository
REF_DIR = os.environ.get("CUTS_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the engine and the oracle once per session (no-op when fresh)."""
    import subprocess
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "cuts_b200", "csrc")],
                   check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    yield


def have_reference() -> bool:
    return os.path.isdir(REF_DIR)
