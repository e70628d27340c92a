import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def reference_root():
    """The reference checkout for tests that read its data files: the
    ICEMPM_REFERENCE environment variable, else the location that
    oracle/build_ref.sh recorded when it built oracle/_ref; None when
    neither names an existing directory (the tests then skip)."""
    root = os.environ.get("ICEMPM_REFERENCE")
    if not root:
        rec = os.path.join(ROOT, "oracle", "_ref", "reference_root")
        if os.path.exists(rec):
            with open(rec) as f:
                root = f.read().strip()
    return root if root and os.path.isdir(root) else None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the in-tree libraries if their sources are newer (no-op when
    prebuilt, as on a GPU box that received the built files)."""
    from icempm_b200 import build

    try:
        build.build_lib()
    except Exception:
        if not os.path.exists(build.LIB):
            raise
    try:
        build.build_oracle()
    except Exception:
        if not os.path.exists(os.path.join(ROOT, "oracle", "libmpm_oracle.so")):
            raise
    yield
