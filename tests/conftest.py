import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_sessionfinish(session, exitstatus):
    """Write the parity tests' measured errors when SF_PARITY_TABLE names a file."""
    path = os.environ.get("SF_PARITY_TABLE")
    if not path:
        return
    import json
    from tests.helpers import PARITY_TABLE
    if PARITY_TABLE:
        old = {}
        if os.path.exists(path):
            try:
                old = json.load(open(path))
            except ValueError:
                old = {}
        old.update(PARITY_TABLE)
        with open(path, "w") as fh:
            json.dump(old, fh, indent=1, sort_keys=True)
