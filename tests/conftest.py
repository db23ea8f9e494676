import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mm-csf_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden_cases():
    import json
    gdir = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(gdir, "manifest.json")) as fh:
        names = json.load(fh)["cases"]
    cases = []
    for n in names:
        with open(os.path.join(gdir, n + ".json")) as fh:
            cases.append(json.load(fh))
    return cases
