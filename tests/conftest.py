import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

GOLDEN = os.path.join(ROOT, "tests", "golden")
# cases stored in the reference's file formats (the regenerated r = 64 cases of
# tests/golden/large_cases.py keep only a spec and are collected separately)
CASES = sorted(d for d in os.listdir(GOLDEN) if os.path.exists(os.path.join(GOLDEN, d, "golden.json"))
               and os.path.exists(os.path.join(GOLDEN, d, "user_parameters")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built CUDA library")


@pytest.fixture(params=CASES)
def case_dir(request):
    return os.path.join(GOLDEN, request.param)
