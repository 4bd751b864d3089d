import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
SAMPLE = os.path.join(GOLDEN, "sample")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def sample_graph():
    import scout_b200 as sb
    off, adj, wide = sb.read_egr(os.path.join(SAMPLE, "sample.egr"))
    return off, adj


@pytest.fixture(scope="session")
def sample_batches():
    import scout_b200 as sb
    return [sb.parse_batch_file(os.path.join(SAMPLE, "batches", f"{k}.mtx"), 2000) for k in range(1, 6)]


@pytest.fixture(scope="session")
def rmat16():
    import scout_b200 as sb
    g = sb.gen_rmat(16, 16, seed=1)
    return g, g.arrays()
