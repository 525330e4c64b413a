import os
import sys

import pytest

# the oracle's OpenMP loops on one thread: every sum in loop order, so its
# results are reproducible bit for bit (set before the library loads)
os.environ["OMP_NUM_THREADS"] = "1"

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built hsolver_b200 extension")


def deck_path(name):
    return os.path.join(GOLDEN, "decks", name + ".in")


def read_deck(name):
    with open(deck_path(name)) as f:
        return f.read()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle
