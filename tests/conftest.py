import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pennant-legion_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
DECKS = os.path.join(PKG, "decks")

for p in (PKG, os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running case")


def golden(name: str) -> str:
    return os.path.join(GOLDEN, name)


def deck(name: str) -> str:
    return os.path.join(DECKS, name)
