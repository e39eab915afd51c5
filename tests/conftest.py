"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


def load_golden(name: str):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


_verifiers = {}


@pytest.fixture(scope="session")
def verifier():
    """verifier(N) -> a cached collatz_b200.Verifier for MAXBITS = N."""
    import collatz_b200 as cb

    def get(maxbits: int = 45, **kw):
        key = (maxbits, tuple(sorted(kw.items())))
        if key not in _verifiers:
            _verifiers[key] = cb.Verifier(maxbits, **kw)
        return _verifiers[key]

    yield get
    for v in _verifiers.values():
        v.close()
    _verifiers.clear()


_tables = {}


@pytest.fixture(scope="session")
def oracle_tables():
    """oracle_tables(N) -> cached oracle.Tables (CPU restatement of precompute)."""
    from oracle import oracle as O

    def get(maxbits: int):
        if maxbits not in _tables:
            _tables[maxbits] = O.Tables(maxbits)
        return _tables[maxbits]

    return get
