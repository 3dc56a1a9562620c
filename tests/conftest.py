import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture
def golden():
    from mac_b200.state import State

    def load(name):
        return State.load_npz(os.path.join(GOLDEN, name + ".npz"))
    return load


@pytest.fixture
def run_oracle(oracle_lib, tmp_path):
    """Runs an oracle stage on a State and returns (State, stats)."""
    from mac_b200.state import State
    counter = [0]

    def run(cmd, s, n=1, rtol=1e-14):
        counter[0] += 1
        src = str(tmp_path / f"in{counter[0]}.state")
        dst = str(tmp_path / f"out{counter[0]}.state")
        s.write(src)
        stats = oracle_lib.run_oracle(cmd, src, dst, n, rtol)
        return State.read(dst), stats
    return run
