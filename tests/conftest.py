import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle_libs():
    """Builds the oracle libraries if they are missing (the reference harness
    only where the reference sources exist)."""
    from oracle import bind
    if not os.path.exists(bind.ORC_LIB) or (
            bind.reference_sources_present() and not os.path.exists(bind.REF_LIB)):
        bind.build(reference=bind.reference_sources_present())
    return bind


@pytest.fixture(scope="session")
def ref_bind(oracle_libs):
    if not oracle_libs.have_reference():
        pytest.skip("reference harness not built (reference sources absent)")
    return oracle_libs


@pytest.fixture(autouse=True)
def _tmp_cwd(tmp_path, monkeypatch):
    """The reference's make_pair appends vapor in/out logs to the working
    directory (src/output/output.cpp:44-65); keep them out of the repo."""
    monkeypatch.chdir(tmp_path)
