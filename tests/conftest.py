import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def restated():
    from oracle.bridge import Restated

    return Restated()


@pytest.fixture(scope="session")
def reference():
    from oracle import bridge

    if not bridge.reference_available():
        try:
            bridge.build(reference=True)
        except Exception:
            pass
    if not bridge.reference_available():
        pytest.skip("compiled FIR reference (oracle/_ref) not available")
    return bridge.Reference()


@pytest.fixture(scope="session")
def gpu_ctx_factory():
    """Creates fir_b200 contexts on cuda:0 (GPU tests only)."""
    from fir_b200 import capi

    made = []

    def make(scanner=None, **opts):
        c = capi.Context(scanner)
        for k, v in opts.items():
            c.set_option(k, v)
        made.append(c)
        return c

    yield make
    for c in made:
        c.close()
