"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def port_built():
    """Builds the C restatement of the oracle (gcc only) once per session."""
    import subprocess
    import oracle
    if not os.path.exists(oracle.PORT_LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True,
                       capture_output=True)
    return True


@pytest.fixture(scope="session")
def gpu_ctx():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from ktplace_b200.gpu import Context
    ctx = Context(0)
    yield ctx
    ctx.close()


def make_design(spec):
    from ktplace_b200 import synth, netlist
    raw = synth.generate(spec)
    return raw, netlist.flatten(raw)


def positions(raw, nl, seed):
    from ktplace_b200 import synth
    return synth.seed_positions(raw, nl.num_movable, seed)
