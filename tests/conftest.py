"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    O.build()
    return O


def oracle_checker(configs, ctx):
    from oracle import oracle as O

    return O.Scene(ctx, np.asarray(configs).shape[1]).check_configs(configs, 0)


@pytest.fixture(scope="session")
def arm():
    from prrtc_b200 import scenes

    return scenes.arm(0)


@pytest.fixture(scope="session")
def dual():
    from prrtc_b200 import scenes

    return scenes.dual_arm(0)


def make_problem(kind, seed):
    from prrtc_b200 import scenes

    return scenes.make_problem(kind, seed, oracle_checker)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from prrtc_b200 import _lib, build

    build.build()  # no-op when the library is newer than every source; rebuilds a stale one
    _lib.load()
    return torch.device("cuda", 0)
