"""Shared fixtures.  Tests marked gpu need a CUDA device and the built
library; everything else runs on the CPU."""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libr3d_b200.so")


@pytest.fixture(scope="session")
def rb():
    import render3d_b200
    return render3d_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def phantom256(rb):
    """The 256^3 scroll phantom of the single-GPU CPU-runnable workload."""
    return rb.phantom(256, seed=1234)


@pytest.fixture(scope="session")
def scroll_tf(rb):
    return rb.scroll_ramp_tf()


@pytest.fixture(scope="session")
def ctx(rb):
    c = rb.Context(0)
    yield c
    c.close()


def elev35(rb, lut, w=512, h=512, yaw=0.6, **kw):
    """Orbit view at 35 degrees elevation (camera above), distance 2."""
    return rb.camera_view(yaw, -35.0 * math.pi / 180.0, 2.0, w, h, lut, **kw)
