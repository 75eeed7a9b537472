"""Test configuration: the `gpu` marker, import paths and shared fixtures.

`-m "not gpu"` runs the oracle pins, host logic and ABI checks on CPU;
`-m gpu` runs the parity tests through the C ABI on an sm_100 device.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "the-powder-toy-rust-wgpu_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU and the built CUDA library")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def tf():
    """The product's host module with its CUDA library loaded."""
    import tpt_field

    if not os.path.exists(tpt_field.LIB_PATH):
        tpt_field.build()
    tpt_field.lib()
    return tpt_field


@pytest.fixture(scope="session")
def cuda(tf):
    import torch

    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    major, minor = torch.cuda.get_device_capability()
    assert (major, minor) == (10, 0), f"need sm_100, got sm_{major}{minor}"
    return torch
