"""GPU test of tpt_air_step_static_scratch, the air step for callers that
cannot allocate device memory (an engine whose memory all comes from its own
pool or graphics API, or code running where cudaMalloc is not allowed). It
takes its four scratch grids from an array inside the library instead of
from the caller.

Checked through the C ABI against tpt_air_step on the same inputs, two calls
in a row, with the bar the air tests use: bit-exact. Kept in its own file,
named to be collected last, and self-contained so it passes alone in a fresh
process as well as after the other tests."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_grids(tf, torch, inst, with_scratch):
    """SimBuffers-like grids of `inst`; without scratch the four scratch
    pointers stay NULL, as a caller that cannot allocate would pass them."""
    b = tf.SimBuffers.from_instance(inst)
    bufs = tf.air_bufs(b)
    if not with_scratch:
        bufs.opv = bufs.ovx = bufs.ovy = bufs.ohv = None
    return b, bufs


def _state(b):
    s = b.air_state()
    return {k: np.ascontiguousarray(v).view(np.uint32) for k, v in s.items()}


@pytest.mark.parametrize("which", ["c1", "stress", "noupdate"])
def test_static_scratch_step_matches_tpt_air_step(which):
    import torch

    import tpt_field as tf
    import workloads as W

    if not torch.cuda.is_available():
        pytest.fail("needs a CUDA device")
    if not __import__("os").path.exists(tf.LIB_PATH):
        tf.build()
    lib = tf.lib()
    if which == "c1":
        inst = W.config_instances(1)[0]
    elif which == "stress":
        inst = W.make_stress_instance(77, 45, 2024)
    else:
        inst = W.make_stress_instance(50, 37, 2025, config=W.AirConfig(air_mode=4))
    prm = tf.SimBuffers.from_instance(inst).config.air_params()

    ref, ref_bufs = _device_grids(tf, torch, inst, with_scratch=True)
    new, new_bufs = _device_grids(tf, torch, inst, with_scratch=False)
    stream = tf._stream(None)
    for call in range(2):
        assert lib.tpt_air_step(ctypes.byref(prm), ctypes.byref(ref_bufs), stream) == 0
        rc = lib.tpt_air_step_static_scratch(ctypes.byref(prm), ctypes.byref(new_bufs), stream)
        assert rc == 0, lib.tpt_last_error_string().decode()
        torch.cuda.synchronize()
        a, b = _state(ref), _state(new)
        for k in a:
            assert np.array_equal(a[k], b[k]), f"call {call + 1}: {k} differs"


def test_static_scratch_rejects_grids_over_the_limit():
    import torch

    import tpt_field as tf

    if not torch.cuda.is_available():
        pytest.fail("needs a CUDA device")
    lib = tf.lib()
    prm = tf.AirParams()
    lib.tpt_air_params_default(ctypes.byref(prm), 600, 600)  # 360000 cells > 512*512
    bufs = tf.AirBufs()
    rc = lib.tpt_air_step_static_scratch(ctypes.byref(prm), ctypes.byref(bufs), None)
    assert rc == -1
    assert b"static scratch" in lib.tpt_last_error_string()
