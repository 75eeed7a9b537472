"""Failure detection on the GPU without a fault: a bounded device wait that
nothing completes gives up after its limit, the library's error word reports
TPT_ERR_DEVICE_TIMEOUT once (then it is cleared), and the context stays
usable: a batch steps bit-exactly afterwards. No kernel traps, faults or
waits without a bound."""
import pytest

pytestmark = pytest.mark.gpu

TPT_ERR_DEVICE_TIMEOUT = -4


def test_bounded_wait_timeout_is_reported_and_cleared(cuda, tf, oracle):
    from test_gpu_batch import check_against_oracle, mixed_instances

    L = tf.lib()
    assert L.tpt_check_device_errors() == 0
    assert L.tpt_selftest_wait_timeout(1 << 22, None) == 0  # about 2 ms of SM clocks
    assert L.tpt_check_device_errors() == TPT_ERR_DEVICE_TIMEOUT
    assert "timed out" in L.tpt_last_error_string().decode()
    assert L.tpt_check_device_errors() == 0  # read and cleared
    insts = mixed_instances()[:2]
    b = tf.Batch(insts)
    b.step(3)
    cuda.cuda.synchronize()
    assert L.tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, 3, "after a timed-out wait")
    b.close()
