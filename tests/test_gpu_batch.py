"""GPU parity of batched instances (tpt_batch_* through the C ABI): a batch
of uneven grids in different modes, stepped through captured CUDA graphs,
must give per instance exactly what the single-grid step gives: bit-exact
air against the FP32 oracle, gravity within the FP32 plan's tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mixed_instances():
    import workloads as W

    insts = [
        W.make_instance(53, 41, 11, mass_density=0.02),
        W.make_instance(120, 33, 12, mass_density=0.02),
        W.make_stress_instance(70, 64, 13),
        W.make_stress_instance(32, 90, 14, config=W.AirConfig(air_mode=4)),
        W.make_stress_instance(45, 45, 15, config=W.AirConfig(aheat_enable=0, convection_mode=1)),
        W.make_stress_instance(64, 40, 16, config=W.AirConfig(gravity_mode=2, newton_grav=0)),
    ]
    return insts


def check_against_oracle(tf, oracle, batch, insts, ticks, ctx):
    from test_gpu_air import assert_bit_exact

    for i, inst in enumerate(insts):
        got = batch.state(i)
        want = oracle.air_steps(inst, ticks)
        assert_bit_exact(got, want, f"{ctx} instance {i}")
        if inst.config.newton_grav:
            dx, dy = oracle.grav_solve(inst.xcells, inst.ycells, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
            scale = max(np.abs(dx).max(), np.abs(dy).max(), 1e-30)
            assert np.abs(got["gx"] - dx).max() <= 1e-5 * scale
            assert np.abs(got["gy"] - dy).max() <= 1e-5 * scale
        else:
            assert not got["gx"].any() and not got["gy"].any()


@pytest.mark.parametrize("ticks", [1, 7, 50, 57])
def test_batch_matches_single_grid_oracle(cuda, tf, oracle, ticks):
    insts = mixed_instances()
    b = tf.Batch(insts)
    b.step(ticks)
    cuda.cuda.synchronize()
    check_against_oracle(tf, oracle, b, insts, ticks, f"{ticks} ticks")
    b.close()


def test_batch_graph_replay_and_continuation(cuda, tf, oracle):
    insts = mixed_instances()
    b = tf.Batch(insts)
    b.step(3)
    b.step(3)   # replays the cached 3-tick graph
    b.step(4)
    cuda.cuda.synchronize()
    check_against_oracle(tf, oracle, b, insts, 10, "3+3+4")
    b.close()


def test_tune_keeps_state_and_results(cuda, tf, oracle):
    insts = mixed_instances()
    b = tf.Batch(insts)
    b.tune()
    t = b.tuning()
    assert t.ctas_per_sm in (1, 2, 3, 4, 6, 8) and t.temporal_depth == 1
    b.step(5)
    cuda.cuda.synchronize()
    check_against_oracle(tf, oracle, b, insts, 5, "tuned")
    b.close()


def test_batch_measured_config_subset(cuda, tf, oracle):
    import workloads as W

    insts = W.config_instances(4, limit=12)
    b = tf.Batch(insts)
    b.step(20)
    cuda.cuda.synchronize()
    check_against_oracle(tf, oracle, b, insts, 20, "C4 subset")
    b.close()


def test_c4_every_instance_20_ticks(cuda, tf, oracle):
    """The whole C4 batch (256 instances, W, H log-uniform 32..512, FP32
    gravity) after 20 ticks: every instance's air bit-exact against the
    oracle and its gx/gy within 1e-5 of max|g| against FP64."""
    import workloads as W

    insts = W.config_instances(4)
    assert len(insts) == 256
    b = tf.Batch(insts)
    b.step(20)
    cuda.cuda.synchronize()
    assert tf.lib().tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, 20, "C4")
    b.close()


def test_batch_field_io_round_trip(cuda, tf):
    import workloads as W

    insts = [W.make_instance(40, 30, 1, mass_density=0.02), W.make_instance(33, 35, 2, mass_density=0.02)]
    b = tf.Batch(insts)
    for i, inst in enumerate(insts):
        assert np.array_equal(b.read(i, tf.FIELD_PV, np.float32), inst.pv)
        assert np.array_equal(b.read(i, tf.FIELD_WALL_BMAP, np.uint32), inst.wall)
        assert np.array_equal(b.read(i, tf.FIELD_GRAV_MASS, np.int32), inst.mass_fx)
    f0, f1 = b.fields(0), b.fields(1)
    assert f0.pv % 256 == 0 and f1.pv % 256 == 0 and f1.pv > f0.pv
    with pytest.raises(tf.TptError):
        b.read(5, tf.FIELD_PV, np.float32)
    with pytest.raises(tf.TptError):
        b.write(0, 99, insts[0].pv)
    b.close()


def test_batch_whole_field_io_matches_per_instance(cuda, tf):
    """tpt_batch_write_field / tpt_batch_read_field against the per-instance
    calls, on uneven grids (row lengths off the 32-element pitch)."""
    insts = mixed_instances()
    b = tf.Batch(insts)  # written through tpt_batch_write_field
    for i, inst in enumerate(insts):
        assert np.array_equal(b.read(i, tf.FIELD_PV, np.float32), inst.pv)
        assert np.array_equal(b.read(i, tf.FIELD_WALL_EMAP, np.uint32), inst.emap)
        assert np.array_equal(b.read(i, tf.FIELD_GRAV_MASS, np.int32), inst.mass_fx)
    total = sum(i.cells for i in insts)
    assert b.total_cells == total
    rng = np.random.default_rng(5)
    vals = rng.standard_normal(total).astype(np.float32)
    b.write_field(tf.FIELD_VY, vals)
    got = b.read_field(tf.FIELD_VY, np.float32)
    assert np.array_equal(got, vals)
    off = 0
    for i, inst in enumerate(insts):
        assert np.array_equal(b.read(i, tf.FIELD_VY, np.float32), vals[off:off + inst.cells])
        off += inst.cells
    for bad in (vals[:-1], np.zeros(total + 1, np.float32)):
        with pytest.raises(tf.TptError, match="cells"):
            b.write_field(tf.FIELD_VY, bad)
    with pytest.raises(tf.TptError, match="field id"):
        b.write_field(99, vals)
    with pytest.raises(tf.TptError):
        b.read_field(tf.FIELD_PV, np.float32, out=np.zeros(3, np.float32))
    b.close()


def test_batch_whole_field_io_then_step(cuda, tf, oracle):
    """Seeding a batch with the whole-field calls and reading it back with
    them gives what the oracle gives per instance."""
    insts = mixed_instances()
    b = tf.Batch(insts)
    b.step(3)
    pv = b.read_field(tf.FIELD_PV, np.float32)
    off = 0
    for inst in insts:
        want = oracle.air_steps(inst, 3)
        assert np.array_equal(pv[off:off + inst.cells].view(np.uint32), want["pv"].view(np.uint32))
        off += inst.cells
    b.close()
