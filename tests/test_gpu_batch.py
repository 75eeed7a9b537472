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


def set_form(tf, b, form, **kw):
    """Switches the batch's air form; tile_x / tile_y default to the form's
    default shape (32x8 tiles, 224-lane x 64-row sweeps), ctas_per_sm to 0,
    temporal_depth to 1, work_queue to 1 (the default tuning's)."""
    t = b.tuning()
    t.air_form = form
    t.tile_x, t.tile_y = (224, 64) if form == tf.AIR_FORM_SWEEP else tf.TILE_SHAPES[0]
    t.ctas_per_sm = 0
    t.temporal_depth = 1
    t.work_queue = 1
    for k, v in kw.items():
        setattr(t, k, v)
    b.set_tuning(t)


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("ticks", [1, 7, 50, 57])
def test_batch_matches_single_grid_oracle(cuda, tf, oracle, ticks, form):
    insts = mixed_instances()
    b = tf.Batch(insts)
    set_form(tf, b, form)
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
    assert t.air_form in (tf.AIR_FORM_TILES, tf.AIR_FORM_SWEEP)
    if t.air_form == tf.AIR_FORM_TILES:
        assert (t.tile_x, t.tile_y) in tf.TILE_SHAPES and t.ctas_per_sm in (0, 2, 4, 6, 8) and t.work_queue in (0, 1)
        assert t.temporal_depth in (1, 2, 4, 10, 20)
    else:
        assert (t.tile_x, t.tile_y) in ((224, 64), (256, 64), (256, 32)) and t.temporal_depth == 1
    b.step(5)
    cuda.cuda.synchronize()
    check_against_oracle(tf, oracle, b, insts, 5, "tuned")
    # a second batch of the same composition takes the cached choice
    b2 = tf.Batch(insts)
    b2.tune()
    assert b2.tuning_dict() == b.tuning_dict()
    b2.close()
    b.close()


@pytest.mark.parametrize("tile_x,tile_y,per_sm", [(64, 8, 0), (96, 16, 1), (128, 32, 0), (224, 64, 0),
                                                  (256, 128, 2), (256, 2048, 0)])
def test_every_sweep_shape_gives_the_same_fields(cuda, tf, oracle, tile_x, tile_y, per_sm):
    """The sweep's tuning knobs change the work layout only: for every shape
    (narrow CTAs that split a grid into many column strips, short strips,
    whole-grid strips) the fields after 9 ticks are bit-exact."""
    insts = mixed_instances()
    b = tf.Batch(insts)
    set_form(tf, b, tf.AIR_FORM_SWEEP, tile_x=tile_x, tile_y=tile_y, ctas_per_sm=per_sm)
    b.step(9)
    cuda.cuda.synchronize()
    assert tf.lib().tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, 9, f"sweep {tile_x}x{tile_y}")
    b.close()


@pytest.mark.parametrize("shape", [(32, 8), (64, 8), (32, 16), (64, 16)])
@pytest.mark.parametrize("per_sm", [0, 1, 2])
def test_every_tile_shape_gives_the_same_fields(cuda, tf, oracle, shape, per_sm):
    """Every tile shape of the tile form (its own kernels, tile list and
    tensor-map boxes) at as many CTAs per SM as fit, one and two: the fields
    after 9 ticks (odd: the copy-back runs) are bit-exact."""
    assert shape in tf.TILE_SHAPES
    insts = mixed_instances()
    b = tf.Batch(insts)
    set_form(tf, b, tf.AIR_FORM_TILES, tile_x=shape[0], tile_y=shape[1], ctas_per_sm=per_sm)
    b.step(9)
    cuda.cuda.synchronize()
    assert tf.lib().tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, 9, f"tiles {shape[0]}x{shape[1]} {per_sm}/SM")
    b.close()


@pytest.mark.parametrize("depth", [2, 3, 5, 50])
@pytest.mark.parametrize("ticks", [1, 2, 7, 57])
def test_temporal_blocking_is_bit_exact(cuda, tf, oracle, depth, ticks):
    """Temporal blocking: blocks of `depth` ticks as A, (depth - 1) fused
    B(t) + A(t + 1) launches and B, with the emap decays deferred to the
    block's last launch (the stress instances' electrified walls decay over
    three ticks), NoUpdate and no-heat instances, blocks cut short by the
    step's tick count: bit-exact after every step length."""
    insts = mixed_instances()
    b = tf.Batch(insts)
    set_form(tf, b, tf.AIR_FORM_TILES, temporal_depth=depth)
    b.step(ticks)
    cuda.cuda.synchronize()
    assert tf.lib().tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, ticks, f"depth {depth}, {ticks} ticks")
    b.close()


def test_steps_longer_than_one_graph(cuda, tf, oracle):
    """A step of more ticks than one captured graph holds (1000) replays it
    and then a graph of the rest; temporal blocks are cut at the graph's end."""
    insts = mixed_instances()[:3]
    for depth in (1, 3):
        b = tf.Batch(insts)
        set_form(tf, b, tf.AIR_FORM_TILES, temporal_depth=depth)
        b.step(1003)
        cuda.cuda.synchronize()
        assert tf.lib().tpt_check_device_errors() == 0
        check_against_oracle(tf, oracle, b, insts, 1003, f"1003 ticks depth {depth}")
        b.close()


@pytest.mark.parametrize("shape", [(32, 8), (64, 16)])
@pytest.mark.parametrize("depth", [1, 3])
@pytest.mark.parametrize("per_sm", [0, 1])
def test_tile_work_queue_gives_the_same_fields(cuda, tf, oracle, shape, depth, per_sm):
    """The tile form's CTAs taking tiles from the atomic work queues (cleared
    by each other's launches), with and without temporal blocking, after
    switching from static striding and back: bit-exact."""
    insts = mixed_instances()
    b = tf.Batch(insts)
    for queue, ticks in ((0, 2), (1, 7), (0, 1), (1, 4)):
        set_form(tf, b, tf.AIR_FORM_TILES, tile_x=shape[0], tile_y=shape[1], temporal_depth=depth,
                 ctas_per_sm=per_sm, work_queue=queue)
        b.step(ticks)
    cuda.cuda.synchronize()
    assert tf.lib().tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, 14, f"queue {shape[0]}x{shape[1]} depth {depth} {per_sm}/SM")
    b.close()


@pytest.mark.parametrize("shape", [(64, 8), (64, 16)])
def test_temporal_blocking_with_other_tile_shapes(cuda, tf, oracle, shape):
    """The block's first and last launches at another tile shape than the
    fused launches' 32x16."""
    insts = mixed_instances()
    b = tf.Batch(insts)
    set_form(tf, b, tf.AIR_FORM_TILES, tile_x=shape[0], tile_y=shape[1], temporal_depth=4)
    for ticks in (3, 6):
        b.step(ticks)
    cuda.cuda.synchronize()
    assert tf.lib().tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, 9, f"depth 4 at {shape[0]}x{shape[1]}")
    b.close()


@pytest.mark.parametrize("per_sm", [1, 3, 6, 8])
@pytest.mark.parametrize("queue", [0, 1])
def test_tile_form_at_every_grid_size(cuda, tf, oracle, per_sm, queue):
    insts = mixed_instances()
    b = tf.Batch(insts)
    set_form(tf, b, tf.AIR_FORM_TILES, ctas_per_sm=per_sm, work_queue=queue)
    b.step(9)
    cuda.cuda.synchronize()
    assert tf.lib().tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, 9, f"tiles {per_sm}/SM queue {queue}")
    b.close()


def test_switching_forms_between_steps(cuda, tf, oracle):
    """The state sits in the canonical buffers between steps whatever the
    form, so a batch may change form from one step to the next."""
    insts = mixed_instances()
    b = tf.Batch(insts)
    for form, shape, ticks in ((1, (224, 64), 3), (0, (32, 8), 4), (1, (256, 32), 1), (0, (64, 16), 2),
                               (0, (32, 16), 1)):
        set_form(tf, b, form, tile_x=shape[0], tile_y=shape[1])
        b.step(ticks)
    cuda.cuda.synchronize()
    check_against_oracle(tf, oracle, b, insts, 11, "form switches")
    b.close()


def test_bad_tunings_are_rejected(cuda, tf):
    b = tf.Batch(mixed_instances()[:2])
    before = b.tuning_dict()
    tiles, sweep = tf.AIR_FORM_TILES, tf.AIR_FORM_SWEEP
    for kw in (
        # tile form: only the four shapes
        dict(air_form=tiles, tile_x=48, tile_y=8), dict(air_form=tiles, tile_x=64, tile_y=32),
        dict(air_form=tiles, tile_x=224, tile_y=64), dict(air_form=tiles, tile_x=32, tile_y=8, ctas_per_sm=64),
        # sweep form: lanes a multiple of 32 in 64..256, rows >= 8, CTAs that fit
        dict(air_form=sweep, tile_x=100, tile_y=64), dict(air_form=sweep, tile_x=32, tile_y=64),
        dict(air_form=sweep, tile_x=288, tile_y=64), dict(air_form=sweep, tile_x=224, tile_y=4),
        dict(air_form=sweep, tile_x=224, tile_y=64, ctas_per_sm=9),
        # temporal depth 1..50, tile form only
        dict(temporal_depth=0), dict(temporal_depth=51),
        dict(air_form=sweep, tile_x=224, tile_y=64, temporal_depth=2),
        dict(air_form=2), dict(work_queue=2),
    ):
        t = b.tuning()
        for k, v in kw.items():
            setattr(t, k, v)
        with pytest.raises(tf.TptError):
            b.set_tuning(t)
    assert b.tuning_dict() == before
    b.close()


def test_packed_narrow_instances_and_modes(cuda, tf, oracle):
    """Many narrow and short instances packed side by side into shared CTAs
    (up to eight strips per CTA), in different air modes, next to one wide
    instance; far-advection samples on every tick."""
    import workloads as W

    insts = []
    for k, (X, Y) in enumerate([(3, 3), (5, 40), (9, 9), (17, 33), (31, 8), (32, 36), (40, 12), (12, 70),
                                (23, 23), (60, 5), (7, 64), (44, 19)]):
        cfg = W.AirConfig(**[dict(), dict(air_mode=4), dict(aheat_enable=0), dict(convection_mode=1),
                             dict(vorticity_coeff=2.5), dict(air_mode=2)][k % 6])
        insts.append(W.make_stress_instance(X, Y, 500 + k, config=cfg))
    insts.append(W.make_stress_instance(300, 20, 599))
    b = tf.Batch(insts)
    set_form(tf, b, tf.AIR_FORM_SWEEP)
    for ticks in (1, 3):
        b.step(ticks)
    cuda.cuda.synchronize()
    check_against_oracle(tf, oracle, b, insts, 4, "packed")
    b.close()


def test_nonfinite_inputs_in_a_batch(cuda, tf, oracle):
    """NaN / Inf state and velocities past the clamp, through the batch's
    sweep (pointwise and pre-pass far samples included)."""
    from test_gpu_air import assert_bit_exact
    from test_oracle_air_numpy import nonfinite_instance

    insts = [nonfinite_instance(), nonfinite_instance(70, 50, 32)]
    for form, depth in ((tf.AIR_FORM_TILES, 1), (tf.AIR_FORM_TILES, 3), (tf.AIR_FORM_SWEEP, 1)):
        b = tf.Batch(insts)
        set_form(tf, b, form, temporal_depth=depth)
        b.step(3)
        cuda.cuda.synchronize()
        for i, inst in enumerate(insts):
            assert_bit_exact(b.state(i), oracle.air_steps(inst, 3), f"form {form} depth {depth} non-finite {i}",
                             nan_equal=True)
        b.close()


def test_batch_measured_config_subset(cuda, tf, oracle):
    import workloads as W

    insts = W.config_instances(4, limit=12)
    b = tf.Batch(insts)
    b.step(20)
    cuda.cuda.synchronize()
    check_against_oracle(tf, oracle, b, insts, 20, "C4 subset")
    b.close()


@pytest.mark.parametrize("form,shape,depth,queue", [(0, (32, 8), 1, 0), (0, (64, 8), 1, 0), (0, (32, 16), 1, 1),
                                                    (0, (32, 8), 4, 1), (1, (224, 64), 1, 0)])
def test_c4_every_instance_20_ticks(cuda, tf, oracle, form, shape, depth, queue):
    """The whole C4 batch (256 instances, W, H log-uniform 32..512, FP32
    gravity) after 20 ticks: every instance's air bit-exact against the
    oracle and its gx/gy within 1e-5 of max|g| against FP64."""
    import workloads as W

    insts = W.config_instances(4)
    assert len(insts) == 256
    b = tf.Batch(insts)
    set_form(tf, b, form, tile_x=shape[0], tile_y=shape[1], temporal_depth=depth, work_queue=queue)
    b.step(20)
    cuda.cuda.synchronize()
    assert tf.lib().tpt_check_device_errors() == 0
    check_against_oracle(tf, oracle, b, insts, 20, f"C4 form {form} {shape[0]}x{shape[1]} depth {depth} queue {queue}")
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
