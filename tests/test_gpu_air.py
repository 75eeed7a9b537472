"""GPU parity of the air step (tpt_air_step through the C ABI) against the
oracle's FP32 restatement of the reference kernels.

Bar: BIT-EXACT. The CUDA air kernels keep the reference's operation order
and are compiled with -fmad=false, so pv/vx/vy/hv must equal the FP32
mirror in every bit after every tick, and the wall masks / emap must be
identical (integer work)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_gpu(tf, torch, inst, ticks, pmap=None, props=None):
    b = tf.SimBuffers.from_instance(inst)
    if pmap is not None:
        b.pmap = torch.from_numpy(pmap.view(np.int32)).cuda()
        b.elem_props = torch.from_numpy(props.view(np.int32)).cuda()
    for _ in range(ticks):
        tf.step_air_gpu(b)
    torch.cuda.synchronize()
    return b.air_state()


def assert_bit_exact(got, want, ctx="", nan_equal=False):
    """Every bit of pv/vx/vy/hv equal (with nan_equal, a NaN matches any NaN:
    NaN payloads are not part of the reference's results); masks and emap
    identical."""
    for k in ("pv", "vx", "vy", "hv"):
        g = np.ascontiguousarray(got[k], np.float32)
        w = np.ascontiguousarray(want[k], np.float32)
        diff = g.view(np.uint32) != w.view(np.uint32)
        if nan_equal:
            diff &= ~(np.isnan(g) & np.isnan(w))
        bad = np.flatnonzero(diff)
        if bad.size:
            i = bad[0]
            raise AssertionError(f"{ctx} {k}: {bad.size} cells differ, first {i}: gpu {g[i]!r} oracle {w[i]!r}, "
                                 f"max abs {np.abs(g - w).max():.3e}")
    for k in ("emap", "bair", "bairh"):
        assert np.array_equal(got[k], want[k]), f"{ctx} {k}"


@pytest.mark.parametrize("ticks", [1, 100, 1000])
def test_c1_default_canvas(cuda, tf, oracle, ticks):
    import workloads as W

    inst = W.config_instances(1)[0]
    assert_bit_exact(run_gpu(tf, cuda, inst, ticks), oracle.air_steps(inst, ticks), f"C1 {ticks}")


def test_c2_large_canvas(cuda, tf, oracle):
    import workloads as W

    inst = W.config_instances(2)[0]
    b = tf.SimBuffers.from_instance(inst)
    cur = inst.copy()
    done = 0
    for t in (1, 2, 10, 30, 100):
        for _ in range(t - done):
            tf.step_air_gpu(b)
        s = oracle.air_steps(cur, t - done)
        for k in ("pv", "vx", "vy", "hv", "emap", "bair", "bairh"):
            setattr(cur, k, s[k])
        done = t
        cuda.cuda.synchronize()
        assert_bit_exact(b.air_state(), s, f"C2 tick {t}")


def test_c2_every_tick_to_1000(cuda, tf, oracle):
    """C2 (400x225) compared against the oracle after every one of its first
    1000 ticks, GPU and oracle stepping in lock step."""
    import workloads as W

    inst = W.config_instances(2)[0]
    b = tf.SimBuffers.from_instance(inst)
    cur = inst.copy()
    for t in range(1, 1001):
        tf.step_air_gpu(b)
        s = oracle.air_steps(cur, 1)
        for k in ("pv", "vx", "vy", "hv", "emap", "bair", "bairh"):
            setattr(cur, k, s[k])
        cuda.cuda.synchronize()
        assert_bit_exact(b.air_state(), s, f"C2 tick {t}")


def test_c2_10000_ticks(cuda, tf, oracle):
    """C2's stated horizon: 10000 ticks, compared at the end point."""
    import workloads as W

    inst = W.config_instances(2)[0]
    b = tf.SimBuffers.from_instance(inst)
    for _ in range(10000):
        tf.step_air_gpu(b)
    cuda.cuda.synchronize()
    assert_bit_exact(b.air_state(), oracle.air_steps(inst, 10000), "C2 10000 ticks")


def test_nonfinite_and_clamp_inputs(cuda, tf, oracle):
    """NaN and +-Inf in every state grid, velocities at and far beyond the
    +-256 clamp: the f32 -> i32 conversions of the walks and samples see NaN
    and out-of-range values, which round toward zero, saturate, and give 0
    for NaN on the GPU as in the oracle."""
    from test_oracle_air_numpy import nonfinite_instance

    inst = nonfinite_instance()
    for ticks in (1, 3):
        assert_bit_exact(run_gpu(tf, cuda, inst, ticks), oracle.air_steps(inst, ticks), f"non-finite t{ticks}",
                         nan_equal=True)


MODES = [
    dict(),
    dict(air_mode=1), dict(air_mode=2), dict(air_mode=3), dict(air_mode=4),
    dict(air_mode=4, aheat_enable=0),
    dict(aheat_enable=0),
    dict(convection_mode=1), dict(convection_mode=0),
    dict(gravity_mode=1), dict(gravity_mode=2), dict(gravity_mode=3, custom_gx=3.0, custom_gy=-40.0),
    dict(convection_mode=1, gravity_mode=2),
    dict(vorticity_coeff=0.0), dict(vorticity_coeff=2.5),
    dict(edge_pressure=12.5, edge_vx=-3.0, edge_vy=1.5, ambient_air_temp=350.0),
]


@pytest.mark.parametrize("shape", [(24, 24), (37, 29), (96, 80), (33, 9)])
@pytest.mark.parametrize("mode", range(len(MODES)))
def test_stress_instances_every_mode(cuda, tf, oracle, shape, mode):
    """Every wall kind, fans, emap decay, element stamps, counter bits,
    far-advection walks up to the +-256 clamp, on grids that are not a
    multiple of the 32x8 tile, in every air / convection / gravity mode."""
    import workloads as W

    X, Y = shape
    cfg = W.AirConfig(**MODES[mode])
    inst = W.make_stress_instance(X, Y, 1000 + 7 * mode + X, config=cfg)
    assert_bit_exact(run_gpu(tf, cuda, inst, 6), oracle.air_steps(inst, 6), f"{shape} {MODES[mode]}")


def test_tiny_and_thin_grids(cuda, tf, oracle):
    import workloads as W

    for X, Y in ((3, 3), (4, 40), (40, 4), (5, 5), (64, 3)):
        inst = W.make_stress_instance(X, Y, 77 + X * Y)
        assert_bit_exact(run_gpu(tf, cuda, inst, 3), oracle.air_steps(inst, 3), f"{X}x{Y}")


def test_hot_air_pass(cuda, tf, oracle):
    """Particle HotAir -> pressure (crates/tpt-sim/src/air_kernel/settle.rs:
    118-161) with GAS/NBLE approach-to-3.5 and out-of-table ids."""
    import workloads as W

    X, Y = 40, 30
    inst = W.make_stress_instance(X, Y, 4242)
    st = W.Stream(99)
    xres, yres = 4 * X, 4 * Y
    pmap = np.zeros(xres * yres, np.uint32)
    occ = st.uniform(0, 1, xres * yres) < 0.3
    types = (st.u64(xres * yres) % np.uint64(120)).astype(np.uint32)
    types[st.uniform(0, 1, xres * yres) < 0.1] = 10
    types[st.uniform(0, 1, xres * yres) < 0.05] = 97
    pmap[occ] = types[occ] | (np.uint32(5) << np.uint32(9))  # id bits above the type
    nel = 110
    props = np.zeros(nel * 32, np.uint32)
    hot = np.zeros(nel, np.float32)
    hot[st.choice_cells(nel, 30)] = st.uniform(-0.002, 0.004, 30).astype(np.float32)
    hot[10], hot[97] = 0.001, -0.0005
    props[11::32] = hot.view(np.uint32)
    got = run_gpu(tf, cuda, inst, 4, pmap, props)
    want = oracle.air_steps(inst, 4, pmap=pmap, props=props, xres=xres, yres=yres)
    assert_bit_exact(got, want, "hot air")


def test_stream_ordering_and_launch_count(cuda, tf, oracle):
    """The step is asynchronous on the given stream and launches the library's
    own kernels (pressure+velocity, advection+heat, settle)."""
    import workloads as W

    inst = W.config_instances(1)[0]
    b = tf.SimBuffers.from_instance(inst)
    s = cuda.cuda.Stream()
    n0 = tf.launch_count()
    with cuda.cuda.stream(s):
        for _ in range(5):
            tf.step_air_gpu(b, stream=s)
    s.synchronize()
    assert tf.launch_count() - n0 == 15
    assert_bit_exact(b.air_state(), oracle.air_steps(inst, 5), "stream")
