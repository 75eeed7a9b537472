"""GPU accuracy of the split-BF16 DFT-as-GEMM gravity (tcgen05) against the
FP64 oracle. Bar (per result): max |g - g64| <= 1e-4 * max |g64| and the L2
error normalised by ||g64|| <= 1e-4, for gx and gy; exact zeros outside the
mask; no device-side wait timed out."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-4


def errors(g, ref):
    g = g.astype(np.float64)
    scale = max(np.abs(ref).max(), 1e-30)
    return np.abs(g - ref).max() / scale, np.linalg.norm(g - ref) / max(np.linalg.norm(ref), 1e-30)


def check_clean(tf):
    rc = tf.lib().tpt_check_device_errors()
    assert rc == 0, tf.lib().tpt_last_error_string().decode()


@pytest.mark.parametrize("X,Y,kind", [(24, 24, "stress"), (37, 29, "stress"), (64, 48, "stress"),
                                      (153, 96, "c1"), (400, 225, "c2"), (32, 130, "stress")])
def test_split_bf16_plan_vs_fp64(cuda, tf, oracle, X, Y, kind):
    import workloads as W
    from test_gpu_grav import solve_gpu

    if kind == "c1":
        inst = W.config_instances(1)[0]
    elif kind == "c2":
        inst = W.config_instances(2)[0]
    else:
        inst = W.make_stress_instance(X, Y, 31 * X + Y)
    gx, gy = solve_gpu(tf, cuda, X, Y, inst.gmask, inst.mass_fx, precision=tf.PRECISION_SPLIT_BF16)
    check_clean(tf)
    dx, dy = oracle.grav_solve(X, Y, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
    for g, d in ((gx, dx), (gy, dy)):
        emax, el2 = errors(g, d)
        assert emax <= TOL and el2 <= TOL, (emax, el2)
    assert np.all(gx[inst.gmask == 0] == 0) and np.all(gy[inst.gmask == 0] == 0)


def test_split_bf16_c3_f32_mass(cuda, tf, oracle):
    import workloads as W
    from test_gpu_grav import solve_gpu

    X = Y = 512
    mass = W.clustered_mass(X, Y, W.instance_seed(3, 0))
    mask = np.full(X * Y, 0xFFFFFFFF, np.uint32)
    gx, gy = solve_gpu(tf, cuda, X, Y, mask, mass_f32=mass, precision=tf.PRECISION_SPLIT_BF16)
    check_clean(tf)
    dx, dy = oracle.grav_solve(X, Y, mask, mass_f32=mass, dtype=np.float64)
    for g, d in ((gx, dx), (gy, dy)):
        emax, el2 = errors(g, d)
        assert emax <= TOL and el2 <= TOL, (emax, el2)


def test_split_bf16_plan_dims_and_repeat(cuda, tf):
    import workloads as W
    from test_gpu_grav import solve_gpu

    inst = W.config_instances(1)[0]
    outs = solve_gpu(tf, cuda, 153, 96, inst.gmask, inst.mass_fx, precision=tf.PRECISION_SPLIT_BF16, repeat=2)
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    s = tf.GravityFft(tf.PRECISION_SPLIT_BF16)
    s._ensure(153, 96)
    assert s.padded_dims() == (306, 192)
    s.close()


def test_split_bf16_batch_mixed_shapes(cuda, tf, oracle):
    """Equal-shape instances share one stacked GEMM per stage; singletons
    run as their own groups; all in the same launches."""
    import workloads as W

    insts = W.config_instances(5, limit=3)  # three 400x225
    insts += [W.make_instance(57, 36, 5, mass_density=0.02), W.make_instance(33, 151, 6, mass_density=0.02),
              W.make_instance(57, 36, 7, mass_density=0.02)]
    b = tf.Batch(insts, tf.PRECISION_SPLIT_BF16)
    b.step(2)
    cuda.cuda.synchronize()
    check_clean(tf)
    for i, inst in enumerate(insts):
        st = b.state(i)
        dx, dy = oracle.grav_solve(inst.xcells, inst.ycells, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
        for g, d in ((st["gx"], dx), (st["gy"], dy)):
            emax, el2 = errors(g, d)
            assert emax <= TOL and el2 <= TOL, (i, emax, el2)
    b.close()


@pytest.mark.parametrize("ymode", ["toeplitz", "dft"])
@pytest.mark.parametrize("X,Y,kind", [(37, 29, "stress"), (153, 96, "c1"), (400, 225, "c2"), (32, 130, "stress"),
                                      (130, 33, "stress")])
def test_split_bf16_forced_y_form_vs_fp64(cuda, tf, oracle, monkeypatch, ymode, X, Y, kind):
    """Both forms of the y stage (y DFT pair, or direct Toeplitz GEMM per x
    frequency with an MN-major R^-1 operand) meet the bar on their own."""
    import workloads as W
    from test_gpu_grav import solve_gpu

    monkeypatch.setenv("TPT_SPLIT_BF16_Y_STAGE", ymode)
    if kind == "c1":
        inst = W.config_instances(1)[0]
    elif kind == "c2":
        inst = W.config_instances(2)[0]
    else:
        inst = W.make_stress_instance(X, Y, 17 * X + Y)
    gx, gy = solve_gpu(tf, cuda, X, Y, inst.gmask, inst.mass_fx, precision=tf.PRECISION_SPLIT_BF16)
    check_clean(tf)
    dx, dy = oracle.grav_solve(X, Y, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
    for g, d in ((gx, dx), (gy, dy)):
        emax, el2 = errors(g, d)
        assert emax <= TOL and el2 <= TOL, (ymode, emax, el2)
    assert np.all(gx[inst.gmask == 0] == 0) and np.all(gy[inst.gmask == 0] == 0)


@pytest.mark.parametrize("ymode", ["toeplitz:2", "toeplitz", "auto"])
def test_split_bf16_batch_mixed_y_forms(cuda, tf, oracle, monkeypatch, ymode):
    """One set whose groups use different y forms: the pair of 400x225 and
    the pair of 57x36 go through T (toeplitz:2), the singletons through the
    y DFT, with both y stages launched in the same solve. Repeating the
    solve gives identical fields."""
    import workloads as W

    monkeypatch.setenv("TPT_SPLIT_BF16_Y_STAGE", ymode)
    insts = W.config_instances(5, limit=2)  # two 400x225
    insts += [W.make_instance(57, 36, 5, mass_density=0.02), W.make_instance(33, 151, 6, mass_density=0.02),
              W.make_instance(57, 36, 7, mass_density=0.02), W.make_instance(200, 40, 8, mass_density=0.02)]
    b = tf.Batch(insts, tf.PRECISION_SPLIT_BF16)
    prof = b.profile_phases(2)
    if ymode == "toeplitz:2":
        assert prof.grav_launches_per_tick == 6  # prep, R, C, C^-1, T, R^-1
    b.step(2)
    cuda.cuda.synchronize()
    check_clean(tf)
    first = [b.state(i) for i in range(len(insts))]
    b.step(1)
    cuda.cuda.synchronize()
    for i, inst in enumerate(insts):
        st = b.state(i)
        dx, dy = oracle.grav_solve(inst.xcells, inst.ycells, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
        for g, d in ((st["gx"], dx), (st["gy"], dy)):
            emax, el2 = errors(g, d)
            assert emax <= TOL and el2 <= TOL, (ymode, i, emax, el2)
        # gravity reads the previous tick's mass, which the air step leaves alone
        assert np.array_equal(st["gx"], first[i]["gx"]) and np.array_equal(st["gy"], first[i]["gy"])
    b.close()


def test_split_bf16_concurrent_y_branches(cuda, tf, oracle, monkeypatch):
    """grav_side_ctas > 0 runs the DFT-pair groups' chain (R, C, C^-1, R^-1)
    on a second stream beside the Toeplitz groups' chain (R, T, R^-1): every
    tile still runs the same code, so the fields are bit-identical to the
    one-stream order for every CTA split, and the autotuner's choice keeps
    them. A batch with one kind of y stage rejects a split."""
    import workloads as W

    monkeypatch.setenv("TPT_SPLIT_BF16_Y_STAGE", "toeplitz:2")
    insts = W.config_instances(5, limit=2)  # two 400x225: Toeplitz
    insts += [W.make_instance(57, 36, 5, mass_density=0.02), W.make_instance(33, 151, 6, mass_density=0.02),
              W.make_instance(57, 36, 7, mass_density=0.02), W.make_instance(200, 40, 8, mass_density=0.02)]
    b = tf.Batch(insts, tf.PRECISION_SPLIT_BF16)
    sms = cuda.cuda.get_device_properties(0).multi_processor_count
    assert b.tuning().grav_side_ctas == 0
    assert b.profile_phases(2).grav_launches_per_tick == 6  # prep, R, C, C^-1, T, R^-1
    b.step(2)
    cuda.cuda.synchronize()
    ref = [(b.state(i)["gx"], b.state(i)["gy"]) for i in range(len(insts))]
    for side in (1, 8, 30, sms // 2):
        t = b.tuning()
        t.grav_side_ctas = side
        b.set_tuning(t)
        # Toeplitz branch R, T, R^-1; DFT-pair branch R, C, C^-1, R^-1; prep
        assert b.profile_phases(2).grav_launches_per_tick == 8
        b.step(3)
        cuda.cuda.synchronize()
        check_clean(tf)
        for i in range(len(insts)):
            st = b.state(i)
            assert np.array_equal(st["gx"], ref[i][0]) and np.array_equal(st["gy"], ref[i][1]), (side, i)
    t = b.tuning()
    t.grav_side_ctas = sms // 2 + 1
    with pytest.raises(tf.TptError, match="grav_side_ctas"):
        b.set_tuning(t)
    b.tune()
    assert b.tuning().grav_side_ctas <= sms // 2
    b.step(2)
    cuda.cuda.synchronize()
    check_clean(tf)
    for i, inst in enumerate(insts):
        st = b.state(i)
        assert np.array_equal(st["gx"], ref[i][0]) and np.array_equal(st["gy"], ref[i][1]), ("tuned", i)
        dx, dy = oracle.grav_solve(inst.xcells, inst.ycells, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
        for g, d in ((st["gx"], dx), (st["gy"], dy)):
            emax, el2 = errors(g, d)
            assert emax <= TOL and el2 <= TOL, (i, emax, el2)
    b.close()
    # one kind of y stage (and the FP32 solve) takes no split
    for prec in (tf.PRECISION_SPLIT_BF16, tf.PRECISION_FP32):
        b = tf.Batch(insts[2:4], prec)
        t = b.tuning()
        t.grav_side_ctas = 4
        with pytest.raises(tf.TptError, match="grav_side_ctas"):
            b.set_tuning(t)
        b.close()


def test_c5_batch_concurrent_branches_full_size(cuda, tf, oracle):
    """The full C5 batch (128 instances, 6.1M cells) in the configuration the
    bench times: autotuned, then with the gravity branches concurrent. gx/gy
    stay bit-identical to the one-stream order on instances of both y forms
    and meet the 1e-4 bar against FP64; the air fields after 5 ticks are
    bit-exact against the oracle."""
    import workloads as W
    from test_gpu_air import assert_bit_exact

    insts = W.config_instances(5)
    b = tf.Batch(insts, tf.PRECISION_SPLIT_BF16)
    sample = (0, 63, 64, 70, 100, 127)
    b.step(2)
    cuda.cuda.synchronize()
    ref = {i: (b.state(i)["gx"], b.state(i)["gy"]) for i in sample}
    b.tune()
    t = b.tuning()
    t.grav_side_ctas = max(1, cuda.cuda.get_device_properties(0).multi_processor_count * 2 // 5)
    b.set_tuning(t)
    b.step(3)
    cuda.cuda.synchronize()
    check_clean(tf)
    for i in sample:
        inst = insts[i]
        st = b.state(i)
        assert np.array_equal(st["gx"], ref[i][0]) and np.array_equal(st["gy"], ref[i][1]), i
        dx, dy = oracle.grav_solve(inst.xcells, inst.ycells, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
        for g, d in ((st["gx"], dx), (st["gy"], dy)):
            emax, el2 = errors(g, d)
            assert emax <= TOL and el2 <= TOL, (i, emax, el2)
        assert_bit_exact(st, oracle.air_steps(inst, 5), f"C5 instance {i}")
    b.close()
