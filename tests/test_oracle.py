"""CPU tests of the oracle: the reference's own known-answer tests, the
brute-force gravity pin and the regression fixtures (no GPU)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_fft_mirror_matches_naive_dft_8x8(oracle):
    # crates/tpt-sim/src/gravity_gpu/fft.rs:357-392: row pass then column pass
    g = load("fft_kat.npz")
    w = h = 8
    bits = oracle.bit_count(max(w, h))
    d = np.zeros(w * h * 2, np.float32)
    d[0::2], d[1::2] = g["re8"], g["im8"]
    oracle.fft_host(d, h, w, w, 1, bits, 1.0)
    oracle.fft_host(d, w, h, 1, w, bits, 1.0)
    assert np.all(np.abs(d[0::2] - g["want_re8"]) < 1e-3)
    assert np.all(np.abs(d[1::2] - g["want_im8"]) < 1e-3)


def test_fft_forward_inverse_scales_by_sample_count(oracle):
    # crates/tpt-sim/src/gravity_gpu/fft.rs:394-415
    g = load("fft_kat.npz")
    w, h = int(g["rt_w"]), int(g["rt_h"])
    bits = oracle.bit_count(max(w, h))
    d = np.zeros(w * h * 2, np.float32)
    d[0::2] = g["rt_in"]
    orig = d.copy()
    for sign in (1.0, -1.0):
        oracle.fft_host(d, h, w, w, 1, bits, sign)
        oracle.fft_host(d, w, h, 1, w, bits, sign)
    assert np.all(np.abs(d[0::2] / (w * h) - orig[0::2]) < 1e-3)


def test_bit_count_and_twiddles(oracle):
    # fft.rs:242-264
    assert [oracle.bit_count(n) for n in (0, 1, 2, 3, 4, 8, 1024)] == [0, 0, 1, 2, 2, 3, 10]
    re, im = oracle.twiddle(16)
    k = np.arange(8)
    assert np.allclose(re, np.cos(-2 * np.pi * k / 16), atol=1e-6)
    assert np.allclose(im, np.sin(-2 * np.pi * k / 16), atol=1e-6)


def test_wall_blocking_matches_reference(oracle):
    # crates/tpt-core/src/walls.rs:378-392 through the mask pass (settle.rs:50-93)
    rows = load("walls_kat.npz")["rows"]
    for wall, emap, air, heat in rows:
        # the mask pass decays emap by one first, so store emap + 1
        e_in = np.array([emap + 1 if emap else 0], np.uint32)
        _, ba, bh = oracle.block_masks(np.array([wall], np.uint32), e_in)
        assert ba[0] == air, (wall, emap)
        if heat >= 0:
            assert (bh[0] == 8) == bool(heat), (wall, emap)


def test_gravity_tool_and_cell_mapping(oracle):
    # crates/tpt-sim/src/engine_commands/mod.rs:140-160
    t = load("tools_kat.npz")
    for s, a, want in t["mass"]:
        assert oracle.tool_gravity_mass(s, bool(a)) == want
    for x, y, want in t["cells"]:
        got = oracle.gravity_tool_cell(int(x), int(y), 612, 384, 153, 96)
        assert (got if got is not None else -1) == want


def test_canvas_alignment(oracle, tf):
    # crates/tpt-core/src/particle.rs:776-784
    for xr, yr, wx, wy, cx, cy in load("align_kat.npz")["rows"]:
        assert (oracle.align_dim(int(xr)), oracle.align_dim(int(yr))) == (wx, wy)
        c = tf.SimulationConfig.new(int(xr), int(yr))
        assert (c.xres, c.yres, c.xcells(), c.ycells()) == (wx, wy, cx, cy)


@pytest.mark.parametrize("X,Y", [(24, 24), (64, 48)])
def test_fft_gravity_equals_brute_force(oracle, X, Y):
    """The removed reference pin (crates/tpt-sim/src/gravity_gpu/mod.rs:38-41):
    the padded FFT convolution equals the direct -M_GRAV sum m d/|d|^3, on
    grids whose transform is larger than 2x the grid, with a mask hole."""
    g = load(f"grav_{X}x{Y}.npz")
    dx, dy = oracle.grav_solve(X, Y, g["gmask"], mass_fx=g["mass_fx"], direct=True)
    gx64, gy64 = oracle.grav_solve(X, Y, g["gmask"], mass_fx=g["mass_fx"], dtype=np.float64)
    gx32, gy32 = oracle.grav_solve(X, Y, g["gmask"], mass_fx=g["mass_fx"])
    scale = max(np.abs(dx).max(), np.abs(dy).max())
    assert scale > 0
    assert np.abs(gx64 - dx).max() / scale < 1e-12 and np.abs(gy64 - dy).max() / scale < 1e-12
    assert np.abs(gx32 - dx).max() / scale < 1e-5 and np.abs(gy32 - dy).max() / scale < 1e-5
    assert np.all(gx32[g["gmask"] == 0] == 0) and np.all(gy32[g["gmask"] == 0] == 0)
    # regression against the committed outputs
    assert np.array_equal(gx32, g["gx32"]) and np.array_equal(gy32, g["gy32"])
    assert np.allclose(gx64, g["gx64"], rtol=0, atol=1e-12 * scale)


def test_air_oracle_regression(oracle):
    import workloads as W

    g = load("air_stress_24x24.npz")
    inst = W.make_stress_instance(24, 24, 0x5EED)
    for k in ("pv", "vx", "vy", "hv", "wall", "emap", "bair", "bairh", "eair", "eairh", "fan_vx", "fan_vy"):
        assert np.array_equal(getattr(inst, k), g[f"in_{k}"]), k
    s32 = oracle.air_steps(inst, 10)
    for k, v in s32.items():
        assert np.array_equal(v, g[f"out32_{k}"]), k
    c1 = load("air_c1_5ticks.npz")
    s = oracle.air_steps(W.config_instances(1)[0], 5)
    for k in ("pv", "vx", "vy", "hv"):
        assert np.array_equal(s[k], c1[f"out32_{k}"]), k


def test_air_fp32_mirror_tracks_fp64_twin(oracle):
    """Per-tick FP32 rounding of the reference maths stays at the 1e-6 level
    over the first ticks (discrete branch flips can amplify it later)."""
    import workloads as W

    inst = W.config_instances(1)[0]
    a = oracle.air_steps(inst, 1)
    b = oracle.air_steps(inst, 1, dtype=np.float64)
    for k in ("pv", "vx", "vy", "hv"):
        assert np.abs(a[k] - b[k]).max() <= 1e-5 * np.abs(b[k]).max(), k


def test_mask_pass_decays_emap_and_keeps_counter_bits(oracle):
    wall = np.array([2, 2, 2, 14, 0, 8], np.uint32)
    emap = np.array([0, 1, 3, 0, 5, 0], np.uint32)
    eair = np.array([0, 0, 0, 0, 1, 0], np.uint32)
    eairh = np.array([0, 0, 0, 0, 8, 3], np.uint32)
    e, ba, bh = oracle.block_masks(wall, emap, eair, eairh)
    assert list(e) == [0, 0, 2, 0, 4, 0]
    assert list(ba) == [1, 1, 0, 0, 1, 1]
    assert list(bh) == [8, 8, 0, 8, 8, 8 | 3]


def test_generators_are_deterministic():
    import workloads as W

    a = W.config_instances(4, limit=3)
    b = W.config_instances(4, limit=3)
    for x, y in zip(a, b):
        assert (x.xcells, x.ycells) == (y.xcells, y.ycells)
        for k in ("pv", "hv", "wall", "mass_fx"):
            assert np.array_equal(getattr(x, k), getattr(y, k))
    shapes = W.config_shapes(4)
    assert len(shapes) == 256 and all(32 <= w <= 512 and 32 <= h <= 512 for w, h in shapes)
    s5 = W.config_shapes(5)
    assert len(s5) == 128 and s5[:64] == [(400, 225)] * 64
    c1 = W.config_instances(1)[0]
    assert (c1.mass_fx != 0).sum() == 2000
    assert c1.pv.dtype == np.float32 and np.abs(c1.pv).max() <= 256


def test_mass_fixed_point_rounding(oracle):
    import workloads as W

    vals = np.array([0.0, 1.0, -1.0, 0.5 / 65536, -0.5 / 65536, 0.49999997 / 65536, 1e-9, 3.7, -2.25,
                     32767.0, -32767.0], np.float32)
    got = W.mass_to_fixed(vals)
    want = np.array([oracle.mass_to_fixed(float(v)) for v in vals], np.int32)
    assert np.array_equal(got, want)


def test_gravity_mask_flood_fill(oracle):
    import workloads as W

    for X, Y, seed in ((24, 24, 1), (40, 31, 2), (64, 48, 3)):
        inst = W.make_stress_instance(X, Y, seed)
        m = oracle.grav_mask(inst.wall, X, Y)
        assert np.array_equal(m, W.grav_mask(inst.wall, X, Y))
        assert (m == 0).any() and (m == 0xFFFFFFFF).any()
