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


def _tick_case(oracle, parts, state_over=None, lut_loss=0.5, solid=(), newton=1.0):
    """One particle-side tick on a 64x64-px (16x16-cell) sandbox with g = (1.5,
    -2.0) everywhere; returns (state', parts')."""
    import workloads as W

    xres = yres = 64
    cells = 16 * 16
    st = {"wall_bmap": np.zeros(cells, np.uint32), "wall_emap": np.zeros(cells, np.uint32),
          "grav_mask": np.full(cells, 0xFFFFFFFF, np.uint32), "mass": np.full(cells, 77, np.int32),
          "mass_prev": np.zeros(cells, np.int32), "gx": np.full(cells, 1.5, np.float32),
          "gy": np.full(cells, -2.0, np.float32)}
    st.update(state_over or {})
    n = len(parts["ty"])
    full = {"ty": np.zeros(n, np.uint32), "x": np.full(n, 20.0, np.float32), "y": np.full(n, 20.0, np.float32),
            "vx": np.full(n, 2.0, np.float32), "vy": np.full(n, -4.0, np.float32), "life": np.zeros(n, np.int32),
            "tmp": np.zeros(n, np.int32), "temp": np.full(n, 295.15, np.float32), "flags": np.zeros(n, np.uint32)}
    full.update({k: np.asarray(v, full[k].dtype) for k, v in parts.items()})
    lut = np.zeros((192, 12), np.uint32)
    lut[:, 7] = np.float32(lut_loss).view(np.uint32)
    for t in solid:
        lut[t, 0] = W.TYPE_SOLID
    seeded = oracle.grav_seed(st, xres, yres)
    return oracle.grav_particles_and_finish(seeded, full, lut.reshape(-1), 192, xres, yres, newton)


def test_gravity_tick_element_masses(oracle):
    # gravity_kernel.rs:297-334: the mass each gravity element adds, in fixed point
    import workloads as W

    cell = 5 * 16 + 5  # pixel (20, 20)
    cases = [  # (ty, life, tmp, temp) -> mass
        ((W.PT_NBHL, 0, 0, 0.0), 0.1),          # NBHL default hole
        ((W.PT_NBHL, 0, 5000, 0.0), 5.0),       # 0.001 * tmp
        ((W.PT_NBHL, 0, 90000, 0.0), 51.2),     # clamped high
        ((W.PT_NWHL, 0, 20, 0.0), -0.1),        # clamped low, negated
        ((W.PT_GRVT, 0, 300, 0.0), 20.0),       # tmp clamped to 100, * 0.2
        ((W.PT_GRVT, 0, -7, 0.0), -1.4),
        ((W.PT_GBMB, 25, 0, 0.0), 20.0),        # armed
        ((W.PT_GBMB, 3, 0, 0.0), -80.0),        # counting down
        ((W.PT_GBMB, 0, 0, 0.0), None),         # inert
        ((W.PT_GPMP, 10, 0, 373.15), 20.0),     # on: 0.2 * (temp - 273.15)
        ((W.PT_GPMP, 9, 0, 373.15), None),      # off
        ((W.PT_SPNG, 0, 0, 0.0), None),         # not a gravity element
    ]
    for (ty, life, tmp, temp), m in cases:
        st, _ = _tick_case(oracle, {"ty": [ty], "life": [life], "tmp": [tmp], "temp": [temp]})
        want = 0 if m is None else oracle.mass_to_fixed(np.float32(m) if ty != W.PT_GRVT else
                                                        np.float32(0.2) * np.float32(min(max(tmp, -100), 100)))
        assert st["mass"][cell] == want and st["mass_prev"][cell] == want, (ty, life, tmp, st["mass"][cell], want)
        assert np.count_nonzero(st["mass"]) == (0 if m is None else 1)  # the stale accumulator is cleared


def test_gravity_tick_accumulates_masks_and_overrides(oracle):
    import workloads as W

    cell = 5 * 16 + 5
    # two holes in one cell add; a masked cell drops its contribution
    st, _ = _tick_case(oracle, {"ty": [W.PT_NBHL, W.PT_NBHL, W.PT_NBHL], "x": [20.0, 21.0, 44.0],
                                "y": [20.0, 22.0, 44.0]},
                       {"grav_mask": np.where(np.arange(256) == 11 * 16 + 11, 0, 0xFFFFFFFF).astype(np.uint32)})
    assert st["mass"][cell] == 2 * oracle.mass_to_fixed(0.1) and st["mass"][11 * 16 + 11] == 0
    # an override replaces the cell's accumulated mass; the snapshot copies it
    ovr = np.zeros(256, np.int32)
    ovr[cell] = -123
    st, _ = _tick_case(oracle, {"ty": [W.PT_NBHL]}, {"override_mass": ovr,
                                                    "override_set": (ovr != 0).astype(np.uint32)})
    assert st["mass"][cell] == -123 and st["mass_prev"][cell] == -123
    # a painted well is folded into the snapshot the solve reads, then consumed
    tool = np.zeros(256, np.float32)
    tool[7] = 2.5
    seeded = oracle.grav_seed({"mass": np.ones(256, np.int32), "mass_prev": np.zeros(256, np.int32),
                               "tool_mass": tool, "wall_bmap": None, "wall_emap": None, "grav_mask": None,
                               "gx": None, "gy": None}, 64, 64)
    assert seeded["mass_prev"][7] == oracle.mass_to_fixed(2.5) and not seeded["tool_mass"].any()
    assert not seeded["mass"].any()


def test_gravity_tick_force_on_particles(oracle):
    # apply_gravity_kernel (gravity_kernel.rs:434-516): Loss then newton * g
    import workloads as W

    f32 = np.float32
    loss = f32(0.5)
    _, p = _tick_case(oracle, {"ty": [1, 27, W.PT_SPNG, W.PT_SPNG, 1, 1, 1, 1, 250],
                               "flags": [0, 0, 0x08, 0, 0x10, 0, 0, 0, 0],
                               "x": [20, 20, 20, 20, 20, 2.0, 61.0, -3.0, 20], "y": [20] * 9},
                      solid=(27,))
    vx, vy = f32(2.0), f32(-4.0)
    assert p["vx"][0] == vx * loss + f32(1.5) and p["vy"][0] == vy * loss + f32(-2.0)   # plain element
    assert p["vx"][1] == vx * loss and p["vy"][1] == vy * loss                           # solid: Loss only
    assert p["vx"][2] == vx + f32(1.5)                                                   # movable sponge: no Loss
    assert p["vx"][3] == vx * loss + f32(1.5)                                            # sponge
    for i in (4, 5, 6, 7, 8):  # rigid pixel, margin, margin, off canvas, id past the table
        assert p["vx"][i] == vx and p["vy"][i] == vy, i
    # unpowered stasis freezes, powered does not
    w = np.zeros(256, np.uint32)
    w[5 * 16 + 5] = W.WL_STASIS
    for emap, frozen in ((3, True), (8, False)):
        e = np.zeros(256, np.uint32)
        e[5 * 16 + 5] = emap
        _, p = _tick_case(oracle, {"ty": [1]}, {"wall_bmap": w, "wall_emap": e})
        assert (p["vx"][0] == vx) == frozen


def test_gravity_tick_fixed_point_literals(oracle):
    # hand-computed: 0.1f * 65536 = 6553.6 -> 6554; 20 * 65536; -80 * 65536; -0.1 -> -6554
    import workloads as W

    cell = 5 * 16 + 5
    for ty, life, tmp, want in ((W.PT_NBHL, 0, 0, 6554), (W.PT_GBMB, 21, 0, 1310720), (W.PT_GBMB, 1, 0, -5242880),
                                (W.PT_NWHL, 0, 0, -6554)):
        st, _ = _tick_case(oracle, {"ty": [ty], "life": [life], "tmp": [tmp]})
        assert st["mass_prev"][cell] == want, (ty, st["mass_prev"][cell])
