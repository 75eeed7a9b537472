"""`.tptrs` save files (crates/tpt-save/src/lib.rs) through the library's
host codec, on CPU.

The reference's own tests for the format (lib.rs:719-857) are ported one by
one. They need payloads the codec does not build itself (signs, version-1
layouts), and those come from a second, independent restatement of the
format below: bincode 1.3.3's default encoding (little-endian fixed-width
integers, u64 lengths, u32 enum indices, one-byte bools and Option tags)
applied to the SaveData field order (lib.rs:67-97, particle.rs:27-44,
166-222, 392-436, sign.rs:27-33). The two restatements must agree byte for
byte. Golden bytes from the reference itself are not available (it needs Rust
and is not built here), so the format is pinned by the reference's tests and
by this agreement.
"""
import struct
import zlib

import numpy as np
import pytest

MAGIC = b"TPTRS001"


# ------------------------------------------------ independent restatement --

def config_new(xres, yres):
    """SimulationConfig::new (particle.rs:224-281), serialised fields only."""
    a = lambda v: (max(v, 64) + 3) // 4 * 4  # noqa: E731  align_dim (particle.rs:383-386)
    x, y = a(xres), a(yres)
    return dict(xres=x, yres=y, paused=False, aheat_enable=False, pretty_powder=False, edge_mode=0, gravity_mode=0,
                air_mode=0, ambient_air_temp=295.15, edge_pressure=0.0, display_mode=0, colour_mode=0,
                render_mode=0x47, fire_intensity=1.0, heat_enable=True, newton_grav=False, water_equal_test=False,
                vorticity_coeff=0.1, convection_mode=2, edge_velocity_x=0.0, edge_velocity_y=0.0,
                custom_gravity_x=0.0, custom_gravity_y=1.0, temperature_scale=0, decorations=True, mouse_x=-1,
                mouse_y=-1, gravity_field_enabled=False, gravity_zones_enabled=False, grid=False, grid_size=1,
                grid_checkerboard=False, hud=True, debug_hud=False, show_brush=True, zoom_enabled=False,
                zoom_window_x=0, zoom_window_y=0, zoom_factor=8, zoom_scope_x=0, zoom_scope_y=0, zoom_scope_size=32,
                heat_display_limit_min=0.0, heat_display_limit_max=9999.0, heat_display_auto_x=0,
                heat_display_auto_y=0, heat_display_auto_w=x, heat_display_auto_h=y)


CONFIG_LAYOUT = [  # (field, format); "?" bool, "o" Option<f32>
    ("xres", "I"), ("yres", "I"), ("paused", "?"), ("aheat_enable", "?"), ("pretty_powder", "?"),
    ("edge_mode", "I"), ("gravity_mode", "I"), ("air_mode", "I"), ("ambient_air_temp", "f"), ("edge_pressure", "f"),
    ("display_mode", "I"), ("colour_mode", "I"), ("render_mode", "I"), ("fire_intensity", "f"),
    ("heat_enable", "?"), ("newton_grav", "?"), ("water_equal_test", "?"), ("vorticity_coeff", "f"),
    ("convection_mode", "I"), ("edge_velocity_x", "f"), ("edge_velocity_y", "f"), ("custom_gravity_x", "f"),
    ("custom_gravity_y", "f"), ("temperature_scale", "I"), ("decorations", "?"), ("mouse_x", "i"), ("mouse_y", "i"),
    ("gravity_field_enabled", "?"), ("gravity_zones_enabled", "?"), ("grid", "?"), ("grid_size", "i"),
    ("grid_checkerboard", "?"), ("hud", "?"), ("debug_hud", "?"), ("show_brush", "?"), ("zoom_enabled", "?"),
    ("zoom_window_x", "i"), ("zoom_window_y", "i"), ("zoom_factor", "i"), ("zoom_scope_x", "i"),
    ("zoom_scope_y", "i"), ("zoom_scope_size", "i"), ("heat_display_limit_min", "o"),
    ("heat_display_limit_max", "o"), ("heat_display_auto_x", "i"), ("heat_display_auto_y", "i"),
    ("heat_display_auto_w", "i"), ("heat_display_auto_h", "i"),
]


def enc_config(c):
    out = b""
    for name, f in CONFIG_LAYOUT:
        v = c[name]
        if f == "o":
            out += b"\x00" if v is None else b"\x01" + struct.pack("<f", v)
        else:
            out += struct.pack("<" + f, v)
    return out


def enc_vec(items, enc):
    return struct.pack("<Q", len(items)) + b"".join(enc(i) for i in items)


def enc_particle(p):  # GpuParticle: 16 four-byte fields
    return struct.pack("<IiIfffffIiiiiIII", *p)


def enc_sign(s):
    t = s["text"].encode()
    return struct.pack("<iiQ", s["x"], s["y"], len(t)) + t + struct.pack("<B", s["ju"])


def enc_rigid(b):
    head = struct.pack("<I?10f", b["id"], b["active"], *b["f"])
    return head + enc_vec(b["pixels"], lambda px: struct.pack("<ffIfiIIii", *px))


def enc_save(d, version_one=False):
    out = struct.pack("<I", d["version"]) + enc_config(d["config"]) + enc_vec(d["particles"], enc_particle)
    for g in ("air_vx", "air_vy", "air_pv", "air_hv", "fan_vx", "fan_vy"):
        out += enc_vec(list(d[g]), lambda v: struct.pack("<f", v))
    for g in ("wall_bmap", "wall_emap"):
        out += enc_vec(list(d[g]), lambda v: struct.pack("<I", v))
    out += enc_vec(d["rigid_bodies"], enc_rigid)
    if not version_one:
        out += enc_vec(d["signs"], enc_sign)
    return out


def file_of(payload):
    return MAGIC + zlib.compress(payload)


def sample_particle(x, y, ty):  # lib.rs:662-681
    return (ty, 42, 2, x, y, 0.5, -0.25, 295.15, 0, 1, 2, 3, 4, 0x00112233, 0, 0)


def sample_save():  # lib.rs:683-717
    c = config_new(128, 96)
    cells = (c["xres"] // 4) * (c["yres"] // 4)
    return dict(version=2, config=c, particles=[sample_particle(10.0, 20.0, 1), sample_particle(11.0, 21.0, 2)],
                air_vx=[0.25] * cells, air_vy=[-0.5] * cells, air_pv=[1.5] * cells, air_hv=[295.15] * cells,
                fan_vx=[0.0] * cells, fan_vy=[0.0] * cells, wall_bmap=[0] * cells, wall_emap=[0] * cells,
                rigid_bodies=[], signs=[dict(x=32, y=48, text="Hot zone", ju=0),
                                        dict(x=90, y=12, text="Max 45 chars", ju=2)])


def dec_signs(payload, offset):
    """The signs vector at `offset` of a payload (the restatement's decoder)."""
    (n,) = struct.unpack_from("<Q", payload, offset)
    offset += 8
    out = []
    for _ in range(n):
        x, y, ln = struct.unpack_from("<iiQ", payload, offset)
        offset += 16
        text = payload[offset:offset + ln].decode()
        offset += ln
        out.append(dict(x=x, y=y, text=text, ju=payload[offset]))
        offset += 1
    return out


def signs_offset(d):
    return len(enc_save(d, version_one=True))


# ---------------------------------------------------------------- tests ----

@pytest.fixture(scope="module")
def SD(tf):
    return tf.SaveData


def test_config_default_is_simulation_config_new(tf):
    c = tf.SaveConfig()
    tf.lib().tpt_save_config_default(c, 100, 30)  # aligned to 100 x 64
    want = config_new(100, 30)
    for name, f in CONFIG_LAYOUT:
        got = getattr(c, name)
        if f == "o":
            assert getattr(c, "has_" + name) == 1
        assert got == pytest.approx(want[name]) if f in "fo" else got == want[name], name
    assert enc_config(want) == enc_config({n: (getattr(c, n) if f != "o" else getattr(c, n))
                                           for n, f in CONFIG_LAYOUT})


def test_encoder_agrees_with_the_restatement_byte_for_byte(SD):
    want = sample_save()
    want["signs"] = []
    s = SD.new(128, 96)
    cells = 32 * 24
    for g in ("air_vx", "air_vy", "air_pv", "air_hv", "fan_vx", "fan_vy"):
        s.set_grid(g, np.array(want[g], np.float32))
    s.set_particles(np.frombuffer(b"".join(enc_particle(p) for p in want["particles"]), np.uint32))
    payload = zlib.decompress(s.to_bytes()[8:])
    assert payload == enc_save(want)
    assert len(want["air_pv"]) == cells


def test_decoder_reads_the_restatements_payload(SD):
    d = sample_save()
    s = SD.from_bytes(file_of(enc_save(d)))
    info = s.info()
    assert (info.version, info.n_particles, info.n_signs, info.n_rigid_bodies) == (2, 2, 2, 0)
    assert s.config.xres == 128 and s.config.yres == 96 and s.config.render_mode == 0x47
    np.testing.assert_array_equal(s.grid("air_hv"), np.float32(295.15))
    p = s.particles()
    assert p[1, 0] == 2 and p[0, 13] == 0x00112233
    assert zlib.decompress(s.to_bytes()[8:]) == enc_save(d)  # signs kept as read


def test_magic_header_is_written(SD):  # lib.rs:719-723
    assert SD.from_bytes(file_of(enc_save(sample_save()))).to_bytes()[:8] == MAGIC


def test_roundtrip_preserves_state(SD):  # lib.rs:725-735
    s = SD.from_bytes(file_of(enc_save(sample_save())))
    r = SD.from_bytes(s.to_bytes())
    assert r.version == 2 and r.config.xres == 128 and r.config.yres == 96
    assert r.info().n_particles == 2 and r.particles()[1, 0] == 2
    assert r.grid("air_pv").size == 32 * 24


def test_roundtrip_preserves_signs(SD):  # lib.rs:737-748
    d = sample_save()
    payload = zlib.decompress(SD.from_bytes(SD.from_bytes(file_of(enc_save(d))).to_bytes()).to_bytes()[8:])
    signs = dec_signs(payload, signs_offset(d))
    assert signs == d["signs"]
    assert signs[0]["text"] == "Hot zone" and signs[1]["ju"] == 2


def test_version_one_payload_loads_without_signs(SD):  # lib.rs:750-778
    d = sample_save()
    d["version"] = 1
    s = SD.from_bytes(file_of(enc_save(d, version_one=True)))
    assert s.version == 1 and s.info().n_signs == 0
    assert s.particles().tobytes() == b"".join(enc_particle(p) for p in d["particles"])
    np.testing.assert_array_equal(s.grid("air_pv"), np.float32(1.5))


def test_payload_with_and_without_pressure(SD):  # lib.rs:780-805
    d = sample_save()
    kept = SD.from_bytes(file_of(enc_save(d))).retain_air_pressure(True)
    np.testing.assert_array_equal(kept.grid("air_vx"), np.float32(0.25))
    dropped = SD.from_bytes(file_of(enc_save(d))).retain_air_pressure(False)
    for g in ("air_vx", "air_vy", "air_pv", "air_hv"):
        assert dropped.grid(g).size == 0
    assert dropped.grid("wall_bmap").size == 32 * 24
    np.testing.assert_array_equal(dropped.grid("fan_vx"), np.float32(0.0))
    assert dropped.info().n_particles == 2 and dropped.info().n_signs == 2


def test_pressureless_payload_roundtrips(SD):  # lib.rs:807-819
    d = sample_save()
    r = SD.from_bytes(SD.from_bytes(file_of(enc_save(d))).retain_air_pressure(False).to_bytes())
    for g in ("air_vx", "air_vy", "air_pv", "air_hv"):
        assert r.grid(g).size == 0
        # restore_into zero-fills an absent grid (fit_f32, lib.rs:104-115)
        np.testing.assert_array_equal(r.restore_grid(g), np.float32(0.0))
    assert r.info().n_particles == 2 and r.info().n_signs == 2


def test_rejects_malformed_files(SD, tf):  # lib.rs:821-849
    good = SD.from_bytes(file_of(enc_save(sample_save()))).to_bytes()
    bad = bytearray(good)
    bad[0] = ord("X")
    for data in (bytes(bad), good[:5], good[:-4], b"", MAGIC):
        with pytest.raises(tf.TptError):
            SD.from_bytes(data)
    for v in (3, 0):
        d = sample_save()
        d["version"] = v
        with pytest.raises(tf.TptError, match="version"):
            SD.from_bytes(file_of(enc_save(d)))


def test_payload_is_zlib_compressed(SD):  # lib.rs:851-857
    d = sample_save()
    b = SD.from_bytes(file_of(enc_save(d))).to_bytes()
    assert b[8] == 0x78 and len(b) < len(enc_save(d))


def test_invalid_values_and_canvas_are_rejected(SD, tf):
    d = sample_save()
    for name, value in (("air_mode", 5), ("edge_mode", 3), ("xres", 0), ("yres", 16385)):
        e = dict(d, config=dict(d["config"], **{name: value}))
        with pytest.raises(tf.TptError):
            SD.from_bytes(file_of(enc_save(e)))
    payload = bytearray(enc_save(d))
    payload[4 + 8] = 2  # `paused` is a bool
    with pytest.raises(tf.TptError, match="bool"):
        SD.from_bytes(file_of(bytes(payload)))
    e = dict(d, signs=[dict(x=0, y=0, text="ok", ju=0)])
    raw = enc_save(e)
    raw = raw[:-3] + b"\xff\xfe" + raw[-1:]  # text bytes that are not UTF-8
    with pytest.raises(tf.TptError, match="UTF-8"):
        SD.from_bytes(file_of(raw))


def test_rigid_bodies_survive_a_roundtrip(SD):
    d = sample_save()
    d["rigid_bodies"] = [dict(id=7, active=True, f=[float(k) for k in range(10)],
                              pixels=[(1.0, -2.0, 5, 300.0, 3, 0, 0xFF, 4, 5), (0.5, 0.5, 6, 273.0, 0, 1, 0, 6, 7)])]
    s = SD.from_bytes(file_of(enc_save(d)))
    assert s.info().n_rigid_bodies == 1
    assert zlib.decompress(s.to_bytes()[8:]) == enc_save(d)


def test_truncations_and_flips_never_crash(SD, tf):
    rng = np.random.default_rng(3)
    payload = enc_save(sample_save())
    for _ in range(300):
        p = bytearray(payload)
        if rng.random() < 0.5:
            p = p[: int(rng.integers(0, len(p)))]
        else:
            for _ in range(int(rng.integers(1, 8))):
                p[int(rng.integers(0, len(p)))] = int(rng.integers(0, 256))
        try:
            SD.from_bytes(file_of(bytes(p))).info()
        except tf.TptError:
            pass


def test_instance_desc_follows_restore_into(SD, tf):
    d = sample_save()
    c = d["config"]
    c.update(air_mode=2, aheat_enable=True, gravity_mode=3, ambient_air_temp=250.0, edge_pressure=3.0,
             vorticity_coeff=0.7, convection_mode=1, edge_velocity_x=1.0, custom_gravity_y=-1.0, newton_grav=True)
    desc = SD.from_bytes(file_of(enc_save(d))).instance_desc()
    a = desc.air
    # copied from the save (lib.rs:266-276) ...
    assert (a.xcells, a.ycells, a.air_mode, a.aheat_enable, a.gravity_mode) == (32, 24, 2, 1, 3)
    assert a.ambient_air_temp == pytest.approx(250.0) and a.edge_pressure == pytest.approx(3.0)
    # ... the rest from SimulationConfig::new
    assert a.vorticity_coeff == pytest.approx(0.1) and a.convection_mode == 2 and a.edge_vx == 0.0
    assert a.custom_gy == pytest.approx(1.0) and desc.newton_grav == 0


def test_restore_grid_fits_the_cell_count(SD):
    s = SD.new(128, 96)
    s.set_grid("air_pv", np.arange(10, dtype=np.float32))  # wrong length: restored as zeros
    np.testing.assert_array_equal(s.restore_grid("air_pv"), np.zeros(32 * 24, np.float32))
    s.set_grid("wall_bmap", np.arange(32 * 24, dtype=np.uint32))
    np.testing.assert_array_equal(s.restore_grid("wall_bmap"), np.arange(32 * 24, dtype=np.uint32))
