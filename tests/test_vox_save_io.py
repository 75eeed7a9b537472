"""`.tpt3` 3-D saves (crates/tpt-save/src/voxel3d.rs) through the library's
host codec, on CPU.

The reference's tests for the format (voxel3d.rs:315-501) are ported one by
one; the payloads they build without validation (`encode_raw`) come from a
second, independent restatement of the layout below (bincode 1.3.3's default
encoding of Voxel3dSaveData, voxel3d.rs:42-90, and Voxel3dConfig,
crates/tpt-core/src/voxel3d/mod.rs:96-122), which must also agree with the
codec byte for byte. The restore of the air state follows
Voxel3dEngine::load_world (crates/tpt-sim/src/voxel3d/engine.rs:523-581).
"""
import struct
import zlib

import numpy as np
import pytest

MAGIC = b"TPT3RS01"
VOXELS, CELLS, MAX_BODIES, BODY_VOXELS = 256 ** 3, 64 ** 3, 64, 32768


def default_config():  # Voxel3dConfig::default (mod.rs:124-141)
    return dict(dim=256, paused=False, ambient_temp_k=293.15, gravity=(0.0, -9.81, 0.0), edge_mode=0,
                air_enabled=True, air_iterations=12, sun_dir=(0.5, 0.70710677, 0.5), exposure=1.0, render_scale=1.0,
                ao_rays=2, shadows=True)


def enc_config(c):
    return (struct.pack("<I?f", c["dim"], c["paused"], c["ambient_temp_k"]) + struct.pack("<3f", *c["gravity"])
            + struct.pack("<I?I", c["edge_mode"], c["air_enabled"], c["air_iterations"])
            + struct.pack("<3f", *c["sun_dir"])
            + struct.pack("<ffI?", c["exposure"], c["render_scale"], c["ao_rays"], c["shadows"]))


def enc_array(a, dt):
    a = np.ascontiguousarray(a, dt)
    return struct.pack("<Q", a.size) + a.astype(np.dtype(dt).newbyteorder("<")).tobytes()


def enc_body(b):
    return (struct.pack("<16f", *b["pos"], *b["quat"], *b["lin_vel"], *b["ang_vel"], *b["half_extents"])
            + struct.pack("<I", b["ty"]) + enc_array(b["local_voxels"], np.uint32))


def enc_save(d):
    out = struct.pack("<I", d["version"]) + enc_config(d["config"]) + enc_array(d["voxels"], np.uint32)
    for k, dt in (("aux_ctype", np.uint32), ("aux_tmp", np.int32), ("aux_tmp2", np.int32), ("aux_tmp3", np.int32),
                  ("air", np.float32)):
        out += enc_array(d[k], dt)
    return out + struct.pack("<Q", len(d["bodies"])) + b"".join(enc_body(b) for b in d["bodies"])


def encode_raw(d):  # voxel3d.rs:289-299
    return MAGIC + zlib.compress(enc_save(d))


def sample_body(local):  # voxel3d.rs:301-311
    return dict(pos=(1.5, 2.5, -3.0), quat=(0.0, 0.0, 0.0, 1.0), lin_vel=(0.5, -0.25, 0.125), ang_vel=(1.0, -2.0, 3.0),
                half_extents=(0.5, 1.0, 1.5), ty=7, local_voxels=local)


def save(config=None, voxels=None, air=(), bodies=(), aux=None, version=4):
    aux = aux or {}
    return dict(version=version, config=config or default_config(),
                voxels=np.zeros(VOXELS, np.uint32) if voxels is None else voxels,
                aux_ctype=aux.get("ctype", []), aux_tmp=aux.get("tmp", []), aux_tmp2=aux.get("tmp2", []),
                aux_tmp3=aux.get("tmp3", []), air=np.asarray(air, np.float32), bodies=list(bodies))


@pytest.fixture(scope="module")
def VS(tf):
    return tf.VoxSave


def test_default_config_and_empty_save_bytes(VS):
    s = VS.new()
    c = s.config
    want = default_config()
    assert (c.dim, c.paused, c.air_enabled, c.air_iterations, c.ao_rays, c.shadows) == (256, 0, 1, 12, 2, 1)
    assert list(c.gravity) == pytest.approx(want["gravity"]) and list(c.sun_dir) == pytest.approx(want["sun_dir"])
    assert zlib.decompress(s.to_bytes()[8:]) == enc_save(save())


def test_empty_roundtrip(VS, tf):  # voxel3d.rs:315-346
    d = save(config=dict(default_config(), paused=True, ambient_temp_k=310.0, gravity=(0.0, -3.5, 0.25)))
    loaded = VS.from_bytes(encode_raw(d))
    c = loaded.config
    assert c.paused == 1 and c.ambient_temp_k == pytest.approx(310.0) and list(c.gravity) == pytest.approx([0, -3.5, 0.25])
    assert loaded.info().len[0] == VOXELS and not loaded.array("voxels").any()
    assert loaded.array("air").size == 0 and loaded.info().n_bodies == 0
    assert zlib.decompress(loaded.to_bytes()[8:]) == enc_save(d)


def test_populated_roundtrip_and_config_survives(VS):  # voxel3d.rs:348-384
    cfg = dict(dim=256, paused=False, ambient_temp_k=293.15, gravity=(1.0, -9.81, -0.5), edge_mode=1,
               air_enabled=True, air_iterations=20, sun_dir=(0.25, 0.5, 0.75), exposure=1.75, render_scale=0.75,
               ao_rays=4, shadows=False)
    vox = np.zeros(VOXELS, np.uint32)
    vox[0], vox[VOXELS // 2], vox[-1] = 1, 0xDEADBEEF, 0x12345678
    air = np.zeros(CELLS, np.float32)
    air[0], air[CELLS // 2], air[-1] = 293.15, -4.5, 1.0e6
    d = save(config=cfg, voxels=vox, air=air,
             bodies=[sample_body(np.full(512, 0x01020304, np.uint32)), sample_body([])])
    loaded = VS.from_bytes(encode_raw(d))
    assert zlib.decompress(loaded.to_bytes()[8:]) == enc_save(d)
    c = loaded.config
    assert (c.edge_mode, c.air_iterations, c.ao_rays, c.shadows) == (1, 20, 4, 0)
    assert loaded.array("air")[CELLS // 2] == np.float32(-4.5) and loaded.info().n_bodies == 2
    np.testing.assert_array_equal(loaded.array("voxels")[[0, VOXELS // 2, VOXELS - 1]], [1, 0xDEADBEEF, 0x12345678])


def test_aux_arrays_roundtrip(VS):  # voxel3d.rs:386-415
    vox = np.zeros(VOXELS, np.uint32)
    vox[7] = 5
    aux = {k: np.zeros(VOXELS, np.uint32 if k == "ctype" else np.int32) for k in ("ctype", "tmp", "tmp2", "tmp3")}
    aux["ctype"][7], aux["tmp"][7], aux["tmp2"][7], aux["tmp3"][7] = 0xDEADBEEF, -123, 456, np.iinfo(np.int32).min
    s = VS.new()
    s.set_array("voxels", vox)
    for k, v in aux.items():
        s.set_array("aux_" + k, v)
    loaded = VS.from_bytes(s.to_bytes())
    assert loaded.array("aux_ctype")[7] == 0xDEADBEEF and loaded.array("aux_tmp")[7] == -123
    assert loaded.array("aux_tmp2")[7] == 456 and loaded.array("aux_tmp3")[7] == np.iinfo(np.int32).min


def test_rejects_bad_magic_and_short_input(VS, tf):  # voxel3d.rs:417-426
    for data in (b"", MAGIC):
        with pytest.raises(tf.TptError):
            VS.from_bytes(data)
    with pytest.raises(tf.TptError, match="bad magic"):
        VS.from_bytes(b"NOTTPT03" + bytes(16))


def test_rejects_unsupported_version(VS, tf):  # voxel3d.rs:428-447
    d = save(voxels=np.zeros(0, np.uint32), version=5)
    with pytest.raises(tf.TptError, match="unsupported voxel save version 5"):
        VS.from_bytes(encode_raw(d))


def test_rejects_wrong_voxel_count(VS, tf):  # voxel3d.rs:449-467
    with pytest.raises(tf.TptError, match=f"expected {VOXELS}"):
        VS.from_bytes(encode_raw(save(voxels=np.zeros(VOXELS - 1, np.uint32))))


def test_to_bytes_rejects_invalid_layout(VS, tf):  # voxel3d.rs:469-480
    s = VS.new()
    s.set_array("voxels", np.zeros(0, np.uint32))
    with pytest.raises(tf.TptError, match="voxels"):
        s.to_bytes()
    s.set_array("voxels", np.zeros(VOXELS, np.uint32))
    s.set_array("air", np.zeros(CELLS + 1, np.float32))
    with pytest.raises(tf.TptError, match="multiple"):
        s.to_bytes()


def test_rejects_invalid_air_and_body_layout(VS, tf):  # voxel3d.rs:482-500
    with pytest.raises(tf.TptError, match="multiple"):
        VS.from_bytes(encode_raw(save(air=np.zeros(CELLS + 1, np.float32))))
    with pytest.raises(tf.TptError, match=f"rigid bodies.*{MAX_BODIES}"):
        VS.from_bytes(encode_raw(save(bodies=[sample_body([])] * (MAX_BODIES + 1))))
    with pytest.raises(tf.TptError, match=f"local grid.*{BODY_VOXELS}"):
        VS.from_bytes(encode_raw(save(bodies=[sample_body(np.zeros(BODY_VOXELS + 1, np.uint32))])))


def test_restore_air_follows_load_world(VS, tf):
    # no air in the save: the cleared AirState
    r = VS.new().restore_air()
    assert not r["vx"].any() and not r["pv"].any() and (r["temp"] == np.float32(293.15)).all()
    # six slots: vx vy vz pv t solid, pv to 1/1024 fixed point with a saturating cast
    air = np.random.default_rng(2).uniform(-3, 3, 6 * CELLS).astype(np.float32)
    air[3 * CELLS: 3 * CELLS + 4] = [1.5, -2.25, np.nan, 3.0e9]
    s = VS.new()
    s.set_array("air", air)
    r = s.restore_air()
    np.testing.assert_array_equal(r["vy"], air[CELLS:2 * CELLS])
    np.testing.assert_array_equal(r["solid"], air[5 * CELLS:])
    assert list(r["pv"][:4]) == [1536, -2304, 0, np.iinfo(np.int32).max]
    want = np.trunc(air[3 * CELLS + 4:4 * CELLS] * np.float32(1024.0)).astype(np.int32)
    np.testing.assert_array_equal(r["pv"][4:], want)
    s.set_array("air", np.zeros(2 * CELLS, np.float32))  # a multiple, but not the six fields load_world takes
    with pytest.raises(tf.TptError, match="air floats"):
        s.restore_air()
