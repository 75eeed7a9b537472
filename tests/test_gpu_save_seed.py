"""Real saves seeding the field step: a `.tptrs` file (the host codec of
crates/tpt-save/src/lib.rs) decoded, restored the way SaveData::restore_into
restores it (lib.rs:262-345), stepped on the GPU as one grid and inside a
batch, bit-exact against the FP32 oracle from the same restored state, and
written back into the save; and a `.tpt3` file seeding the 3-D field step."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _save_bytes(tf, seed, xres, yres, air_mode=0, aheat=1, drop_pressure=False):
    import workloads as W

    inst = W.make_stress_instance(xres // 4, yres // 4, seed)
    s = tf.SaveData.new(xres, yres)
    c = s.config
    c.air_mode, c.aheat_enable, c.vorticity_coeff = air_mode, aheat, 0.9  # vorticity is not restored
    s.config = c
    for name, key in (("air_pv", "pv"), ("air_vx", "vx"), ("air_vy", "vy"), ("air_hv", "hv"), ("fan_vx", "fan_vx"),
                      ("fan_vy", "fan_vy"), ("wall_bmap", "wall"), ("wall_emap", "emap")):
        s.set_grid(name, getattr(inst, key))
    s.retain_air_pressure(not drop_pressure)
    return s.to_bytes()


@pytest.mark.parametrize("drop_pressure", [False, True])
def test_save_seeds_one_grid(cuda, tf, oracle, drop_pressure):
    from test_gpu_air import assert_bit_exact

    inst = tf.SaveData.from_bytes(_save_bytes(tf, 21, 612, 384, drop_pressure=drop_pressure)).to_instance()
    assert inst.config.vorticity_coeff == pytest.approx(0.1)
    if drop_pressure:
        assert not inst.pv.any() and not inst.hv.any()
    b = tf.SimBuffers.from_instance(inst)
    for _ in range(12):
        tf.step_air_gpu(b)
    cuda.cuda.synchronize()
    assert_bit_exact(b.air_state(), oracle.air_steps(inst, 12), "save-seeded grid")


def test_saves_seed_a_batch_and_are_written_back(cuda, tf, oracle):
    from test_gpu_air import assert_bit_exact

    raws = [_save_bytes(tf, 30 + k, x, y, air_mode=m) for k, (x, y, m) in
            enumerate(((612, 384, 0), (256, 200, 2), (1600, 900, 0)))]
    saves = [tf.SaveData.from_bytes(r) for r in raws]
    insts = [s.to_instance() for s in saves]
    batch = tf.Batch(insts)
    batch.step(9)
    cuda.cuda.synchronize()
    for i, (s, inst) in enumerate(zip(saves, insts)):
        got = batch.state(i)
        assert_bit_exact(got, oracle.air_steps(inst, 9), f"save {i}")
        s.set_field_state(got)
        back = tf.SaveData.from_bytes(s.to_bytes())
        np.testing.assert_array_equal(back.grid("air_pv").view(np.uint32), got["pv"].view(np.uint32))
        np.testing.assert_array_equal(back.grid("wall_emap"), got["emap"])
    batch.close()


def test_tpt3_save_seeds_the_3d_field_step(cuda, tf, oracle):
    """A `.tpt3` world (crates/tpt-save/src/voxel3d.rs) written the way the
    engine saves it (read_air_fields, engine.rs:391-430: pv in pressure
    units), decoded, restored as load_world restores it and stepped one
    tick, bit-exact against the oracle from the same restored state."""
    import voxel3d as V
    import workloads as W

    w = W.voxel_world(0x3D33, active=0.5)
    s = tf.VoxSave.new()
    s.set_array("voxels", w["voxel"])
    s.set_array("aux_tmp", w["aux_tmp"])
    s.set_array("air", np.concatenate([w["vx"], w["vy"], w["vz"], w["pv"].astype(np.float32) / np.float32(1024.0),
                                       w["temp"], w["solid"]]))
    d = tf.VoxSave.from_bytes(s.to_bytes()).to_world()
    np.testing.assert_array_equal(d["pv"], w["pv"])  # the fixed-point round trip is exact
    assert d["sim_count"][0] > 0
    bufs, air = V.upload(d)
    plan = V.Plan()
    V.field_step(plan, [(bufs, air)], 12)
    V.gravity_gather(plan, bufs)
    cuda.cuda.synchronize()
    want = {k: v.copy() for k, v in d.items()}
    oracle.vox_field_step(want, 12)
    oracle.vox_grav_gather(want)
    got = V.download(bufs, air)
    for k in ("pv", "p", "p_tmp", "vx", "vy", "vz", "solid", "temp", "grav_mass", "grav_potential", "grav_force_z"):
        assert np.array_equal(np.ascontiguousarray(got[k]).view(np.uint32),
                              np.ascontiguousarray(want[k]).view(np.uint32)), k
