"""CPU tests of the C ABI: the library loads, exports every entry point the
header declares, validates arguments before touching a GPU, and its host
helpers match the oracle (no compute call needs a GPU here)."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(tpt_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol(tf):
    names = header_functions()
    assert len(names) >= 20
    lib = tf.lib()
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(tf.EXPORTS) == names
    assert b"sm_100a" in lib.tpt_version()


def test_arguments_are_validated_before_any_device_work(tf):
    lib = tf.lib()
    assert lib.tpt_air_step(None, None, None) == -2
    assert b"NULL" in lib.tpt_last_error_string()
    p = tf.AirParams()
    lib.tpt_air_params_default(ctypes.byref(p), 10, 10)
    p.air_mode = 9
    assert lib.tpt_air_step(ctypes.byref(p), ctypes.byref(tf.AirBufs()), None) == -5
    p.air_mode = 0
    p.xcells = 5000
    assert lib.tpt_air_step(ctypes.byref(p), ctypes.byref(tf.AirBufs()), None) == -1
    p.xcells = 0  # empty grid: the reference returns silently (mod.rs:124-126)
    assert lib.tpt_air_step(ctypes.byref(p), ctypes.byref(tf.AirBufs()), None) == 0
    h = ctypes.c_void_p()
    assert lib.tpt_grav_plan_create(0, 10, 0, ctypes.byref(h)) == -1
    assert lib.tpt_grav_plan_create(10, 10, 7, ctypes.byref(h)) == -5
    assert lib.tpt_grav_plan_create(10, 10, 0, None) == -2
    assert lib.tpt_batch_create(0, None, 0, ctypes.byref(h)) == -1
    d = (tf.InstanceDesc * 1)()
    d[0].air.xcells, d[0].air.ycells = 2, 10
    assert lib.tpt_batch_create(1, d, 0, ctypes.byref(h)) == -1
    assert lib.tpt_grav_solve(None, None, 1.0, None, None, None, None) == -2
    assert lib.tpt_grav_step(None, None, None, None) == -2
    assert lib.tpt_batch_step(None, 1, None) == -2
    assert lib.tpt_grav_plan_destroy(None) == 0 and lib.tpt_batch_destroy(None) == 0
    # 3-D field step
    assert lib.tpt_vox_plan_create(0, None) == -2
    assert lib.tpt_vox_plan_create(9, ctypes.byref(h)) == -5
    w = tf.VoxWorld()
    assert lib.tpt_vox_air_clear(None, None) == -2
    assert lib.tpt_vox_air_clear(ctypes.byref(w), None) == -2
    assert lib.tpt_vox_air_gather(None, ctypes.byref(w), None) == -2
    assert lib.tpt_vox_air_solve(None, ctypes.byref(w), 12, None) == -2
    assert lib.tpt_vox_grav_solve(None, ctypes.byref(w), None) == -2
    assert lib.tpt_vox_grav_clear_mass(None, ctypes.byref(w), None) == -2
    assert lib.tpt_vox_grav_gather(None, ctypes.byref(w), None) == -2
    assert lib.tpt_vox_field_step(None, ctypes.byref(w), 1, 12, None) == -2
    assert lib.tpt_vox_plan_form(None) == -2 and lib.tpt_vox_plan_destroy(None) == 0


def test_default_params_match_reference(tf):
    # crates/tpt-core/src/particle.rs:290-345
    p = tf.AirParams()
    tf.lib().tpt_air_params_default(ctypes.byref(p), 153, 96)
    assert (p.xcells, p.ycells, p.air_mode, p.aheat_enable, p.convection_mode, p.gravity_mode) == (153, 96, 0, 0, 2, 0)
    assert abs(p.ambient_air_temp - 295.15) < 1e-4 and abs(p.vorticity_coeff - 0.1) < 1e-7
    assert (p.edge_pressure, p.edge_vx, p.edge_vy, p.custom_gx, p.custom_gy) == (0.0, 0.0, 0.0, 0.0, 1.0)
    c = tf.SimulationConfig()
    assert (c.xcells(), c.ycells()) == (153, 96)


def test_host_helpers_match_oracle(tf, oracle):
    import workloads as W

    inst = W.make_stress_instance(40, 31, 11)
    m = tf.rebuild_gravity_mask(inst.wall, 40, 31)
    assert np.array_equal(m, oracle.grav_mask(inst.wall, 40, 31))
    ba = np.zeros(40 * 31, np.uint32)
    bh = np.zeros(40 * 31, np.uint32)
    e = inst.emap.copy()
    rc = tf.lib().tpt_wall_masks_host(tf._ptr(inst.wall), tf._ptr(e), tf._ptr(ba), tf._ptr(bh), 40 * 31)
    assert rc == 0
    wa, wh = W.wall_masks(inst.wall, inst.emap)
    assert np.array_equal(ba, wa) and np.array_equal(bh, wh)
    for v in (0.0, 1.0, -1.0, 0.3, -0.7, 7.62939453125e-06, 1e6, -1e6, 1e9):
        assert tf.mass_to_fixed(v) == oracle.mass_to_fixed(v) or abs(v) >= 32768.0


def test_python_mirror_fails_loudly_without_a_gpu(tf):
    """No CPU fallback: a compute call without an sm_100 device raises."""
    import torch

    if torch.cuda.is_available():
        return
    p = tf.AirParams()
    tf.lib().tpt_air_params_default(ctypes.byref(p), 8, 8)
    b = tf.AirBufs()
    for name, _ in tf.AirBufs._fields_[:16]:
        setattr(b, name, 16)  # never dereferenced: the device check comes first
    rc = tf.lib().tpt_air_step(ctypes.byref(p), ctypes.byref(b), None)
    assert rc in (-3, -7)


def test_python_struct_mirrors_match_the_header(tf):
    """The ctypes mirrors of the C structs the batch API passes by pointer
    (tpt_batch_tuning, tpt_batch_profile) list the header's fields in the
    header's order, so a field appended to one side only fails here on CPU."""
    import os
    import re

    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "tpt_field.h")).read()

    def fields(struct):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct), hdr, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        names = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            decl = re.sub(r"^\w+\s+", "", decl)  # the type
            names += [n.strip() for n in decl.split(",")]
        return names

    assert fields("tpt_batch_tuning") == [n for n, _ in tf.BatchTuning._fields_]
    assert fields("tpt_batch_profile") == [n for n, _ in tf.BatchProfile._fields_]
