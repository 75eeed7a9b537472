"""GPU gravity tick with particles (`tpt_grav_step`) against the oracle's
restatement of gravity_kernel.rs:217-527 on seeded sandboxes:

  mass accumulator and snapshot   bit-exact (integer atomics)
  particle velocities             bit-exact, given the solved field
  gx/gy                           the solve of the well-seeded snapshot,
                                  max err <= 1e-5 (FP32) / 1e-4 (split-BF16)
                                  of max|g| against the FP64 oracle
  painted wells                   consumed
over two ticks in a row (the second solve reads the first tick's mass)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _to_gpu(cuda, d):
    # u32 grids travel as i32 tensors of the same bits
    return {k: (None if v is None else cuda.from_numpy(np.ascontiguousarray(
        v.view(np.int32) if v.dtype == np.uint32 else v)).cuda()) for k, v in d.items()}


def _to_np(d, like):
    return {k: (None if v is None else v.cpu().numpy().view(like[k].dtype)) for k, v in d.items()}


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("xres,yres", [(256, 192), (612, 384)])
def test_grav_step_matches_oracle(cuda, tf, oracle, precision, xres, yres):
    import workloads as W

    X, Y = xres // 4, yres // 4
    state = W.gravity_state(xres, yres, 11 + xres)
    parts = W.gravity_particles(xres, yres, 20000, 12 + yres)
    lut = W.move_lut(192, 13)
    solver = tf.GravityFft(precision)
    gs, gp = _to_gpu(cuda, state), _to_gpu(cuda, parts)
    glut = cuda.from_numpy(lut.view(np.int32)).cuda()
    want_s, want_p = state, parts
    for tick in range(2):
        solver.step(gs, gp, glut, 192, xres, yres, 1.0)
        cuda.cuda.synchronize()
        assert tf.lib().tpt_check_device_errors() == 0
        got_s, got_p = _to_np(gs, state), _to_np(gp, parts)
        seeded = oracle.grav_seed(want_s, xres, yres)
        # the field is the solve of the snapshot with the wells folded in
        dx, dy = oracle.grav_solve(X, Y, seeded["grav_mask"], mass_fx=seeded["mass_prev"], dtype=np.float64)
        tol = 1e-4 if precision else 1e-5
        for g, d in ((got_s["gx"], dx), (got_s["gy"], dy)):
            assert np.abs(g.astype(np.float64) - d).max() <= tol * max(np.abs(d).max(), 1e-30), tick
        seeded["gx"], seeded["gy"] = got_s["gx"], got_s["gy"]
        want_s, want_p = oracle.grav_particles_and_finish(seeded, want_p, lut, 192, xres, yres, 1.0)
        for k in ("mass", "mass_prev", "tool_mass"):
            assert np.array_equal(got_s[k], want_s[k]), (tick, k)
        for k in ("vx", "vy"):
            assert np.array_equal(got_p[k].view(np.uint32), want_p[k].view(np.uint32)), (tick, k)
        assert not got_s["tool_mass"].any()
        assert np.count_nonzero(got_s["mass_prev"]) > 10
    solver.close()


def test_grav_step_rejects_bad_arguments(cuda, tf):
    import ctypes
    import workloads as W

    solver = tf.GravityFft(0)
    solver._ensure(16, 16)
    st = tf.GravState(xres=64, yres=60)  # 16 x 15 cells: not the plan's size
    for k in tf.GRAV_STATE_FIELDS:
        setattr(st, k, 16)  # non-NULL placeholders: the size check comes first
    pa = tf.Particles()
    assert tf.lib().tpt_grav_step(solver._plan, ctypes.byref(st), ctypes.byref(pa), None) == -1
    st.yres = 64
    st.mass = None
    assert tf.lib().tpt_grav_step(solver._plan, ctypes.byref(st), ctypes.byref(pa), None) == -2
    st.mass, st.override_set = 16, None  # override pair half set
    assert tf.lib().tpt_grav_step(solver._plan, ctypes.byref(st), ctypes.byref(pa), None) == -2
    st.override_set = 16
    pa.num_slots = 5  # slots without arrays
    assert tf.lib().tpt_grav_step(solver._plan, ctypes.byref(st), ctypes.byref(pa), None) == -2
    solver.close()
