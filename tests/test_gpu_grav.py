"""GPU parity of the gravity solve (tpt_grav_solve / _f32 through the C ABI).

FP32 plan: its FFT differs from the reference's in summation order and
twiddle rounding, so the bar is the per-tick tolerance
    max |g_gpu - g_ref| <= 1e-5 * max |g_ref|
against both the oracle's FP32 mirror of the reference solve and the FP64
oracle, and exact zeros where the mask is 0."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-5


def solve_gpu(tf, torch, X, Y, mask, mass_fx=None, mass_f32=None, precision=0, repeat=1):
    cfg = tf.SimulationConfig(xres=4 * X, yres=4 * Y, newton_grav=True)
    b = tf.SimBuffers(cfg)
    b.grav_mask.copy_(torch.from_numpy(np.ascontiguousarray(mask, np.uint32).view(np.int32)))
    solver = tf.GravityFft(precision)
    if mass_f32 is not None:
        m = torch.from_numpy(np.ascontiguousarray(mass_f32, np.float32)).cuda()
    else:
        m = torch.from_numpy(np.ascontiguousarray(mass_fx, np.int32)).cuda()
    outs = []
    for _ in range(repeat):
        solver.solve(b, m)
        torch.cuda.synchronize()
        outs.append((b.grav_fx.cpu().numpy().copy(), b.grav_fy.cpu().numpy().copy()))
    solver.close()
    return outs if repeat > 1 else outs[0]


def rel_max(a, b):
    return np.abs(a.astype(np.float64) - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("X,Y,seed", [(24, 24, 1), (64, 48, 2), (37, 29, 3), (153, 96, 4), (5, 7, 5),
                                      (16, 3, 6), (600, 40, 7), (40, 520, 8)])
def test_fp32_plan_stress(cuda, tf, oracle, X, Y, seed):
    """Shapes of both FFT forms: padded lengths 32..1024 (one warp per 1-D
    transform; 5x7 and 16x3 are padded up to 32) and longer ones (600 and 520
    cells: 2048-point transforms in shared memory)."""
    import workloads as W

    g = W.make_stress_instance(X, Y, seed)
    gx, gy = solve_gpu(tf, cuda, X, Y, g.gmask, g.mass_fx)
    rx, ry = oracle.grav_solve(X, Y, g.gmask, mass_fx=g.mass_fx)
    dx, dy = oracle.grav_solve(X, Y, g.gmask, mass_fx=g.mass_fx, dtype=np.float64)
    scale = max(np.abs(dx).max(), np.abs(dy).max())
    assert np.abs(gx - rx).max() <= TOL * scale and np.abs(gy - ry).max() <= TOL * scale
    assert np.abs(gx - dx).max() <= TOL * scale and np.abs(gy - dy).max() <= TOL * scale
    assert np.all(gx[g.gmask == 0] == 0) and np.all(gy[g.gmask == 0] == 0)


@pytest.mark.parametrize("cfg", [1, 2])
def test_fp32_plan_measured_configs(cuda, tf, oracle, cfg):
    import workloads as W

    inst = W.config_instances(cfg)[0]
    X, Y = inst.xcells, inst.ycells
    gx, gy = solve_gpu(tf, cuda, X, Y, inst.gmask, inst.mass_fx)
    rx, ry = oracle.grav_solve(X, Y, inst.gmask, mass_fx=inst.mass_fx)
    dx, dy = oracle.grav_solve(X, Y, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
    scale = max(np.abs(dx).max(), np.abs(dy).max())
    for a, r, d in ((gx, rx, dx), (gy, ry, dy)):
        assert np.abs(a - r).max() <= TOL * scale
        assert np.abs(a - d).max() <= TOL * scale


def test_fp32_plan_f32_mass_c3(cuda, tf, oracle):
    import workloads as W

    X = Y = 512
    mass = W.clustered_mass(X, Y, W.instance_seed(3, 0))
    mask = np.full(X * Y, 0xFFFFFFFF, np.uint32)
    gx, gy = solve_gpu(tf, cuda, X, Y, mask, mass_f32=mass)
    dx, dy = oracle.grav_solve(X, Y, mask, mass_f32=mass, dtype=np.float64)
    assert rel_max(gx, dx) <= TOL and rel_max(gy, dy) <= TOL


def test_empty_mass_and_closed_mask(cuda, tf):
    X, Y = 30, 20
    mask = np.full(X * Y, 0xFFFFFFFF, np.uint32)
    gx, gy = solve_gpu(tf, cuda, X, Y, mask, np.zeros(X * Y, np.int32))
    assert not gx.any() and not gy.any()
    m = np.ones(X * Y, np.int32) * 65536
    gx, gy = solve_gpu(tf, cuda, X, Y, np.zeros(X * Y, np.uint32), m)
    assert not gx.any() and not gy.any()


def test_repeated_solves_are_identical(cuda, tf):
    import workloads as W

    inst = W.config_instances(1)[0]
    outs = solve_gpu(tf, cuda, inst.xcells, inst.ycells, inst.gmask, inst.mass_fx, repeat=3)
    for gx, gy in outs[1:]:
        assert np.array_equal(gx, outs[0][0]) and np.array_equal(gy, outs[0][1])


def test_step_gravity_rebuilds_mask_after_wall_change(cuda, tf, oracle):
    import workloads as W

    inst = W.make_stress_instance(48, 40, 5)
    b = tf.SimBuffers.from_instance(inst)
    b.grav_mask.zero_()
    b.grav_mask_dirty = True
    solver = tf.GravityFft()
    tf.step_gravity(b, solver)
    cuda.cuda.synchronize()
    assert np.array_equal(b.grav_mask.cpu().numpy().view(np.uint32), oracle.grav_mask(inst.wall, 48, 40))
    rx, ry = oracle.grav_solve(48, 40, inst.gmask, mass_fx=inst.mass_fx, dtype=np.float64)
    gx = b.grav_fx.cpu().numpy()
    assert rel_max(gx, rx) <= TOL
    b.config.newton_grav = False
    tf.step_gravity(b, solver)
    assert not b.grav_fx.any().item() and not b.grav_fy.any().item()
