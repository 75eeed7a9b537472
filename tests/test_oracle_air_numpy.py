"""The C++ oracle's 2-D air tick against a second, independent restatement
(oracle/air_numpy.py: vectorised numpy, f32 per operation, written from the
reference's Rust kernels). No reference test pins the air arithmetic, so the
two restatements pin each other: they must agree in every bit after every
tick, on every wall kind, air / convection / gravity mode and grid shape the
GPU parity tests use, on the C1 workload, and on non-finite inputs."""
import numpy as np
import pytest

from test_gpu_air import MODES  # noqa: E402  (the mode list the GPU parity tests run)


def _same(a, b, ctx, nan_equal=False):
    for k in ("pv", "vx", "vy", "hv"):
        g = np.ascontiguousarray(a[k], np.float32)
        w = np.ascontiguousarray(b[k], np.float32)
        diff = g.view(np.uint32) != w.view(np.uint32)
        if nan_equal:
            diff &= ~(np.isnan(g) & np.isnan(w))
        bad = np.flatnonzero(diff)
        assert bad.size == 0, f"{ctx} {k}: {bad.size} cells differ, first {bad[0]}: {g[bad[0]]!r} vs {w[bad[0]]!r}"
    for k in ("emap", "bair", "bairh"):
        assert np.array_equal(np.asarray(a[k], np.uint32), np.asarray(b[k], np.uint32)), f"{ctx} {k}"


@pytest.fixture(scope="module")
def npo():
    import air_numpy

    return air_numpy


@pytest.mark.parametrize("shape", [(24, 24), (37, 29), (96, 80), (33, 9)])
@pytest.mark.parametrize("mode", range(len(MODES)))
def test_stress_every_mode_both_restatements_agree(oracle, npo, shape, mode):
    import workloads as W

    X, Y = shape
    inst = W.make_stress_instance(X, Y, 1000 + 7 * mode + X, config=W.AirConfig(**MODES[mode]))
    for ticks in (1, 6):
        _same(npo.air_steps(inst, ticks), oracle.air_steps(inst, ticks), f"{shape} {MODES[mode]} t{ticks}")


def test_c1_workload_100_ticks(oracle, npo):
    import workloads as W

    inst = W.config_instances(1)[0]
    _same(npo.air_steps(inst, 100), oracle.air_steps(inst, 100), "C1 100 ticks")


def test_tiny_grids(oracle, npo):
    import workloads as W

    for X, Y in ((3, 3), (4, 40), (40, 4), (5, 5), (64, 3)):
        inst = W.make_stress_instance(X, Y, 77 + X * Y)
        _same(npo.air_steps(inst, 3), oracle.air_steps(inst, 3), f"{X}x{Y}")


def nonfinite_instance(X=40, Y=30, seed=31):
    """A stress instance with NaN and +-Inf in pv/vx/vy/hv and velocities at
    and beyond the +-256 clamp, so the walks run to their longest and the
    f32 -> i32 conversions see NaN and out-of-range values."""
    import workloads as W

    inst = W.make_stress_instance(X, Y, seed)
    n = X * Y
    idx = np.arange(n)
    inst.vx[idx % 97 == 5] = np.nan
    inst.vy[idx % 89 == 7] = np.inf
    inst.vx[idx % 83 == 11] = -np.inf
    inst.pv[idx % 71 == 3] = np.nan
    inst.hv[idx % 67 == 2] = np.nan
    inst.vx[idx % 13 == 1] = 256.0
    inst.vy[idx % 17 == 2] = -256.0
    inst.vx[idx % 19 == 3] = 1.0e30
    return inst


def test_nonfinite_and_clamp_inputs(oracle, npo):
    inst = nonfinite_instance()
    for ticks in (1, 3):
        _same(npo.air_steps(inst, ticks), oracle.air_steps(inst, ticks), f"non-finite t{ticks}", nan_equal=True)


def test_f32_to_i32_conversion(npo):
    v = np.array([0.0, -0.0, 0.99, -0.99, 2.5, -2.5, 2147483520.0, 3e9, -3e9, np.inf, -np.inf, np.nan],
                 np.float32)
    want = [0, 0, 0, 0, 2, -2, 2147483520, 2147483647, -2147483648, 2147483647, -2147483648, 0]
    assert npo.f2i(v).tolist() == want


def test_smoothing_weight_sum(npo):
    # advect.rs:215-247: nine taps, centre 1, edges e^-2, corners e^-4, summed
    # in f32 in dy-major order
    s = np.float32(0)
    for w in (0.01831564, 0.13533528, 0.01831564, 0.13533528, 1.0, 0.13533528, 0.01831564, 0.13533528,
              0.01831564):
        s = np.float32(s + np.float32(w))
    assert npo.WSUM == s and abs(float(s) - (1.0 + 4 * 0.13533528 + 4 * 0.01831564)) < 1e-6


def test_far_advect_walk_known_answers(npo):
    """advect.rs:66-152 by hand on a 10x10 grid, cell (5, 5), v = (-4, 0):
    0.7*|v| = 2.8 > 1 and the backtrace x = 7.8 lies in [2, 8), so the walk
    takes int(2.8) = 2 steps of +1 along x: it stops before the first blocked
    or out-of-grid cell, or takes the full backtrace when none is met."""
    g = npo.Grid(10, 10)
    dx = np.zeros((10, 10), np.float32)
    dy = np.zeros((10, 10), np.float32)
    dx[5, 5] = -4.0

    def target(blocked_cells):
        blk = np.zeros((10, 10), bool)
        for (x, y) in blocked_cells:
            blk[y, x] = True
        tx, ty = npo.far_advect_target(dx, dy, blk, g)
        return float(tx[5, 5]), float(ty[5, 5])

    assert target([]) == (np.float32(5) - np.float32(-4.0) * np.float32(0.7), 5.0)
    assert target([(7, 5)]) == (6.0, 5.0)  # second step hits: back to (6, 5)
    assert target([(6, 5)]) == (5.0, 5.0)  # first step hits: stays on the cell
    assert target([(8, 5)]) == (np.float32(7.8), 5.0)  # beyond the walk: full backtrace
    # counter bits 0..7 of block_airh do not block the heat walk; bit 3 does
    bairh = np.zeros((10, 10), np.uint32)
    bairh[5, 7] = 0x7
    tx, _ = npo.far_advect_target(dx, dy, (bairh & np.uint32(0x8)) != 0, g)
    assert float(tx[5, 5]) == np.float32(7.8)
    bairh[5, 7] = 0x8
    tx, _ = npo.far_advect_target(dx, dy, (bairh & np.uint32(0x8)) != 0, g)
    assert float(tx[5, 5]) == 6.0
    # a backtrace landing outside [2, X-2) is not walked at all
    dx[5, 5] = -5.0  # x = 8.5 >= 8
    tx, _ = npo.far_advect_target(dx, dy, np.ones((10, 10), bool), g)
    assert float(tx[5, 5]) == np.float32(5) - np.float32(-5.0) * np.float32(0.7)
