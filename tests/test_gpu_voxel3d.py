"""GPU 3-D field step (crates/tpt-sim/src/voxel3d) against the oracle's
restatement of its kernels, bit-exact, on seeded 64^3 worlds, in the three forms
of the solve (batched launches per sweep index, the cluster launch, and the
reference's per-pass, per-sweep launches):

  air gather       solid and temp of the listed bricks' cells; the other
                   cells keep their values; empty and full brick lists
  air solve        pv (i32), the p / p_tmp pair as the reference's
                   alternation leaves it, vx / vy / vz; 0, 1, 2, 3, 12 sweeps
  gravity solve    potential pair and forces after 24 sweeps
  gravity gather   fixed-point mass (wrapping integer sums)
  field step       three worlds in one call, two ticks in a row
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORMS = {"cluster": 1, "per_sweep": 2, "batched": 3}
AIR_KEYS = ("pv", "p", "p_tmp", "vx", "vy", "vz")
GRAV_KEYS = ("grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y", "grav_force_z", "grav_mass")


@pytest.fixture(scope="module")
def world():
    import workloads as W

    return W.voxel_world(0x3D01)


def _copy(d):
    return {k: v.copy() for k, v in d.items()}


def _same(got, want, keys, what=""):
    for k in keys:
        g, w = np.ascontiguousarray(got[k]), np.ascontiguousarray(want[k])
        assert g.dtype.itemsize == 4 and w.dtype.itemsize == 4
        gb, wb = g.view(np.uint32), w.view(np.uint32)
        bad = np.flatnonzero(gb != wb)
        assert bad.size == 0, f"{what}{k}: {bad.size} cells differ, first {bad[0]}: got {g[bad[0]]!r} want {w[bad[0]]!r}"


@pytest.fixture(scope="module")
def plans(tf, cuda):
    import voxel3d as V

    return {name: V.Plan(form) for name, form in FORMS.items()}


def test_auto_plan_takes_the_batched_form(tf, cuda):
    import voxel3d as V

    assert V.Plan(tf.VOX_AUTO).form == tf.VOX_BATCHED


@pytest.mark.parametrize("active", [0.0, 0.3, 1.0])
def test_air_gather(cuda, oracle, plans, world, active):
    import voxel3d as V
    import workloads as W

    d = _copy(world)
    n = int(round(active * W.VOX_BRICKS))
    d["sim_list"] = np.random.default_rng(5).permutation(W.VOX_BRICKS)[:n].astype(np.uint32)
    d["sim_count"] = np.array([n, 1, 1], np.uint32)
    bufs, air = V.upload(d)
    air.gather(plans["cluster"], bufs)
    oracle.vox_air_gather(d)
    _same(V.download(bufs, air), d, ("solid", "temp"))


@pytest.mark.parametrize("active", [0.0, 0.3, 1.0])
def test_grav_gather(cuda, oracle, plans, world, active):
    import voxel3d as V
    import workloads as W

    d = _copy(world)
    n = int(round(active * W.VOX_BRICKS))
    d["sim_list"] = np.random.default_rng(6).permutation(W.VOX_BRICKS)[:n].astype(np.uint32)
    d["sim_count"] = np.array([n, 1, 1], np.uint32)
    bufs, air = V.upload(d)
    V.gravity_gather(plans["cluster"], bufs)
    oracle.vox_grav_gather(d)
    _same(V.download(bufs, air), d, ("grav_mass",))


def test_grav_gather_repeated_bricks(cuda, oracle, plans, world):
    """A brick listed k times adds its mass k times, as the reference's
    per-listed-brick atomics do (the device sums cells in memory order)."""
    import voxel3d as V
    import workloads as W

    d = _copy(world)
    uniq = np.random.default_rng(8).permutation(W.VOX_BRICKS)[:3000].astype(np.uint32)
    lst = np.concatenate([uniq, uniq[:1000], uniq[:10]])
    np.random.default_rng(9).shuffle(lst)
    d["sim_list"] = np.zeros(W.VOX_BRICKS, np.uint32)
    d["sim_list"][:lst.size] = lst
    d["sim_count"] = np.array([lst.size, 1, 1], np.uint32)
    bufs, air = V.upload(d)
    V.gravity_gather(plans["batched"], bufs)
    V.gravity_gather(plans["batched"], bufs)  # twice in a row: the brick table is rebuilt per call
    oracle.vox_grav_gather(d)
    oracle.vox_grav_gather(d)
    _same(V.download(bufs, air), d, ("grav_mass",))


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("iterations", [0, 1, 2, 3, 12])
def test_air_solve(cuda, oracle, plans, world, form, iterations):
    import voxel3d as V

    d = _copy(world)
    bufs, air = V.upload(d)
    air.iterations = iterations
    air.solve(plans[form])
    oracle.vox_air_solve(d, iterations)
    _same(V.download(bufs, air), d, AIR_KEYS, f"{form} n={iterations}: ")


@pytest.mark.parametrize("form", sorted(FORMS))
def test_grav_solve(cuda, oracle, plans, world, form):
    import voxel3d as V

    d = _copy(world)
    bufs, air = V.upload(d)
    V.gravity_solve(plans[form], bufs)
    oracle.vox_grav_solve(d, 24)
    _same(V.download(bufs, air), d, GRAV_KEYS, f"{form}: ")
    V.gravity_clear_mass(plans[form], bufs)
    assert not bufs.grav_mass.any()


@pytest.mark.parametrize("form", sorted(FORMS))
def test_field_step_three_worlds_two_ticks(cuda, oracle, plans, world, form):
    import voxel3d as V
    import workloads as W

    rng = np.random.default_rng(7)
    hosts = []
    for w in range(3):
        d = _copy(world)
        n = [W.VOX_BRICKS, 5000, 0][w]
        d["sim_list"] = rng.permutation(W.VOX_BRICKS)[:n].astype(np.uint32)
        d["sim_count"] = np.array([n, 1, 1], np.uint32)
        d["vx"] = (d["vx"] * np.float32(0.5 + w)).clip(-8, 8).astype(np.float32)
        d["grav_mass"] = np.roll(d["grav_mass"], 4099 * w)
        hosts.append(d)
    devs = [V.upload(d) for d in hosts]
    for tick in range(2):
        V.field_step(plans[form], devs, 12)
        for d in hosts:
            oracle.vox_field_step(d, 12)
        for w, (d, (bufs, air)) in enumerate(zip(hosts, devs)):
            _same(V.download(bufs, air), d, AIR_KEYS + GRAV_KEYS + ("solid", "temp"), f"{form} tick {tick} world {w}: ")
