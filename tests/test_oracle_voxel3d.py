"""The oracle's 3-D field step (crates/tpt-sim/src/voxel3d) on CPU.

The reference holds no golden vectors for these kernels; its tests for this
path are the constant pins in gravity.rs:295-309. The oracle is checked
against:
  - those pins (FOUR_PI_G against 4*pi*M_GRAV, the grid sizes);
  - hand-computed cases of every branch (voxel mass per element, pv rim /
    interior / clamp, gather means, sweep values);
  - a second, independent restatement below (vectorised numpy, f32 per
    operation), bit for bit on a seeded world.
"""
import math

import numpy as np
import pytest

N, SZ, SY = 64, 64, 4096
f32 = np.float32


# ---------------------------------------------------- numpy restatement ----

def _coords():
    i = np.arange(N ** 3)
    return i & 63, i >> 12, (i >> 6) & 63  # x, y, z


def _nb(a, i, d):
    """a[i + d] where in range, else 0 (the caller masks)."""
    j = np.clip(i + d, 0, N ** 3 - 1)
    return a[j]


def np_air_solve(d, iterations):
    x, y, z = _coords()
    i = np.arange(N ** 3)
    vx, vy, vz = d["vx"], d["vy"], d["vz"]
    # air_kernel.rs:294-326
    rim = (x < 2) | (x >= 62) | (y < 2) | (y >= 62) | (z < 2) | (z >= 62)
    pv = d["pv"]
    dp = ((_nb(vx, i, -1) - _nb(vx, i, 1)) + (_nb(vy, i, -SY) - _nb(vy, i, SY))) + (_nb(vz, i, -SZ) - _nb(vz, i, SZ))
    mixed = pv.astype(f32) * f32(0.9999)
    nxt = mixed + ((dp * f32(0.3)) * f32(0.5)) * f32(1024.0)
    inner = np.where(nxt > f32(262144.0), 262144, np.where(nxt < f32(-262144.0), -262144,
                                                             np.trunc(nxt).astype(np.int64)))
    rimv = np.trunc(pv.astype(f32) * f32(0.2)).astype(np.int64)
    pv_new = np.where(rim, rimv, inner).astype(np.int32)
    snap = (vx.copy(), vy.copy(), vz.copy())
    # air_kernel.rs:361-398
    fixed = (x == 0) | (y == 0) | (z == 0) | (x == 63) | (y == 63) | (z == 63) | (d["solid"] > f32(0.5))
    div = f32(0.5) * (((_nb(vx, i, 1) - _nb(vx, i, -1)) + (_nb(vy, i, SY) - _nb(vy, i, -SY)))
                      + (_nb(vz, i, SZ) - _nb(vz, i, -SZ)))
    pin, pout = d["p"].copy(), d["p_tmp"].copy()
    for _ in range(iterations):
        nb = (((((_nb(pin, i, -1) + _nb(pin, i, 1)) + _nb(pin, i, -SZ)) + _nb(pin, i, SZ)) + _nb(pin, i, -SY))
              + _nb(pin, i, SY))
        pout = np.where(fixed, f32(0.0), (nb - div) / f32(6.0)).astype(f32)
        pin, pout = pout, pin
    p_final = pin
    if iterations % 2 == 0:
        p, p_tmp = pin, pout
    else:
        p, p_tmp = pout, pin
    # air_kernel.rs:414-536
    def avg(a):
        s, c = a.copy(), np.ones(N ** 3, f32)
        for ok, dd in ((x > 0, -1), (x < 63, 1), (z > 0, -SZ), (z < 63, SZ), (y > 0, -SY), (y < 63, SY)):
            s = np.where(ok, s + _nb(a, i, dd), s)
            c = np.where(ok, c + f32(1.0), c)
        return s / c

    def grad(lo_ok, hi_ok, dd):
        lo = np.where(lo_ok, _nb(p_final, i, -dd), p_final)
        hi = np.where(hi_ok, _nb(p_final, i, dd), p_final)
        return (hi - lo) * f32(0.5)

    buoy = (avg(d["temp"]) - f32(293.15)) * f32(0.02)
    out = []
    for a, (lo_ok, hi_ok, dd) in enumerate(((x > 0, x < 63, 1), (y > 0, y < 63, SY), (z > 0, z < 63, SZ))):
        old = snap[a]
        g = grad(lo_ok, hi_ok, dd)
        nxt = ((old + buoy) - g) * f32(0.99) if a == 1 else (old - g) * f32(0.99)
        nxt = nxt * (f32(1.0) - f32(0.1)) + avg(old) * f32(0.1)
        up = np.where(old > 0, np.where(lo_ok, _nb(old, i, -dd), old),
                      np.where(old < 0, np.where(hi_ok, _nb(old, i, dd), old), old))
        nxt = nxt * (f32(1.0) - f32(0.25)) + up * f32(0.25)
        nxt = np.minimum(np.maximum(nxt, f32(-8.0)), f32(8.0))
        out.append(np.where(d["solid"] > f32(0.5), f32(0.0), nxt).astype(f32))
    return {"pv": pv_new, "p": p, "p_tmp": p_tmp, "vx": out[0], "vy": out[1], "vz": out[2]}


def np_grav_solve(d, iterations=24):
    x, y, z = _coords()
    i = np.arange(N ** 3)
    boundary = (x == 0) | (x == 63) | (y == 0) | (y == 63) | (z == 0) | (z == 63)
    src = f32(8.385539) * (d["grav_mass"].astype(f32) * f32(1.0 / 1024.0))
    uin, uout = d["grav_potential"].copy(), d["grav_potential_tmp"].copy()
    for _ in range(iterations):
        s = (((((_nb(uin, i, -1) + _nb(uin, i, 1)) + _nb(uin, i, -SZ)) + _nb(uin, i, SZ)) + _nb(uin, i, -SY))
             + _nb(uin, i, SY))
        uout = np.where(boundary, uin * f32(0.0) + f32(0.0), (s - src) * f32(1.0 / 6.0)).astype(f32)
        uin, uout = uout, uin
    u = uin
    fx = np.where(boundary, u * f32(0.0) + f32(0.0), (_nb(u, i, -1) - _nb(u, i, 1)) * f32(0.5))
    fy = np.where(boundary, u * f32(0.0) + f32(0.0), (_nb(u, i, -SY) - _nb(u, i, SY)) * f32(0.5))
    fz = np.where(boundary, u * f32(0.0) + f32(0.0), (_nb(u, i, -SZ) - _nb(u, i, SZ)) * f32(0.5))
    return {"grav_potential": u, "grav_potential_tmp": uout, "grav_force_x": fx.astype(f32),
            "grav_force_y": fy.astype(f32), "grav_force_z": fz.astype(f32)}


def _cells_of(bricks):
    b = np.asarray(bricks, np.int64)
    bx, bz, by = b & 31, (b >> 5) & 31, (b >> 10) & 31
    out = []
    for s in range(8):
        cx, cz, cy = bx * 2 + (s & 1), bz * 2 + ((s >> 1) & 1), by * 2 + ((s >> 2) & 1)
        out.append((cy << 12) | (cz << 6) | cx)
    return np.concatenate(out) if out else np.zeros(0, np.int64)


def _per_cell(a):
    """Sum of a per-voxel array over each 4^3 cell, as a 64^3 cell array."""
    v = a.reshape(64, 4, 64, 4, 64, 4)  # y, ly, z, lz, x, lx
    return v.sum(axis=(1, 3, 5)).reshape(-1)


def voxel_mass_np(ty, life, tmp, temp_k):
    out = np.zeros(ty.shape, np.int64)
    t = np.trunc(np.clip(tmp.astype(f32), f32(-100), f32(100))).astype(f32)
    grvt = np.trunc((f32(0.2) * t) * f32(1024.0))
    add = np.where(tmp != 0, np.clip(f32(0.001) * tmp.astype(f32), f32(0.1), f32(51.2)), f32(0.1)).astype(f32)
    out = np.where(ty == 39, grvt, out)
    out = np.where(ty == 40, np.trunc(add * f32(1024.0)), out)
    out = np.where(ty == 41, np.trunc((-add) * f32(1024.0)), out)
    gbmb = np.where(life > 20, 20480, np.where(life >= 1, -81920, 0))
    out = np.where(ty == 42, gbmb, out)
    gpmp = np.where(life == 10, np.trunc((f32(0.2) * (temp_k - f32(273.15))) * f32(1024.0)), 0)
    out = np.where(ty == 43, gpmp, out)
    return out.astype(np.int64)


def np_gathers(d):
    w = d["voxel"]
    ty = w & 0xFF
    temp_q = (w >> 8) & 0xFFFF
    life = (w >> 24) & 0xFF
    occ = _per_cell((ty != 0).astype(np.int64))
    tq = _per_cell(np.where(ty != 0, temp_q, 0).astype(np.int64))
    m = voxel_mass_np(ty, life, d["aux_tmp"], temp_q.astype(f32) * f32(0.125))
    mass = _per_cell(np.where(ty != 0, m, 0))
    cells = _cells_of(d["sim_list"][: int(d["sim_count"][0])])
    solid, temp, gm = d["solid"].copy(), d["temp"].copy(), d["grav_mass"].astype(np.int64)
    solid[cells] = occ[cells].astype(f32) * f32(1.0 / 64.0)
    temp[cells] = np.where(occ[cells] > 0, (tq[cells].astype(f32) * f32(0.125)) / occ[cells].astype(f32),
                           f32(293.15))
    gm[cells] = gm[cells] + mass[cells]
    gm = ((gm + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
    return {"solid": solid, "temp": temp, "grav_mass": gm}


# ---------------------------------------------------------------- tests ----

def _bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


@pytest.fixture(scope="module")
def world():
    import workloads as W

    return W.voxel_world(0x3D02, active=0.4)


def test_reference_constant_pins():
    # gravity.rs:296-303: FOUR_PI_G is 4*pi*M_GRAV to 1e-5 (M_GRAV 0.6673)
    assert abs(8.385539 - 4.0 * math.pi * 0.6673) < 1e-5
    # gravity.rs:305-309, air.rs:44-46: one 64^3 grid for air and gravity
    import workloads as W

    assert W.VOX_CELLS == 262144 == 64 ** 3 and W.VOX_VOXELS == 256 ** 3 and W.VOX_BRICKS == 32 ** 3


@pytest.mark.parametrize("iterations", [0, 1, 2, 5, 12])
def test_air_solve_matches_numpy_restatement(oracle, world, iterations):
    d = {k: v.copy() for k, v in world.items()}
    want = np_air_solve(d, iterations)
    oracle.vox_air_solve(d, iterations)
    for k, v in want.items():
        assert _bits_equal(d[k], v), k


def test_grav_solve_matches_numpy_restatement(oracle, world):
    d = {k: v.copy() for k, v in world.items()}
    want = np_grav_solve(d)
    oracle.vox_grav_solve(d, 24)
    for k, v in want.items():
        assert _bits_equal(d[k], v), k


def test_gathers_match_numpy_restatement(oracle, world):
    d = {k: v.copy() for k, v in world.items()}
    want = np_gathers(d)
    oracle.vox_air_gather(d)
    oracle.vox_grav_gather(d)
    for k, v in want.items():
        assert _bits_equal(d[k], v), k


def _blank_world():
    nv, nc = 256 ** 3, 64 ** 3
    return {"voxel": np.zeros(nv, np.uint32), "aux_tmp": np.zeros(nv, np.int32),
            "sim_list": np.zeros(32768, np.uint32), "sim_count": np.array([0, 1, 1], np.uint32),
            **{k: np.zeros(nc, f32) for k in ("vx", "vy", "vz", "p", "p_tmp", "temp", "solid", "grav_potential",
                                               "grav_potential_tmp", "grav_force_x", "grav_force_y",
                                               "grav_force_z")},
            "pv": np.zeros(nc, np.int32), "grav_mass": np.zeros(nc, np.int32)}


def _vox_index(x, y, z):
    return (y << 16) | (z << 8) | x


def test_gather_known_answers(oracle):
    d = _blank_world()
    d["solid"][:] = 7.0  # untouched cells keep it
    d["temp"][:] = 7.0
    brick = (3 << 10) | (5 << 5) | 7  # bx 7, bz 5, by 3: voxels x 56.., z 40.., y 24..
    d["sim_list"][0] = brick
    d["sim_count"][0] = 1

    def put(x, y, z, ty, temp_q=0, life=0, tmp=0):
        i = _vox_index(56 + x, 24 + y, 40 + z)
        d["voxel"][i] = ty | (temp_q << 8) | (life << 24)
        d["aux_tmp"][i] = tmp

    # cell (0,0,0): three voxels at 300, 301, 302 K
    put(0, 0, 0, 1, 2400)
    put(1, 2, 3, 1, 2408)
    put(3, 3, 3, 1, 2416)
    # cell (1,0,0): every voxel at the top of the range
    for ly in range(4):
        for lz in range(4):
            for lx in range(4):
                put(4 + lx, ly, lz, 2, 0xFFFF)
    # cell (0,1,1) (x 0-3, y 4-7, z 4-7): one of each gravity case
    cases = [  # (ty, temp_q, life, tmp, fixed-point mass)
        (39, 0, 0, 150, 20480),      # GRVT, tmp clamped to 100: 0.2*100*1024
        (39, 0, 0, -37, -7577),      # 0.2*-37*1024 = -7577.6
        (40, 0, 0, 0, 102),          # NBHL, tmp 0: 0.1*1024 = 102.4
        (40, 0, 0, 100000, 52428),   # clamp 51.2: 52428.8
        (41, 0, 0, 5, -102),         # NWHL, clamp 0.1 from below
        (42, 0, 30, 0, 20480),       # GBMB fuse
        (42, 0, 5, 0, -81920),       # GBMB push
        (42, 0, 0, 0, 0),            # GBMB inert
        (43, 2985, 10, 0, 20474),    # GPMP life 10 at 373.125 K: 0.2*99.975*1024
        (43, 2985, 11, 0, 0),        # GPMP off
        (5, 2985, 10, 77, 0),        # not a gravity element
    ]
    for n, (ty, tq, life, tmp, _) in enumerate(cases):
        put(n % 4, 4 + n // 4, 4 + (n // 2) % 4, ty, tq, life, tmp)
    oracle.vox_air_gather(d)
    oracle.vox_grav_gather(d)
    c000 = (6 << 12) | (10 << 6) | 14
    c100 = c000 + 1
    c011 = ((6 + 1) << 12) | ((10 + 1) << 6) | 14
    assert d["solid"][c000] == f32(3 / 64) and d["temp"][c000] == f32(301.0)
    assert d["solid"][c100] == f32(1.0) and d["temp"][c100] == f32(8191.875)
    assert d["solid"][c011] == f32(len(cases) / 64)
    assert d["grav_mass"][c011] == sum(c[4] for c in cases) == 20480 - 7577 + 102 + 52428 - 102 + 20480 - 81920 + 20474
    empty = c000 + 64  # cell (0, 0, 1): nothing in it
    assert d["solid"][empty] == 0.0 and d["temp"][empty] == f32(293.15)
    assert (d["solid"] == 7.0).sum() == 64 ** 3 - 8  # only the listed brick's 8 cells change


def test_pv_and_sweep_known_answers(oracle):
    d = _blank_world()
    rim = (0 << 12) | (5 << 6) | 5          # y = 0
    inner = (10 << 12) | (10 << 6) | 10
    clampc = (20 << 12) | (20 << 6) | 20
    d["pv"][rim] = -999                      # trunc(-199.8)
    d["pv"][inner] = 1000
    d["vx"][inner - 1] = 1.0                 # dp = 1: 999.9 + 153.6
    d["pv"][clampc] = 262144
    d["vx"][clampc - 1] = 8.0                # beyond the clamp
    d["p"][:] = 1.0
    oracle.vox_air_solve(d, 1)
    assert d["pv"][rim] == -199 and d["pv"][inner] == 1153 and d["pv"][clampc] == 262144
    c = (30 << 12) | (30 << 6) | 30          # far from walls and sources: (6 - 0) / 6
    assert d["p_tmp"][c] == 1.0 and d["p"][c] == 1.0   # one sweep writes p_tmp; p keeps p_0
    face, edge = (0 << 12) | (30 << 6) | 30, (1 << 12) | (30 << 6) | 30
    assert d["p_tmp"][face] == 0.0 and d["p_tmp"][edge] == 1.0  # sweep 1 still reads p_0 = 1 on the face
    d2 = _blank_world()
    d2["p"][:] = 1.0
    oracle.vox_air_solve(d2, 2)              # sweep 2 reads the pinned face: (1+1+1+1+0+1) / 6
    assert d2["p"][edge] == f32(f32(5.0) / f32(6.0)) and d2["p_tmp"][edge] == 1.0 and d2["p"][face] == 0.0


def test_grav_sweep_known_answer(oracle):
    d = _blank_world()
    c = (32 << 12) | (32 << 6) | 32
    d["grav_mass"][c] = 1024                 # rho = 1
    d["grav_potential"][0] = np.nan          # a pinned face cell stays NaN (u * 0 + 0)
    oracle.vox_grav_solve(d, 2)
    u1 = f32((f32(0.0) - f32(8.385539)) * f32(1.0 / 6.0))
    assert d["grav_potential_tmp"][c] == u1
    assert d["grav_potential"][c + 1] == f32(u1 * f32(1.0 / 6.0))   # (u1 - 0) / 6 beside it
    assert np.isnan(d["grav_potential"][0]) and np.isnan(d["grav_force_x"][0])
    assert d["grav_force_x"][c + 1] == f32((d["grav_potential"][c] - d["grav_potential"][c + 2]) * f32(0.5))
