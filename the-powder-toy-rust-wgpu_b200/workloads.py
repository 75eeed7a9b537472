"""Seeded synthetic sandbox instances for the coarse-grid field step.

The reference publishes no dataset or benchmark input for this path; its
`--bench` runner steps whatever canvas the user drew. These generators stand
in for it with the shapes and value ranges of the five workloads the field
step is measured on:

  C1  153x96 cells (the default 612x384 canvas), 2000 mass cells
  C2  400x225 cells (1600x900 canvas), mass on 3% of cells
  C3  gravity only, 512x512 cells, clustered f32 mass
  C4  256 instances, W,H log-uniform in [32, 512], mass on 2%
  C5  64 x (400x225) + 64 heavy-tailed (Pareto 1.5 on [32, 512])

Every random draw comes from a counter-based SplitMix64 stream, so an
instance depends only on (config id, instance index) and the numbers are the
same on every machine and numpy version. Seed of config c: 0x74707400 + c;
instance i uses substream i.

Grids use the reference layout (row-major `cy * xcells + cx`) and the
reference's types: f32 fields, u32 walls/masks, i32 fixed-point mass.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# Wall ids (crates/tpt-core/src/constants.rs:700-735).
WL_WALLELEC = 1
WL_EWALL = 2
WL_FAN = 5
WL_WALL = 8
WL_GRAV = 14
WL_BLOCKAIR = 16

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
CONFIG_SEED_BASE = 0x74707400
MASS_SCALE = np.float32(65536.0)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on a uint64 array (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = np.asarray(x, dtype=np.uint64)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


class Stream:
    """Counter-based stream: draw k is splitmix64(seed + (k+1) * golden)."""

    def __init__(self, seed: int):
        self.seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.counter = 0

    def u64(self, n: int) -> np.ndarray:
        k = np.arange(self.counter + 1, self.counter + 1 + n, dtype=np.uint64)
        self.counter += n
        with np.errstate(over="ignore"):
            return splitmix64(self.seed + k * GOLDEN)

    def uniform(self, lo: float, hi: float, n: int) -> np.ndarray:
        u = (self.u64(n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def choice_cells(self, cells: int, n: int) -> np.ndarray:
        """n distinct cell indices, uniformly."""
        n = min(n, cells)
        keys = self.u64(cells)
        return np.argsort(keys, kind="stable")[:n]


def instance_seed(config_id: int, instance: int) -> int:
    base = splitmix64(np.array([CONFIG_SEED_BASE + config_id], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        return int(splitmix64(np.array([base + np.uint64(instance + 1)], dtype=np.uint64))[0])


# ---------------------------------------------------------------- masks --

def wall_masks(wall: np.ndarray, emap: np.ndarray, eair=None, eairh=None):
    """`bmap_blockair` / `bmap_blockairh` from wall ids and emap.

    Follows `air_block_masks_kernel` (crates/tpt-sim/src/air_kernel/settle.rs:
    62-91) without the emap decrement: blocked = wall in {WALL, WALLELEC,
    BLOCKAIR} or (EWALL and emap == 0); heat = blocked or GRAV -> 0x8.
    """
    w = wall.astype(np.uint32) & np.uint32(0xFF)
    e = emap.astype(np.uint32) & np.uint32(0xFF)
    blocked = (w == WL_WALL) | (w == WL_WALLELEC) | (w == WL_BLOCKAIR) | ((w == WL_EWALL) & (e == 0))
    bair = blocked.astype(np.uint32)
    bairh = np.where(blocked | (w == WL_GRAV), np.uint32(8), np.uint32(0)).astype(np.uint32)
    if eair is not None:
        bair |= eair.astype(np.uint32)
    if eairh is not None:
        bairh |= eairh.astype(np.uint32)
    return bair, bairh


def grav_mask(wall: np.ndarray, xcells: int, ycells: int) -> np.ndarray:
    """Gravity propagation mask: cells 4-connected to the border through
    non-WL_GRAV cells -> 0xFFFFFFFF, others 0 (the flood fill of
    crates/tpt-sim/src/gravity_kernel.rs:658-712)."""
    from scipy import ndimage

    w = (wall.reshape(ycells, xcells).astype(np.uint32) & np.uint32(0xFF)) != WL_GRAV
    lab, _ = ndimage.label(w, structure=[[0, 1, 0], [1, 1, 1], [0, 1, 0]])
    border = np.unique(np.concatenate([lab[0, :], lab[-1, :], lab[:, 0], lab[:, -1]]))
    border = border[border != 0]
    reach = np.isin(lab, border)
    return np.where(reach, np.uint32(0xFFFFFFFF), np.uint32(0)).astype(np.uint32).reshape(-1)


def mass_to_fixed(m: np.ndarray) -> np.ndarray:
    """Round half away from zero of m*65536 in f32 arithmetic, truncated to
    i32 (crates/tpt-sim/src/gravity_kernel.rs:217-229)."""
    s = np.asarray(m, dtype=np.float32) * MASS_SCALE
    s = np.where(s >= np.float32(0), s + np.float32(0.5), s - np.float32(0.5)).astype(np.float32)
    return np.trunc(s).astype(np.int32)


# ------------------------------------------------------------ instances --

@dataclasses.dataclass
class AirConfig:
    """The `SimulationConfig` fields of the field step; defaults are the
    reference's (crates/tpt-core/src/particle.rs:290-345) except
    aheat_enable, which the measured workloads turn on."""

    air_mode: int = 0
    aheat_enable: int = 1
    convection_mode: int = 2
    gravity_mode: int = 0
    edge_pressure: float = 0.0
    edge_vx: float = 0.0
    edge_vy: float = 0.0
    ambient_air_temp: float = 295.15
    vorticity_coeff: float = 0.1
    custom_gx: float = 0.0
    custom_gy: float = 1.0
    newton_grav: int = 1


@dataclasses.dataclass
class Instance:
    xcells: int
    ycells: int
    config: AirConfig
    pv: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    hv: np.ndarray
    wall: np.ndarray
    emap: np.ndarray
    bair: np.ndarray
    bairh: np.ndarray
    eair: np.ndarray
    eairh: np.ndarray
    fan_vx: np.ndarray
    fan_vy: np.ndarray
    mass_fx: np.ndarray
    gmask: np.ndarray

    @property
    def cells(self) -> int:
        return self.xcells * self.ycells

    def copy(self) -> "Instance":
        return dataclasses.replace(
            self,
            config=dataclasses.replace(self.config),
            **{f.name: getattr(self, f.name).copy() for f in dataclasses.fields(self)
               if isinstance(getattr(self, f.name), np.ndarray)},
        )


def blob_field(st: Stream, X: int, Y: int, blobs: int = 8) -> np.ndarray:
    """pv = clamp(sum of `blobs` Gaussians, +-256): centres uniform over the
    interior, sigma ~ U(3, 12) cells, amplitude ~ U(-200, 200)."""
    cx = st.uniform(1.0, max(X - 1, 2), blobs)
    cy = st.uniform(1.0, max(Y - 1, 2), blobs)
    sg = st.uniform(3.0, 12.0, blobs)
    amp = st.uniform(-200.0, 200.0, blobs)
    xs = np.arange(X, dtype=np.float64)[None, :]
    ys = np.arange(Y, dtype=np.float64)[:, None]
    f = np.zeros((Y, X), dtype=np.float64)
    for b in range(blobs):
        f += amp[b] * np.exp(-((xs - cx[b]) ** 2 + (ys - cy[b]) ** 2) / (2.0 * sg[b] ** 2))
    return np.clip(f, -256.0, 256.0).astype(np.float32).reshape(-1)


def make_instance(X: int, Y: int, seed: int, *, mass_cells: int | None = None,
                  mass_density: float | None = None, wall_fraction: float = 0.05,
                  config: AirConfig | None = None) -> Instance:
    """A measured-workload instance: blob pv, zero velocity, hv = 273.15 +
    U(20, 30) K, WL_WALL on the 1-cell border ring (EDGE_SOLID,
    crates/tpt-sim/src/buffers/layout.rs:284-318) plus `wall_fraction` of the
    interior, masks from the walls, mass m ~ U(0, 1) on `mass_cells` (or
    `mass_density` of all) distinct cells in fixed point."""
    st = Stream(seed)
    n = X * Y
    pv = blob_field(st, X, Y)
    vx = np.zeros(n, np.float32)
    vy = np.zeros(n, np.float32)
    hv = (273.15 + st.uniform(20.0, 30.0, n)).astype(np.float32)
    wall = np.zeros((Y, X), np.uint32)
    wall[0, :] = WL_WALL
    wall[-1, :] = WL_WALL
    wall[:, 0] = WL_WALL
    wall[:, -1] = WL_WALL
    u = st.uniform(0.0, 1.0, n).reshape(Y, X)
    inner = np.zeros((Y, X), bool)
    inner[1:-1, 1:-1] = True
    wall[inner & (u < wall_fraction)] = WL_WALL
    wall = wall.reshape(-1)
    emap = np.zeros(n, np.uint32)
    eair = np.zeros(n, np.uint32)
    eairh = np.zeros(n, np.uint32)
    bair, bairh = wall_masks(wall, emap)
    if mass_cells is None:
        mass_cells = int(round((mass_density or 0.0) * n))
    idx = st.choice_cells(n, mass_cells)
    m = st.uniform(0.0, 1.0, len(idx))
    mass_fx = np.zeros(n, np.int32)
    mass_fx[idx] = mass_to_fixed(m.astype(np.float32))
    return Instance(X, Y, config or AirConfig(), pv, vx, vy, hv, wall, emap, bair, bairh, eair, eairh,
                    np.zeros(n, np.float32), np.zeros(n, np.float32), mass_fx, grav_mask(wall, X, Y))


def make_stress_instance(X: int, Y: int, seed: int, config: AirConfig | None = None) -> Instance:
    """Edge-case instance: nonzero and large velocities (far-advection walks up
    to the +-256 cap), every wall kind the field step reads (WALL, WALLELEC,
    EWALL with emap 0..3, FAN with fan velocity, GRAV, BLOCKAIR), element
    stamps, block_airh counter bits, hot and cold hv, and signed mass."""
    st = Stream(seed)
    n = X * Y
    pv = blob_field(st, X, Y)
    big = st.uniform(0.0, 1.0, n) < 0.05
    vx = st.uniform(-8.0, 8.0, n)
    vy = st.uniform(-8.0, 8.0, n)
    vx = np.where(big, st.uniform(-256.0, 256.0, n), vx).astype(np.float32)
    vy = np.where(big, st.uniform(-256.0, 256.0, n), vy).astype(np.float32)
    hv = st.uniform(250.0, 3000.0, n).astype(np.float32)
    kinds = np.array([WL_WALL, WL_WALLELEC, WL_EWALL, WL_FAN, WL_GRAV, WL_BLOCKAIR, 3, 9], np.uint32)
    pick = kinds[(st.u64(n) % np.uint64(len(kinds))).astype(np.int64)]
    u = st.uniform(0.0, 1.0, n)
    wall = np.where(u < 0.12, pick, np.uint32(0)).astype(np.uint32)
    # a GRAV ring enclosing a pocket, so the gravity mask has a hole
    if X >= 16 and Y >= 16:
        w2 = wall.reshape(Y, X)
        x0, y0, x1, y1 = X // 4, Y // 4, X // 4 + 6, Y // 4 + 6
        w2[y0, x0:x1 + 1] = WL_GRAV
        w2[y1, x0:x1 + 1] = WL_GRAV
        w2[y0:y1 + 1, x0] = WL_GRAV
        w2[y0:y1 + 1, x1] = WL_GRAV
        w2[y0 + 1:y1, x0 + 1:x1] = 0
        wall = w2.reshape(-1)
    emap = (st.u64(n) % np.uint64(4)).astype(np.uint32) * (wall == WL_EWALL)
    emap = emap.astype(np.uint32)
    eair = (st.uniform(0.0, 1.0, n) < 0.01).astype(np.uint32)
    eairh = np.where(st.uniform(0.0, 1.0, n) < 0.01, np.uint32(8), np.uint32(0)).astype(np.uint32)
    bair, bairh = wall_masks(wall, emap, eair, eairh)
    # thermal-pass counter bits (low 3 bits) that do not block heat
    bairh = bairh | ((st.u64(n) % np.uint64(8)).astype(np.uint32) * (st.uniform(0, 1, n) < 0.1))
    bairh = bairh.astype(np.uint32)
    fan_vx = np.where(wall == WL_FAN, st.uniform(-2.0, 2.0, n), 0.0).astype(np.float32)
    fan_vy = np.where(wall == WL_FAN, st.uniform(-2.0, 2.0, n), 0.0).astype(np.float32)
    idx = st.choice_cells(n, max(1, n // 20))
    m = st.uniform(-1.0, 3.0, len(idx))
    mass_fx = np.zeros(n, np.int32)
    mass_fx[idx] = mass_to_fixed(m.astype(np.float32))
    return Instance(X, Y, config or AirConfig(), pv, vx, vy, hv, wall, emap, bair, bairh, eair, eairh,
                    fan_vx, fan_vy, mass_fx, grav_mask(wall, X, Y))


def clustered_mass(X: int, Y: int, seed: int, clusters: int = 50) -> np.ndarray:
    """C3 mass: `clusters` Gaussian clusters (sigma ~ U(2, 20) cells, peak ~
    U(0.5, 5)) plus 1% of cells with U(0, 1) noise, as f32."""
    st = Stream(seed)
    cx = st.uniform(0.0, X, clusters)
    cy = st.uniform(0.0, Y, clusters)
    sg = st.uniform(2.0, 20.0, clusters)
    pk = st.uniform(0.5, 5.0, clusters)
    xs = np.arange(X, dtype=np.float64)[None, :]
    ys = np.arange(Y, dtype=np.float64)[:, None]
    m = np.zeros((Y, X))
    for c in range(clusters):
        m += pk[c] * np.exp(-((xs - cx[c]) ** 2 + (ys - cy[c]) ** 2) / (2.0 * sg[c] ** 2))
    m = m.reshape(-1)
    idx = st.choice_cells(X * Y, int(round(0.01 * X * Y)))
    m[idx] += st.uniform(0.0, 1.0, len(idx))
    return m.astype(np.float32)


# -------------------------------------------------------------- configs --

def config_shapes(config_id: int) -> list[tuple[int, int]]:
    """Instance grid shapes (xcells, ycells) of a measured workload."""
    if config_id == 1:
        return [(153, 96)]
    if config_id == 2:
        return [(400, 225)]
    if config_id == 3:
        return [(512, 512)]
    if config_id == 4:
        st = Stream(CONFIG_SEED_BASE + 4)
        lo, hi = math.log(32.0), math.log(512.0)
        w = np.rint(np.exp(st.uniform(lo, hi, 256))).astype(int)
        h = np.rint(np.exp(st.uniform(lo, hi, 256))).astype(int)
        return [(int(a), int(b)) for a, b in zip(w, h)]
    if config_id == 5:
        st = Stream(CONFIG_SEED_BASE + 5)
        u1 = st.uniform(0.0, 1.0, 64)
        u2 = st.uniform(0.0, 1.0, 64)
        pw = np.clip(np.floor(32.0 * (1.0 - u1) ** (-1.0 / 1.5)), 32, 512).astype(int)
        ph = np.clip(np.floor(32.0 * (1.0 - u2) ** (-1.0 / 1.5)), 32, 512).astype(int)
        return [(400, 225)] * 64 + [(int(a), int(b)) for a, b in zip(pw, ph)]
    raise ValueError(f"unknown config {config_id}")


def config_instances(config_id: int, limit: int | None = None) -> list[Instance]:
    """The seeded instances of workload C1, C2, C4 or C5."""
    shapes = config_shapes(config_id)
    if limit is not None:
        shapes = shapes[:limit]
    out = []
    for i, (X, Y) in enumerate(shapes):
        seed = instance_seed(config_id, i)
        if config_id == 1:
            out.append(make_instance(X, Y, seed, mass_cells=2000))
        elif config_id == 2:
            out.append(make_instance(X, Y, seed, mass_density=0.03))
        else:
            out.append(make_instance(X, Y, seed, mass_density=0.02))
    return out


CONFIG_TICKS = {1: 1000, 2: 10000, 3: 1, 4: 1000, 5: 1000}


# ------------------------------------------------ gravity tick particles --

# Element ids the gravity tick branches on (crates/tpt-core/src/constants.rs).
PT_GRVT, PT_NBHL, PT_NWHL, PT_GBMB, PT_GPMP, PT_SPNG = 39, 40, 41, 42, 43, 78
TYPE_SOLID = 0x4
WL_STASIS = 18


def move_lut(n_types: int, seed: int) -> np.ndarray:
    """A movement table of `n_types` 12-word records (the layout of the
    reference's `build_move_lut`): word 0 the element properties (TYPE_SOLID
    on about a third of the ids), word 7 the f32 bits of Loss in [0.5, 1]."""
    st = Stream(seed)
    lut = np.zeros((n_types, 12), np.uint32)
    props = (st.u64(n_types) % np.uint64(3) == np.uint64(0)).astype(np.uint32) * np.uint32(TYPE_SOLID)
    loss = st.uniform(0.5, 1.0, n_types).astype(np.float32)
    lut[:, 0] = props
    lut[:, 7] = loss.view(np.uint32)
    return lut.reshape(-1)


def gravity_particles(xres: int, yres: int, n: int, seed: int, n_types: int = 192) -> dict:
    """Seeded particle slots for the gravity tick: every gravity element with
    its mass cases (GRVT tmp beyond the clamp, NBHL/NWHL tmp 0 and beyond the
    range, GBMB armed / counting / inert, GPMP on and off), SPNG with and
    without FLAG_MOVABLE, rigid pixels, empty slots, ids past the table,
    positions off the canvas and in the 4-px margin, several particles per
    cell. Struct of arrays, numpy."""
    st = Stream(seed)
    kinds = np.array([0, PT_GRVT, PT_NBHL, PT_NWHL, PT_GBMB, PT_GPMP, PT_SPNG, 1, 5, 27, n_types + 3],
                     np.uint32)
    ty = kinds[(st.u64(n) % np.uint64(len(kinds))).astype(np.int64)]
    x = st.uniform(-6.0, xres + 6.0, n).astype(np.float32)
    y = st.uniform(-6.0, yres + 6.0, n).astype(np.float32)
    # a cluster of particles in a few cells, so several add to one cell
    k = n // 8
    x[:k] = (40.0 + (st.u64(k) % np.uint64(3)).astype(np.float64) * 4.0).astype(np.float32)
    y[:k] = np.float32(48.0)
    vx = st.uniform(-20.0, 20.0, n).astype(np.float32)
    vy = st.uniform(-20.0, 20.0, n).astype(np.float32)
    life = (st.u64(n) % np.uint64(40)).astype(np.int32)
    life[(st.u64(n) % np.uint64(4)) == 0] = 10
    tmp = (st.u64(n) % np.uint64(120001)).astype(np.int64) - 60000
    tmp[(st.u64(n) % np.uint64(5)) == 0] = 0
    temp = st.uniform(0.0, 9999.0, n).astype(np.float32)
    flags = np.zeros(n, np.uint32)
    r = st.u64(n) % np.uint64(8)
    flags[r == 0] |= np.uint32(0x08)
    flags[r == 1] |= np.uint32(0x10)
    return {"ty": ty, "x": x, "y": y, "vx": vx, "vy": vy, "life": life, "tmp": tmp.astype(np.int32),
            "temp": temp, "flags": flags}


def gravity_state(xres: int, yres: int, seed: int) -> dict:
    """Seeded gravity grids of one sandbox for the tick: walls with WL_GRAV
    pockets (masked cells) and WL_STASIS with powered and unpowered emap,
    painted wells, overrides on a few cells, a stale accumulator."""
    X, Y = xres // 4, yres // 4
    st = Stream(seed)
    cells = X * Y
    wall = np.zeros(cells, np.uint32)
    r = st.u64(cells) % np.uint64(40)
    wall[r == 0] = WL_STASIS
    g = np.zeros((Y, X), bool)
    g[Y // 3:Y // 3 + 3, X // 4:X // 4 + 6] = True  # a ring of GRAV walls
    g[Y // 3 + 1, X // 4 + 1:X // 4 + 5] = False
    wall[g.reshape(-1)] = WL_GRAV
    emap = (st.u64(cells) % np.uint64(16)).astype(np.uint32)
    tool = np.zeros(cells, np.float32)
    tool[(st.u64(cells) % np.uint64(97)) == 0] = st.uniform(-5.0, 5.0, 1)[0]
    ovr_set = ((st.u64(cells) % np.uint64(61)) == 0).astype(np.uint32)
    ovr = (st.u64(cells) % np.uint64(200001)).astype(np.int64) - 100000
    return {"wall_bmap": wall, "wall_emap": emap, "grav_mask": grav_mask(wall, X, Y),
            "mass": (st.u64(cells) % np.uint64(1000)).astype(np.int32),  # stale: the tick clears it
            "mass_prev": (st.u64(cells) % np.uint64(70000)).astype(np.int32),
            "tool_mass": tool, "override_mass": ovr.astype(np.int32), "override_set": ovr_set,
            "gx": np.zeros(cells, np.float32), "gy": np.zeros(cells, np.float32)}


# ---------------------------------------------------------------- 3-D ----
# The 3-D sandbox (crates/tpt-sim/src/voxel3d): a 64^3 coarse grid
# ((y << 12) | (z << 6) | x) over 256^3 voxels ((y << 16) | (z << 8) | x) in
# 8^3 bricks ((by << 10) | (bz << 5) | bx).
VOX_AXIS = 64
VOX_CELLS = 64 ** 3
VOX_VOXELS = 256 ** 3
VOX_BRICKS = 32 ** 3


def voxel_world(seed: int, active: float = 0.3, fill: float = 0.4) -> dict:
    """A seeded 3-D world for the field step, numpy arrays in the reference
    layout and types:

      voxel     u32 words ty | temp_q << 8 | life << 24 (step/mod.rs:125-133):
                empty voxels (ty 0) with probability 1 - fill, else one of
                the gravity elements GRVT..GPMP or another element id;
                temp_q over the whole u16 range, life over u8 with 10 (the
                GPMP trigger) and the GBMB thresholds frequent
      aux_tmp   i32 per voxel: 0, inside and far outside the clamps
      sim_list  `active` of the 32768 brick ids, in random order (the order
                the device compaction's atomics give); sim_count [n, 1, 1]
      vx vy vz  f32 in [-8, 8] (the advection clamp), some exact zeros
      p p_tmp   f32 pressure pair, temp f32 250..600 K, solid k/64
      pv        i32 in the +-262144 clamp, a few at the limits
      grav_*    i32 mass on 2% of cells, f32 potential pair, stale forces
    """
    st = Stream(seed)
    nv = VOX_VOXELS
    kinds = np.array([1, 5, 27, PT_GRVT, PT_NBHL, PT_NWHL, PT_GBMB, PT_GPMP, 100, 255], np.uint32)
    ty = kinds[(st.u64(nv) % np.uint64(len(kinds))).astype(np.int64)]
    ty[st.uniform(0.0, 1.0, nv) >= fill] = 0
    temp_q = (st.u64(nv) & np.uint64(0xFFFF)).astype(np.uint32)
    warm = (st.u64(nv) % np.uint64(3)) == 0
    temp_q[warm] = (2345 + (st.u64(int(warm.sum())) % np.uint64(800))).astype(np.uint32)
    life = (st.u64(nv) & np.uint64(0xFF)).astype(np.uint32)
    r = st.u64(nv) % np.uint64(6)
    life[r == 0] = 10
    life[r == 1] = 0
    life[r == 2] = (st.u64(int((r == 2).sum())) % np.uint64(25)).astype(np.uint32)
    voxel = ty | (temp_q << np.uint32(8)) | (life << np.uint32(24))
    aux = (st.u64(nv) % np.uint64(120001)).astype(np.int64) - 60000
    r = st.u64(nv) % np.uint64(4)
    aux[r == 0] = 0
    aux[r == 1] = aux[r == 1] % 201 - 100
    n_active = int(round(active * VOX_BRICKS))
    sim_list = st.choice_cells(VOX_BRICKS, n_active).astype(np.uint32)

    nc = VOX_CELLS
    v = [st.uniform(-8.0, 8.0, nc).astype(np.float32) for _ in range(3)]
    for a in v:
        a[(st.u64(nc) % np.uint64(10)) == 0] = 0.0
    solid = ((st.u64(nc) % np.uint64(65)).astype(np.float32) * np.float32(1.0 / 64.0)).astype(np.float32)
    solid[(st.u64(nc) % np.uint64(3)) != 0] = 0.0
    pv = (st.u64(nc) % np.uint64(524289)).astype(np.int64) - 262144
    r = st.u64(nc) % np.uint64(50)
    pv[r == 0] = 262144
    pv[r == 1] = -262144
    mass = np.zeros(nc, np.int64)
    hot = st.choice_cells(nc, nc // 50)
    mass[hot] = (st.u64(len(hot)) % np.uint64(200001)).astype(np.int64) - 100000
    return {
        "voxel": voxel.astype(np.uint32), "aux_tmp": aux.astype(np.int32), "sim_list": sim_list,
        "sim_count": np.array([n_active, 1, 1], np.uint32),
        "vx": v[0], "vy": v[1], "vz": v[2],
        "p": st.uniform(-2.0, 2.0, nc).astype(np.float32), "p_tmp": st.uniform(-2.0, 2.0, nc).astype(np.float32),
        "temp": st.uniform(250.0, 600.0, nc).astype(np.float32), "solid": solid, "pv": pv.astype(np.int32),
        "grav_mass": mass.astype(np.int32),
        "grav_potential": st.uniform(-50.0, 50.0, nc).astype(np.float32),
        "grav_potential_tmp": st.uniform(-50.0, 50.0, nc).astype(np.float32),
        "grav_force_x": np.full(nc, 7.0, np.float32), "grav_force_y": np.full(nc, 7.0, np.float32),
        "grav_force_z": np.full(nc, 7.0, np.float32),
    }


VOX_FIELDS = ("voxel", "aux_tmp", "sim_list", "sim_count", "vx", "vy", "vz", "p", "p_tmp", "temp", "solid", "pv",
              "grav_mass", "grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y", "grav_force_z")
