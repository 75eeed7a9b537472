"""ctypes wrapper of the CPU oracle (liboracle.so). TEST INFRASTRUCTURE ONLY:
used by tests/, the smoke check and bench.py's CPU-baseline leg as the
checker; the product never imports it.

The oracle restates the reference's field-step kernels (air:
crates/tpt-sim/src/air_kernel/*.rs, gravity: crates/tpt-sim/src/gravity_gpu/
*.rs) in an FP32 mirror and an FP64 twin; see tpt_oracle.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class AirParams(ctypes.Structure):
    """Same layout as `tpt_air_params` in include/tpt_field.h."""

    _fields_ = [
        ("xcells", ctypes.c_uint32), ("ycells", ctypes.c_uint32),
        ("air_mode", ctypes.c_uint32), ("aheat_enable", ctypes.c_uint32),
        ("convection_mode", ctypes.c_uint32), ("gravity_mode", ctypes.c_uint32),
        ("edge_pressure", ctypes.c_float), ("edge_vx", ctypes.c_float), ("edge_vy", ctypes.c_float),
        ("ambient_air_temp", ctypes.c_float), ("vorticity_coeff", ctypes.c_float),
        ("custom_gx", ctypes.c_float), ("custom_gy", ctypes.c_float),
    ]


class VoxWorld(ctypes.Structure):
    """Same layout as `tpt_vox_world` in include/tpt_field.h (host pointers here)."""

    _fields_ = [(n, ctypes.c_void_p) for n in (
        "voxel", "aux_tmp", "sim_list", "sim_count", "vx", "vy", "vz", "p", "p_tmp", "temp", "solid", "pv",
        "grav_mass", "grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y", "grav_force_z")]


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        u32, f32, i32 = ctypes.c_uint32, ctypes.c_float, ctypes.c_int
        _lib.ora_air_steps_f32.argtypes = [ctypes.POINTER(AirParams), i32] + [P] * 12 + [P, P, u32, u32, u32]
        _lib.ora_air_steps_f64.argtypes = _lib.ora_air_steps_f32.argtypes
        _lib.ora_grav_solve_f32.argtypes = [u32, u32, P, P, f32, P, P, P]
        _lib.ora_grav_solve_f64.argtypes = [u32, u32, P, P, f32, P, P, P]
        _lib.ora_grav_direct_f64.argtypes = [u32, u32, P, P, f32, P, P, P]
        _lib.ora_fft_host_f32.argtypes = [P, u32, u32, u32, u32, u32, f32]
        _lib.ora_bit_count.argtypes = [u32]
        _lib.ora_bit_count.restype = u32
        _lib.ora_twiddle_f32.argtypes = [u32, P, P]
        _lib.ora_grav_mask.argtypes = [P, P, u32, u32]
        _lib.ora_mass_to_fixed.argtypes = [f32]
        _lib.ora_mass_to_fixed.restype = ctypes.c_int32
        _lib.ora_block_masks.argtypes = [ctypes.c_size_t, P, P, P, P, P, P]
        _lib.ora_tool_gravity_mass.argtypes = [f32, i32]
        _lib.ora_tool_gravity_mass.restype = f32
        _lib.ora_gravity_tool_cell.argtypes = [ctypes.c_int32] * 6
        _lib.ora_gravity_tool_cell.restype = ctypes.c_int64
        _lib.ora_align_dim.argtypes = [u32]
        _lib.ora_align_dim.restype = u32
        _lib.ora_set_threads.argtypes = [i32]
        _lib.ora_grav_seed.argtypes = [P, u32]
        _lib.ora_grav_particles.argtypes = [P, P, u32, u32]
        _lib.ora_grav_finish.argtypes = [P, u32]
        _lib.ora_num_threads.restype = i32
        W = ctypes.POINTER(VoxWorld)
        _lib.ora_vox_air_clear.argtypes = [W]
        _lib.ora_vox_air_gather.argtypes = [W, u32]
        _lib.ora_vox_air_solve.argtypes = [W, u32]
        _lib.ora_vox_grav_solve.argtypes = [W, u32]
        _lib.ora_vox_grav_clear_mass.argtypes = [W]
        _lib.ora_vox_grav_gather.argtypes = [W, u32]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def params_of(inst) -> AirParams:
    c = inst.config
    return AirParams(inst.xcells, inst.ycells, c.air_mode, c.aheat_enable, c.convection_mode, c.gravity_mode,
                     c.edge_pressure, c.edge_vx, c.edge_vy, c.ambient_air_temp, c.vorticity_coeff,
                     c.custom_gx, c.custom_gy)


def set_threads(n: int) -> None:
    lib().ora_set_threads(int(n))


def num_threads() -> int:
    return int(lib().ora_num_threads())


def air_steps(inst, ticks: int, dtype=np.float32, pmap=None, props=None, xres=0, yres=0):
    """Runs `ticks` air steps on a copy of `inst`'s state; returns the new
    state dict (pv, vx, vy, hv in `dtype`; emap, bair, bairh as u32)."""
    L = lib()
    f = L.ora_air_steps_f32 if dtype == np.float32 else L.ora_air_steps_f64
    st = {k: getattr(inst, k).astype(dtype).copy() for k in ("pv", "vx", "vy", "hv", "fan_vx", "fan_vy")}
    for k in ("wall", "emap", "bair", "bairh", "eair", "eairh"):
        st[k] = getattr(inst, k).astype(np.uint32).copy()
    prm = params_of(inst)
    nprops = 0 if props is None else len(props) // 32
    rc = f(ctypes.byref(prm), int(ticks), _p(st["pv"]), _p(st["vx"]), _p(st["vy"]), _p(st["hv"]),
           _p(st["wall"]), _p(st["emap"]), _p(st["bair"]), _p(st["bairh"]), _p(st["eair"]), _p(st["eairh"]),
           _p(st["fan_vx"]), _p(st["fan_vy"]), _p(pmap), _p(props), nprops, xres, yres)
    assert rc == 0
    return st


def grav_solve(X, Y, mask, mass_fx=None, mass_f32=None, mass_scale_inv=1.0 / 65536.0, dtype=np.float32,
               direct=False):
    """FP32 mirror (dtype f32), FP64 FFT twin (f64) or FP64 direct sum
    (direct=True) of the gravity solve; returns (gx, gy)."""
    L = lib()
    n = X * Y
    if direct:
        dtype = np.float64
    gx = np.zeros(n, dtype)
    gy = np.zeros(n, dtype)
    mi = None if mass_fx is None else np.ascontiguousarray(mass_fx, np.int32)
    mf = None if mass_f32 is None else np.ascontiguousarray(mass_f32, np.float32)
    mk = np.ascontiguousarray(mask, np.uint32)
    if direct:
        fn = L.ora_grav_direct_f64
    else:
        fn = L.ora_grav_solve_f32 if dtype == np.float32 else L.ora_grav_solve_f64
    rc = fn(X, Y, _p(mi), _p(mf), float(mass_scale_inv), _p(mk), _p(gx), _p(gy))
    assert rc == 0
    return gx, gy


def fft_host(data: np.ndarray, rows, n, inner, stride, tw_bits, sign):
    """In-place host mirror of the reference's bitrev + stage kernels on an
    interleaved complex f32 buffer (crates/tpt-sim/src/gravity_gpu/fft.rs:274)."""
    assert data.dtype == np.float32 and data.flags.c_contiguous
    lib().ora_fft_host_f32(_p(data), rows, n, inner, stride, tw_bits, float(sign))


def bit_count(n: int) -> int:
    return int(lib().ora_bit_count(n))


def twiddle(max_len: int):
    half = max(max_len // 2, 1)
    re = np.zeros(half, np.float32)
    im = np.zeros(half, np.float32)
    lib().ora_twiddle_f32(max_len, _p(re), _p(im))
    return re, im


def grav_mask(wall: np.ndarray, X: int, Y: int) -> np.ndarray:
    out = np.zeros(X * Y, np.uint32)
    w = np.ascontiguousarray(wall, np.uint32)
    lib().ora_grav_mask(_p(w), _p(out), X, Y)
    return out


def mass_to_fixed(m: float) -> int:
    return int(lib().ora_mass_to_fixed(float(m)))


def block_masks(wall, emap, eair=None, eairh=None):
    n = len(wall)
    w = np.ascontiguousarray(wall, np.uint32)
    e = np.ascontiguousarray(emap, np.uint32).copy()
    ba = np.zeros(n, np.uint32)
    bh = np.zeros(n, np.uint32)
    ea = None if eair is None else np.ascontiguousarray(eair, np.uint32)
    eh = None if eairh is None else np.ascontiguousarray(eairh, np.uint32)
    lib().ora_block_masks(n, _p(w), _p(e), _p(ba), _p(bh), _p(ea), _p(eh))
    return e, ba, bh


def tool_gravity_mass(strength: float, attract: bool) -> float:
    return float(lib().ora_tool_gravity_mass(float(strength), int(attract)))


def gravity_tool_cell(x, y, xres, yres, xcells, ycells):
    r = int(lib().ora_gravity_tool_cell(x, y, xres, yres, xcells, ycells))
    return None if r < 0 else r


def align_dim(v: int) -> int:
    return int(lib().ora_align_dim(v))


# ---- gravity tick around the solve (gravity_kernel.rs:217-527) ------------
class _Particles(ctypes.Structure):  # tpt_particles with host pointers
    _fields_ = [("num_slots", ctypes.c_uint32)] + [(n, ctypes.c_void_p) for n in (
        "ty", "x", "y", "vx", "vy", "life", "tmp", "temp", "flags", "move_lut")] + [("n_types", ctypes.c_uint32)]


class _GravState(ctypes.Structure):  # tpt_grav_state with host pointers
    _fields_ = [("xres", ctypes.c_uint32), ("yres", ctypes.c_uint32)] + [(n, ctypes.c_void_p) for n in (
        "wall_bmap", "wall_emap", "grav_mask", "mass", "mass_prev", "tool_mass", "override_mass", "override_set",
        "gx", "gy")] + [("newton_grav", ctypes.c_float)]


_STATE_TYPES = {"wall_bmap": np.uint32, "wall_emap": np.uint32, "grav_mask": np.uint32, "mass": np.int32,
                "mass_prev": np.int32, "tool_mass": np.float32, "override_mass": np.int32,
                "override_set": np.uint32, "gx": np.float32, "gy": np.float32}
_PART_TYPES = {"ty": np.uint32, "x": np.float32, "y": np.float32, "vx": np.float32, "vy": np.float32,
               "life": np.int32, "tmp": np.int32, "temp": np.float32, "flags": np.uint32}


def _state(state: dict, xres: int, yres: int, newton: float):
    arrs = {k: (None if state.get(k) is None else np.ascontiguousarray(state[k], t).copy())
            for k, t in _STATE_TYPES.items()}
    st = _GravState(xres=xres, yres=yres, newton_grav=float(newton), **{k: _p(a) for k, a in arrs.items()})
    return st, arrs


def grav_seed(state: dict, xres: int, yres: int) -> dict:
    """Wells folded into mass_prev, accumulator cleared (before the solve)."""
    st, arrs = _state(state, xres, yres, 1.0)
    lib().ora_grav_seed(ctypes.byref(st), (xres // 4) * (yres // 4))
    return arrs


def grav_particles_and_finish(state: dict, parts: dict, move_lut, n_types: int, xres: int, yres: int,
                              newton: float = 1.0):
    """Force on the particles (with the gx/gy given in `state`), mass build,
    overrides, snapshot copy. Returns (state', parts')."""
    st, arrs = _state(state, xres, yres, newton)
    pa = {k: np.ascontiguousarray(parts[k], t).copy() for k, t in _PART_TYPES.items()}
    lut = np.ascontiguousarray(move_lut, np.uint32)
    q = _Particles(num_slots=len(pa["ty"]), n_types=n_types, move_lut=_p(lut), **{k: _p(a) for k, a in pa.items()})
    lib().ora_grav_particles(ctypes.byref(st), ctypes.byref(q), xres // 4, yres // 4)
    lib().ora_grav_finish(ctypes.byref(st), (xres // 4) * (yres // 4))
    return arrs, pa


# ------------------------------------------------------------ 3-D ------
# The 3-D sandbox's field step (crates/tpt-sim/src/voxel3d), in place on a
# dict of numpy arrays with the keys of workloads.voxel_world.

def _vox(d: dict) -> VoxWorld:
    w = VoxWorld()
    for name, _ in VoxWorld._fields_:
        if name in d:
            a = d[name]
            assert a.flags["C_CONTIGUOUS"]
            setattr(w, name, a.ctypes.data)
    return w


def vox_air_clear(d: dict) -> None:
    lib().ora_vox_air_clear(ctypes.byref(_vox(d)))


def vox_air_gather(d: dict) -> None:
    lib().ora_vox_air_gather(ctypes.byref(_vox(d)), int(d["sim_count"][0]))


def vox_air_solve(d: dict, iterations: int = 12) -> None:
    lib().ora_vox_air_solve(ctypes.byref(_vox(d)), int(iterations))


def vox_grav_solve(d: dict, iterations: int = 24) -> None:
    lib().ora_vox_grav_solve(ctypes.byref(_vox(d)), int(iterations))


def vox_grav_clear_mass(d: dict) -> None:
    lib().ora_vox_grav_clear_mass(ctypes.byref(_vox(d)))


def vox_grav_gather(d: dict) -> None:
    lib().ora_vox_grav_gather(ctypes.byref(_vox(d)), int(d["sim_count"][0]))


def vox_field_step(d: dict, iterations: int = 12) -> None:
    """The reference tick's field part (engine.rs:195-208): air gather, air
    solve, gravity solve, clear mass."""
    vox_air_gather(d)
    vox_air_solve(d, iterations)
    vox_grav_solve(d)
    vox_grav_clear_mass(d)
