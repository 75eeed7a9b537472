"""Python host side of the B200 field step: ctypes bindings of
libtpt_field.so (include/tpt_field.h) and a mirror of the reference's
interface for this path.

Reference interface mirrored here (paths relative to the reference project):

  SimulationConfig   crates/tpt-core/src/particle.rs:166-345 (hot-path fields)
  SimBuffers         crates/tpt-sim/src/buffers/mod.rs:186-230 (air, wall and
                     gravity grids; device tensors in the reference layout)
  step_air_gpu       crates/tpt-sim/src/air_kernel/mod.rs:120
  GravityFft.solve   crates/tpt-sim/src/gravity_gpu/mod.rs:114
  step_gravity       crates/tpt-sim/src/gravity_kernel.rs:826-920 (mask
                     rebuild on a wall change, then the solve)

Every call goes to the CUDA library; there is no CPU fallback. Importing
works anywhere, but the first call raises `TptError` if the library is not
built or no sm_100 GPU is present.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtpt_field.so")

TPT_OK = 0
ERRORS = {
    -1: "TPT_ERR_INVALID_DIMS", -2: "TPT_ERR_NULL_POINTER", -3: "TPT_ERR_CUDA",
    -4: "TPT_ERR_DEVICE_TIMEOUT", -5: "TPT_ERR_INVALID_ARG", -6: "TPT_ERR_OUT_OF_MEMORY",
    -7: "TPT_ERR_UNSUPPORTED",
}
PRECISION_FP32 = 0
PRECISION_SPLIT_BF16 = 1

(FIELD_PV, FIELD_VX, FIELD_VY, FIELD_HV, FIELD_BLOCK_AIR, FIELD_BLOCK_AIRH, FIELD_WALL_BMAP, FIELD_WALL_EMAP,
 FIELD_ELEM_BLOCK_AIR, FIELD_ELEM_BLOCK_AIRH, FIELD_FAN_VX, FIELD_FAN_VY, FIELD_GRAV_MASS, FIELD_GRAV_MASK,
 FIELD_GX, FIELD_GY) = range(16)

# Every symbol include/tpt_field.h declares.
EXPORTS = [
    "tpt_air_params_default", "tpt_air_step", "tpt_air_step_static_scratch", "tpt_wall_masks_host", "tpt_grav_plan_create",
    "tpt_grav_plan_destroy", "tpt_grav_plan_dims", "tpt_grav_solve", "tpt_grav_solve_f32",
    "tpt_grav_mask_rebuild", "tpt_mass_to_fixed", "tpt_grav_step", "tpt_batch_create", "tpt_batch_destroy", "tpt_batch_fields",
    "tpt_batch_write", "tpt_batch_read", "tpt_batch_write_field", "tpt_batch_read_field", "tpt_batch_step", "tpt_batch_tune", "tpt_batch_get_tuning",
    "tpt_batch_set_tuning", "tpt_batch_profile_phases", "tpt_vox_plan_create", "tpt_vox_plan_destroy",
    "tpt_vox_plan_form", "tpt_vox_air_clear", "tpt_vox_air_gather", "tpt_vox_air_solve", "tpt_vox_grav_solve",
    "tpt_vox_grav_clear_mass", "tpt_vox_grav_gather", "tpt_vox_field_step", "tpt_save_config_default",
    "tpt_save_create", "tpt_save_decode", "tpt_save_encode", "tpt_save_destroy", "tpt_save_get_info",
    "tpt_save_get_config", "tpt_save_set_config", "tpt_save_set_version", "tpt_save_grid_read",
    "tpt_save_grid_write", "tpt_save_grid_restore", "tpt_save_particles_read", "tpt_save_particles_write",
    "tpt_save_retain_air_pressure", "tpt_save_instance_desc", "tpt_vox_save_config_default", "tpt_vox_save_create",
    "tpt_vox_save_decode", "tpt_vox_save_encode", "tpt_vox_save_destroy", "tpt_vox_save_get_info",
    "tpt_vox_save_get_config", "tpt_vox_save_set_config", "tpt_vox_save_array_read", "tpt_vox_save_array_write",
    "tpt_vox_save_restore_air", "tpt_check_device_errors", "tpt_selftest_wait_timeout",
    "tpt_last_error_string", "tpt_kernel_launch_count", "tpt_version",
]
SAVE_GRIDS = ("air_vx", "air_vy", "air_pv", "air_hv", "fan_vx", "fan_vy", "wall_bmap", "wall_emap")
VOX_SAVE_ARRAYS = ("voxels", "aux_ctype", "aux_tmp", "aux_tmp2", "aux_tmp3", "air")
VOX_AUTO, VOX_CLUSTER, VOX_PER_SWEEP, VOX_BATCHED = 0, 1, 2, 3


class TptError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class AirParams(ctypes.Structure):
    _fields_ = [
        ("xcells", ctypes.c_uint32), ("ycells", ctypes.c_uint32),
        ("air_mode", ctypes.c_uint32), ("aheat_enable", ctypes.c_uint32),
        ("convection_mode", ctypes.c_uint32), ("gravity_mode", ctypes.c_uint32),
        ("edge_pressure", ctypes.c_float), ("edge_vx", ctypes.c_float), ("edge_vy", ctypes.c_float),
        ("ambient_air_temp", ctypes.c_float), ("vorticity_coeff", ctypes.c_float),
        ("custom_gx", ctypes.c_float), ("custom_gy", ctypes.c_float),
    ]


class AirBufs(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "pv", "vx", "vy", "hv", "opv", "ovx", "ovy", "ohv", "block_air", "block_airh", "wall_bmap", "wall_emap",
        "elem_block_air", "elem_block_airh", "fan_vx", "fan_vy", "pmap", "elem_props")] + [
        ("xres", ctypes.c_uint32), ("yres", ctypes.c_uint32), ("n_elements", ctypes.c_uint32)]


class Particles(ctypes.Structure):
    """tpt_particles: particle slots, struct of arrays (device pointers)."""
    _fields_ = [("num_slots", ctypes.c_uint32)] + [(n, ctypes.c_void_p) for n in (
        "ty", "x", "y", "vx", "vy", "life", "tmp", "temp", "flags", "move_lut")] + [("n_types", ctypes.c_uint32)]


class GravState(ctypes.Structure):
    """tpt_grav_state: one sandbox's gravity grids (device pointers)."""
    _fields_ = [("xres", ctypes.c_uint32), ("yres", ctypes.c_uint32)] + [(n, ctypes.c_void_p) for n in (
        "wall_bmap", "wall_emap", "grav_mask", "mass", "mass_prev", "tool_mass", "override_mass", "override_set",
        "gx", "gy")] + [("newton_grav", ctypes.c_float)]


PARTICLE_FIELDS = ("ty", "x", "y", "vx", "vy", "life", "tmp", "temp", "flags")
GRAV_STATE_FIELDS = ("wall_bmap", "wall_emap", "grav_mask", "mass", "mass_prev", "tool_mass", "override_mass",
                     "override_set", "gx", "gy")


class InstanceDesc(ctypes.Structure):
    _fields_ = [("air", AirParams), ("newton_grav", ctypes.c_uint32)]


class InstanceFields(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "pv", "vx", "vy", "hv", "block_air", "block_airh", "wall_bmap", "wall_emap", "elem_block_air",
        "elem_block_airh", "fan_vx", "fan_vy", "grav_mass", "grav_mask", "gx", "gy")] + [("pitch", ctypes.c_uint32)]


class BatchProfile(ctypes.Structure):
    _fields_ = [("air_ms", ctypes.c_float), ("grav_ms", ctypes.c_float), ("ticks", ctypes.c_uint32),
                ("air_launches_per_tick", ctypes.c_uint32), ("grav_launches_per_tick", ctypes.c_uint32),
                ("cells", ctypes.c_uint64), ("grav_cells", ctypes.c_uint64), ("grav_flops_per_tick", ctypes.c_double)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("tile_x", ctypes.c_uint32), ("tile_y", ctypes.c_uint32), ("temporal_depth", ctypes.c_uint32),
                ("ctas_per_sm", ctypes.c_uint32), ("grav_side_ctas", ctypes.c_uint32), ("air_form", ctypes.c_uint32),
                ("work_queue", ctypes.c_uint32)]


AIR_FORM_TILES, AIR_FORM_SWEEP = 0, 1
# (tile_x, tile_y) of the tile form's shapes, the default first
TILE_SHAPES = ((32, 8), (64, 8), (32, 16), (64, 16))


_lib = None


class VoxWorld(ctypes.Structure):
    """tpt_vox_world: one 3-D world's device buffers."""

    _fields_ = [(n, ctypes.c_void_p) for n in (
        "voxel", "aux_tmp", "sim_list", "sim_count", "vx", "vy", "vz", "p", "p_tmp", "temp", "solid", "pv",
        "grav_mass", "grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y", "grav_force_z")]


class SaveConfig(ctypes.Structure):
    """tpt_save_config: every serialised SimulationConfig field, in order."""

    u8, u32, i32, f32 = ctypes.c_uint8, ctypes.c_uint32, ctypes.c_int32, ctypes.c_float
    _fields_ = [
        ("xres", u32), ("yres", u32), ("paused", u8), ("aheat_enable", u8), ("pretty_powder", u8), ("_pad0", u8),
        ("edge_mode", u32), ("gravity_mode", u32), ("air_mode", u32), ("ambient_air_temp", f32),
        ("edge_pressure", f32), ("display_mode", u32), ("colour_mode", u32), ("render_mode", u32),
        ("fire_intensity", f32), ("heat_enable", u8), ("newton_grav", u8), ("water_equal_test", u8), ("_pad1", u8),
        ("vorticity_coeff", f32), ("convection_mode", u32), ("edge_velocity_x", f32), ("edge_velocity_y", f32),
        ("custom_gravity_x", f32), ("custom_gravity_y", f32), ("temperature_scale", u32), ("decorations", u8),
        ("_pad2", u8 * 3), ("mouse_x", i32), ("mouse_y", i32), ("gravity_field_enabled", u8),
        ("gravity_zones_enabled", u8), ("grid", u8), ("_pad3", u8), ("grid_size", i32), ("grid_checkerboard", u8),
        ("hud", u8), ("debug_hud", u8), ("show_brush", u8), ("zoom_enabled", u8), ("_pad4", u8 * 3),
        ("zoom_window_x", i32), ("zoom_window_y", i32), ("zoom_factor", i32), ("zoom_scope_x", i32),
        ("zoom_scope_y", i32), ("zoom_scope_size", i32), ("has_heat_display_limit_min", u8),
        ("has_heat_display_limit_max", u8), ("_pad5", u8 * 2), ("heat_display_limit_min", f32),
        ("heat_display_limit_max", f32), ("heat_display_auto_x", i32), ("heat_display_auto_y", i32),
        ("heat_display_auto_w", i32), ("heat_display_auto_h", i32),
    ]


class VoxSaveConfig(ctypes.Structure):
    """tpt_vox_save_config: Voxel3dConfig's serialised fields, in order."""

    u8, u32, f32 = ctypes.c_uint8, ctypes.c_uint32, ctypes.c_float
    _fields_ = [("dim", u32), ("paused", u8), ("_pad0", u8 * 3), ("ambient_temp_k", f32), ("gravity", f32 * 3),
                ("edge_mode", u32), ("air_enabled", u8), ("_pad1", u8 * 3), ("air_iterations", u32),
                ("sun_dir", f32 * 3), ("exposure", f32), ("render_scale", f32), ("ao_rays", u32), ("shadows", u8),
                ("_pad2", u8 * 3)]


class VoxSaveInfo(ctypes.Structure):
    _fields_ = [("version", ctypes.c_uint32), ("len", ctypes.c_uint64 * 6), ("n_bodies", ctypes.c_uint64)]


class SaveInfo(ctypes.Structure):
    _fields_ = [("version", ctypes.c_uint32), ("xcells", ctypes.c_uint32), ("ycells", ctypes.c_uint32),
                ("n_particles", ctypes.c_uint64), ("n_rigid_bodies", ctypes.c_uint64), ("n_signs", ctypes.c_uint64),
                ("grid_len", ctypes.c_uint64 * 8)]


def build() -> None:
    """Compiles libtpt_field.so for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    """The loaded CUDA library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise TptError(-7, f"{LIB_PATH} is not built (run build())")
        L = ctypes.CDLL(LIB_PATH)
        P, u32, i32, f32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
        L.tpt_air_params_default.argtypes = [ctypes.POINTER(AirParams), u32, u32]
        L.tpt_air_params_default.restype = None
        L.tpt_air_step.argtypes = [ctypes.POINTER(AirParams), ctypes.POINTER(AirBufs), P]
        L.tpt_air_step_static_scratch.argtypes = [ctypes.POINTER(AirParams), ctypes.POINTER(AirBufs), P]
        L.tpt_wall_masks_host.argtypes = [P, P, P, P, ctypes.c_size_t]
        L.tpt_grav_plan_create.argtypes = [u32, u32, i32, ctypes.POINTER(P)]
        L.tpt_grav_plan_destroy.argtypes = [P]
        L.tpt_grav_plan_dims.argtypes = [P, ctypes.POINTER(u32), ctypes.POINTER(u32)]
        L.tpt_grav_solve.argtypes = [P, P, f32, P, P, P, P]
        L.tpt_grav_solve_f32.argtypes = [P, P, P, P, P, P]
        L.tpt_grav_mask_rebuild.argtypes = [P, P, u32, u32]
        L.tpt_mass_to_fixed.argtypes = [f32]
        L.tpt_mass_to_fixed.restype = ctypes.c_int32
        L.tpt_grav_step.argtypes = [P, ctypes.POINTER(GravState), ctypes.POINTER(Particles), P]
        L.tpt_batch_create.argtypes = [u32, ctypes.POINTER(InstanceDesc), i32, ctypes.POINTER(P)]
        L.tpt_batch_destroy.argtypes = [P]
        L.tpt_batch_fields.argtypes = [P, u32, ctypes.POINTER(InstanceFields)]
        L.tpt_batch_write.argtypes = [P, u32, i32, P, ctypes.c_size_t, P]
        L.tpt_batch_read.argtypes = [P, u32, i32, P, ctypes.c_size_t, P]
        L.tpt_batch_write_field.argtypes = [P, i32, P, ctypes.c_size_t, P]
        L.tpt_batch_read_field.argtypes = [P, i32, P, ctypes.c_size_t, P]
        L.tpt_batch_step.argtypes = [P, u32, P]
        L.tpt_batch_tune.argtypes = [P, P]
        L.tpt_batch_get_tuning.argtypes = [P, ctypes.POINTER(BatchTuning)]
        L.tpt_batch_set_tuning.argtypes = [P, ctypes.POINTER(BatchTuning)]
        L.tpt_batch_profile_phases.argtypes = [P, u32, P, ctypes.POINTER(BatchProfile)]
        W = ctypes.POINTER(VoxWorld)
        L.tpt_vox_plan_create.argtypes = [i32, ctypes.POINTER(P)]
        L.tpt_vox_plan_destroy.argtypes = [P]
        L.tpt_vox_plan_form.argtypes = [P]
        L.tpt_vox_air_clear.argtypes = [W, P]
        L.tpt_vox_air_gather.argtypes = [P, W, P]
        L.tpt_vox_air_solve.argtypes = [P, W, u32, P]
        L.tpt_vox_grav_solve.argtypes = [P, W, P]
        L.tpt_vox_grav_clear_mass.argtypes = [P, W, P]
        L.tpt_vox_grav_gather.argtypes = [P, W, P]
        L.tpt_vox_field_step.argtypes = [P, W, u32, u32, P]
        SC, S = ctypes.POINTER(SaveConfig), P
        L.tpt_save_config_default.argtypes = [SC, u32, u32]
        L.tpt_save_config_default.restype = None
        L.tpt_save_create.argtypes = [SC, ctypes.POINTER(P)]
        L.tpt_save_decode.argtypes = [P, ctypes.c_size_t, ctypes.POINTER(P)]
        L.tpt_save_encode.argtypes = [S, ctypes.POINTER(P), ctypes.POINTER(ctypes.c_size_t)]
        L.tpt_save_destroy.argtypes = [S]
        L.tpt_save_get_info.argtypes = [S, ctypes.POINTER(SaveInfo)]
        L.tpt_save_get_config.argtypes = [S, SC]
        L.tpt_save_set_config.argtypes = [S, SC]
        L.tpt_save_set_version.argtypes = [S, u32]
        L.tpt_save_grid_read.argtypes = [S, i32, P, ctypes.c_size_t]
        L.tpt_save_grid_write.argtypes = [S, i32, P, ctypes.c_size_t]
        L.tpt_save_grid_restore.argtypes = [S, i32, P, ctypes.c_uint64]
        L.tpt_save_particles_read.argtypes = [S, P, ctypes.c_size_t]
        L.tpt_save_particles_write.argtypes = [S, P, ctypes.c_size_t]
        L.tpt_save_retain_air_pressure.argtypes = [S, i32]
        L.tpt_save_instance_desc.argtypes = [S, ctypes.POINTER(InstanceDesc)]
        VC = ctypes.POINTER(VoxSaveConfig)
        L.tpt_vox_save_config_default.argtypes = [VC]
        L.tpt_vox_save_config_default.restype = None
        L.tpt_vox_save_create.argtypes = [VC, ctypes.POINTER(P)]
        L.tpt_vox_save_decode.argtypes = [P, ctypes.c_size_t, ctypes.POINTER(P)]
        L.tpt_vox_save_encode.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(ctypes.c_size_t)]
        L.tpt_vox_save_destroy.argtypes = [P]
        L.tpt_vox_save_get_info.argtypes = [P, ctypes.POINTER(VoxSaveInfo)]
        L.tpt_vox_save_get_config.argtypes = [P, VC]
        L.tpt_vox_save_set_config.argtypes = [P, VC]
        L.tpt_vox_save_array_read.argtypes = [P, i32, P, ctypes.c_size_t]
        L.tpt_vox_save_array_write.argtypes = [P, i32, P, ctypes.c_size_t]
        L.tpt_vox_save_restore_air.argtypes = [P] * 7
        L.tpt_selftest_wait_timeout.argtypes = [u32, P]
        L.tpt_last_error_string.restype = ctypes.c_char_p
        L.tpt_kernel_launch_count.restype = ctypes.c_uint64
        L.tpt_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != TPT_OK:
        raise TptError(rc, lib().tpt_last_error_string().decode())


def launch_count() -> int:
    return int(lib().tpt_kernel_launch_count())


def _ptr(t) -> ctypes.c_void_p | None:
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data_as(ctypes.c_void_p)
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream) -> ctypes.c_void_p | None:
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


# ----------------------------------------------------- reference mirror --

@dataclasses.dataclass
class SimulationConfig:
    """Hot-path fields of the reference `SimulationConfig` with its defaults
    (crates/tpt-core/src/particle.rs:290-345). `xres`/`yres` are pixels; the
    air grid is (xres/4) x (yres/4) cells."""

    xres: int = 612
    yres: int = 384
    air_mode: int = 0
    aheat_enable: bool = False
    convection_mode: int = 2
    gravity_mode: int = 0
    edge_pressure: float = 0.0
    edge_velocity_x: float = 0.0
    edge_velocity_y: float = 0.0
    ambient_air_temp: float = 295.15
    vorticity_coeff: float = 0.1
    custom_gravity_x: float = 0.0
    custom_gravity_y: float = 1.0
    newton_grav: bool = False

    @classmethod
    def new(cls, xres: int, yres: int, **kw) -> "SimulationConfig":
        """`SimulationConfig::new` (crates/tpt-core/src/particle.rs:290-293,
        381-383): each side clamped to at least 64 px and rounded up to a
        multiple of the 4-px cell."""
        def align(v: int) -> int:
            v = max(int(v), 64)
            return (v + 3) // 4 * 4
        return cls(xres=align(xres), yres=align(yres), **kw)

    def xcells(self) -> int:
        return self.xres // 4

    def ycells(self) -> int:
        return self.yres // 4

    def num_cells(self) -> int:
        return self.xcells() * self.ycells()

    def air_params(self) -> AirParams:
        return AirParams(self.xcells(), self.ycells(), int(self.air_mode), int(bool(self.aheat_enable)),
                         int(self.convection_mode), int(self.gravity_mode), self.edge_pressure,
                         self.edge_velocity_x, self.edge_velocity_y, self.ambient_air_temp, self.vorticity_coeff,
                         self.custom_gravity_x, self.custom_gravity_y)


_F32 = ("air_pv", "air_vx", "air_vy", "air_hv", "air_opv", "air_ovx", "air_ovy", "air_ohv", "fan_vx", "fan_vy",
        "grav_fx", "grav_fy")
_U32 = ("block_air", "block_airh", "wall_bmap", "wall_emap", "elem_block_air", "elem_block_airh", "grav_mask")


class SimBuffers:
    """Device grids of one canvas, in the reference layout and names
    (`gpu_air_pv`, ... of crates/tpt-sim/src/buffers/mod.rs:186-230), held as
    torch CUDA tensors. `grav_mass_prev` is the fixed-point mass the solve
    reads; `grav_mask_dirty` triggers the flood fill on the next gravity step
    (crates/tpt-sim/src/gravity_kernel.rs:868-881)."""

    def __init__(self, config: SimulationConfig, device="cuda"):
        import torch

        self.config = config
        n = config.num_cells()
        for k in _F32:
            setattr(self, k, torch.zeros(n, dtype=torch.float32, device=device))
        for k in _U32:
            setattr(self, k, torch.zeros(n, dtype=torch.int32, device=device))  # u32 bit patterns
        self.grav_mass_prev = torch.zeros(n, dtype=torch.int32, device=device)
        self.pmap = None
        self.elem_props = None
        self.grav_mask_dirty = True

    @classmethod
    def from_instance(cls, inst, device="cuda") -> "SimBuffers":
        """Uploads a `workloads.Instance` (host numpy grids)."""
        import torch

        c = inst.config
        cfg = SimulationConfig(xres=inst.xcells * 4, yres=inst.ycells * 4, air_mode=c.air_mode,
                               aheat_enable=bool(c.aheat_enable), convection_mode=c.convection_mode,
                               gravity_mode=c.gravity_mode, edge_pressure=c.edge_pressure,
                               edge_velocity_x=c.edge_vx, edge_velocity_y=c.edge_vy,
                               ambient_air_temp=c.ambient_air_temp, vorticity_coeff=c.vorticity_coeff,
                               custom_gravity_x=c.custom_gx, custom_gravity_y=c.custom_gy,
                               newton_grav=bool(c.newton_grav))
        b = cls(cfg, device)

        def put(name, arr, dt):
            getattr(b, name).copy_(torch.from_numpy(np.ascontiguousarray(arr).view(dt)))

        put("air_pv", inst.pv, np.float32)
        put("air_vx", inst.vx, np.float32)
        put("air_vy", inst.vy, np.float32)
        put("air_hv", inst.hv, np.float32)
        put("fan_vx", inst.fan_vx, np.float32)
        put("fan_vy", inst.fan_vy, np.float32)
        for name, arr in (("block_air", inst.bair), ("block_airh", inst.bairh), ("wall_bmap", inst.wall),
                          ("wall_emap", inst.emap), ("elem_block_air", inst.eair),
                          ("elem_block_airh", inst.eairh), ("grav_mask", inst.gmask)):
            put(name, arr.astype(np.uint32), np.int32)
        b.grav_mass_prev.copy_(torch.from_numpy(inst.mass_fx.astype(np.int32)))
        b.grav_mask_dirty = False
        return b

    def air_state(self) -> dict:
        """Host copies of the state grids (f32 and u32 numpy arrays)."""
        out = {k: getattr(self, a).cpu().numpy() for k, a in (("pv", "air_pv"), ("vx", "air_vx"), ("vy", "air_vy"),
                                                                ("hv", "air_hv"))}
        for k, a in (("emap", "wall_emap"), ("bair", "block_air"), ("bairh", "block_airh")):
            out[k] = getattr(self, a).cpu().numpy().view(np.uint32)
        return out


def air_bufs(b: SimBuffers) -> AirBufs:
    x = AirBufs()
    for name, attr in (("pv", "air_pv"), ("vx", "air_vx"), ("vy", "air_vy"), ("hv", "air_hv"), ("opv", "air_opv"),
                       ("ovx", "air_ovx"), ("ovy", "air_ovy"), ("ohv", "air_ohv"), ("block_air", "block_air"),
                       ("block_airh", "block_airh"), ("wall_bmap", "wall_bmap"), ("wall_emap", "wall_emap"),
                       ("elem_block_air", "elem_block_air"), ("elem_block_airh", "elem_block_airh"),
                       ("fan_vx", "fan_vx"), ("fan_vy", "fan_vy")):
        setattr(x, name, _ptr(getattr(b, attr)))
    if b.pmap is not None:
        x.pmap = _ptr(b.pmap)
        x.elem_props = _ptr(b.elem_props)
        x.xres = b.config.xres
        x.yres = b.config.yres
        x.n_elements = b.elem_props.numel() // 32
    return x


def step_air_gpu(bufs: SimBuffers, stream=None) -> None:
    """One air step on the device (crates/tpt-sim/src/air_kernel/mod.rs:120)."""
    prm = bufs.config.air_params()
    check(lib().tpt_air_step(ctypes.byref(prm), ctypes.byref(air_bufs(bufs)), _stream(stream)))


class GravityFft:
    """Gravity solver with a plan cached per canvas size, rebuilt lazily on a
    size change (crates/tpt-sim/src/gravity_gpu/mod.rs:99-135)."""

    def __init__(self, precision: int = PRECISION_FP32):
        self.precision = precision
        self._plan = None
        self._dims = None

    def _ensure(self, xcells: int, ycells: int):
        if self._dims != (xcells, ycells):
            self.close()
            p = ctypes.c_void_p()
            check(lib().tpt_grav_plan_create(xcells, ycells, self.precision, ctypes.byref(p)))
            self._plan, self._dims = p, (xcells, ycells)

    def padded_dims(self):
        n1, n2 = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().tpt_grav_plan_dims(self._plan, ctypes.byref(n1), ctypes.byref(n2)))
        return n1.value, n2.value

    def solve(self, bufs: SimBuffers, mass, mass_scale_inv: float = 1.0 / 65536.0, stream=None) -> None:
        """Solves into bufs.grav_fx / grav_fy from a fixed-point i32 `mass`
        grid, or from an f32 grid (then `mass_scale_inv` is unused)."""
        import torch

        X, Y = bufs.config.xcells(), bufs.config.ycells()
        if X == 0 or Y == 0:
            return
        self._ensure(X, Y)
        if mass.dtype == torch.float32:
            check(lib().tpt_grav_solve_f32(self._plan, _ptr(mass), _ptr(bufs.grav_mask), _ptr(bufs.grav_fx),
                                           _ptr(bufs.grav_fy), _stream(stream)))
        else:
            check(lib().tpt_grav_solve(self._plan, _ptr(mass), float(mass_scale_inv), _ptr(bufs.grav_mask),
                                       _ptr(bufs.grav_fx), _ptr(bufs.grav_fy), _stream(stream)))

    def step(self, state: dict, parts: dict, move_lut, n_types: int, xres: int, yres: int,
             newton_grav: float = 1.0, stream=None) -> None:
        """One gravity tick with particles (`step_gravity_gpu`,
        crates/tpt-sim/src/gravity_kernel.rs:826-1010, after the mask
        rebuild): wells into `mass_prev`, the solve into `gx`/`gy`, Loss and
        the force on the particles' `vx`/`vy`, the mass grid rebuilt from the
        particles and copied into `mass_prev`. `state` maps GRAV_STATE_FIELDS
        to device tensors (tool_mass and the override pair may be missing or
        None); `parts` maps PARTICLE_FIELDS to device tensors of one length."""
        self._ensure(xres // 4, yres // 4)
        st = GravState(xres=xres, yres=yres, newton_grav=float(newton_grav),
                       **{k: (_ptr(state[k]) if state.get(k) is not None else None) for k in GRAV_STATE_FIELDS})
        n = int(parts["ty"].numel()) if parts else 0
        pa = Particles(num_slots=n, n_types=int(n_types), move_lut=_ptr(move_lut),
                       **{k: _ptr(parts[k]) for k in PARTICLE_FIELDS})
        check(lib().tpt_grav_step(self._plan, ctypes.byref(st), ctypes.byref(pa), _stream(stream)))

    def close(self):
        if self._plan is not None:
            lib().tpt_grav_plan_destroy(self._plan)
            self._plan, self._dims = None, None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rebuild_gravity_mask(wall_bmap: np.ndarray, xcells: int, ycells: int) -> np.ndarray:
    """Host flood fill (crates/tpt-sim/src/gravity_kernel.rs:658-712)."""
    w = np.ascontiguousarray(wall_bmap, np.uint32)
    out = np.zeros(xcells * ycells, np.uint32)
    check(lib().tpt_grav_mask_rebuild(_ptr(w), _ptr(out), xcells, ycells))
    return out


def step_gravity(bufs: SimBuffers, solver: GravityFft, stream=None) -> None:
    """The field part of `step_gravity_gpu` (crates/tpt-sim/src/gravity_kernel.rs:
    826-920): skipped unless newton_grav; the mask is rebuilt after a wall
    change, then the previous tick's mass is solved."""
    import torch

    if not bufs.config.newton_grav:
        bufs.grav_fx.zero_()
        bufs.grav_fy.zero_()
        return
    if bufs.grav_mask_dirty:
        wall = bufs.wall_bmap.cpu().numpy().view(np.uint32)
        m = rebuild_gravity_mask(wall, bufs.config.xcells(), bufs.config.ycells())
        bufs.grav_mask.copy_(torch.from_numpy(m.view(np.int32)))
        bufs.grav_mask_dirty = False
    solver.solve(bufs, bufs.grav_mass_prev, 1.0 / 65536.0, stream)


def mass_to_fixed(m: float) -> int:
    return int(lib().tpt_mass_to_fixed(float(m)))


# ------------------------------------------------------------- batches --

class Batch:
    """Many independent instances stepped together (tpt_batch_*)."""

    def __init__(self, instances, precision: int = PRECISION_FP32, stream=None):
        n = len(instances)
        descs = (InstanceDesc * n)()
        for i, inst in enumerate(instances):
            c = inst.config
            descs[i].air = AirParams(inst.xcells, inst.ycells, c.air_mode, c.aheat_enable, c.convection_mode,
                                     c.gravity_mode, c.edge_pressure, c.edge_vx, c.edge_vy, c.ambient_air_temp,
                                     c.vorticity_coeff, c.custom_gx, c.custom_gy)
            descs[i].newton_grav = int(bool(c.newton_grav))
        self.n = n
        self.shapes = [(inst.xcells, inst.ycells) for inst in instances]
        self.precision = precision
        self._h = ctypes.c_void_p()
        check(lib().tpt_batch_create(n, descs, precision, ctypes.byref(self._h)))
        self.write_all(instances, stream)

    GRIDS = (("pv", FIELD_PV), ("vx", FIELD_VX), ("vy", FIELD_VY), ("hv", FIELD_HV), ("bair", FIELD_BLOCK_AIR),
             ("bairh", FIELD_BLOCK_AIRH), ("wall", FIELD_WALL_BMAP), ("emap", FIELD_WALL_EMAP),
             ("eair", FIELD_ELEM_BLOCK_AIR), ("eairh", FIELD_ELEM_BLOCK_AIRH), ("fan_vx", FIELD_FAN_VX),
             ("fan_vy", FIELD_FAN_VY), ("mass_fx", FIELD_GRAV_MASS), ("gmask", FIELD_GRAV_MASK))

    def write(self, i: int, field: int, arr: np.ndarray, stream=None):
        a = np.ascontiguousarray(arr)
        assert a.itemsize == 4
        check(lib().tpt_batch_write(self._h, i, field, _ptr(a), a.nbytes, _stream(stream)))

    def read(self, i: int, field: int, dtype, out: np.ndarray | None = None, stream=None) -> np.ndarray:
        X, Y = self.shapes[i] if 0 <= i < self.n else (1, 1)  # the library rejects a bad index
        a = np.empty(X * Y, dtype) if out is None else out
        check(lib().tpt_batch_read(self._h, i, field, _ptr(a), a.nbytes, _stream(stream)))
        return a

    @property
    def total_cells(self) -> int:
        return sum(X * Y for X, Y in self.shapes)

    def write_field(self, field: int, arr: np.ndarray, stream=None):
        """One grid of every instance, dense and back to back in instance order."""
        a = np.ascontiguousarray(arr)
        assert a.itemsize == 4
        check(lib().tpt_batch_write_field(self._h, field, _ptr(a), a.nbytes, _stream(stream)))

    def read_field(self, field: int, dtype, out: np.ndarray | None = None, stream=None) -> np.ndarray:
        a = np.empty(self.total_cells, dtype) if out is None else out
        check(lib().tpt_batch_read_field(self._h, field, _ptr(a), a.nbytes, _stream(stream)))
        return a

    def write_all(self, instances, stream=None):
        import torch

        for name, fid in self.GRIDS:
            self.write_field(fid, np.concatenate([np.ascontiguousarray(getattr(inst, name)).ravel()
                                                  for inst in instances]), stream)
        torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()

    def step(self, ticks: int, stream=None):
        check(lib().tpt_batch_step(self._h, int(ticks), _stream(stream)))

    def tune(self, stream=None):
        check(lib().tpt_batch_tune(self._h, _stream(stream)))

    def profile_phases(self, ticks: int, stream=None) -> BatchProfile:
        out = BatchProfile()
        check(lib().tpt_batch_profile_phases(self._h, int(ticks), _stream(stream), ctypes.byref(out)))
        return out

    def tuning(self) -> BatchTuning:
        t = BatchTuning()
        check(lib().tpt_batch_get_tuning(self._h, ctypes.byref(t)))
        return t

    def tuning_dict(self) -> dict:
        t = self.tuning()
        return {name: getattr(t, name) for name, _ in BatchTuning._fields_}

    def set_tuning(self, t: BatchTuning):
        check(lib().tpt_batch_set_tuning(self._h, ctypes.byref(t)))

    def fields(self, i: int) -> InstanceFields:
        f = InstanceFields()
        check(lib().tpt_batch_fields(self._h, i, ctypes.byref(f)))
        return f

    def state(self, i: int, stream=None) -> dict:
        import torch

        out = {
            "pv": self.read(i, FIELD_PV, np.float32, stream=stream), "vx": self.read(i, FIELD_VX, np.float32, stream=stream),
            "vy": self.read(i, FIELD_VY, np.float32, stream=stream), "hv": self.read(i, FIELD_HV, np.float32, stream=stream),
            "emap": self.read(i, FIELD_WALL_EMAP, np.uint32, stream=stream),
            "bair": self.read(i, FIELD_BLOCK_AIR, np.uint32, stream=stream),
            "bairh": self.read(i, FIELD_BLOCK_AIRH, np.uint32, stream=stream),
            "gx": self.read(i, FIELD_GX, np.float32, stream=stream), "gy": self.read(i, FIELD_GY, np.float32, stream=stream),
        }
        torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
        return out

    def close(self):
        if self._h:
            lib().tpt_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ save files --

class SaveData:
    """A `.tptrs` save (crates/tpt-save/src/lib.rs:67-97), decoded and encoded by
    the library on the host: `SaveData.from_bytes` / `to_bytes` mirror the
    reference's calls, `grid(name)` / `set_grid(name, array)` give the eight
    cell grids (names in SAVE_GRIDS), `particles()` the raw 64-byte records
    (numpy uint32, 16 words each), `instance_desc()` the field-step
    configuration restore_into gives the engine, `restore_grid(name)` the
    grid restore_into loads (zeros on a cell-count mismatch)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle

    @classmethod
    def from_bytes(cls, data: bytes) -> "SaveData":
        h = ctypes.c_void_p()
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        check(lib().tpt_save_decode(buf, len(data), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def new(cls, xres: int, yres: int) -> "SaveData":
        """An empty version-2 save of SimulationConfig::new(xres, yres)."""
        c = SaveConfig()
        lib().tpt_save_config_default(ctypes.byref(c), xres, yres)
        h = ctypes.c_void_p()
        check(lib().tpt_save_create(ctypes.byref(c), ctypes.byref(h)))
        return cls(h)

    def to_bytes(self) -> bytes:
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        check(lib().tpt_save_encode(self._h, ctypes.byref(p), ctypes.byref(n)))
        return ctypes.string_at(p, n.value)

    def info(self) -> SaveInfo:
        out = SaveInfo()
        check(lib().tpt_save_get_info(self._h, ctypes.byref(out)))
        return out

    @property
    def version(self) -> int:
        return int(self.info().version)

    @version.setter
    def version(self, v: int) -> None:
        check(lib().tpt_save_set_version(self._h, int(v)))

    @property
    def config(self) -> SaveConfig:
        c = SaveConfig()
        check(lib().tpt_save_get_config(self._h, ctypes.byref(c)))
        return c

    @config.setter
    def config(self, c: SaveConfig) -> None:
        check(lib().tpt_save_set_config(self._h, ctypes.byref(c)))

    def grid(self, name: str) -> np.ndarray:
        g = SAVE_GRIDS.index(name)
        out = np.empty(int(self.info().grid_len[g]), np.uint32 if name.startswith("wall") else np.float32)
        check(lib().tpt_save_grid_read(self._h, g, _ptr(out), out.nbytes))
        return out

    def set_grid(self, name: str, values) -> None:
        a = np.ascontiguousarray(values, np.uint32 if name.startswith("wall") else np.float32)
        check(lib().tpt_save_grid_write(self._h, SAVE_GRIDS.index(name), _ptr(a), a.nbytes))

    def restore_grid(self, name: str) -> np.ndarray:
        d = self.instance_desc()
        out = np.empty(d.air.xcells * d.air.ycells, np.uint32 if name.startswith("wall") else np.float32)
        check(lib().tpt_save_grid_restore(self._h, SAVE_GRIDS.index(name), _ptr(out), out.size))
        return out

    def particles(self) -> np.ndarray:
        n = int(self.info().n_particles)
        out = np.empty((n, 16), np.uint32)
        check(lib().tpt_save_particles_read(self._h, _ptr(out), out.nbytes))
        return out

    def set_particles(self, records) -> None:
        a = np.ascontiguousarray(records, np.uint32).reshape(-1, 16)
        check(lib().tpt_save_particles_write(self._h, _ptr(a), a.nbytes))

    def retain_air_pressure(self, include: bool) -> "SaveData":
        check(lib().tpt_save_retain_air_pressure(self._h, int(bool(include))))
        return self

    def instance_desc(self) -> InstanceDesc:
        d = InstanceDesc()
        check(lib().tpt_save_instance_desc(self._h, ctypes.byref(d)))
        return d

    def to_instance(self):
        """The field-step state SaveData::restore_into gives the engine
        (lib.rs:262-345), as a workloads.Instance for SimBuffers.from_instance
        or Batch: the restored configuration, the eight grids fitted to the
        canvas, the wall masks rebuilt from the walls (rebuild_spatial_maps)
        and the gravity mask flood-filled from them; no element stamps and no
        mass (particles are outside the field step)."""
        import workloads as W

        d = self.instance_desc()
        a = d.air
        cfg = W.AirConfig(air_mode=a.air_mode, aheat_enable=a.aheat_enable, convection_mode=a.convection_mode,
                          gravity_mode=a.gravity_mode, edge_pressure=a.edge_pressure, edge_vx=a.edge_vx,
                          edge_vy=a.edge_vy, ambient_air_temp=a.ambient_air_temp,
                          vorticity_coeff=a.vorticity_coeff, custom_gx=a.custom_gx, custom_gy=a.custom_gy,
                          newton_grav=d.newton_grav)
        g = {n: self.restore_grid(n) for n in SAVE_GRIDS}
        X, Y = int(a.xcells), int(a.ycells)
        bair, bairh = W.wall_masks(g["wall_bmap"], g["wall_emap"])
        zero = np.zeros(X * Y, np.uint32)
        return W.Instance(X, Y, cfg, pv=g["air_pv"], vx=g["air_vx"], vy=g["air_vy"], hv=g["air_hv"],
                          wall=g["wall_bmap"], emap=g["wall_emap"], bair=bair, bairh=bairh, eair=zero,
                          eairh=zero.copy(), fan_vx=g["fan_vx"], fan_vy=g["fan_vy"],
                          mass_fx=np.zeros(X * Y, np.int32), gmask=W.grav_mask(g["wall_bmap"], X, Y))

    def set_field_state(self, state: dict) -> None:
        """Writes air state back into the save's grids: `state` maps pv, vx,
        vy, hv (and optionally wall, emap) to dense cell arrays, as
        SimBuffers.air_state() or Batch.state() return them."""
        names = {"pv": "air_pv", "vx": "air_vx", "vy": "air_vy", "hv": "air_hv", "wall": "wall_bmap",
                 "emap": "wall_emap", "fan_vx": "fan_vx", "fan_vy": "fan_vy"}
        for k, v in state.items():
            if k in names:
                self.set_grid(names[k], v)

    def close(self) -> None:
        if self._h:
            lib().tpt_save_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VoxSave:
    """A `.tpt3` 3-D save (crates/tpt-save/src/voxel3d.rs:63-90), decoded and
    encoded by the library on the host. `array(name)` / `set_array(name, a)`
    for the names in VOX_SAVE_ARRAYS (voxels and ctype as uint32, the tmp
    arrays as int32, air as float32); `restore_air()` the AirState fields
    Voxel3dEngine::load_world restores; `to_world()` a world dict (the keys
    of workloads.voxel_world) for voxel3d.upload."""

    _DT = {"voxels": np.uint32, "aux_ctype": np.uint32, "aux_tmp": np.int32, "aux_tmp2": np.int32,
           "aux_tmp3": np.int32, "air": np.float32}

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle

    @classmethod
    def from_bytes(cls, data: bytes) -> "VoxSave":
        h = ctypes.c_void_p()
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        check(lib().tpt_vox_save_decode(buf, len(data), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def new(cls, config: VoxSaveConfig | None = None) -> "VoxSave":
        """Voxel3dSaveData::empty of `config` (Voxel3dConfig::default if None)."""
        if config is None:
            config = VoxSaveConfig()
            lib().tpt_vox_save_config_default(ctypes.byref(config))
        h = ctypes.c_void_p()
        check(lib().tpt_vox_save_create(ctypes.byref(config), ctypes.byref(h)))
        return cls(h)

    def to_bytes(self) -> bytes:
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        check(lib().tpt_vox_save_encode(self._h, ctypes.byref(p), ctypes.byref(n)))
        return ctypes.string_at(p, n.value)

    def info(self) -> VoxSaveInfo:
        out = VoxSaveInfo()
        check(lib().tpt_vox_save_get_info(self._h, ctypes.byref(out)))
        return out

    @property
    def config(self) -> VoxSaveConfig:
        c = VoxSaveConfig()
        check(lib().tpt_vox_save_get_config(self._h, ctypes.byref(c)))
        return c

    @config.setter
    def config(self, c: VoxSaveConfig) -> None:
        check(lib().tpt_vox_save_set_config(self._h, ctypes.byref(c)))

    def array(self, name: str) -> np.ndarray:
        a = VOX_SAVE_ARRAYS.index(name)
        out = np.empty(int(self.info().len[a]), self._DT[name])
        check(lib().tpt_vox_save_array_read(self._h, a, _ptr(out), out.nbytes))
        return out

    def set_array(self, name: str, values) -> None:
        a = np.ascontiguousarray(values, self._DT[name])
        check(lib().tpt_vox_save_array_write(self._h, VOX_SAVE_ARRAYS.index(name), _ptr(a), a.nbytes))

    def restore_air(self) -> dict:
        n = 64 ** 3
        out = {k: np.empty(n, np.float32) for k in ("vx", "vy", "vz", "temp", "solid")}
        out["pv"] = np.empty(n, np.int32)
        check(lib().tpt_vox_save_restore_air(self._h, *[_ptr(out[k]) for k in ("vx", "vy", "vz", "pv", "temp",
                                                                              "solid")]))
        return out

    def to_world(self) -> dict:
        """The field-step state of the loaded world: the voxels, aux_tmp (zeros
        when absent), the restored air, a zero Jacobi pair and zero gravity
        fields (load_world resets them), and as the brick list every brick
        holding a non-empty voxel, in id order."""
        n = 64 ** 3
        vox = self.array("voxels")
        tmp = self.array("aux_tmp")
        if tmp.size == 0:
            tmp = np.zeros(vox.size, np.int32)
        occupied = ((vox & 0xFF) != 0).reshape(32, 8, 32, 8, 32, 8).any(axis=(1, 3, 5)).reshape(-1)
        bricks = np.flatnonzero(occupied).astype(np.uint32)
        w = {"voxel": vox, "aux_tmp": tmp, "sim_list": bricks,
             "sim_count": np.array([bricks.size, 1, 1], np.uint32),
             "p": np.zeros(n, np.float32), "p_tmp": np.zeros(n, np.float32), "grav_mass": np.zeros(n, np.int32)}
        w.update(self.restore_air())
        for k in ("grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y", "grav_force_z"):
            w[k] = np.zeros(n, np.float32)
        return w

    def close(self) -> None:
        if self._h:
            lib().tpt_vox_save_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
