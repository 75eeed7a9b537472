"""The 3-D sandbox's coarse field step on B200: a mirror of the reference's
interface for this path, over the CUDA library (include/tpt_field.h).

Reference interface mirrored here (paths relative to the reference project):

  AirState           crates/tpt-sim/src/voxel3d/air.rs:52-80 (vx, vy, vz, p,
                     p_tmp, t, solid, pv; `iterations`), its clear on creation
                     (air.rs:93-123), gather (:126-148), solve (:162-222),
                     read_pv / write_pv (:226-255)
  gravity.solve      crates/tpt-sim/src/voxel3d/gravity.rs:228-260
  gravity.clear_mass gravity.rs:264-273
  gravity.gather     gravity.rs:276-289
  Voxel3dBuffers     crates/tpt-sim/src/voxel3d/buffers.rs:56-190 (the voxel,
                     brick-list and gravity buffers this path reads or writes)

The grids are torch CUDA tensors in the reference layout: 64^3 cells indexed
(y << 12) | (z << 6) | x, 256^3 voxels indexed (y << 16) | (z << 8) | x. Every
call goes to the CUDA library; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

import tpt_field as tf

CELLS = 64 ** 3
VOXELS = 256 ** 3
BRICKS = 32 ** 3
AIR_JACOBI_ITERATIONS = 12   # air_kernel.rs:47
GRAVITY_ITERATIONS = 24      # gravity.rs:49


class Plan:
    """How the Jacobi solves run: `tf.VOX_BATCHED` (one launch per sweep
    index for every world of a call, air and gravity together; what
    `tf.VOX_AUTO` picks), `tf.VOX_CLUSTER` (one 16-CTA cluster per field, the
    grid in distributed shared memory) or `tf.VOX_PER_SWEEP` (the
    reference's launch structure: one launch per pass, sweep and world)."""

    def __init__(self, form: int = tf.VOX_AUTO):
        h = ctypes.c_void_p()
        tf.check(tf.lib().tpt_vox_plan_create(int(form), ctypes.byref(h)))
        self._h = h

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def form(self) -> int:
        rc = tf.lib().tpt_vox_plan_form(self._h)
        if rc < 0:
            tf.check(rc)
        return rc

    def close(self) -> None:
        if self._h:
            tf.lib().tpt_vox_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Voxel3dBuffers:
    """The voxel state and gravity fields of one world (torch CUDA tensors):
    voxel_a (u32 bit patterns in int32), aux_tmp, sim_list, sim_count
    ([n, 1, 1]), grav_mass (1/1024 fixed point), grav_potential,
    grav_potential_tmp, grav_force_x/y/z. New buffers are zero."""

    def __init__(self, device="cuda"):
        import torch

        z = dict(device=device)
        self.voxel_a = torch.zeros(VOXELS, dtype=torch.int32, **z)
        self.aux_tmp = torch.zeros(VOXELS, dtype=torch.int32, **z)
        self.sim_list = torch.zeros(BRICKS, dtype=torch.int32, **z)
        self.sim_count = torch.tensor([0, 1, 1], dtype=torch.int32, **z)
        self.grav_mass = torch.zeros(CELLS, dtype=torch.int32, **z)
        for k in ("grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y", "grav_force_z"):
            setattr(self, k, torch.zeros(CELLS, dtype=torch.float32, **z))


class AirState:
    """Device-resident 64^3 air field (air.rs:52-80); a new state is cleared
    on the device to the neutral field (zero velocity, pressure, solid and
    pv; 293.15 K)."""

    def __init__(self, device="cuda", stream=None):
        import torch

        for k in ("vx", "vy", "vz", "p", "p_tmp", "t", "solid"):
            setattr(self, k, torch.empty(CELLS, dtype=torch.float32, device=device))
        self.pv = torch.empty(CELLS, dtype=torch.int32, device=device)
        self.iterations = AIR_JACOBI_ITERATIONS
        tf.check(tf.lib().tpt_vox_air_clear(ctypes.byref(world(None, self)), tf._stream(stream)))

    def gather(self, plan: Plan, bufs: Voxel3dBuffers, stream=None) -> None:
        """Solid fraction and mean temperature of every listed brick's cells."""
        tf.check(tf.lib().tpt_vox_air_gather(plan.handle, ctypes.byref(world(bufs, self)), tf._stream(stream)))

    def solve(self, plan: Plan, stream=None) -> None:
        """pv update, `iterations` Jacobi pressure sweeps, advection."""
        tf.check(tf.lib().tpt_vox_air_solve(plan.handle, ctypes.byref(world(None, self)), int(self.iterations),
                                            tf._stream(stream)))

    def read_pv(self) -> np.ndarray:
        return self.pv.cpu().numpy()

    def write_pv(self, values) -> None:
        import torch

        self.pv.copy_(torch.as_tensor(np.asarray(values, np.int32)))


def world(bufs: Voxel3dBuffers | None, air: AirState | None) -> tf.VoxWorld:
    """The tpt_vox_world of a buffer set and an air state (either may be None)."""
    w = tf.VoxWorld()
    if bufs is not None:
        w.voxel = bufs.voxel_a.data_ptr()
        w.aux_tmp = bufs.aux_tmp.data_ptr()
        w.sim_list = bufs.sim_list.data_ptr()
        w.sim_count = bufs.sim_count.data_ptr()
        for k in ("grav_mass", "grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y",
                  "grav_force_z"):
            setattr(w, k, getattr(bufs, k).data_ptr())
    if air is not None:
        for k in ("vx", "vy", "vz", "p", "p_tmp", "solid", "pv"):
            setattr(w, k, getattr(air, k).data_ptr())
        w.temp = air.t.data_ptr()
    return w


def gravity_solve(plan: Plan, bufs: Voxel3dBuffers, stream=None) -> None:
    """24 Jacobi sweeps of the potential from grav_mass, then the force."""
    tf.check(tf.lib().tpt_vox_grav_solve(plan.handle, ctypes.byref(world(bufs, None)), tf._stream(stream)))


def gravity_clear_mass(plan: Plan, bufs: Voxel3dBuffers, stream=None) -> None:
    tf.check(tf.lib().tpt_vox_grav_clear_mass(plan.handle, ctypes.byref(world(bufs, None)), tf._stream(stream)))


def gravity_gather(plan: Plan, bufs: Voxel3dBuffers, stream=None) -> None:
    """Adds the fixed-point mass of every listed brick's gravity elements."""
    tf.check(tf.lib().tpt_vox_grav_gather(plan.handle, ctypes.byref(world(bufs, None)), tf._stream(stream)))


def field_step(plan: Plan, worlds, air_iterations: int = AIR_JACOBI_ITERATIONS, stream=None) -> None:
    """Air gather, air solve, gravity solve and clear mass for every
    (Voxel3dBuffers, AirState) pair of `worlds`; in the cluster form the
    solves of all worlds are one launch."""
    arr = (tf.VoxWorld * len(worlds))(*[world(b, a) for b, a in worlds])
    tf.check(tf.lib().tpt_vox_field_step(plan.handle, arr, len(worlds), int(air_iterations), tf._stream(stream)))


def upload(d: dict, device="cuda") -> tuple[Voxel3dBuffers, AirState]:
    """Device buffers holding a host world (the dict of workloads.voxel_world)."""
    import torch

    bufs = Voxel3dBuffers.__new__(Voxel3dBuffers)
    air = AirState.__new__(AirState)
    air.iterations = AIR_JACOBI_ITERATIONS

    def dev(a):
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        return torch.from_numpy(a.copy()).to(device)

    bufs.voxel_a = dev(d["voxel"])
    bufs.aux_tmp = dev(d["aux_tmp"])
    lst = np.zeros(BRICKS, np.uint32)
    lst[: len(d["sim_list"])] = d["sim_list"]
    bufs.sim_list = dev(lst)
    bufs.sim_count = dev(d["sim_count"])
    for k in ("grav_mass", "grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y", "grav_force_z"):
        setattr(bufs, k, dev(d[k]))
    for k in ("vx", "vy", "vz", "p", "p_tmp", "solid", "pv"):
        setattr(air, k, dev(d[k]))
    air.t = dev(d["temp"])
    return bufs, air


def download(bufs: Voxel3dBuffers, air: AirState) -> dict:
    """Host copies of every field, keyed like workloads.voxel_world."""
    out = {k: getattr(air, k).cpu().numpy() for k in ("vx", "vy", "vz", "p", "p_tmp", "solid", "pv")}
    out["temp"] = air.t.cpu().numpy()
    for k in ("grav_mass", "grav_potential", "grav_potential_tmp", "grav_force_x", "grav_force_y", "grav_force_z"):
        out[k] = getattr(bufs, k).cpu().numpy()
    return out
