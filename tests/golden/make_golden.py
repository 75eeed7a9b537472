"""Generates the golden fixtures under tests/golden/ (run from the repo root:
`python tests/golden/make_golden.py`).

Two kinds of vectors:

1. Known answers taken from the reference's own unit tests (paths relative
   to the reference project), written here as data:
     fft_kat.npz     crates/tpt-sim/src/gravity_gpu/fft.rs:357-415 (8x8 naive
                     DFT pattern; 4x8 forward+inverse round trip)
     walls_kat.npz   crates/tpt-core/src/walls.rs:378-392 (air/heat blocking)
     tools_kat.npz   crates/tpt-sim/src/engine_commands/mod.rs:140-160
                     (tool mass sign, pixel -> cell on 612x384)
     align_kat.npz   crates/tpt-core/src/particle.rs:776-780 (4-px alignment)
   The expected DFT is numpy's float64 FFT of the same pattern (the
   reference compares its mirror with a naive DFT at tolerance 1e-3).

2. Oracle regression vectors (the reference cannot run here: no Rust
   toolchain, no wgpu): small seeded inputs and the CPU oracle's FP32/FP64
   outputs, so any later change of the oracle shows up as a diff:
     air_stress_24x24.npz, air_c1_crop.npz, grav_24x24.npz, grav_64x48.npz
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "the-powder-toy-rust-wgpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
OUT = os.path.dirname(os.path.abspath(__file__))


def fft_kat():
    w = h = 8
    re = np.array([[((x * 7 + y * 3) % 11) - 5.0 for x in range(w)] for y in range(h)], np.float32)
    im = np.array([[((x * 5 + y * 9) % 7) - 3.0 for x in range(w)] for y in range(h)], np.float32)
    want = np.fft.fft2(re.astype(np.float64) + 1j * im.astype(np.float64))
    rt_in = np.array([(i * 0.25) - 1.0 for i in range(4 * 8)], np.float32)
    np.savez(os.path.join(OUT, "fft_kat.npz"), re8=re.reshape(-1), im8=im.reshape(-1),
             want_re8=want.real.reshape(-1), want_im8=want.imag.reshape(-1), rt_in=rt_in, rt_w=4, rt_h=8)


def walls_kat():
    # (wall id, emap, blocks air, blocks heat) from walls.rs:378-392
    rows = [(8, 0, 1, 1), (1, 0, 1, -1), (16, 0, 1, -1), (9, 0, 0, 0), (14, 0, 0, 1), (2, 0, 1, -1), (2, 8, 0, 0)]
    np.savez(os.path.join(OUT, "walls_kat.npz"), rows=np.array(rows, np.int64))


def tools_kat():
    # tool_gravity_mass(strength, attract) -> mass, engine_commands/mod.rs:142-147
    mass = [(1.0, 1, 5.0), (1.0, 0, -5.0), (0.5, 1, 2.5), (0.5, 0, -2.5)]
    # gravity_tool_cell(x, y, 612, 384, 153, 96) -> cell or -1, mod.rs:151-159
    cells = [(0, 0, 0), (3, 0, 0), (4, 0, 1), (7, 5, 153 + 1), (-1, 0, -1), (0, -1, -1), (612, 0, -1), (0, 384, -1)]
    np.savez(os.path.join(OUT, "tools_kat.npz"), mass=np.array(mass, np.float64), cells=np.array(cells, np.int64))


def align_kat():
    # SimulationConfig::new(xres, yres) -> (xres, yres, xcells, ycells), particle.rs:776-784
    rows = [(100, 101, 100, 104, 25, 26), (1, 7, 64, 64, 16, 16), (612, 384, 612, 384, 153, 96)]
    np.savez(os.path.join(OUT, "align_kat.npz"), rows=np.array(rows, np.int64))


def oracle_vectors():
    import oracle as O
    import workloads as W

    O.build()
    inst = W.make_stress_instance(24, 24, 0x5EED)
    s32 = O.air_steps(inst, 10)
    s64 = O.air_steps(inst, 10, dtype=np.float64)
    np.savez_compressed(
        os.path.join(OUT, "air_stress_24x24.npz"),
        **{f"in_{k}": getattr(inst, k) for k in ("pv", "vx", "vy", "hv", "wall", "emap", "bair", "bairh", "eair",
                                                  "eairh", "fan_vx", "fan_vy")},
        **{f"out32_{k}": v for k, v in s32.items()}, **{f"out64_{k}": v for k, v in s64.items()})
    c1 = W.config_instances(1)[0]
    s32 = O.air_steps(c1, 5)
    np.savez_compressed(os.path.join(OUT, "air_c1_5ticks.npz"), **{f"out32_{k}": s32[k] for k in ("pv", "vx", "vy", "hv")})
    for (X, Y) in ((24, 24), (64, 48)):
        g = W.make_stress_instance(X, Y, 0x6A7 + X)
        gx32, gy32 = O.grav_solve(X, Y, g.gmask, mass_fx=g.mass_fx)
        gx64, gy64 = O.grav_solve(X, Y, g.gmask, mass_fx=g.mass_fx, dtype=np.float64)
        dx, dy = O.grav_solve(X, Y, g.gmask, mass_fx=g.mass_fx, direct=True)
        np.savez_compressed(os.path.join(OUT, f"grav_{X}x{Y}.npz"), mass_fx=g.mass_fx, gmask=g.gmask, wall=g.wall,
                            gx32=gx32, gy32=gy32, gx64=gx64, gy64=gy64, dx=dx, dy=dy)


if __name__ == "__main__":
    fft_kat()
    walls_kat()
    tools_kat()
    align_kat()
    oracle_vectors()
    print("wrote", sorted(f for f in os.listdir(OUT) if f.endswith(".npz")))
