"""Second, independent restatement of the 2-D air tick in vectorised numpy.
TEST INFRASTRUCTURE ONLY: the parity tests use it to check the C++ oracle
(tpt_oracle.cpp); the product never imports it.

Written from the reference's kernel source, not from the C++ oracle, so a
misreading in one restatement shows up as a bit difference against the other:

  pressure / velocity   crates/tpt-sim/src/air_kernel/pressure.rs:9-299
  smooth / advect       crates/tpt-sim/src/air_kernel/advect.rs:10-360
  heat / convection     crates/tpt-sim/src/air_kernel/heat.rs:29-253
  copy-back / masks     crates/tpt-sim/src/air_kernel/settle.rs:21-93
  pass order            crates/tpt-sim/src/air_kernel/mod.rs:120-263

Every operation is an f32 numpy operation on whole grids (numpy rounds each
elementwise operation to f32 and never fuses a multiply into an add), in the
order the Rust expressions evaluate: left to right, `a + b * c` as
`a + (b * c)`. Branches become `np.where` selections; the far-advection step
walk runs all walking cells in lock step. The one deliberate departure from
the reference is shared with the C++ oracle and the CUDA kernels: the heat
pass reads every neighbour's vx/vy as the smoothing pass left them
(read-before-write), where the reference races with its own in-place writes
(heat.rs:92-94 against heat.rs:249-250).

f32 -> i32 conversions (`as i32` in the kernels, WGSL `i32(f32)`) round
toward zero and saturate to the i32 range; NaN converts to 0, as CUDA's
cvt.rzi does (WGSL leaves the NaN case to the implementation).
"""
from __future__ import annotations

import numpy as np

F = np.float32
U = np.uint32

# advect.rs:215-225: w(0,0) = 1, w(+-1,0) = e^-2, w(+-1,+-1) = e^-4, indexed [dy][dx]
# with 0 = -1, 1 = 0, 2 = +1.
_W_CORNER, _W_EDGE, _W_CENTRE = F(0.01831564), F(0.13533528), F(1.0)


def _tap_weight(dx: int, dy: int) -> np.float32:
    w = _W_CORNER
    if dx == 1:
        w = _W_EDGE
    if dy == 1:
        w = _W_EDGE
    if dx == 1 and dy == 1:
        w = _W_CENTRE
    return w


def _wsum() -> np.float32:
    s = F(0.0)
    for dy in range(3):
        for dx in range(3):
            s = F(s + _tap_weight(dx, dy))
    return s


WSUM = _wsum()


def f2i(v: np.ndarray) -> np.ndarray:
    """f32 -> i32: truncate toward zero, saturate, NaN -> 0."""
    v = np.asarray(v, np.float32)
    out = np.zeros(v.shape, np.int64)
    ok = ~np.isnan(v)
    t = np.trunc(v[ok].astype(np.float64))
    out[ok] = np.clip(t, -2147483648.0, 2147483647.0).astype(np.int64)
    return out


def _shift(a: np.ndarray, dx: int, dy: int, fill) -> np.ndarray:
    """b[y, x] = a[y + dy, x + dx] inside the grid, `fill` outside."""
    Y, X = a.shape
    b = np.full_like(a, fill)
    ys0, ys1 = max(0, -dy), min(Y, Y - dy)
    xs0, xs1 = max(0, -dx), min(X, X - dx)
    if ys0 < ys1 and xs0 < xs1:
        b[ys0:ys1, xs0:xs1] = a[ys0 + dy:ys1 + dy, xs0 + dx:xs1 + dx]
    return b


def _clampf(v, lo, hi):
    # mod.rs:92-102: compare and assign (NaN passes through)
    out = np.where(v < F(lo), F(lo), v)
    return np.where(out > F(hi), F(hi), out).astype(np.float32)


def _absf(v):
    # `if v < 0 { v = 0 - v }` keeps -0.0 as -0.0 (np.abs would not)
    return np.where(v < F(0.0), F(0.0) - v, v).astype(np.float32)


class Grid:
    def __init__(self, X: int, Y: int):
        self.X, self.Y = X, Y
        self.xs = np.broadcast_to(np.arange(X, dtype=np.int64)[None, :], (Y, X))
        self.ys = np.broadcast_to(np.arange(Y, dtype=np.int64)[:, None], (Y, X))

    def in_border(self):  # pressure.rs:9-15 (BORDER = 2, mod.rs:75)
        x, y, X, Y = self.xs, self.ys, self.X, self.Y
        return (x < 2) | (y < 2) | (x + 2 >= X) | (y + 2 >= Y)

    def interior(self):  # pressure.rs:20-26
        x, y, X, Y = self.xs, self.ys, self.X, self.Y
        return (x >= 1) & (y >= 1) & (x + 1 < X) & (y + 1 < Y)


# ---------------------------------------------------------------- pressure.rs

def _effective(v, blk, g: Grid, edge, axis_x: bool):
    """effective_vx / effective_vy (pressure.rs:119-158) of every cell: border
    mix toward the edge velocity, then the three-cell wall clear
    (wall_cleared_vx/vy, pressure.rs:43-85)."""
    x, y, X, Y = g.xs, g.ys, g.X, g.Y
    out = np.where(g.in_border(), F(edge) + (v - F(edge)) * F(0.9), v).astype(np.float32)
    if axis_x:
        row_ok = (y >= 1) & (y + 1 < Y)
        here = (x >= 1) & (x + 1 < X) & blk
        left = (x >= 2) & _shift(blk, -1, 0, False)
        right = (x + 2 < X) & _shift(blk, 1, 0, False)
    else:
        row_ok = (x >= 1) & (x + 1 < X)
        here = (y >= 1) & (y + 1 < Y) & blk
        left = (y >= 2) & _shift(blk, 0, -1, False)
        right = (y + 2 < Y) & _shift(blk, 0, 1, False)
    cleared = row_ok & (here | left | right)
    return np.where(cleared, F(0.0), out).astype(np.float32)


def pressure(pv, vx, vy, blk, g: Grid, ep, evx, evy):
    """air_pressure_kernel (pressure.rs:173-238) -> opv."""
    ex = _effective(vx, blk, g, evx, True)
    ey = _effective(vy, blk, g, evy, False)
    cur = np.where(g.in_border(), F(ep) + (pv - F(ep)) * F(0.8), pv).astype(np.float32)
    # dp = evx(x-1) - evx(x+1) + evy(y-1) - evy(y+1), left to right
    dp = _shift(ex, -1, 0, F(0)) - _shift(ex, 1, 0, F(0))
    dp = dp + _shift(ey, 0, -1, F(0))
    dp = dp - _shift(ey, 0, 1, F(0))
    nxt = F(ep) + (cur - F(ep)) * F(0.9999)
    nxt = nxt + dp * F(0.15)
    return np.where(g.interior(), nxt, cur).astype(np.float32)


def velocity(opv, vx, vy, blk, g: Grid, evx, evy):
    """air_velocity_kernel (pressure.rs:247-299) -> ovx, ovy."""
    cx = _effective(vx, blk, g, evx, True)
    cy = _effective(vy, blk, g, evy, False)
    dx = _shift(opv, -1, 0, F(0)) - _shift(opv, 1, 0, F(0))
    dy = _shift(opv, 0, -1, F(0)) - _shift(opv, 0, 1, F(0))
    nx = F(evx) + (cx - F(evx)) * F(0.999)
    nx = nx + dx * F(0.2)
    ny = F(evy) + (cy - F(evy)) * F(0.999)
    ny = ny + dy * F(0.2)
    # adjacent_blocked_x/y (pressure.rs:92-114), blocked_at = 0 outside the grid
    adj_x = _shift(blk, -1, 0, False) | blk | _shift(blk, 1, 0, False)
    adj_y = _shift(blk, 0, -1, False) | blk | _shift(blk, 0, 1, False)
    nx = np.where(adj_x, F(0.0), nx)
    ny = np.where(adj_y, F(0.0), ny)
    inner = g.interior()
    return (np.where(inner, nx, cx).astype(np.float32), np.where(inner, ny, cy).astype(np.float32))


# ------------------------------------------------------------------ advect.rs

def vorticity_bmap(vx, vy, blk, g: Grid):
    """advect.rs:10-42 for every cell."""
    x, y, X, Y = g.xs, g.ys, g.X, g.Y
    win = (x > 1) & (x + 2 < X) & (y > 1) & (y + 2 < Y)
    dvydx = _shift(vy, 1, 0, F(0)) - _shift(vy, -1, 0, F(0))
    dvydx = np.where(blk | _shift(blk, 1, 0, False) | _shift(blk, -1, 0, False), F(0.0), dvydx)
    dvxdy = _shift(vx, 0, 1, F(0)) - _shift(vx, 0, -1, F(0))
    dvxdy = np.where(blk | _shift(blk, 0, 1, False) | _shift(blk, 0, -1, False), F(0.0), dvxdy)
    return np.where(win, (dvydx - dvxdy) * F(0.5), F(0.0)).astype(np.float32)


def smooth3(fields, open_mask, g: Grid):
    """The 3x3 normalised smoothing of advect.rs:192-253 / heat.rs:60-104:
    a neighbour counts when it is an interior cell and `open_mask` is set
    there; otherwise the tap repeats the centre value. Sums run dy-major,
    dx-minor; the result is divided by the sum of all nine weights."""
    X, Y = g.X, g.Y
    x, y = g.xs, g.ys
    sums = [np.zeros((Y, X), np.float32) for _ in fields]
    for dy in range(3):
        for dx in range(3):
            # nx = saturating_sub(x + dx, 1): taps below 0 land on column 0,
            # which is never interior, so they repeat the centre like any
            # non-interior tap.
            ox, oy = dx - 1, dy - 1
            nx, ny = x + ox, y + oy
            itap = (nx >= 1) & (ny >= 1) & (nx + 1 < X) & (ny + 1 < Y)
            use = itap & _shift(open_mask, ox, oy, False)
            w = _tap_weight(dx, dy)
            for k, f in enumerate(fields):
                t = np.where(use, _shift(f, ox, oy, F(0)), f)
                sums[k] = (sums[k] + t * w).astype(np.float32)
    return [(s / WSUM).astype(np.float32) for s in sums]


def far_advect_target(dx, dy, blocked, g: Grid):
    """advect.rs:66-152 for every cell; `blocked` is the mask the walk tests
    (block_air != 0, or block_airh & 0x8 for the heat pass)."""
    X, Y = g.X, g.Y
    xf = g.xs.astype(np.float32)
    yf = g.ys.astype(np.float32)
    ad = F(0.7)
    tx = (xf - dx * ad).astype(np.float32)
    ty = (yf - dy * ad).astype(np.float32)
    adx = _absf((dx * ad).astype(np.float32))
    ady = _absf((dy * ad).astype(np.float32))
    limx, limy = F(X) - F(2.0), F(Y) - F(2.0)
    walk = ((adx > F(1.0)) | (ady > F(1.0))) & (tx >= F(2.0)) & (tx < limx) & (ty >= F(2.0)) & (ty < limy)
    if not walk.any():
        return tx, ty
    wy_, wx_ = np.nonzero(walk)
    ddx, ddy = dx[walk], dy[walk]
    abs_dx = np.where(ddx < F(0), F(0) - ddx, ddx).astype(np.float32)
    abs_dy = np.where(ddy < F(0), F(0) - ddy, ddy).astype(np.float32)
    major_x = abs_dx > abs_dy
    with np.errstate(divide="ignore", invalid="ignore"):
        sx = np.where(major_x, np.where(ddx < F(0), F(1.0), F(-1.0)), F(0.0) - ddx / abs_dy).astype(np.float32)
        sy = np.where(major_x, F(0.0) - ddy / abs_dx, np.where(ddy < F(0), F(1.0), F(-1.0))).astype(np.float32)
    limit = np.where(major_x, f2i(adx[walk]), f2i(ady[walk]))
    cx_ = wx_.astype(np.float32)
    cy_ = wy_.astype(np.float32)
    stopped = np.zeros(len(wx_), bool)
    active = limit > 0
    step = 0
    while active.any():
        a = active
        cx_[a] = cx_[a] + sx[a]
        cy_[a] = cy_[a] + sy[a]
        ix = f2i(cx_[a] + F(0.5))
        iy = f2i(cy_[a] + F(0.5))
        inside = (ix >= 0) & (iy >= 0) & (ix < X) & (iy < Y)
        hit = np.ones(len(ix), bool)
        hit[inside] = blocked[iy[inside], ix[inside]]
        idx = np.flatnonzero(a)
        h = idx[hit]
        cx_[h] = cx_[h] - sx[h]
        cy_[h] = cy_[h] - sy[h]
        stopped[h] = True
        active[h] = False
        step += 1
        active &= step < limit
    otx, oty = tx.copy(), ty.copy()
    # walked to the end without a wall: the full backtrace (already in tx/ty)
    sel = stopped
    otx[wy_[sel], wx_[sel]] = cx_[sel]
    oty[wy_[sel], wx_[sel]] = cy_[sel]
    return otx, oty


def smooth_advect(ovx, ovy, opv, blk, wall, fan_vx, fan_vy, g: Grid, vcoef, air_mode):
    """air_smooth_advect_kernel (advect.rs:174-360) -> vx, vy, pv."""
    X, Y = g.X, g.Y
    x, y = g.xs, g.ys
    nvx, nvy, npv = smooth3([ovx, ovy, opv], ~blk, g)
    tx0, ty0 = far_advect_target(nvx, nvy, blk, g)
    i0, j0 = f2i(tx0), f2i(ty0)
    fx = (tx0 - i0.astype(np.float32)).astype(np.float32)
    fy = (ty0 - j0.astype(np.float32)).astype(np.float32)
    ok = (~blk) & (i0 >= 2) & (i0 < X - 3) & (j0 >= 2) & (j0 < Y - 3) & (fx >= F(0)) & (fy >= F(0))
    ii, jj = np.clip(i0, 0, X - 2), np.clip(j0, 0, Y - 2)
    w00 = (F(1.0) - fx) * (F(1.0) - fy)
    w10 = fx * (F(1.0) - fy)
    w01 = (F(1.0) - fx) * fy
    w11 = fx * fy

    def bil(a):
        s = a[jj, ii] * w00 + a[jj, ii + 1] * w10
        s = s + a[jj + 1, ii] * w01
        return s + a[jj + 1, ii + 1] * w11

    nvx = np.where(ok, nvx * F(0.7) + F(0.3) * bil(ovx), nvx).astype(np.float32)
    nvy = np.where(ok, nvy * F(0.7) + F(0.3) * bil(ovy), nvy).astype(np.float32)
    if F(vcoef) > F(0.0):  # advect.rs:297-328
        win = (x > 1) & (x + 2 < X) & (y > 1) & (y + 2 < Y)
        vort = vorticity_bmap(ovx, ovy, blk, g)
        w = vort
        wxp = _absf(_shift(vort, 1, 0, F(0)))
        wxm = _absf(_shift(vort, -1, 0, F(0)))
        wyp = _absf(_shift(vort, 0, 1, F(0)))
        wym = _absf(_shift(vort, 0, -1, F(0)))
        dwx = (wxp - wxm) * F(0.5)
        dwy = (wyp - wym) * F(0.5)
        norm = np.sqrt(dwx * dwx + dwy * dwy).astype(np.float32)
        k = F(F(vcoef) / F(5.0))
        den = norm + F(0.001)
        ax = (k * dwy) / den * w
        ay = (k * (F(0.0) - dwx)) / den * w
        nvx = np.where(win, nvx + ax, nvx).astype(np.float32)
        nvy = np.where(win, nvy + ay, nvy).astype(np.float32)
    fan = wall == U(5)  # WL_FAN
    nvx = np.where(fan, nvx + fan_vx, nvx).astype(np.float32)
    nvy = np.where(fan, nvy + fan_vy, nvy).astype(np.float32)
    nvx = _clampf(nvx, -256.0, 256.0)
    nvy = _clampf(nvy, -256.0, 256.0)
    npv = _clampf(npv, -256.0, 256.0)
    if air_mode == 1:
        npv = np.zeros_like(npv)
    if air_mode == 2:
        nvx, nvy = np.zeros_like(nvx), np.zeros_like(nvy)
    if air_mode == 3:
        nvx, nvy, npv = np.zeros_like(nvx), np.zeros_like(nvy), np.zeros_like(npv)
    return nvx, nvy, npv


# -------------------------------------------------------------------- heat.rs

def heat_convect(hv, vx, vy, bairh, g: Grid, amb, aheat, conv, gmode, cgx, cgy):
    """air_heat_convect_kernel (heat.rs:29-253) with read-before-write
    neighbours -> (ohv, vx, vy)."""
    X, Y = g.X, g.Y
    x, y = g.xs, g.ys
    hblk = (bairh & U(0x8)) != U(0)
    dh, svx, svy = smooth3([hv, vx, vy], ~hblk, g)
    tx, ty = far_advect_target(svx, svy, hblk, g)
    i0, j0 = f2i(tx), f2i(ty)
    fx = (tx - i0.astype(np.float32)).astype(np.float32)
    fy = (ty - j0.astype(np.float32)).astype(np.float32)
    ok = (~hblk) & (i0 >= 0) & (i0 < X - 1) & (j0 >= 0) & (j0 < Y - 1) & (fx >= F(0)) & (fy >= F(0))
    ii, jj = np.clip(i0, 0, X - 2), np.clip(j0, 0, Y - 2)

    def samp(a, b):
        return np.where(hblk[b, a], dh, hv[b, a])

    s00, s10, s01, s11 = samp(ii, jj), samp(ii + 1, jj), samp(ii, jj + 1), samp(ii + 1, jj + 1)
    w00 = (F(1.0) - fx) * (F(1.0) - fy)
    w10 = fx * (F(1.0) - fy)
    w01 = (F(1.0) - fx) * fy
    w11 = fx * fy
    s = s00 * w00 + s10 * w10
    s = s + s01 * w01
    s = s + s11 * w11
    dh = np.where(ok, dh * F(0.7) + F(0.3) * s, dh).astype(np.float32)
    dh = np.where(hblk, hv, dh)
    dh = _clampf(dh, 0.0, 9999.0)
    border = (x < 2) | (y < 2) | (x + 2 >= X) | (y + 2 >= Y)
    dh = np.where(border, F(amb), dh)
    if aheat == 0:
        dh = np.full_like(dh, F(amb))
    # convection (heat.rs:182-251)
    inner = (x >= 2) & (x + 2 < X) & (y >= 2) & (y + 2 < Y)
    gx = np.zeros((Y, X), np.float32)
    gy = np.zeros((Y, X), np.float32)
    if gmode == 0:
        gy[:] = F(1.0)
    elif gmode == 2:
        rx = (F(X) * F(0.5) - (x.astype(np.float32) + F(0.5))).astype(np.float32)
        ry = (F(Y) * F(0.5) - (y.astype(np.float32) + F(0.5))).astype(np.float32)
        rd = np.sqrt(rx * rx + ry * ry).astype(np.float32)
        pos = rd > F(0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            gx = np.where(pos, rx / rd, F(0.0)).astype(np.float32)
            gy = np.where(pos, ry / rd, F(0.0)).astype(np.float32)
    elif gmode == 3:
        gx[:] = F(cgx)
        gy[:] = F(cgy)
    cvx = (F(0.0) - gx).astype(np.float32)
    cvy = (F(0.0) - gy).astype(np.float32)
    nx, ny = vx.copy(), vy.copy()
    if conv == 1:
        wgt = (hv - _shift(hv, -1, 0, F(0))) * cvx + (hv - _shift(hv, 0, -1, F(0))) * cvy
        wgt = (wgt / F(5000.0)).astype(np.float32)
        up_open = ~_shift(hblk, 0, -1, False)
        push = (wgt > F(0.0)) & up_open
        nx = np.where(push, nx + wgt * cvx, nx).astype(np.float32)
        ny = np.where(push, ny + wgt * cvy, ny).astype(np.float32)
    elif conv == 2:
        gm = np.sqrt(cvx * cvx + cvy * cvy).astype(np.float32)
        big = gm > F(10.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            cvx = np.where(big, cvx / (F(0.1) * gm), cvx).astype(np.float32)
            cvy = np.where(big, cvy / (F(0.1) * gm), cvy).astype(np.float32)
        wgt = ((hv - F(amb)) / F(10000.0)).astype(np.float32)
        wgt = np.where(wgt > F(0.01), F(0.01), wgt).astype(np.float32)
        nx = (nx + wgt * cvx).astype(np.float32)
        ny = (ny + wgt * cvy).astype(np.float32)
    nx = _clampf(nx, -256.0, 256.0)
    ny = _clampf(ny, -256.0, 256.0)
    return dh, np.where(inner, nx, vx).astype(np.float32), np.where(inner, ny, vy).astype(np.float32)


# ------------------------------------------------------------------ settle.rs

def block_masks(wall, emap, eair, eairh):
    """air_block_masks_kernel (settle.rs:50-93) -> (emap, bair, bairh)."""
    w = wall & U(0xFF)
    emap = np.where(emap != U(0), emap - U(1), emap).astype(np.uint32)
    e = emap & U(0xFF)
    blocked = (w == U(8)) | (w == U(1)) | (w == U(16)) | ((w == U(2)) & (e == U(0)))
    bair = blocked.astype(np.uint32) | eair
    bairh = np.where(blocked | (w == U(14)), U(0x8), U(0)).astype(np.uint32) | eairh
    return emap, bair.astype(np.uint32), bairh.astype(np.uint32)


# ---------------------------------------------------------------- one tick

def air_tick(st: dict, X: int, Y: int, cfg) -> dict:
    """One step_air_gpu (mod.rs:120-263) without HotAir. `st` holds the
    grids (pv, vx, vy, hv f32; wall, emap, bair, bairh, eair, eairh u32;
    fan_vx, fan_vy f32) as (Y, X) arrays; returns the new state."""
    g = Grid(X, Y)
    s = {k: v.copy() for k, v in st.items()}
    blk = s["bair"] != U(0)
    if cfg.air_mode != 4:
        opv = pressure(s["pv"], s["vx"], s["vy"], blk, g, cfg.edge_pressure, cfg.edge_vx, cfg.edge_vy)
        ovx, ovy = velocity(opv, s["vx"], s["vy"], blk, g, cfg.edge_vx, cfg.edge_vy)
        s["vx"], s["vy"], s["pv"] = smooth_advect(ovx, ovy, opv, blk, s["wall"], s["fan_vx"], s["fan_vy"], g,
                                                  cfg.vorticity_coeff, cfg.air_mode)
    if cfg.aheat_enable:
        s["hv"], s["vx"], s["vy"] = heat_convect(s["hv"], s["vx"], s["vy"], s["bairh"], g, cfg.ambient_air_temp,
                                                 cfg.aheat_enable, cfg.convection_mode, cfg.gravity_mode,
                                                 cfg.custom_gx, cfg.custom_gy)
    s["emap"], s["bair"], s["bairh"] = block_masks(s["wall"], s["emap"], s["eair"], s["eairh"])
    return s


def air_steps(inst, ticks: int) -> dict:
    """`ticks` air steps of a workloads.Instance; returns flat grids like the
    C++ oracle's air_steps."""
    X, Y = inst.xcells, inst.ycells
    st = {k: np.asarray(getattr(inst, k), np.float32).reshape(Y, X).copy()
          for k in ("pv", "vx", "vy", "hv", "fan_vx", "fan_vy")}
    for k in ("wall", "emap", "bair", "bairh", "eair", "eairh"):
        st[k] = np.asarray(getattr(inst, k), np.uint32).reshape(Y, X).copy()
    with np.errstate(all="ignore"):  # NaN / Inf inputs propagate as IEEE says
        for _ in range(ticks):
            st = air_tick(st, X, Y, inst.config)
    return {k: v.reshape(-1) for k, v in st.items()}
