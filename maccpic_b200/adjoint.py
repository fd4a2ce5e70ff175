"""Gradients of the reconnected flux through em2's time step.

em2 has no adjoint; this module adds one.  It differentiates

    flux(T) = max(psi) - min(psi) along the centre row of the sheet at ny/4,
    psi = -integral of By dx,   after T steps of em2's step,

with respect to the parameters of the initial double-Harris state: the flux
perturbation amplitude psi0 (in B0 d_i), the guide field B_g (in B0) and the
sheet half-thickness L (in d_i).

Two implementations of the same FP64 step live here:

* :func:`step` -- a plain-PyTorch restatement of em2's move / curnt /
  fields (pic/move.f90, pic/curnt.f90, pic/fields.f90) on periodic (ny, nx)
  arrays.  For a periodic state (the loader's fields are) the guard cells of
  em2's (0:nx+2, 0:ny+2) arrays are exact periodic images, so this is the
  same step; it differs from em2 only in solving the Poisson correction
  exactly (FFT of the periodic 5-point Laplacian) where em2's CG stops at
  mean r^2 < 1e-9.  Run under autograd it is the reference tape.
* :class:`Em2Step` -- a torch.autograd.Function whose backward is written
  out by hand: the Poisson projection is self-adjoint; smooth2 is a
  symmetric periodic stencil and is its own transpose; the Yee half-steps
  transpose into the negated transposed curls; the deposit's transpose is a
  gather of the current adjoint at the particles (plus the derivative of the
  quadratic weights); the gather's transpose is a scatter of the force
  adjoint onto the grid; the Boris rotation is reversed stage by stage.
  :func:`flux_and_gradient` chains it over T steps with checkpoints every K
  steps and recomputation between them.

Particles carry (x, y, ux, uy, uz) with u = gamma v, x, y in cells.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace

import torch

TWO_PI = 2.0 * math.pi


@dataclass
class StepConst:
    nx: int
    ny: int
    dx: float
    dt: float
    c: float
    isav: int
    qm: tuple      # per species q/m
    qd: tuple      # per species q*dn/(dx*dy)


# ---------------------------------------------------------------------------
# quadratic weights (pic/move.f90:76-148), periodic node indices
# ---------------------------------------------------------------------------
def w_half(x):
    """Cell-centred nodes (Ex/Bx along x): em2 index int(x+1); returns the
    periodic index of the middle node, the three weights and d/dx of them."""
    ix = torch.floor(x + 1.0)
    s = 0.75 - (x + 0.5 - ix) ** 2
    sp = 0.5 * (1.0 + x - ix) ** 2
    sm = 0.5 * (ix - x) ** 2
    ds = -2.0 * (x + 0.5 - ix)
    dsp = 1.0 + x - ix
    dsm = -(ix - x)
    return (ix - 1).long(), (sm, s, sp), (dsm, ds, dsp)


def w_node(x):
    """Integer nodes (rho along x and y): em2 index int(x+1.5)."""
    ix = torch.floor(x + 1.5)
    s = 0.75 - (x + 1.0 - ix) ** 2
    sp = 0.5 * (1.5 + x - ix) ** 2
    sm = 0.5 * (-0.5 - x + ix) ** 2
    ds = -2.0 * (x + 1.0 - ix)
    dsp = 1.5 + x - ix
    dsm = -(-0.5 - x + ix)
    return (ix - 1).long(), (sm, s, sp), (dsm, ds, dsp)


def _stencil_index(ic, jc, nx, ny):
    """9 flat indices (b rows, a cols) around (ic, jc), periodic."""
    out = []
    for b in (-1, 0, 1):
        j = torch.remainder(jc + b, ny)
        for a in (-1, 0, 1):
            i = torch.remainder(ic + a, nx)
            out.append(j * nx + i)
    return out


def gather(F, wx, wy, nx, ny):
    """sum_ab wx[a] wy[b] F[jc+b, ic+a]; F (ny, nx); wx, wy from w_half/w_node."""
    ic, sx, _ = wx
    jc, sy, _ = wy
    flat = F.reshape(-1)
    idx = _stencil_index(ic, jc, nx, ny)
    out = 0.0
    k = 0
    for b in range(3):
        for a in range(3):
            out = out + sx[a] * sy[b] * flat[idx[k]]
            k += 1
    return out


def gather_grad(F, wx, wy, nx, ny):
    """(d/dx, d/dy) of gather(F, ...) through the weights."""
    ic, sx, dsx = wx
    jc, sy, dsy = wy
    flat = F.reshape(-1)
    idx = _stencil_index(ic, jc, nx, ny)
    gx = 0.0
    gy = 0.0
    k = 0
    for b in range(3):
        for a in range(3):
            v = flat[idx[k]]
            gx = gx + dsx[a] * sy[b] * v
            gy = gy + sx[a] * dsy[b] * v
            k += 1
    return gx, gy


def scatter(q, wx, wy, nx, ny):
    """The transpose of gather: sum over particles of q * wx[a] wy[b] at the
    nine nodes (a (ny, nx) array)."""
    ic, sx, _ = wx
    jc, sy, _ = wy
    idx = _stencil_index(ic, jc, nx, ny)
    out = torch.zeros(ny * nx, dtype=q.dtype, device=q.device)
    k = 0
    for b in range(3):
        for a in range(3):
            out.index_add_(0, idx[k], q * sx[a] * sy[b])
            k += 1
    return out.reshape(ny, nx)


# staggering of each component: (x weights, y weights)
STAG = {"ex": ("h", "n"), "bx": ("h", "n"), "ey": ("n", "h"), "by": ("n", "h"),
        "ez": ("h", "h"), "bz": ("h", "h"), "rho": ("n", "n")}


def _w(kind, x):
    return w_half(x) if kind == "h" else w_node(x)


# ---------------------------------------------------------------------------
# grid operators on periodic (ny, nx) arrays (pic/fields.f90, pic/smooth.f90)
# ---------------------------------------------------------------------------
def xm(a):  # a[j, i-1]
    return torch.roll(a, 1, dims=-1)


def xp(a):  # a[j, i+1]
    return torch.roll(a, -1, dims=-1)


def ym(a):  # a[j-1, i]
    return torch.roll(a, 1, dims=-2)


def yp(a):  # a[j+1, i]
    return torch.roll(a, -1, dims=-2)


def b_half(E, B, k):
    """pic/fields.f90:184-200: B += curl E times (ctxh, ctyh)."""
    ex, ey, ez = E
    bx, by, bz = B
    ctxh, ctyh = k.dt * k.c / k.dx * 0.5, k.dt * k.c / k.dx * 0.5
    return (bx - ctyh * (ez - ym(ez)),
            by + ctxh * (ez - xm(ez)),
            bz - ctxh * (xp(ey) - ey) + ctyh * (yp(ex) - ex))


def b_half_T(lE, lB, k):
    """Transpose of b_half: lB passes through, lE gains the negated
    transposed curl of lB."""
    lbx, lby, lbz = lB
    ctxh, ctyh = k.dt * k.c / k.dx * 0.5, k.dt * k.c / k.dx * 0.5
    lex, ley, lez = lE
    # d(-ctyh*(ez - ym ez))/dez: -ctyh*(1 - yp); d(ctxh*(ez - xm ez)): ctxh*(1 - xp)
    lez = lez - ctyh * (lbx - yp(lbx)) + ctxh * (lby - xp(lby))
    ley = ley - ctxh * (xm(lbz) - lbz)
    lex = lex + ctyh * (ym(lbz) - lbz)
    return (lex, ley, lez), lB


def e_full(E, B, J, k):
    """pic/fields.f90:207-224 with J = jm + jp."""
    ex, ey, ez = E
    bx, by, bz = B
    jx, jy, jz = J
    ctx, cty, tem = k.dt * k.c / k.dx, k.dt * k.c / k.dx, 0.5 * k.dt
    return (ex + cty * (bz - ym(bz)) - tem * jx,
            ey - ctx * (bz - xm(bz)) - tem * jy,
            ez + ctx * (xp(by) - by) - cty * (yp(bx) - bx) - tem * jz)


def e_full_T(lE, lB, k):
    lex, ley, lez = lE
    ctx, cty, tem = k.dt * k.c / k.dx, k.dt * k.c / k.dx, 0.5 * k.dt
    lbx, lby, lbz = lB
    lbz = lbz + cty * (lex - yp(lex)) - ctx * (ley - xp(ley))
    lby = lby + ctx * (xm(lez) - lez)
    lbx = lbx - cty * (ym(lez) - lez)
    lJ = (-tem * lex, -tem * ley, -tem * lez)
    return lE, (lbx, lby, lbz), lJ


def smooth2(a):
    """pic/smooth.f90:143-177 on a periodic array (symmetric: its own transpose)."""
    d = (4 * a + 2 * (xm(a) + xp(a) + ym(a) + yp(a)) + xm(ym(a)) + xm(yp(a)) + xp(ym(a))
         + xp(yp(a))) / 16.0
    return (20 * d - xm(d) - xp(d) - ym(d) - yp(d) - xm(ym(d)) - xm(yp(d)) - xp(ym(d))
            - xp(yp(d))) / 12.0


def _lap_eig(nx, ny, dtype, device):
    kx = torch.arange(nx, dtype=dtype, device=device)
    ky = torch.arange(ny, dtype=dtype, device=device)
    lam = (2 * torch.cos(TWO_PI * kx / nx))[None, :] + (2 * torch.cos(TWO_PI * ky / ny))[:, None] - 4.0
    lam[0, 0] = 1.0
    return lam


def lap_solve(f):
    """u with L u = f (periodic 5-point Laplacian, mean-free part), exactly."""
    ny, nx = f.shape
    lam = _lap_eig(nx, ny, f.dtype, f.device)
    fh = torch.fft.fft2(f)
    uh = fh / lam
    uh[0, 0] = 0.0
    return torch.fft.ifft2(uh).real


def poisson(E, rho, k):
    """pic/fields.f90:384-442: E -= grad L^-1 ((div E - rho) dx^2)."""
    ex, ey, ez = E
    dx = k.dx
    f = ((ex - xm(ex)) / dx + (ey - ym(ey)) / dx - rho) * dx * dx
    u = lap_solve(f)
    return (ex - (xp(u) - u) / dx, ey - (yp(u) - u) / dx, ez)


def poisson_T(lE, k):
    """Transpose of poisson: the projection is self-adjoint in E; the rho
    adjoint is -dx^2 L^-1 div(lE)."""
    lex, ley, lez = lE
    dx = k.dx
    div = (lex - xm(lex)) / dx + (ley - ym(ley)) / dx
    w = lap_solve(div * dx * dx)
    return (lex - (xp(w) - w) / dx, ley - (yp(w) - w) / dx, lez), -w


# ---------------------------------------------------------------------------
# the step
# ---------------------------------------------------------------------------
def _boris(u, aE, aB, c):
    """Relativistic Boris on u = gamma v (pic/move.f90:176-203); returns
    u_new and the intermediates the reverse pass uses."""
    um = [u[i] + aE[i] for i in range(3)]
    g = torch.sqrt(1.0 + um[0] ** 2 + um[1] ** 2 + um[2] ** 2)
    t = [aB[i] / (c * g) for i in range(3)]
    up = [um[0] + um[1] * t[2] - um[2] * t[1],
          um[1] + um[2] * t[0] - um[0] * t[2],
          um[2] + um[0] * t[1] - um[1] * t[0]]
    f = 2.0 / (1.0 + t[0] ** 2 + t[1] ** 2 + t[2] ** 2)
    s = [f * t[i] for i in range(3)]
    upl = [um[0] + up[1] * s[2] - up[2] * s[1],
           um[1] + up[2] * s[0] - up[0] * s[2],
           um[2] + up[0] * s[1] - up[1] * s[0]]
    un = [upl[i] + aE[i] for i in range(3)]
    return un, (um, g, t, up, f, s)


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _boris_T(lun, aB, c, mids):
    """Reverse of _boris: adjoints of u, aE, aB from that of u_new."""
    um, g, t, up, f, s = mids
    laE = list(lun)
    lupl = list(lun)
    # upl = um + up x s
    lum = list(lupl)
    lup = _cross(s, lupl)              # d(up x s)/d up applied: s x lambda
    ls = _cross(lupl, up)              # lambda x up
    # s = f t
    lt = [f * ls[i] for i in range(3)]
    lf = ls[0] * t[0] + ls[1] * t[1] + ls[2] * t[2]
    # f = 2/(1+|t|^2): df/dt = -f^2 t
    lt = [lt[i] - f * f * t[i] * lf for i in range(3)]
    # up = um + um x t
    tx = _cross(t, lup)                # d(um x t)/d um: t x lambda
    lum = [lum[i] + lup[i] + tx[i] for i in range(3)]
    lt2 = _cross(lup, um)              # lambda x um
    lt = [lt[i] + lt2[i] for i in range(3)]
    # t = aB/(c g)
    laB = [lt[i] / (c * g) for i in range(3)]
    lg = -(lt[0] * t[0] + lt[1] * t[1] + lt[2] * t[2]) / g
    # g = sqrt(1+|um|^2)
    lum = [lum[i] + lg * um[i] / g for i in range(3)]
    # um = u + aE
    laE = [laE[i] + lum[i] for i in range(3)]
    return lum, laE, laB


def _vel(un):
    g = torch.sqrt(1.0 + un[0] ** 2 + un[1] ** 2 + un[2] ** 2)
    return [un[i] / g for i in range(3)], g


def _vel_T(lv, un, g):
    dot = (lv[0] * un[0] + lv[1] * un[1] + lv[2] * un[2])
    return [lv[i] / g - un[i] * dot / g ** 3 for i in range(3)]


def _deposit(x, y, v, q, k):
    """J of particles at (x, y) with velocity v and charge factor q."""
    nx, ny = k.nx, k.ny
    J = []
    for comp, vi in zip(("ex", "ey", "ez"), v):
        sx, sy = STAG[comp]
        J.append(scatter(q * vi, _w(sx, x), _w(sy, y), nx, ny))
    return J


def step(E, B, parts, k: StepConst, it: int):
    """One em2 main-loop pass: move, curnt, it+1 -> fields(it).  parts: list
    of (x, y, ux, uy, uz) per species.  Plain PyTorch, differentiable."""
    nx, ny = k.nx, k.ny
    J = [torch.zeros_like(E[0]) for _ in range(3)]
    rho = torch.zeros_like(E[0])
    out_parts = []
    names_e, names_b = ("ex", "ey", "ez"), ("bx", "by", "bz")
    for s, (x, y, ux, uy, uz) in enumerate(parts):
        ae = 0.5 * k.qm[s] * k.dt / k.c
        aE = [ae * gather(E[i], _w(STAG[names_e[i]][0], x), _w(STAG[names_e[i]][1], y), nx, ny)
              for i in range(3)]
        aB = [ae * gather(B[i], _w(STAG[names_b[i]][0], x), _w(STAG[names_b[i]][1], y), nx, ny)
              for i in range(3)]
        un, _ = _boris([ux, uy, uz], aE, aB, k.c)
        v, _ = _vel(un)
        q = k.qd[s]
        Jm = _deposit(x, y, v, q, k)
        xn = torch.remainder(x + v[0] * k.dt / k.dx, nx)
        yn = torch.remainder(y + v[1] * k.dt / k.dx, ny)
        Jp = _deposit(xn, yn, v, q, k)
        J = [J[i] + Jm[i] + Jp[i] for i in range(3)]
        rho = rho + scatter(q * torch.ones_like(xn), w_node(xn), w_node(yn), nx, ny)
        out_parts.append((xn, yn, un[0], un[1], un[2]))
    B1 = b_half(E, B, k)
    E1 = e_full(E, B1, J, k)
    B2 = b_half(E1, B1, k)
    rho_s = smooth2(rho)
    if it % k.isav == 0:
        E1 = tuple(smooth2(a) for a in E1)
        B2 = tuple(smooth2(a) for a in B2)
    E2 = poisson(E1, rho_s, k)
    return E2, B2, out_parts


def step_T(E, B, parts, lE2, lB2, lparts, k: StepConst, it: int):
    """Hand-written reverse of :func:`step`: from the adjoints of its outputs,
    those of its inputs (E, B, particles)."""
    nx, ny = k.nx, k.ny
    names_e, names_b = ("ex", "ey", "ez"), ("bx", "by", "bz")
    # ---- fields (linear) in reverse --------------------------------------
    lE1, lrho_s = poisson_T(tuple(lE2), k)
    lB2 = tuple(lB2)
    if it % k.isav == 0:
        lE1 = tuple(smooth2(a) for a in lE1)
        lB2 = tuple(smooth2(a) for a in lB2)
    lrho = smooth2(lrho_s)
    # B2 = b_half(E1, B1)
    lE1, lB1 = b_half_T(lE1, lB2, k)
    # E1 = e_full(E, B1, J)
    lE, lB1, lJ = e_full_T(lE1, lB1, k)
    # B1 = b_half(E, B)
    lE, lB = b_half_T(lE, lB1, k)
    lE = list(lE)
    lB = list(lB)
    # ---- particles: recompute the forward pieces, then reverse them -------
    lparts_in = []
    for s, (x, y, ux, uy, uz) in enumerate(parts):
        lxn, lyn, lux_n, luy_n, luz_n = lparts[s]
        ae = 0.5 * k.qm[s] * k.dt / k.c
        wE = [(_w(STAG[n][0], x), _w(STAG[n][1], y)) for n in names_e]
        wB = [(_w(STAG[n][0], x), _w(STAG[n][1], y)) for n in names_b]
        aE = [ae * gather(E[i], *wE[i], nx, ny) for i in range(3)]
        aB = [ae * gather(B[i], *wB[i], nx, ny) for i in range(3)]
        un, mids = _boris([ux, uy, uz], aE, aB, k.c)
        v, gn = _vel(un)
        q = k.qd[s]
        xn = torch.remainder(x + v[0] * k.dt / k.dx, nx)
        yn = torch.remainder(y + v[1] * k.dt / k.dx, ny)
        # rho(xn) and jp(xn, v): deposit transpose = gather of the adjoints
        lv = [torch.zeros_like(x) for _ in range(3)]
        lx = torch.zeros_like(x)
        ly = torch.zeros_like(x)
        lxn = lxn.clone()
        lyn = lyn.clone()
        gx, gy = gather_grad(lrho, w_node(xn), w_node(yn), nx, ny)
        lxn = lxn + q * gx
        lyn = lyn + q * gy
        for i, n in enumerate(names_e):
            wxn, wyn = _w(STAG[n][0], xn), _w(STAG[n][1], yn)
            wxo, wyo = _w(STAG[n][0], x), _w(STAG[n][1], y)
            lv[i] = lv[i] + q * (gather(lJ[i], wxn, wyn, nx, ny) + gather(lJ[i], wxo, wyo, nx, ny))
            gxn, gyn = gather_grad(lJ[i], wxn, wyn, nx, ny)
            gxo, gyo = gather_grad(lJ[i], wxo, wyo, nx, ny)
            lxn = lxn + q * v[i] * gxn
            lyn = lyn + q * v[i] * gyn
            lx = lx + q * v[i] * gxo
            ly = ly + q * v[i] * gyo
        # move: xn = x + vx dt/dx (the periodic wrap has unit derivative)
        lx = lx + lxn
        ly = ly + lyn
        lv[0] = lv[0] + lxn * k.dt / k.dx
        lv[1] = lv[1] + lyn * k.dt / k.dx
        # v = un / gamma(un)
        lun = _vel_T(lv, un, gn)
        lun = [lun[0] + lux_n, lun[1] + luy_n, lun[2] + luz_n]
        # Boris, reversed
        lu, laE, laB = _boris_T(lun, aB, k.c, mids)
        # gather transpose = scatter onto the grid; weight derivatives to x, y
        for i in range(3):
            lE[i] = lE[i] + scatter(ae * laE[i], *wE[i], nx, ny)
            lB[i] = lB[i] + scatter(ae * laB[i], *wB[i], nx, ny)
            gxe, gye = gather_grad(E[i], *wE[i], nx, ny)
            gxb, gyb = gather_grad(B[i], *wB[i], nx, ny)
            lx = lx + ae * (laE[i] * gxe + laB[i] * gxb)
            ly = ly + ae * (laE[i] * gye + laB[i] * gyb)
        lparts_in.append((lx, ly, lu[0], lu[1], lu[2]))
    return tuple(lE), tuple(lB), lparts_in


def flux(B, k: StepConst, row: int | None = None):
    """Reconnected flux max(psi) - min(psi) along the centre row of the sheet
    at ny/4 (By averaged over the two rows either side of it)."""
    by = B[1]
    j = k.ny // 4 - 1 if row is None else row
    b = 0.5 * (by[j] + by[j + 1])
    psi = -torch.cumsum(b, 0) * k.dx
    return psi.max() - psi.min()


# ---------------------------------------------------------------------------
# autograd.Function with the hand-written backward, and the T-step driver
# ---------------------------------------------------------------------------
def _flatten(E, B, parts):
    return list(E) + list(B) + [t for p in parts for t in p]


def flatten_state(E, B, parts):
    """(E, B, particles) as the flat tensor list CudaRun takes and returns
    adjoints for: Ex, Ey, Ez, Bx, By, Bz, then x, y, ux, uy, uz per species."""
    return _flatten(E, B, parts)


def _unflatten(ts, nsp):
    E, B = tuple(ts[0:3]), tuple(ts[3:6])
    parts = [tuple(ts[6 + 5 * s: 11 + 5 * s]) for s in range(nsp)]
    return E, B, parts


class Em2Step(torch.autograd.Function):
    """One em2 step; backward = step_T (recomputes the step's intermediates)."""

    @staticmethod
    def forward(ctx, k, it, nsp, *ts):
        E, B, parts = _unflatten(list(ts), nsp)
        with torch.no_grad():
            E2, B2, p2 = step(E, B, parts, k, it)
        ctx.k, ctx.it, ctx.nsp = k, it, nsp
        ctx.save_for_backward(*ts)
        return tuple(_flatten(E2, B2, p2))

    @staticmethod
    def backward(ctx, *gs):
        ts = ctx.saved_tensors
        E, B, parts = _unflatten(list(ts), ctx.nsp)
        gs = [g if g is not None else torch.zeros_like(t) for g, t in zip(gs, ts)]
        lE2, lB2, lparts = _unflatten(gs, ctx.nsp)
        with torch.no_grad():
            lE, lB, lp = step_T(E, B, parts, lE2, lB2, lparts, ctx.k, ctx.it)
        return (None, None, None) + tuple(_flatten(lE, lB, lp))


def run_forward(E, B, parts, k, steps, it0=0):
    with torch.no_grad():
        for n in range(steps):
            E, B, parts = step(E, B, parts, k, it0 + n + 1)
    return E, B, parts


def flux_and_gradient(E0, B0, parts0, k: StepConst, steps: int, checkpoint: int = 50):
    """flux(T) and its adjoint with respect to the initial fields and
    particles, by the hand-written reverse sweep with checkpoints every
    `checkpoint` steps (states in between are recomputed)."""
    nsp = len(parts0)
    ckpts = {0: (E0, B0, parts0)}
    E, B, parts = E0, B0, parts0
    with torch.no_grad():
        for n in range(steps):
            E, B, parts = step(E, B, parts, k, n + 1)
            if (n + 1) % checkpoint == 0 and n + 1 < steps:
                ckpts[n + 1] = (E, B, parts)
    Bf = [b.detach().requires_grad_(True) for b in B]
    with torch.enable_grad():
        F = flux(Bf, k)
        gB = torch.autograd.grad(F, Bf, allow_unused=True)
    gB = [g if g is not None else torch.zeros_like(b) for g, b in zip(gB, Bf)]
    lE = tuple(torch.zeros_like(e) for e in E)
    lB = tuple(gB)
    lparts = [tuple(torch.zeros_like(t) for t in p) for p in parts]
    starts = sorted(ckpts)
    with torch.no_grad():
        for si in range(len(starts) - 1, -1, -1):
            s0 = starts[si]
            s1 = starts[si + 1] if si + 1 < len(starts) else steps
            # recompute the segment's states from its checkpoint
            seg = [ckpts[s0]]
            Es, Bs, ps = ckpts[s0]
            for n in range(s0, s1 - 1):
                Es, Bs, ps = step(Es, Bs, ps, k, n + 1)
                seg.append((Es, Bs, ps))
            for n in range(s1 - 1, s0 - 1, -1):
                Es, Bs, ps = seg[n - s0]
                lE, lB, lparts = step_T(Es, Bs, ps, lE, lB, lparts, k, n + 1)
    return F.detach(), lE, lB, lparts


def _reference_tape(E0, B0, parts0, k, steps):
    """flux(T) and its gradient by autograd through :func:`step` (small
    sizes only: the whole tape is kept)."""
    leaves = [t.detach().clone().requires_grad_(True) for t in _flatten(E0, B0, parts0)]
    E, B, parts = _unflatten(leaves, len(parts0))
    for n in range(steps):
        E, B, parts = step(E, B, parts, k, n + 1)
    F = flux(B, k)
    g = torch.autograd.grad(F, leaves, allow_unused=True)
    g = [gi if gi is not None else torch.zeros_like(li) for gi, li in zip(g, leaves)]
    return F.detach(), _unflatten(g, len(parts0))


# ---------------------------------------------------------------------------
# differentiable initial state (maccpic_b200/loader.py with fixed draws)
# ---------------------------------------------------------------------------
@dataclass
class Draws:
    """The random numbers of one sampled state, kept fixed (common random
    numbers) while the parameters vary."""
    xu: torch.Tensor        # x uniform in [0, 1)
    yu: torch.Tensor        # background y uniform / sheet quantile in (0, 1)
    sheet: torch.Tensor     # 0 background, +1 sheet at ny/4, -1 sheet at 3ny/4
    normals: list           # per species (3, n) standard normals


def make_draws(cfg, n=None, seed=None, device="cpu"):
    import numpy as np
    n = n if n is not None else cfg.nx * cfg.ny * cfg.ppc
    rng = np.random.Generator(np.random.Philox(key=[cfg.seed if seed is None else seed, 0xAD]))
    lc = cfg.L / cfg.dx
    sheet_w = cfg.csden * 2.0 * lc * 2.0
    n_sheet = int(round(n * sheet_w / (cfg.ny + sheet_w)))
    sheet = np.zeros(n)
    which = rng.random(n_sheet) < 0.5
    sheet[n - n_sheet:] = np.where(which, 1.0, -1.0)
    xu = rng.random(n)
    yu = rng.random(n)
    normals = [rng.standard_normal((3, n)) for _ in range(2)]
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device)
    return Draws(t(xu), t(yu), t(sheet), [t(a) for a in normals])


def initial_state_torch(cfg, theta, draws: Draws):
    """(E, B, parts) of the double-Harris workload as a differentiable
    function of theta = (psi0 / (B0 d_i), B_g / B0, L / d_i), with the
    particle counts, categories and macro charge of the nominal config."""
    psi0_r, guide_r, l_r = theta
    nx, ny, dx = cfg.nx, cfg.ny, cfg.dx
    dev = draws.xu.device
    f64 = torch.float64
    lx, ly = nx * dx, ny * dx
    b0, di = cfg.b0, cfg.di
    L = l_r * di
    y1, y2 = ly / 4, 3 * ly / 4
    psi0 = psi0_r * b0 * di

    def psi(xc, yc):
        x = xc * dx
        y = torch.remainder(yc * dx, ly)
        eq = b0 * (L * torch.log(torch.cosh((y - y1) / L)) - L * torch.log(torch.cosh((y - y2) / L)) - y)
        return eq + psi0 * torch.cos(TWO_PI * (x - lx / 2) / lx) * torch.sin(TWO_PI * y / ly) ** 2

    i = torch.arange(nx, dtype=f64, device=dev)[None, :]
    j = torch.arange(ny, dtype=f64, device=dev)[:, None]
    # periodic arrays: Bx[j,i] at (i+1/2, j), By[j,i] at (i, j+1/2) (cells)
    bx = (psi(i + 0.5, j + 0.5) - psi(i + 0.5, j - 0.5)) / dx
    by = -(psi(i + 0.5, j + 0.5) - psi(i - 0.5, j + 0.5)) / dx
    bz = guide_r * b0 * torch.ones_like(bx)
    zero = torch.zeros_like(bx)
    E = (zero, zero.clone(), zero.clone())
    B = (bx, by, bz)
    # particles (positions shared by the two species)
    lc = L / dx
    n = draws.xu.numel()
    x = draws.xu * nx
    bg = draws.sheet == 0
    centre = torch.where(draws.sheet > 0, torch.tensor(ny / 4.0, dtype=f64, device=dev),
                         torch.tensor(3.0 * ny / 4.0, dtype=f64, device=dev))
    ys = centre + lc * torch.atanh((2.0 * draws.yu - 1.0).clamp(-1 + 1e-15, 1 - 1e-15))
    y = torch.where(bg, draws.yu * ny, torch.remainder(ys, ny))
    te, ti = cfg.temperatures()
    vdiff = b0 / (L * cfg.csden)
    ve = vdiff / (1.0 + cfg.ti_over_te)
    vi = vdiff * cfg.ti_over_te / (1.0 + cfg.ti_over_te)
    sign = torch.where(bg, torch.zeros_like(x), -draws.sheet)
    parts = []
    for s, (temp_over_m, vdrift) in enumerate([(te, -ve), (ti / cfg.mass_ratio, vi)]):
        uth = math.sqrt(temp_over_m)
        ux, uy, uz = (draws.normals[s][k] * uth for k in range(3))
        g1 = torch.sqrt(1.0 + ux * ux + uy * uy + uz * uz)
        vx, vy, vz = ux / g1, uy / g1, uz / g1
        V = sign * vdrift
        g0 = torch.sqrt(1.0 - V * V)
        den = 1.0 + V * vz
        vz2 = (V + vz) / den
        vx2 = vx * g0 / den
        vy2 = vy * g0 / den
        gam = 1.0 / torch.sqrt(1.0 - vx2 * vx2 - vy2 * vy2 - vz2 * vz2)
        parts.append((x, y, vx2 * gam, vy2 * gam, vz2 * gam))
    return E, B, parts


def step_const(cfg, draws=None) -> StepConst:
    qm, q, dn, am = cfg.species_constants()
    qd = tuple(q[s] * dn[s] / (cfg.dx * cfg.dx) for s in range(2))
    return StepConst(nx=cfg.nx, ny=cfg.ny, dx=cfg.dx, dt=cfg.dt, c=1.0, isav=cfg.isav,
                     qm=tuple(qm), qd=qd)


def theta_gradient(cfg, theta, steps: int, checkpoint: int = 50, draws=None, device="cpu"):
    """flux(T) and d flux(T) / d theta: hand-written reverse sweep through the
    steps, autograd only through the initial-state map theta -> state."""
    draws = draws or make_draws(cfg, device=device)
    k = step_const(cfg)
    th = torch.tensor(theta, dtype=torch.float64, device=device, requires_grad=True)
    with torch.enable_grad():
        E0, B0, P0 = initial_state_torch(cfg, (th[0], th[1], th[2]), draws)
        flat0 = _flatten(E0, B0, P0)
    F, lE, lB, lP = flux_and_gradient(*(_unflatten([t.detach() for t in flat0], 2)), k,
                                      steps, checkpoint)
    lam = _flatten(lE, lB, lP)
    used = [(t, l) for t, l in zip(flat0, lam) if t.requires_grad]
    g = torch.autograd.grad([t for t, _ in used], th, grad_outputs=[l for _, l in used],
                            allow_unused=True)[0]
    return float(F), g.detach().cpu().numpy()


def flux_of_theta(cfg, theta, steps: int, draws, device="cpu"):
    k = step_const(cfg)
    th = torch.tensor(theta, dtype=torch.float64, device=device)
    E0, B0, P0 = initial_state_torch(cfg, (th[0], th[1], th[2]), draws)
    E, B, P = run_forward(E0, B0, P0, k, steps)
    return float(flux(B, k))


# ---------------------------------------------------------------------------
# the same derivative through the CUDA step (libem2g: em2g_adj_*)
# ---------------------------------------------------------------------------
def _guarded_block(E, B):
    """(13, ny+3, nx+3) em2 field block on the device from periodic E, B:
    index (ix, iy) holds periodic node (ix-1, iy-1); rho and J zero."""
    ny, nx = E[0].shape
    iy = (torch.arange(ny + 3, device=E[0].device) - 1) % ny
    ix = (torch.arange(nx + 3, device=E[0].device) - 1) % nx
    out = torch.zeros((13, ny + 3, nx + 3), dtype=torch.float64, device=E[0].device)
    for k, a in enumerate(list(E) + list(B)):
        out[k] = a[iy][:, ix]
    return out


class CudaAdjoint:
    """One FP64 em2g context with the exact Poisson solve and its adjoint:
    forward(T) advances the state keeping what the reverse sweep needs,
    backward(seed) returns the adjoints of the state forward started from.
    The state enters as (E, B, parts) in this module's periodic, u = gamma v
    form; its first step number is it0.  load() replaces the state, so one
    object (and its device buffers: E, B of every step and the checkpointed
    particles) serves many gradients of runs of the same shape."""

    def __init__(self, k: StepConst, E, B, parts, max_steps: int, checkpoint: int,
                 isav: int, smooth_current: int = 0, it0: int = 0, keep_all_fields=False,
                 field_slots=None, memory_fraction: float = 0.5):
        import ctypes as C
        from . import _lib
        from ._lib import check
        from .em2 import Em2Gpu, RunParams
        self.k, self.nsp = k, len(parts)
        self._L = _lib.lib()
        n = [int(p[0].numel()) for p in parts]
        # em2's species constants from StepConst: q*dn/(dx dy) = qd with dn = 1
        rp = RunParams(nx=k.nx, ny=k.ny, dx=k.dx, dy=k.dx, dt=k.dt, c=k.c, nsp=self.nsp,
                       qm=list(k.qm), q=[qd * k.dx * k.dx for qd in k.qd],
                       dn=[1.0] * self.nsp, am=[1.0] * self.nsp, np_max=n, isav=isav,
                       precision=_lib.FP64, poisson=1, smooth_current=smooth_current)
        self.g = Em2Gpu(rp)
        self.dev = E[0].device
        self.n = n
        self.max_steps, self.checkpoint, self.isav = int(max_steps), int(checkpoint), isav
        self.smooth_current = smooth_current
        # the library works on torch's stream: uploads follow their producers
        self.g.set_stream(torch.cuda.current_stream(self.dev))
        self.load(E, B, parts, it0)
        h = C.c_void_p()
        check(self._L.em2g_adj_create(self.g._h, self.max_steps, self.checkpoint, C.byref(h)))
        self._h = h
        # checkpoints every K steps; E and B of the last `field_slots` steps
        # kept by the forward sweep and the steps before them recomputed a
        # segment at a time in the reverse sweep.  field_slots=None takes as
        # many steps as fit in `memory_fraction` of the device memory still
        # free (at least K, at most max_steps); keep_all_fields takes one
        # per step (no recomputation)
        if keep_all_fields:
            field_slots = self.max_steps
        elif field_slots is None:
            field_slots = self.slots_that_fit(memory_fraction)
        self.set_field_slots(field_slots)

    def slot_bytes(self) -> int:
        """Device bytes of one step's E and B slot."""
        return 6 * 8 * self.k.nx * self.k.ny

    def slots_that_fit(self, memory_fraction: float = 0.5) -> int:
        """Field slots that `memory_fraction` of the free device memory holds
        beside the ones allocated now, clamped to checkpoint .. max_steps."""
        free, _ = torch.cuda.mem_get_info(self.dev)
        have = self.field_slots()
        n = have + int(free * memory_fraction) // self.slot_bytes()
        return max(min(self.checkpoint, self.max_steps), min(self.max_steps, n))

    def set_field_slots(self, n: int):
        """Steps whose E and B the forward sweep keeps (checkpoint ..
        max_steps); the reverse sweep recomputes the steps before them."""
        from ._lib import check
        check(self._L.em2g_adj_field_slots(self._h, int(n)))

    def field_slots(self) -> int:
        import ctypes as C
        from ._lib import check
        n = C.c_int()
        check(self._L.em2g_adj_get_field_slots(self._h, C.byref(n)))
        return n.value

    def load(self, E, B, parts, it0: int = 0):
        """Replace the context's state (same grid and particle counts)."""
        import ctypes as C
        from ._lib import check
        if [int(p[0].numel()) for p in parts] != self.n or tuple(E[0].shape) != (self.k.ny,
                                                                                 self.k.nx):
            raise ValueError("state of another shape than this adjoint's")
        fld = _guarded_block([e.detach() for e in E], [b.detach() for b in B]).contiguous()
        check(self._L.em2g_set_fields_device(self.g._h, C.c_void_p(fld.data_ptr())))
        for s, (x, y, ux, uy, uz) in enumerate(parts):
            u = torch.stack([ux, uy, uz]).detach()
            gam = torch.sqrt(1.0 + (u * u).sum(0))
            st = torch.stack([x.detach(), y.detach(), u[0] / gam, u[1] / gam, u[2] / gam,
                              gam]).contiguous()
            self.g.set_particles_device(s, st)
        self.g.it = it0
        torch.cuda.synchronize(self.dev)

    def close(self):
        from ._lib import check
        if getattr(self, "_h", None) is not None and self._h.value:
            check(self._L.em2g_adj_destroy(self._h))
            self._h = None
        if getattr(self, "g", None) is not None:
            self.g.close()
            self.g = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def forward(self, steps: int):
        from ._lib import check
        check(self._L.em2g_adj_forward(self._h, int(steps)))

    def final_EB(self):
        """Periodic E and B of the current state (device tensors)."""
        import ctypes as C
        from ._lib import check
        k = self.k
        out = torch.empty((13, k.ny + 3, k.nx + 3), dtype=torch.float64, device=self.dev)
        check(self._L.em2g_get_fields_device(self.g._h, C.c_void_p(out.data_ptr())))
        torch.cuda.synchronize(self.dev)
        f = [out[c, 1:k.ny + 1, 1:k.nx + 1].clone() for c in range(6)]
        return tuple(f[:3]), tuple(f[3:])

    def final_B(self):
        """Periodic B of the current state (device tensors)."""
        return self.final_EB()[1]

    def backward(self, lE, lB):
        """Adjoints of the initial state from those of the final E, B
        (periodic tensors); the final particles' adjoints are zero."""
        import ctypes as C
        from ._lib import check
        k = self.k
        seed = torch.stack([t.to(torch.float64) for t in list(lE) + list(lB)]).contiguous()
        check(self._L.em2g_adj_seed_fields_device(self._h, C.c_void_p(seed.data_ptr())))
        check(self._L.em2g_adj_backward(self._h))
        out = torch.empty((6, k.ny, k.nx), dtype=torch.float64, device=self.dev)
        check(self._L.em2g_adj_get_fields_device(self._h, C.c_void_p(out.data_ptr())))
        parts = []
        for s in range(self.nsp):
            lp = torch.empty((5, self.n[s]), dtype=torch.float64, device=self.dev)
            check(self._L.em2g_adj_get_particles_device(
                self._h, s, *[C.c_void_p(lp[c].data_ptr()) for c in range(5)]))
            parts.append(tuple(lp[c] for c in range(5)))
        return tuple(out[:3]), tuple(out[3:]), parts


class CudaRun(torch.autograd.Function):
    """T steps of the CUDA FP64 step (exact Poisson solve) as one autograd
    node: forward maps the initial (E, B, particles) -- the flat tensors of
    :func:`flatten_state`, particles as x, y, u = gamma v -- to the final E and B;
    backward is the hand-written adjoint (em2g_adj_backward), which takes
    the adjoints of the final E, B and returns those of the initial state.
    The final particles are not outputs (their adjoints are zero).

        Ef_Bf = CudaRun.apply(adj, steps, *flatten_state(E0, B0, P0))
        flux(Ef_Bf[3:], k).backward()   # reaches what E0, B0, P0 came from
    """

    @staticmethod
    def forward(ctx, adj, steps, *flat):
        E, B, P = _unflatten([t.detach() for t in flat], adj.nsp)
        adj.load(E, B, P)
        adj.forward(int(steps))
        Ef, Bf = adj.final_EB()
        ctx.adj = adj
        return (*Ef, *Bf)

    @staticmethod
    def backward(ctx, *g):
        adj = ctx.adj
        g = [t if t is not None else
             torch.zeros((adj.k.ny, adj.k.nx), dtype=torch.float64, device=adj.dev) for t in g]
        lE, lB, lP = adj.backward(g[:3], g[3:])
        return (None, None, *_flatten(lE, lB, lP))


def theta_gradient_cuda(cfg, theta, steps: int, checkpoint: int = 50, draws=None,
                        device="cuda", workspace: "CudaAdjoint | None" = None):
    """flux(T) and d flux(T) / d theta with the CUDA step and its adjoint
    (exact Poisson solve), by autograd through :class:`CudaRun`: the
    initial-state map theta -> state is differentiated by autograd, the T
    steps by the hand-written adjoint.  `workspace`: a CudaAdjoint of this
    config's shape with max_steps >= steps and this checkpoint interval,
    reused instead of allocating a new one."""
    import contextlib
    draws = draws or make_draws(cfg, device=device)
    k = step_const(cfg)
    th = torch.tensor(theta, dtype=torch.float64, device=device, requires_grad=True)
    if workspace is not None:
        if workspace.max_steps < steps or workspace.checkpoint != checkpoint:
            raise ValueError("workspace made for fewer steps or another checkpoint interval")
        ctx = contextlib.nullcontext(workspace)
    else:
        with torch.no_grad():
            E0, B0, P0 = initial_state_torch(cfg, tuple(theta), draws)
        ctx = CudaAdjoint(k, E0, B0, P0, steps, checkpoint, cfg.isav, cfg.smooth_current)
    with ctx as adj:
        with torch.enable_grad():
            E0, B0, P0 = initial_state_torch(cfg, (th[0], th[1], th[2]), draws)
            out = CudaRun.apply(adj, steps, *_flatten(E0, B0, P0))
            F = flux(out[3:], k)
            F.backward()
    return float(F.detach()), th.grad.detach().cpu().numpy()


def fd_check_cuda(cfg, theta, steps: int, h: float = 1e-3, checkpoint: int = 50, draws=None,
                  device="cuda", workspace: "CudaAdjoint | None" = None):
    """The adjoint gradient of flux(T) against central finite differences of
    the same CUDA forward, (flux(theta + h e_i) - flux(theta - h e_i)) / 2h,
    with common random numbers (the same draws for every evaluation).
    Returns {"flux", "adjoint", "fd", "rel_error"} (rel_error per component:
    |adjoint - fd| / max(|fd|, 1e-3 max|fd|))."""
    import numpy as np
    draws = draws or make_draws(cfg, device=device)
    F, g = theta_gradient_cuda(cfg, theta, steps, checkpoint, draws, device, workspace)
    k = step_const(cfg)
    fd = []
    for i in range(3):
        vals = []
        for sgn in (1.0, -1.0):
            th = list(theta)
            th[i] += sgn * h
            with torch.no_grad():
                E0, B0, P0 = initial_state_torch(cfg, tuple(th), draws)
            if workspace is not None:
                workspace.load(E0, B0, P0)
                workspace.g.step(steps)
                vals.append(float(flux(workspace.final_B(), k)))
            else:
                with CudaAdjoint(k, E0, B0, P0, 1, 1, cfg.isav, cfg.smooth_current) as adj:
                    adj.g.step(steps)
                    vals.append(float(flux(adj.final_B(), k)))
        fd.append((vals[0] - vals[1]) / (2 * h))
    fd = np.array(fd)
    floor = 1e-3 * np.abs(fd).max()
    rel = np.abs(g - fd) / np.maximum(np.abs(fd), floor)
    return {"flux": F, "adjoint": g.tolist(), "fd": fd.tolist(), "rel_error": rel.tolist()}


def flux_of_theta_cuda(cfg, theta, steps: int, draws, device="cuda"):
    """flux(T) by the CUDA FP64 step with the exact Poisson solve."""
    k = step_const(cfg)
    th = torch.tensor(theta, dtype=torch.float64, device=device)
    E0, B0, P0 = initial_state_torch(cfg, (th[0], th[1], th[2]), draws)
    with CudaAdjoint(k, E0, B0, P0, 1, 1, cfg.isav, cfg.smooth_current) as adj:
        adj.g.step(steps)
        return float(flux(adj.final_B(), k))
