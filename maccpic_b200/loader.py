"""Seeded double-Harris initial state (the shared start for GPU and oracle).

em2 builds its start with a quiet-start lattice loader (pic/creator.f90,
pic/smear.f90, pic/setv.f90) fixed at compile time.  The workloads here are
instead sampled from a seed, with em2's normalisation (density in units of
the background, pic/README.md:218; macro charge of pic/input.f90:61-69):

* grid NX x NY, cells dx = dy, doubly periodic;
* Bx = B0 [tanh((y-y1)/L) - tanh((y-y2)/L) - 1], sheets at y1 = Ly/4 and
  y2 = 3Ly/4, from a flux function psi on the Ez nodes so that the discrete
  div B is zero; plus a flux perturbation
  dpsi = psi0 cos(2 pi (x - Lx/2)/Lx) sin^2(2 pi y / Ly)
  (smooth in y, largest on both sheets); optional uniform guide field Bz;
* density n_b [1 + csden (sech^2((y-y1)/L) + sech^2((y-y2)/L))], n_b = 1;
  electrons and ions share positions (quasi-neutral start, as em2 does);
* background particles: Maxwellian at rest; sheet particles: Maxwellian
  drifting along z, V_i - V_e = B0/(L csden) with V_i/V_e = -Ti/Te
  (pic/RECONNECTION_MODEL.md, sections 5.1-5.2), signs following the
  current of the sign convention above, added relativistically
  (pic/creator.f90:227-235);
* velocities are taken as the leapfrog values at t = -dt/2.

Units: lengths in c/wpe, time 1/wpe, c = 1; positions in cells.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from ._lib import NFIELD, FIELD_ID
from .em2 import RunParams


@dataclass
class HarrisConfig:
    nx: int = 256
    ny: int = 128
    dx: float = 0.5
    dt: float = 0.05
    mass_ratio: float = 25.0
    ppc: int = 16               # particles per cell per species (NX*NY*ppc each)
    wpe_over_wce: float = 2.0   # B0 = 1/(wpe/wce)
    csden: float = 5.0          # n0 / n_b
    l_over_di: float = 0.5      # sheet half-thickness in d_i
    ti_over_te: float = 5.0
    psi0_over_b0di: float = 0.1
    guide_over_b0: float = 0.0
    isav: int = 20
    steps: int = 2000
    seed: int = 0
    smooth_current: int = 0     # binomial current filter every step (not in em2)
    check_steps: int | None = None  # length of the FP32-vs-FP64 check (None: steps)

    @property
    def b0(self):
        return 1.0 / self.wpe_over_wce

    @property
    def di(self):
        # ion inertial length at the sheet density n0 = csden * n_b
        return math.sqrt(self.mass_ratio / self.csden)

    @property
    def L(self):
        return self.l_over_di * self.di

    def temperatures(self):
        # pressure balance B0^2/2 = n0 (Te + Ti)
        tsum = self.b0 ** 2 / (2.0 * self.csden)
        te = tsum / (1.0 + self.ti_over_te)
        return te, tsum - te

    def species_constants(self):
        """(qm, q, dn, am) as com_den and init compute them, for the
        background density of this config's sampling."""
        nb_ppc = self.background_ppc()
        rm = [1.0, self.mass_ratio]
        qm = [-1.0, 1.0 / self.mass_ratio]
        q = [self.dx * self.dx / (nb_ppc * qm[s]) / rm[s] for s in range(2)]
        am = [q[0] / -1.0, q[1] / (1.0 / self.mass_ratio)]
        return qm, q, [1.0, 1.0], am

    def background_ppc(self):
        """Particles per cell at density n_b (= em2's npcel)."""
        lc = self.L / self.dx  # half-thickness in cells
        sheet_cells = self.csden * 2.0 * lc * 2.0  # two sheets, integral of csden sech^2
        return self.ppc * self.ny / (self.ny + sheet_cells)

    def run_params(self, np_max=None, **kw) -> RunParams:
        qm, q, dn, am = self.species_constants()
        n = self.nx * self.ny * self.ppc
        kw.setdefault("smooth_current", self.smooth_current)
        return RunParams(nx=self.nx, ny=self.ny, dx=self.dx, dy=self.dx, dt=self.dt,
                         qm=qm, q=q, dn=dn, am=am,
                         np_max=np_max or [n, n], isav=self.isav, **kw)
# the benchmark and test workloads (synthetic, seeded)
PRESETS = {
    "harris_256x128_ppc16": HarrisConfig(),
    "harris_2048x1024_ppc64": HarrisConfig(nx=2048, ny=1024, ppc=64, steps=1000),
    "harris_512x256_ppc32": HarrisConfig(nx=512, ny=256, ppc=32, steps=800),
    # profiling size: particle buffers (0.4-0.8 GB) well above the 126 MB L2
    "harris_1024x512_ppc32": HarrisConfig(nx=1024, ny=512, ppc=32, steps=100),
    "harris_4096x2048_ppc100": HarrisConfig(nx=4096, ny=2048, ppc=100, mass_ratio=100.0,
                                            dt=0.04, steps=2000, smooth_current=1,
                                            check_steps=200),
}


def initial_fields(cfg: HarrisConfig) -> np.ndarray:
    """(13, ny+3, nx+3) block: B from a flux function, E = 0, rho = J = 0."""
    nx, ny, dx = cfg.nx, cfg.ny, cfg.dx
    lx, ly = nx * dx, ny * dx
    y1, y2, L, b0 = ly / 4, 3 * ly / 4, cfg.L, cfg.b0
    psi0 = cfg.psi0_over_b0di * b0 * cfg.di

    def psi(xc, yc):
        # xc, yc in cells; psi with Bx = dpsi/dy, By = -dpsi/dx
        x = xc * dx
        y = np.mod(yc * dx, ly)
        eq = b0 * (L * np.log(np.cosh((y - y1) / L)) - L * np.log(np.cosh((y - y2) / L)) - y)
        # psi_eq(Ly) - psi_eq(0) vanishes to exp(-Ly/2L); y in [0, Ly)
        pert = psi0 * np.cos(2 * np.pi * (x - lx / 2) / lx) * np.sin(2 * np.pi * y / ly) ** 2
        return eq + pert

    fld = np.zeros((NFIELD, ny + 3, nx + 3))
    ix = np.arange(nx + 3)[None, :]
    iy = np.arange(ny + 3)[:, None]
    # psi on Ez nodes: (ix - 1/2, iy - 1/2) in cells
    # Bx(ix,iy) at (ix-1/2, iy-1) = [psi(ix, iy) - psi(ix, iy-1)] / dy
    bx = (psi(ix - 0.5, iy - 0.5) - psi(ix - 0.5, iy - 1.5)) / dx
    # By(ix,iy) at (ix-1, iy-1/2) = -[psi(ix, iy) - psi(ix-1, iy)] / dx
    by = -(psi(ix - 0.5, iy - 0.5) - psi(ix - 1.5, iy - 0.5)) / dx
    fld[FIELD_ID["bx"]] = bx
    fld[FIELD_ID["by"]] = by
    fld[FIELD_ID["bz"]] = cfg.guide_over_b0 * b0
    return fld


def sample_particles(cfg: HarrisConfig, n: int | None = None):
    """Two species blocks (6, n): x, y (cells), vx, vy, vz, gamma."""
    nx, ny, dx = cfg.nx, cfg.ny, cfg.dx
    n = n if n is not None else nx * ny * cfg.ppc
    rng = np.random.Generator(np.random.Philox(key=[cfg.seed, 0xE2]))
    lc = cfg.L / dx
    sheet_w = cfg.csden * 2.0 * lc * 2.0
    n_sheet = int(round(n * sheet_w / (ny + sheet_w)))
    n_bg = n - n_sheet
    y = np.empty(n)
    y[:n_bg] = rng.random(n_bg) * ny
    u = rng.random(n_sheet)
    which = rng.random(n_sheet) < 0.5
    centre = np.where(which, ny / 4.0, 3.0 * ny / 4.0)
    # inverse CDF of sech^2: y = c + L atanh(2u - 1)
    ys = centre + lc * np.arctanh(np.clip(2.0 * u - 1.0, -1 + 1e-15, 1 - 1e-15))
    y[n_bg:] = np.mod(ys, ny)
    x = rng.random(n) * nx
    # floating wrap can give exactly n; keep positions in [0, n)
    x[x >= nx] = 0.0
    y[y >= ny] = 0.0
    te, ti = cfg.temperatures()
    vdiff = cfg.b0 / (cfg.L * cfg.csden)  # |V_i - V_e|
    ve = vdiff / (1.0 + cfg.ti_over_te)
    vi = vdiff * cfg.ti_over_te / (1.0 + cfg.ti_over_te)
    # sheet 1 (y1) carries Jz < 0 with this Bx sign: ions drift -z, electrons +z
    sign = np.zeros(n)
    sign[n_bg:] = np.where(which, -1.0, 1.0)
    out = []
    for s, (temp_over_m, vdrift) in enumerate([(te, -ve), (ti / cfg.mass_ratio, vi)]):
        srng = np.random.Generator(np.random.Philox(key=[cfg.seed, 0xE2 + 1 + s]))
        uth = math.sqrt(temp_over_m)
        ux, uy, uz = (srng.standard_normal(n) * uth for _ in range(3))
        g1 = np.sqrt(1.0 + ux * ux + uy * uy + uz * uz)
        vx, vy, vz = ux / g1, uy / g1, uz / g1
        V = sign * vdrift
        g0 = np.sqrt(1.0 - V * V)
        den = 1.0 + V * vz
        vz2 = (V + vz) / den
        vx2 = vx * g0 / den
        vy2 = vy * g0 / den
        gam = 1.0 / np.sqrt(1.0 - vx2 * vx2 - vy2 * vy2 - vz2 * vz2)
        out.append(np.stack([x, y, vx2, vy2, vz2, gam]))
    return out


def initial_state(cfg: HarrisConfig, n: int | None = None):
    """(fields, [electrons, ions]) for the config."""
    return initial_fields(cfg), sample_particles(cfg, n)


def sample_particles_torch(cfg: HarrisConfig, device="cuda", n: int | None = None,
                           dtype=None):
    """The same distribution as :func:`sample_particles`, drawn on the GPU
    with torch's Philox generator (for workloads too large for host RAM).
    Returns two (6, n) tensors (x, y, vx, vy, vz, gamma) on ``device``."""
    import torch
    dtype = dtype or torch.float64
    nx, ny, dx = cfg.nx, cfg.ny, cfg.dx
    n = n if n is not None else nx * ny * cfg.ppc
    gen = torch.Generator(device=device)
    gen.manual_seed(cfg.seed * 7919 + 0xE2)
    lc = cfg.L / dx
    sheet_w = cfg.csden * 2.0 * lc * 2.0
    n_sheet = int(round(n * sheet_w / (ny + sheet_w)))
    n_bg = n - n_sheet
    f64 = torch.float64
    y = torch.empty(n, dtype=f64, device=device)
    y[:n_bg] = torch.rand(n_bg, generator=gen, dtype=f64, device=device) * ny
    u = torch.rand(n_sheet, generator=gen, dtype=f64, device=device)
    which = torch.rand(n_sheet, generator=gen, dtype=f64, device=device) < 0.5
    centre = torch.where(which, torch.tensor(ny / 4.0, dtype=f64, device=device),
                         torch.tensor(3.0 * ny / 4.0, dtype=f64, device=device))
    ys = centre + lc * torch.atanh((2.0 * u - 1.0).clamp(-1 + 1e-15, 1 - 1e-15))
    y[n_bg:] = torch.remainder(ys, ny)
    x = torch.rand(n, generator=gen, dtype=f64, device=device) * nx
    x[x >= nx] = 0.0
    y[y >= ny] = 0.0
    te, ti = cfg.temperatures()
    vdiff = cfg.b0 / (cfg.L * cfg.csden)
    ve = vdiff / (1.0 + cfg.ti_over_te)
    vi = vdiff * cfg.ti_over_te / (1.0 + cfg.ti_over_te)
    sign = torch.zeros(n, dtype=f64, device=device)
    sign[n_bg:] = torch.where(which, -1.0, 1.0).to(f64)
    out = []
    for temp_over_m, vdrift in [(te, -ve), (ti / cfg.mass_ratio, vi)]:
        uth = math.sqrt(temp_over_m)
        ux, uy, uz = (torch.randn(n, generator=gen, dtype=f64, device=device) * uth
                      for _ in range(3))
        g1 = torch.sqrt(1.0 + ux * ux + uy * uy + uz * uz)
        vx, vy, vz = ux / g1, uy / g1, uz / g1
        del ux, uy, uz, g1
        V = sign * vdrift
        g0 = torch.sqrt(1.0 - V * V)
        den = 1.0 + V * vz
        vz2 = (V + vz) / den
        vx2 = vx * g0 / den
        vy2 = vy * g0 / den
        del vx, vy, vz, V, g0, den
        gam = 1.0 / torch.sqrt(1.0 - vx2 * vx2 - vy2 * vy2 - vz2 * vz2)
        out.append(torch.stack([x, y, vx2, vy2, vz2, gam]).to(dtype))
        del vx2, vy2, vz2, gam
    return out


def setv_torch(cfg: HarrisConfig, fields, parts, device="cuda") -> None:
    """em2's start-up as its fresh run does it (pic/main.f90 -> setv): take
    the drawn velocities as those at t = 0 and push them back to t = -dt/2
    on the GPU with the initial E and B and linear weights
    (pic/setv.f90:36-128, ``em2g_setv_device``), in place on each species'
    (6, n) float64 CUDA tensor.  Without it the drawn velocities are taken
    as the t = -dt/2 values directly."""
    import torch
    from .em2 import setv_device
    fld = torch.as_tensor(np.ascontiguousarray(fields), dtype=torch.float64, device=device)
    rp = cfg.run_params()
    for s, p in enumerate(parts):
        setv_device(rp, s, fld, p)


def sample_particles_torch_slices(cfg: HarrisConfig, device="cuda", slice_size: int = 1 << 24):
    """The double-Harris distribution of :func:`sample_particles_torch`,
    drawn slice by slice on the GPU for workloads whose whole FP64 state
    (48 bytes per particle and species) would not fit beside the run: yields
    (electrons, ions), two (6, m) float64 tensors per slice, m = slice_size
    except for the last, NX*NY*ppc particles in all per species.  Slice k
    has its own Philox stream (seed, k), so any slice can be drawn again
    alone; each slice splits its particles between background and sheets in
    the proportion of the whole."""
    import dataclasses
    n = cfg.nx * cfg.ny * cfg.ppc
    for k, first in enumerate(range(0, n, slice_size)):
        m = min(slice_size, n - first)
        sub = dataclasses.replace(cfg, seed=cfg.seed * 1000003 + 7 * k + 1)
        yield sample_particles_torch(sub, device=device, n=m)
