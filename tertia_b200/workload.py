"""Synthetic workloads of the quasi-static layer loop.

No input deck ships with the reference (vlpl3d.cpp:45 reads a v.ini that is
not in the tree), so the runs are defined here: a uniform plasma seeded on
the reference lattice and a sampled bi-Gaussian driver.  The five named
configurations are the benchmark's workloads:

  c0: 128 x 128 transverse, 256 layers, 1e5 beam particles, CIC, FP64 (CPU case)
  c1: 512 x 512, 1024 layers, thermal sigma_p 0.01, 1e6 beam particles, 10 steps
  c2: 1024 x 1024, 2048 layers, n_b/n_0 = 1, 4e6 beam particles (precision study)
  c3: 256 x 256, 2048 layers, 1e6 beam particles, 64 xi-bins (adjoint)
  c4: 1024 x 1024, 4096 layers, 1e7 driver + 1e6 witness particles, 20 steps

Lengths are in 1/k_p: with Density = 1 the spectral solver's
dens = |n q/m| = 1 (movefieldshydrolinlayersplit.cpp:244-252).  The driver's
centre sits 4 sigma_xi behind the front layer; xi is measured from it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .abi import QsConfig, default_config, QS_SHAPE_CIC, QS_SHAPE_NGP, PRECISIONS


@dataclass
class BeamSpec:
    n: int
    sigma_r: float = 0.5
    sigma_xi: float = 1.0
    nb_over_n0: float = 0.5
    gamma: float = 1000.0
    xi_center: float = 0.0     # relative to the driver centre
    seed: int = 1


@dataclass
class Workload:
    name: str
    cfg: QsConfig
    beams: list = field(default_factory=list)
    steps: int = 1
    description: str = ""


def _cfg(n, layers, h=0.05, **kw):
    c = default_config(ny=n, nz=n, nx=layers, hx=h, hy=h, hz=h)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def make_workload(name: str, precision: str | None = None) -> Workload:
    """The named benchmark configurations (see module docstring)."""
    if name == "c0":
        w = Workload("c0", _cfg(128, 256, shape=QS_SHAPE_CIC, precision=PRECISIONS["fp64"]),
                     [BeamSpec(100_000)], 1,
                     "128x128x256 FP64 CIC, 1e5 beam particles, 1 beam step")
    elif name == "c1":
        w = Workload("c1", _cfg(512, 1024, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01),
                     [BeamSpec(1_000_000)], 10,
                     "512x512x1024 FP32, thermal 0.01, 1e6 beam particles, 10 beam steps")
    elif name == "c2":
        w = Workload("c2", _cfg(1024, 2048), [BeamSpec(4_000_000, nb_over_n0=1.0)], 1,
                     "1024x1024x2048 precision study, n_b/n_0 = 1, 4e6 beam particles")
    elif name == "c3":
        w = Workload("c3", _cfg(256, 2048), [BeamSpec(1_000_000)], 1,
                     "256x256x2048 adjoint, 64 xi-bins, 1e6 beam particles")
    elif name == "c4":
        w = Workload("c4", _cfg(1024, 4096, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01),
                     [BeamSpec(10_000_000),
                      BeamSpec(1_000_000, sigma_r=0.3, sigma_xi=0.3, xi_center=-5.5, seed=2)],
                     20, "1024x1024x4096, 1e7 driver + 1e6 witness, 20 beam steps")
    else:
        raise ValueError(f"unknown workload {name}")
    if precision is not None:
        w.cfg.precision = PRECISIONS[precision]
    return w


def driver_center_x(cfg: QsConfig, sigma_xi: float = 1.0) -> float:
    """Longitudinal box coordinate X = i*hx of the driver centre."""
    return cfg.nx * cfg.hx - 4.0 * sigma_xi


def sample_beam(cfg: QsConfig, spec: BeamSpec, driver_sigma_xi: float = 1.0) -> dict:
    """Sample a bi-Gaussian bunch into (cell, fraction) form.

    The weight makes the peak of the deposited density n_b/n_0 in plasma
    units (plasma cell density = Density, weight Density/ppc per particle).
    Particles outside the box are clipped into the edge cells.
    """
    rng = np.random.default_rng(spec.seed)
    n = spec.n
    xc = driver_center_x(cfg, driver_sigma_xi) + spec.xi_center
    yc = cfg.ny * cfg.hy / 2.0
    zc = cfg.nz * cfg.hz / 2.0
    X = xc + spec.sigma_xi * rng.standard_normal(n)
    Y = yc + spec.sigma_r * rng.standard_normal(n)
    Z = zc + spec.sigma_r * rng.standard_normal(n)
    gx = np.clip(X / cfg.hx, 0.0, cfg.nx - 1e-9)
    gy = np.clip(Y / cfg.hy, 0.0, cfg.ny - 1e-9)
    gz = np.clip(Z / cfg.hz, 0.0, cfg.nz - 1e-9)
    i = np.floor(gx).astype(np.int32)
    j = np.floor(gy).astype(np.int32)
    k = np.floor(gz).astype(np.int32)
    vol = (2.0 * math.pi) ** 1.5 * spec.sigma_xi * spec.sigma_r ** 2
    w = spec.nb_over_n0 * cfg.plasma_density * vol / (n * cfg.hx * cfg.hy * cfg.hz)
    p0 = math.sqrt(spec.gamma ** 2 - 1.0)
    return dict(i=i, j=j, k=k, x=gx - i, y=gy - j, z=gz - k,
                px=np.full(n, p0), py=np.zeros(n), pz=np.zeros(n),
                w=np.full(n, w))


def concat_beams(parts: list) -> dict:
    return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}


def workload_beam(w: Workload) -> dict:
    sig = w.beams[0].sigma_xi
    return concat_beams([sample_beam(w.cfg, b, sig) for b in w.beams])


def lattice_offsets(ppc: int):
    """In-cell (y, z) of the seeded plasma particles in list order (head
    first), Mesh::SeedParticles (mesh.cpp:436-470): seeds are created for
    iseed = nseed-1 .. 0 and each is pushed to the list head."""
    out = []
    nseed = ppc
    iside = int(math.pow(nseed - 1, 0.5) + 1.0) if nseed > 0 else 1
    for iseed in range(nseed):             # head first = iseed 0
        if nseed == 1:
            y = z = 0.5
        elif nseed in (2, 3):
            y = z = 0.5
        elif nseed == 4:
            y = 1.0 / 3.0 * (1.0 + iseed % 2)
            z = 1.0 / 3.0 * (1.0 + iseed // 2)
        else:
            iz = iseed // iside
            iy = iseed - iside * iz
            y = 1.0 / iside * (iy + 0.5)
            z = 1.0 / iside * (iz + 0.5)
        out.append((y, z))
    return out


def front_plasma(cfg: QsConfig, seed: int = 7, thermal: bool = True) -> dict:
    """Front-layer plasma on the reference lattice, grouped by cell, with
    P0 + N(0, Pspread) momenta drawn from numpy (used by the parity tests to
    hand identical arrays to the oracle and the GPU path)."""
    ppc = cfg.ppc
    ncell = cfg.ny * cfg.nz
    offs = np.array(lattice_offsets(ppc))
    cell = np.repeat(np.arange(ncell, dtype=np.int32), ppc)
    y = np.tile(offs[:, 0], ncell)
    z = np.tile(offs[:, 1], ncell)
    n = ncell * ppc
    rng = np.random.default_rng(seed)
    def mom(p0, s):
        if thermal and s > 0:
            return p0 + s * rng.standard_normal(n)
        return np.full(n, float(p0))
    px = mom(cfg.plasma_px0, cfg.pspread_x)
    py = mom(cfg.plasma_py0, cfg.pspread_y)
    pz = mom(cfg.plasma_pz0, cfg.pspread_z)
    w = np.full(n, cfg.plasma_density / ppc)
    return dict(cell=cell, y=y, z=z, px=px, py=py, pz=pz, w=w)


def small_config(n=32, layers=48, h=0.2, hx=0.1, **kw) -> QsConfig:
    """A coarse deck that the oracle finishes in seconds (parity tests)."""
    c = default_config(ny=n, nz=n, nx=layers, hx=hx, hy=h, hz=h)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def small_beam(cfg: QsConfig, n=4000, sigma_r=0.5, sigma_xi=1.0, nb=0.5, seed=1,
               sigma_p=0.0) -> dict:
    spec = BeamSpec(n, sigma_r=sigma_r, sigma_xi=sigma_xi, nb_over_n0=nb, seed=seed)
    # keep the driver centre 2.5 sigma behind the front on short boxes
    b = sample_beam(cfg, spec, driver_sigma_xi=min(sigma_xi, cfg.nx * cfg.hx / 6.5))
    if sigma_p > 0:
        rng = np.random.default_rng(seed + 100)
        b["py"] = sigma_p * rng.standard_normal(n)
        b["pz"] = sigma_p * rng.standard_normal(n)
    return b
