"""The synthetic workloads (host only): the named configurations' sizes, the
reference lattice of the seeded plasma (mesh.cpp:436-470), the beam sampler's
bounds, determinism and charge calibration, and the front plasma's layout."""
import math

import numpy as np
import pytest

from tertia_b200 import workload as wl
from tertia_b200.abi import PRECISIONS


@pytest.mark.parametrize("name,n,layers,beams", [
    ("c0", 128, 256, [100_000]),
    ("c1", 512, 1024, [1_000_000]),
    ("c2", 1024, 2048, [4_000_000]),
    ("c3", 256, 2048, [1_000_000]),
    ("c4", 1024, 4096, [10_000_000, 1_000_000]),
])
def test_named_configurations(name, n, layers, beams):
    w = wl.make_workload(name)
    c = w.cfg
    assert (c.ny, c.nz, c.nx) == (n, n, layers)
    assert c.ppc == 4 and c.n_iter == 1 and c.nx_split == 1
    assert c.hx == c.hy == c.hz == 0.05
    assert [b.n for b in w.beams] == beams


def test_thermal_spread_and_precision():
    assert wl.make_workload("c1").cfg.pspread_x == 0.01
    assert wl.make_workload("c4").cfg.pspread_z == 0.01
    assert wl.make_workload("c0").cfg.precision == PRECISIONS["fp64"]
    assert wl.make_workload("c3", "fp32").cfg.precision == PRECISIONS["fp32"]
    with pytest.raises(ValueError):
        wl.make_workload("c9")


def test_four_particles_sit_at_thirds_of_the_cell():
    offs = wl.lattice_offsets(4)
    assert sorted(offs) == sorted([(1 / 3, 1 / 3), (2 / 3, 1 / 3), (1 / 3, 2 / 3), (2 / 3, 2 / 3)])
    assert wl.lattice_offsets(1) == [(0.5, 0.5)]


def test_beam_sampler_bounds_determinism_and_charge():
    cfg = wl.small_config(n=32, layers=64)
    spec = wl.BeamSpec(20_000, sigma_r=0.5, sigma_xi=1.0, nb_over_n0=0.5, seed=3)
    a = wl.sample_beam(cfg, spec)
    b = wl.sample_beam(cfg, spec)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert np.all((a["i"] >= 0) & (a["i"] < cfg.nx))
    assert np.all((a["j"] >= 0) & (a["j"] < cfg.ny))
    assert np.all((a["k"] >= 0) & (a["k"] < cfg.nz))
    for k in ("x", "y", "z"):
        assert np.all((a[k] >= 0) & (a[k] < 1))
    # total charge: n_b/n_0 * Density over the bunch volume (2 pi)^1.5 sigma_xi sigma_r^2
    vol = (2 * math.pi) ** 1.5 * spec.sigma_xi * spec.sigma_r ** 2
    total = a["w"].sum() * cfg.hx * cfg.hy * cfg.hz
    assert total == pytest.approx(spec.nb_over_n0 * cfg.plasma_density * vol, rel=1e-12)
    assert np.all(a["px"] == math.sqrt(spec.gamma ** 2 - 1))
    c = wl.sample_beam(cfg, wl.BeamSpec(20_000, seed=4))
    assert not np.array_equal(a["y"], c["y"])


def test_front_plasma_layout():
    cfg = wl.small_config(n=16, layers=8, pspread_x=0.01, pspread_y=0.01, pspread_z=0.01)
    p = wl.front_plasma(cfg, seed=5)
    ncell = cfg.ny * cfg.nz
    assert p["cell"].size == ncell * cfg.ppc
    assert np.all(np.diff(p["cell"]) >= 0)                       # grouped by cell
    assert np.all(np.bincount(p["cell"], minlength=ncell) == cfg.ppc)
    assert np.all(p["w"] == cfg.plasma_density / cfg.ppc)
    assert abs(np.std(p["px"] - cfg.plasma_px0) - 0.01) < 1e-3
    cold = wl.front_plasma(cfg, thermal=False)
    assert np.all(cold["py"] == cfg.plasma_py0)
