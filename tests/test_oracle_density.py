"""The oracle's plasma density profiles (Specie::Density, plasma.cpp:6-399)
against closed forms of the reference formulas, and the front-layer weights
of Mesh::SeedParticles (mesh.cpp:413-471).  Host only."""
import ctypes as C
import math

import numpy as np
import pytest

from tertia_b200 import abi
from tertia_b200.abi import density_profile

PI_REF = 3.1415927   # the reference's PI (domain.h:10)


@pytest.fixture(scope="module")
def orc(oracle_lib):
    return oracle_lib


def dens(orc, prof, x, y=0.0, z=0.0):
    return orc.density(prof, x, y, z)


def test_profile_layout_and_default():
    from tertia_b200 import build as qb
    qb.build()
    L = abi.load_library()
    assert C.sizeof(abi.QsDensityProfile) == 192
    assert abi.QsDensityProfile.curvature_end.offset == 184
    p = abi.QsDensityProfile()
    assert L.qs_density_profile_default(C.byref(p)) == 0
    assert p.as_dict() == density_profile().as_dict()


def test_trapezoid(orc):
    p = density_profile(density=2.0, begin=1.0, plateau_begin=3.0, plateau_end=5.0, end=9.0)
    assert dens(orc, p, 0.5) == 0.0 and dens(orc, p, 9.5) == 0.0 and dens(orc, p, -1.0) == 0.0
    assert dens(orc, p, 2.0) == pytest.approx(1.0, rel=1e-15)
    assert dens(orc, p, 4.0) == 2.0
    assert dens(orc, p, 7.0) == pytest.approx(1.0, rel=1e-15)
    # any unknown distribution number is the trapezoid (the reference's default label)
    q = density_profile(distribution=42, density=2.0, begin=1.0, plateau_begin=3.0,
                        plateau_end=5.0, end=9.0)
    assert dens(orc, q, 2.0) == dens(orc, p, 2.0)


def test_gaussian_channel(orc):
    p = density_profile(distribution=abi.DIST_GAUSS_CHANNEL, density=1.0, density1=3.0,
                        begin=0.0, plateau_begin=0.0, plateau_end=10.0, end=20.0, delta=0.5,
                        radius=2.0)
    assert dens(orc, p, 5.0) == pytest.approx(2.0 * 0.5, rel=1e-15)       # axis: t = delta
    t = 0.5 * math.exp(-1.0)                                              # r = radius
    assert dens(orc, p, 5.0, 2.0, 0.0) == pytest.approx(2.0 * (1 - t), rel=1e-14)
    assert dens(orc, p, 15.0, 0.0, 0.0) == pytest.approx(3.0 * 0.5 * 0.5, rel=1e-14)
    assert dens(orc, p, 5.0, 20.0, 0.0) == pytest.approx(2.0, rel=1e-15)  # arg >= 10: t = 0


def test_empty_channel_and_parallelepiped(orc):
    p = density_profile(distribution=abi.DIST_EMPTY_CHANNEL, density=1.5, delta=0.1, radius=1.0)
    assert dens(orc, p, 1.0, 0.5, 0.5) == pytest.approx(0.15, rel=1e-15)
    assert dens(orc, p, 1.0, 1.0, 0.5) == 1.5
    q = density_profile(distribution=abi.DIST_PARALLELEPIPED, density=0.7, x0=2.0, radius=1.0,
                        radius_y=0.5)
    assert dens(orc, q, 2.9, 0.4, -0.9) == 0.7
    assert dens(orc, q, 2.9, 0.6, 0.0) == 0.0


def test_ellipsoid_cos_gauss_tanh(orc):
    p = density_profile(distribution=abi.DIST_GAUSS_ELLIPSOID, density=2.0, x0=5.0, radius=1.0,
                        radius_x=2.0, begin=0.0, end=10.0)
    assert dens(orc, p, 7.0, 0.5, 0.0) == pytest.approx(2.0 * math.exp(-1.0 - 0.25), rel=1e-14)
    assert dens(orc, p, 5.0, 4.1, 0.0) == 0.0                              # arg > 16
    q = density_profile(distribution=abi.DIST_COS_GAUSS, density=1.0, x0=5.0, radius=0.5,
                        radius_x=1.0, begin=0.0, end=20.0, plateau_end=20.0)
    assert dens(orc, q, 5.0) == pytest.approx(1.0, rel=1e-15)
    # x < x0 has no front factor
    a = -0.5
    want = 0.5 * (1 + math.cos(math.sqrt(PI_REF / 2.) * a)) * math.exp(-0.5)
    assert dens(orc, q, 4.5, 0.5, 0.0) == pytest.approx(want, rel=1e-14)
    r = density_profile(distribution=abi.DIST_TANH_STEP, density=3.0, x0=2.0, radius=1.0,
                        radius_x=0.5, begin=0.0, end=10.0)
    assert dens(orc, r, 2.0, 0.2, 0.2) == pytest.approx(1.5, rel=1e-15)
    assert dens(orc, r, 2.0, 1.0, 0.2) == 0.0


def test_ramps(orc):
    e = density_profile(distribution=abi.DIST_EXPONENTIAL, density=1.0, delta=1.0, begin=0.0,
                        plateau_begin=2.0, plateau_end=6.0, end=8.0)
    assert dens(orc, e, 4.0) == pytest.approx(1.5, rel=1e-15)
    assert dens(orc, e, 1.0) == pytest.approx(0.5 * (1 + math.tanh(2.5)), rel=1e-15)
    assert dens(orc, e, 7.0) == pytest.approx(2.0 * 0.5, rel=1e-15)
    s = density_profile(distribution=abi.DIST_LINEAR_STEP, density=1.0, delta=0.5, begin=0.0,
                        plateau_begin=2.0, plateau_end=6.0, end=8.0)
    assert dens(orc, s, 1.0) == 1.0
    assert dens(orc, s, 4.0) == pytest.approx(1.25, rel=1e-15)
    assert dens(orc, s, 7.0) == pytest.approx(1.5, rel=1e-15)
    g = density_profile(distribution=abi.DIST_GRADIENT, density=1.0, delta=2.0, begin=0.0,
                        plateau_begin=2.0, plateau_end=6.0, end=8.0)
    assert dens(orc, g, 4.0) == pytest.approx(math.exp(1.0), rel=1e-15)
    assert dens(orc, g, 1.0) == pytest.approx(0.5, rel=1e-15)


def test_periodic_and_rod(orc):
    p = density_profile(distribution=abi.DIST_PERIODIC, density=1.0, density1=4.0, begin=0.0,
                        plateau_begin=1.0, plateau_end=100.0, end=110.0, xperiod=1.0, delta=0.25,
                        scale=0.5)
    assert dens(orc, p, 5.9) == 4.0
    assert dens(orc, p, 5.5) == 1.0
    assert dens(orc, p, 0.5) == pytest.approx(math.exp(-1.0), rel=1e-15)
    rod = density_profile(distribution=abi.DIST_ROD, density=2.0, begin=0.0, end=10.0,
                          radius=0.5, yperiod=2.0)
    assert dens(orc, rod, 1.0, 0.4, 0.0) == 2.0
    assert dens(orc, rod, 1.0, 0.6, 0.0) == 0.0
    assert dens(orc, rod, 1.0, 4.3, 0.0) == 2.0                            # 4.3 -> 0.3
    inv = density_profile(distribution=abi.DIST_ROD, density=2.0, begin=0.0, end=10.0,
                          radius=1.0, radius_y=-0.5, radius_z=-0.5)
    assert dens(orc, inv, 1.0, 0.2, 0.0) == 0.0                            # inside a hole
    assert dens(orc, inv, 1.0, 0.7, 0.0) == 2.0


def test_curved_channel(orc):
    p = density_profile(distribution=abi.DIST_CURVED_CHANNEL, density=1.0, delta=1.0, radius=1.0,
                        y0=0.0, xperiod=4.0, y_curvature=0.5, begin=0.0, plateau_begin=0.0,
                        plateau_end=100.0, end=200.0, curvature_begin=0.0, curvature_end=50.0)
    x = 1.0                                                               # sin(pi/2) = 1
    yc = 0.5 * math.sin(2. * PI_REF * x / 4.0)
    assert dens(orc, p, x, yc, 0.0) == pytest.approx(0.0, abs=1e-15)     # channel centre
    assert dens(orc, p, 60.0, 0.0, 0.0) == pytest.approx(0.0, abs=1e-15)  # past the curvature


def test_front_weights_follow_the_profile(orc):
    from tertia_b200 import workload as wl
    cfg = wl.small_config(n=32, layers=8)
    o = orc.Oracle(cfg)
    p = density_profile(distribution=abi.DIST_EMPTY_CHANNEL, density=2.0, delta=0.0, radius=0.3,
                        begin=0.0, plateau_begin=cfg.hx * cfg.nx + 1.0, plateau_end=1e9, end=1e10)
    o.set_density_profile(p)
    o.set_phase(0.5)
    w = o.front_weights().reshape(cfg.nz, cfg.ny)
    x = cfg.hx * cfg.nx + 0.5
    ramp = (x - 0.0) / (cfg.hx * cfg.nx + 1.0)
    j = np.arange(cfg.ny)
    k = np.arange(cfg.nz)
    yy = cfg.hy * j[None, :] - cfg.ny * cfg.hy / 2
    zz = cfg.hz * k[:, None] - cfg.nz * cfg.hz / 2
    inside = yy ** 2 + zz ** 2 < 0.09
    assert inside.sum() > 4
    assert np.all(w[inside] == 0.0)
    np.testing.assert_allclose(w[~inside], 2.0 * ramp / cfg.ppc, rtol=1e-14)
    o.set_density_profile(None)
    np.testing.assert_allclose(o.front_weights(), cfg.plasma_density / cfg.ppc, rtol=1e-15)
    o.close()
