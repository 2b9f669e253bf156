"""Known answer: the linear response of a uniform plasma.

The Guess step's per-mode map of a source-free mode (no beam) is, on
(Rho, Ex), the matrix [[P, a], [b, P]] with the analytic propagator
P = (4 - d hx^2) / (4 + d hx^2) (movefieldshydrolinlayersplit.cpp:843-849),
a = 4 hx (k^2 + d) / D, b = -4 d hx / ((k^2 + d) D), D = 4 + d hx^2.  Since
P^2 - a b = 1 it is a rotation by theta = arccos(P) per layer, the discrete
plasma oscillation (theta = 2 atan(hx sqrt(d) / 2)).

So behind a weak driver the on-axis wake of the full march (push, deposit,
corrector) obeys the three-term recurrence of that rotation,
Ex(i-1) + Ex(i+1) = 2 cos(theta) Ex(i), up to corrections of the order of
the driver's density n_b/n_0 (measured in the oracle: theta of the march
exceeds the propagator's by 0.04 n_b/n_0 relative, 4e-6 at n_b/n_0 = 1e-4).
Checked for the oracle's per-mode map, for the oracle's march and for the
GPU path in FP64 and FP32.
"""
import numpy as np
import pytest

from tertia_b200 import workload as wl
from tertia_b200.abi import PRECISIONS


def propagator(cfg, d=1.0):
    return (4.0 - d * cfg.hx ** 2) / (4.0 + d * cfg.hx ** 2)


def weak_wake_case():
    """A 32 x 32 box of 640 layers, cold uniform plasma (d = 1), and a wide
    weak driver (sigma_r 2, sigma_xi 0.5, n_b/n_0 1e-4)."""
    cfg = wl.small_config(n=32, layers=640, h=0.2, hx=0.05)
    spec = wl.BeamSpec(20000, sigma_r=2.0, sigma_xi=0.5, nb_over_n0=1e-4, seed=3)
    beam = wl.sample_beam(cfg, spec, driver_sigma_xi=1.0)
    return cfg, beam


def march_cos_theta(cfg, ex):
    """cos(theta) of the on-axis wake behind the driver, from the three-term
    recurrence (median over the layers where |Ex| is not near a node)."""
    xc = wl.driver_center_x(cfg, 1.0)
    e = np.asarray(ex)[: int((xc - 3.0) / cfg.hx)]
    ratio = (e[:-2] + e[2:]) / (2.0 * e[1:-1])
    sel = np.abs(e[1:-1]) > 0.3 * np.abs(e).max()
    assert sel.sum() > 100
    return float(np.median(ratio[sel]))


def test_predictor_map_is_the_rotation_of_the_propagator(oracle_lib):
    """Oracle per-mode map with no beam and no currents: (Rho, Ex) of every
    mode rotate by theta with cos(theta) = P; the scaled energy is kept."""
    ny = nz = 16
    hx, d, ylen, zlen = 0.05, 1.0, 3.2, 3.2
    rng = np.random.default_rng(1)
    n = ny * nz
    P = {k: np.zeros(n) for k in ("RhoP", "JxP", "JyP", "JzP", "ExP", "EyP", "EzP")}
    P["RhoP"] = rng.standard_normal(n)
    P["ExP"] = rng.standard_normal(n)
    beam = {k: np.zeros(n) for k in ("RhoBeam", "RhoBeamP", "JxBeam")}
    out = oracle_lib.predictor_modes(ny, nz, hx, d, ylen, zlen, P, beam)
    j, k = np.meshgrid(np.arange(ny), np.arange(nz))
    ky = np.pi / ylen * (j.ravel() + 0.5)
    kz = np.pi / zlen * (k.ravel() + 0.5)
    k2 = ky ** 2 + kz ** 2
    D = 4.0 + d * hx ** 2
    p = (4.0 - d * hx ** 2) / D
    a = 4.0 * hx * (k2 + d) / D
    b = -4.0 * d * hx / ((k2 + d) * D)
    np.testing.assert_allclose(p * p - a * b, 1.0, rtol=0, atol=1e-14)
    np.testing.assert_allclose(out["Rho"], p * P["RhoP"] + a * P["ExP"], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(out["Ex"], b * P["RhoP"] + p * P["ExP"], rtol=1e-13, atol=1e-13)
    e0 = P["RhoP"] ** 2 / a - P["ExP"] ** 2 / b
    e1 = out["Rho"] ** 2 / a - out["Ex"] ** 2 / b
    np.testing.assert_allclose(e1, e0, rtol=1e-12)


def test_oracle_march_follows_the_propagator(oracle_lib):
    cfg, beam = weak_wake_case()
    o = oracle_lib.Oracle(cfg)
    o.load_beam(beam)
    o.load_front_plasma(wl.front_plasma(cfg, thermal=False))
    o.step()
    c = march_cos_theta(cfg, o.onaxis_ex())
    P = propagator(cfg)
    theta, theta_m = np.arccos(P), np.arccos(c)
    assert abs(theta_m / theta - 1.0) < 1e-5, (theta_m, theta)
    # the discrete plasma frequency, not the continuum one: theta = 2 atan(hx/2)
    assert abs(theta - 2.0 * np.arctan(cfg.hx / 2.0)) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-5), ("fp32", 1e-4)])
def test_gpu_march_follows_the_propagator(prec, tol):
    from tertia_b200.mesh import Mesh
    cfg, beam = weak_wake_case()
    cfg.precision = PRECISIONS[prec]
    with Mesh(cfg) as m:
        m.load_beam(beam)
        m.load_front_plasma(wl.front_plasma(cfg, thermal=False))
        m.step()
        c = march_cos_theta(cfg, m.onaxis_ex())
    theta, theta_m = np.arccos(propagator(cfg)), np.arccos(c)
    assert abs(theta_m / theta - 1.0) < tol, (theta_m, theta)
