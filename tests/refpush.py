"""Vectorised numpy restatement of one plasma sub-push (test helper).

An independent second restatement of MoveParticlesLayerSplit
(movepart_splitlayer.cpp:882-1522, NGP, single sub-step |dy|,|dz| <= 1)
used to cross-check the C++ oracle: numpy ufuncs are IEEE without
contraction, so the two agree bit for bit.
"""
import numpy as np


def push_ngp(cfg, cell, y, z, px, py, pz, w, P, C):
    My, Mz = cfg.ny, cfg.nz
    hx = cfg.hx / cfg.nx_split
    j = cell % My
    k = cell // My
    g = lambda F, c: F[c].reshape(-1)[cell]
    ex = 0.5 * (g(P, 0) + g(C, 0)); ey = 0.5 * (g(P, 1) + g(C, 1)); ez = 0.5 * (g(P, 2) + g(C, 2))
    bx = 0.5 * (g(P, 3) + g(C, 3)); by = 0.5 * (g(P, 4) + g(C, 4)); bz = 0.5 * (g(P, 5) + g(C, 5))
    gammap = np.sqrt(1. + px * px + py * py + pz * pz)
    Vx = px / gammap
    Vxp, Vyp, Vzp = Vx, py / gammap, pz / gammap
    q2m = cfg.plasma_q2m
    sE = q2m * hx / 2.
    ex = ex * sE; ey = ey * sE; ez = ez * sE
    px = px + ex / (1. - Vx); py = py + ey / (1. - Vx); pz = pz + ez / (1. - Vx)
    gamma = np.sqrt(1. + px * px + py * py + pz * pz)
    gr = 1. / gamma
    bx = bx + cfg.bx_ext; by = by + cfg.by_ext; bz = bz + cfg.bz_ext
    bx = bx * gr * q2m / (1. - Vx) * hx / 2.
    by = by * gr * q2m / (1. - Vx) * hx / 2.
    bz = bz * gr * q2m / (1. - Vx) * hx / 2.
    co = 2. / (1. + (bx * bx) + (by * by) + (bz * bz))
    p3x = (py * bz - pz * by + px) * co
    p3y = (pz * bx - px * bz + py) * co
    p3z = (px * by - py * bx + pz) * co
    pxn = p3y * bz - p3z * by; pyn = p3z * bx - p3x * bz; pzn = p3x * by - p3y * bx
    px = px + (ex / (1. - Vx) + pxn); py = py + (ey / (1. - Vx) + pyn); pz = pz + (ez / (1. - Vx) + pzn)
    gamma = np.sqrt(1. + px * px + py * py + pz * pz)
    Vxm, Vym, Vzm = px / gamma, py / gamma, pz / gamma
    Vx = 0.5 * (Vxm + Vxp); Vy = 0.5 * (Vym + Vyp); Vz = 0.5 * (Vzm + Vzp)
    djx = w * cfg.plasma_djx0 * Vxm * (1. / (1. - Vx))
    djy = w * cfg.plasma_djy0 * Vym * (1. / (1. - Vx))
    djz = w * cfg.plasma_djz0 * Vzm * (1. / (1. - Vx))
    drho = w * cfg.plasma_drho0 * (1. / (1. - Vx))
    dy = Vy * hx / cfg.hy / (1. - Vx)
    dz = Vz * hx / cfg.hz / (1. - Vx)
    assert np.all(np.abs(dy) <= 1) and np.all(np.abs(dz) <= 1)
    yt = y + (dy * 1. + j)
    zt = z + (dz * 1. + k)
    yt = np.where(yt > My, yt - My, yt); yt = np.where(yt < 0, yt + My, yt)
    zt = np.where(zt > Mz, zt - Mz, zt); zt = np.where(zt < 0, zt + Mz, zt)
    jj = yt.astype(np.int64); kk = zt.astype(np.int64)
    yt = yt - jj; zt = zt - kk
    dcell = (jj % My) + My * (kk % Mz)
    dep = np.zeros((4, My * Mz))
    for q, v in enumerate((djx, djy, djz, drho)):
        np.add.at(dep[q], dcell, v)
    return dict(px=px, py=py, pz=pz, y=yt, z=zt, dep=dep.reshape(4, Mz, My), dep_cell=dcell)
