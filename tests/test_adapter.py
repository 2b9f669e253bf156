"""The C++ adapter of INTEGRATION.md (include/mesh_qs.h, class MeshQS with the
reference's Mesh method names) compiled against libqsb200.so: it builds and
links on the host, and on the GPU one beam step of the c0 deck through it
gives the same on-axis field as the Python binding of the same library."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "adapter", "run_step.cpp")


def build_driver(out_dir):
    from tertia_b200 import build as qb
    lib = qb.build()
    exe = os.path.join(out_dir, "run_step")
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           SRC, "-o", exe, "-L", os.path.dirname(lib), "-lqsb200",
           f"-Wl,-rpath,{os.path.dirname(lib)}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_adapter_compiles_and_links(tmp_path):
    exe = build_driver(str(tmp_path))
    assert os.path.exists(exe)


def write_inputs(path, cfg, beam, front, steps):
    iv = np.array([cfg.ny, cfg.nz, cfg.nx, cfg.n_iter, cfg.nx_split, cfg.ppc, cfg.precision,
                   cfg.shape, steps], dtype=np.int32)
    dv = np.array([cfg.hx, cfg.hy, cfg.hz, cfg.ts, cfg.plasma_density, cfg.wavelength])
    with open(path, "wb") as f:
        iv.tofile(f)
        dv.tofile(f)
        np.array([len(beam["x"])], dtype=np.int64).tofile(f)
        for k in "ijk":
            np.asarray(beam[k], dtype=np.int32).tofile(f)
        for k in ("x", "y", "z", "px", "py", "pz", "w"):
            np.asarray(beam[k], dtype=np.float64).tofile(f)
        np.array([len(front["y"])], dtype=np.int64).tofile(f)
        np.asarray(front["cell"], dtype=np.int32).tofile(f)
        for k in ("y", "z", "px", "py", "pz", "w"):
            np.asarray(front[k], dtype=np.float64).tofile(f)


@pytest.mark.gpu
def test_adapter_runs_a_c0_step(tmp_path):
    from tertia_b200 import workload as wl
    from tertia_b200.mesh import Mesh
    exe = build_driver(str(tmp_path))
    w = wl.make_workload("c0")      # 128 x 128 x 256, FP64, CIC
    cfg = w.cfg
    beam = wl.workload_beam(w)
    front = wl.front_plasma(cfg, seed=1, thermal=False)
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "ex.bin")
    write_inputs(inp, cfg, beam, front, steps=1)
    r = subprocess.run([exe, inp, out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ex_cpp = np.fromfile(out, dtype=np.float64)
    with Mesh(cfg) as m:
        m.load_beam(beam)
        m.load_front_plasma(front)
        m.move_beam_particles()
        m.move_all_split_layers()
        ex_py = m.onaxis_ex()
    assert ex_cpp.shape == ex_py.shape
    assert np.max(np.abs(ex_py)) > 1e-2
    err = np.linalg.norm(ex_cpp - ex_py) / np.linalg.norm(ex_py)
    assert err < 1e-12, err
