"""Python mirror of the reference's Mesh call surface over the C ABI.

Method names follow the reference (mesh.h:55-76, step.cpp:24):
MoveAllSplitLayers, MoveSplitLayer, GuessFieldsHydroLinLayerSplit,
MoveParticlesLayerSplit, IterateFieldsHydroLinLayerSplit, MoveBeamParticles,
Step; the snake_case names are the same calls.  Every call raises QsError
carrying the library's qs_status where the reference would have exit()ed.
All arrays are host numpy arrays; the device copies live in the handle.
"""
from __future__ import annotations

import ctypes as C
import functools

import numpy as np

from . import abi
from .abi import QsConfig, QsError, load_library


def _p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _changes_state(f):
    """Count the calls that change the box's state (beam, plasma, fields,
    checkpoints): `Mesh.state_version` lets a caller that kept results of an
    earlier call (the autograd wrapper) see that the mesh has moved on."""
    @functools.wraps(f)
    def g(self, *a, **k):
        self.state_version += 1
        return f(self, *a, **k)
    return g


class Mesh:
    """One quasi-static box on one GPU (a qs_handle)."""

    def __init__(self, cfg: QsConfig):
        self._L = load_library()
        self.cfg = cfg.copy()
        h = C.c_void_p()
        st = self._L.qs_create(C.byref(self.cfg), C.byref(h))
        if st != 0:
            raise QsError(st, self._L.qs_last_error(None).decode())
        self._h = h
        self.plane = cfg.ny * cfg.nz
        self.state_version = 0

    # -------------------------------------------------------------- plumbing
    def _chk(self, st: int, what: str):
        if st != 0:
            msg = self._L.qs_last_error(self._h).decode() if self._h else ""
            raise QsError(st, f"{what}: {msg}")

    def close(self):
        if getattr(self, "_h", None):
            self._L.qs_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        self._chk(self._L.qs_sync(self._h), "qs_sync")

    def stream(self) -> int:
        s = C.c_void_p()
        self._chk(self._L.qs_get_stream(self._h, C.byref(s)), "qs_get_stream")
        return s.value or 0

    def kernel_launches(self) -> int:
        return int(self._L.qs_kernel_launches(self._h))

    def profile_enable(self, on: bool = True):
        self._chk(self._L.qs_profile_enable(self._h, int(on)), "qs_profile_enable")

    def profile_read(self) -> dict:
        n = len(abi.KERNEL_CLASSES)
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int64)
        self._chk(self._L.qs_profile_read(self._h, _p(ms, C.c_double), _p(cnt, C.c_int64), n),
                  "qs_profile_read")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(abi.KERNEL_CLASSES)}

    # -------------------------------------------------------------- state
    @_changes_state
    def load_beam(self, b: dict):
        n = len(b["x"])
        ii, jj, kk = (_i32(b[k]) for k in "ijk")
        f = [_f64(b[k]) for k in ("x", "y", "z", "px", "py", "pz", "w")]
        self._chk(self._L.qs_load_beam(self._h, n, _p(ii, C.c_int32), _p(jj, C.c_int32),
                                       _p(kk, C.c_int32), *[_p(a, C.c_double) for a in f]),
                  "qs_load_beam")

    def get_beam(self) -> dict:
        n = int(self._L.qs_beam_count(self._h))
        out = {k: np.empty(n, dtype=np.int32) for k in "ijk"}
        out.update({k: np.empty(n) for k in ("x", "y", "z", "px", "py", "pz", "w")})
        self._chk(self._L.qs_get_beam(self._h, n, *[_p(out[k], C.c_int32) for k in "ijk"],
                                      *[_p(out[k], C.c_double) for k in
                                        ("x", "y", "z", "px", "py", "pz", "w")]),
                  "qs_get_beam")
        return out

    @_changes_state
    def load_front_plasma(self, p: dict):
        n = len(p["y"])
        cell = _i32(p["cell"])
        f = [_f64(p[k]) for k in ("y", "z", "px", "py", "pz", "w")]
        self._chk(self._L.qs_load_front_plasma(self._h, n, _p(cell, C.c_int32),
                                               *[_p(a, C.c_double) for a in f]),
                  "qs_load_front_plasma")

    @_changes_state
    def seed_front_plasma(self, step: int):
        self._chk(self._L.qs_seed_front_plasma(self._h, int(step)), "qs_seed_front_plasma")

    @_changes_state
    def set_density_profile(self, prof):
        """Specie density profile (abi.QsDensityProfile, or None for the
        uniform cfg.plasma_density)."""
        self._chk(self._L.qs_set_density_profile(self._h, C.byref(prof) if prof is not None
                                                 else None), "qs_set_density_profile")

    def plasma_density(self, x: float, y: float, z: float) -> float:
        out = C.c_double()
        self._chk(self._L.qs_plasma_density(self._h, x, y, z, C.byref(out)), "qs_plasma_density")
        return out.value

    @_changes_state
    def set_phase(self, phase: float):
        self._chk(self._L.qs_set_phase(self._h, float(phase)), "qs_set_phase")

    def get_phase(self) -> float:
        out = C.c_double()
        self._chk(self._L.qs_get_phase(self._h, C.byref(out)), "qs_get_phase")
        return out.value

    def pack_size(self) -> int:
        """Doubles in the hand-off buffer: 12 ny nz + 12 Np."""
        return int(self._L.qs_layer_pack_size(self._h))

    def pack_layer(self, out: np.ndarray | None = None) -> np.ndarray:
        """PackLayer: the tail layer and the plasma in flight after a march, in
        the reference's hand-off buffer layout.  `out` (contiguous float64 of
        pack_size() values, pinned host memory for the fastest copy) is filled
        in place when given."""
        n = self.pack_size()
        if out is None:
            out = np.empty(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"pack_layer: out must be contiguous float64 of {n} values")
        self._chk(self._L.qs_pack_layer(self._h, _p(out, C.c_double), n), "qs_pack_layer")
        return out

    @_changes_state
    def unpack_layer(self, buf):
        """UnpackLayer: the received layer is the front of the next march."""
        b = _f64(buf)
        self._chk(self._L.qs_unpack_layer(self._h, _p(b, C.c_double), b.size), "qs_unpack_layer")

    @_changes_state
    def clear_front_layer(self):
        self._chk(self._L.qs_clear_front_layer(self._h), "qs_clear_front_layer")

    def get_plasma(self) -> dict:
        n = int(self._L.qs_plasma_count(self._h))
        out = {"cell": np.empty(n, dtype=np.int32)}
        out.update({k: np.empty(n) for k in ("y", "z", "px", "py", "pz", "w")})
        self._chk(self._L.qs_get_plasma(self._h, n, _p(out["cell"], C.c_int32),
                                        *[_p(out[k], C.c_double) for k in
                                          ("y", "z", "px", "py", "pz", "w")]), "qs_get_plasma")
        return out

    def _plane(self):
        return np.empty(self.plane, dtype=np.float64)

    def _shape(self, a):
        return a.reshape(self.cfg.nz, self.cfg.ny)

    @_changes_state
    def set_layer(self, which: int, field: int, data):
        d = _f64(data).reshape(-1)
        self._chk(self._L.qs_set_layer(self._h, which, field, _p(d, C.c_double)), "qs_set_layer")

    def get_layer(self, which: int, field: int):
        out = self._plane()
        self._chk(self._L.qs_get_layer(self._h, which, field, _p(out, C.c_double)), "qs_get_layer")
        return self._shape(out)

    def get_field3d(self, field: int, layer: int):
        out = self._plane()
        self._chk(self._L.qs_get_field3d(self._h, field, layer, _p(out, C.c_double)),
                  "qs_get_field3d")
        return self._shape(out)

    @_changes_state
    def set_beam_currents(self, field: int, layer: int, data):
        d = _f64(data).reshape(-1)
        self._chk(self._L.qs_set_beam_currents(self._h, field, layer, _p(d, C.c_double)),
                  "qs_set_beam_currents")

    def get_beam_currents(self, field: int, layer: int):
        out = self._plane()
        self._chk(self._L.qs_get_beam_currents(self._h, field, layer, _p(out, C.c_double)),
                  "qs_get_beam_currents")
        return self._shape(out)

    def onaxis_ex(self):
        out = np.empty(self.cfg.nx)
        self._chk(self._L.qs_get_onaxis_ex(self._h, _p(out, C.c_double)), "qs_get_onaxis_ex")
        return out

    def psi(self):
        out = np.empty(self.cfg.nx)
        self._chk(self._L.qs_get_psi(self._h, _p(out, C.c_double)), "qs_get_psi")
        return out

    def charge_sums(self) -> dict:
        """FP64 per-layer sums over the transverse plane (qs_get_charge_sums):
        rho (nx) of the corrected density, jx (nx) of the full push's Jx
        deposit, rho_beam (nx + 1) of the beam's RhoBeam."""
        r, j, b = np.empty(self.cfg.nx), np.empty(self.cfg.nx), np.empty(self.cfg.nx + 1)
        self._chk(self._L.qs_get_charge_sums(self._h, _p(r, C.c_double), _p(j, C.c_double),
                                             _p(b, C.c_double)), "qs_get_charge_sums")
        return {"rho": r, "jx": j, "rho_beam": b}

    def save_fields(self, path: str):
        """Mesh::Save's field file (save.cpp:520-838) as a QSF1 file at
        `path` (read it with tertia_b200.fields_io.read_qsf)."""
        self._chk(self._L.qs_save_fields(self._h, str(path).encode()), "qs_save_fields")

    def save_movie_frame(self, path: str):
        """Mesh::SaveCadrMovie2's central slices as a QSF1 file at `path`."""
        self._chk(self._L.qs_save_movie_frame(self._h, str(path).encode()),
                  "qs_save_movie_frame")

    # -------------------------------------------------------------- the path
    @_changes_state
    def step(self):
        self._chk(self._L.qs_step(self._h), "qs_step")

    @_changes_state
    def move_beam_particles(self):
        self._chk(self._L.qs_move_beam_particles(self._h), "qs_move_beam_particles")

    @_changes_state
    def move_all_split_layers(self):
        self._chk(self._L.qs_move_all_split_layers(self._h), "qs_move_all_split_layers")

    @_changes_state
    def begin_march(self):
        self._chk(self._L.qs_begin_march(self._h), "qs_begin_march")

    @_changes_state
    def layer_begin(self, i: int, s: int = 0):
        self._chk(self._L.qs_layer_begin(self._h, i, s), "qs_layer_begin")

    @_changes_state
    def move_split_layer(self, i: int, s: int = 0):
        self._chk(self._L.qs_move_split_layer(self._h, i, s), "qs_move_split_layer")

    @_changes_state
    def guess_fields(self, i: int, s: int = 0):
        self._chk(self._L.qs_guess_fields(self._h, i, s), "qs_guess_fields")

    @_changes_state
    def move_particles_layer(self, i: int, s: int, full: int):
        self._chk(self._L.qs_move_particles_layer(self._h, i, s, int(full)),
                  "qs_move_particles_layer")

    @_changes_state
    def iterate_fields(self, i: int, s: int, it: int) -> float:
        e = C.c_double(0.0)
        self._chk(self._L.qs_iterate_fields(self._h, i, s, it, C.byref(e)), "qs_iterate_fields")
        return e.value

    @_changes_state
    def layer_end(self, i: int, s: int = 0):
        self._chk(self._L.qs_layer_end(self._h, i, s), "qs_layer_end")

    def transform2d(self, x, kind_z: int, kind_y: int):
        x = _f64(x)
        nz, ny = x.shape[-2:]
        if (nz, ny) != (self.cfg.nz, self.cfg.ny):
            raise ValueError("planes must be nz x ny")
        batch = int(np.prod(x.shape[:-2])) if x.ndim > 2 else 1
        out = np.empty_like(x)
        self._chk(self._L.qs_transform2d(self._h, kind_z, kind_y, batch, _p(x, C.c_double),
                                         _p(out, C.c_double)), "qs_transform2d")
        return out

    def transform2d_dev(self, kind_z: int, kind_y: int, batch: int, d_in: int, d_out: int):
        """qs_transform2d_dev on device pointers (float, or double in FP64),
        enqueued on the handle's stream."""
        self._chk(self._L.qs_transform2d_dev(self._h, kind_z, kind_y, batch, C.c_void_p(d_in),
                                             C.c_void_p(d_out)), "qs_transform2d_dev")

    @_changes_state
    def step_host(self, b: dict, want_beam: bool = True, out: dict | None = None):
        """One step through host buffers (beam in, beam and on-axis Ex out).
        `out` may supply the output arrays (e.g. views of pinned memory)."""
        n = len(b["x"])
        ii, jj, kk = (_i32(b[k]) for k in "ijk")
        f = [_f64(b[k]) for k in ("x", "y", "z", "px", "py", "pz", "w")]
        if out is None:
            out = {k: np.empty(n, dtype=np.int32) for k in "ijk"}
            out.update({k: np.empty(n) for k in ("x", "y", "z", "px", "py", "pz")})
        ex = np.empty(self.cfg.nx)
        outs_i = [_p(out[k], C.c_int32) if want_beam else None for k in "ijk"]
        outs_f = [_p(out[k], C.c_double) if want_beam else None
                  for k in ("x", "y", "z", "px", "py", "pz")]
        self._chk(self._L.qs_step_host(self._h, n, _p(ii, C.c_int32), _p(jj, C.c_int32),
                                       _p(kk, C.c_int32), *[_p(a, C.c_double) for a in f],
                                       *outs_i, *outs_f, _p(ex, C.c_double)), "qs_step_host")
        out["w"] = f[-1]
        return (out if want_beam else None), ex

    # -------------------------------------------------------------- adjoint
    @_changes_state
    def adjoint_checkpoints(self, every: int):
        """Store layer checkpoints every `every` layers in the next marches."""
        self._chk(self._L.qs_adjoint_checkpoints(self._h, int(every)), "qs_adjoint_checkpoints")

    @_changes_state
    def adjoint(self, dloss_donaxis_ex) -> np.ndarray:
        """d loss / d (beam weight) of every beam particle, given d loss / d
        (on-axis Ex of each layer) for the last march."""
        d = _f64(dloss_donaxis_ex).reshape(-1)
        if d.size != self.cfg.nx:
            raise ValueError("dloss_donaxis_ex needs one entry per layer")
        out = np.empty(int(self._L.qs_beam_count(self._h)))
        self._chk(self._L.qs_adjoint(self._h, _p(d, C.c_double), _p(out, C.c_double)),
                  "qs_adjoint")
        return out

    # reference-named aliases (mesh.h:55-76, step.cpp:24)
    Step = step
    MoveBeamParticles = move_beam_particles
    MoveAllSplitLayers = move_all_split_layers
    MoveSplitLayer = move_split_layer
    GuessFieldsHydroLinLayerSplit = guess_fields

    def MoveParticlesLayerSplit(self, iLayer, iSplit, iFullStep, part=1.0):
        if part != 1.0:
            raise QsError(abi.QS_ERR_UNSUPPORTED, "part != 1 is not used by the split march")
        self.move_particles_layer(iLayer, iSplit, iFullStep)

    def IterateFieldsHydroLinLayerSplit(self, iLayer, iSplit, N_iter):
        return self.iterate_fields(iLayer, iSplit, N_iter)
