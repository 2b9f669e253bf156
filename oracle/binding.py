"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the checker of the GPU path: tests, the smoke check and the
CPU-baseline leg of bench.py load it; the product never does.  It restates
the reference's live FP64 host path (movepart_splitlayer.cpp,
movefieldshydrolinlayersplit.cpp, movebeam.cpp); see qs_oracle.h for the
parity status.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile oracle/liboracle.so with the committed Makefile."""
    if force or not os.path.exists(_LIB_PATH) or _stale():
        subprocess.run(["make", "-C", _HERE, "ORACLE_CXX=g++", "-B" if force else "liboracle.so"],
                       check=True, capture_output=True)
    return _LIB_PATH


REF_LIB_PATH = os.path.join(_HERE, "_ref", "libref_linearized.so")
# the reference checkout the recipe compiles from: QS_REFERENCE_DIR, else the
# path where this build environment mounts it
REFERENCE = os.environ.get("QS_REFERENCE_DIR", "/root/reference")


REFPIN_LIB_PATH = os.path.join(_HERE, "_ref", "librefpin.so")


def build_reference() -> str | None:
    """Compile, where the reference checkout is present, its CUDA twins of the
    per-mode spectral maps and its host plasma push and beam push into
    oracle/_ref/; returns the spectral-map library path or None."""
    if os.path.isdir(os.path.join(REFERENCE, "CUDA_WRAP")):
        subprocess.run(["make", "-C", _HERE, "ref", "refpin", f"REFERENCE={REFERENCE}"],
                       check=True, capture_output=True)
    return REF_LIB_PATH if os.path.exists(REF_LIB_PATH) else None


def refpin_lib():
    """The reference's own host plasma push and beam push (oracle/ref_pin.cpp
    over the reference files), or None when they were not built."""
    if not os.path.exists(REFPIN_LIB_PATH):
        return None
    from tertia_b200.abi import QsConfig
    L = C.CDLL(REFPIN_LIB_PATH)
    L.refpin_push_layer.argtypes = [C.POINTER(QsConfig), C.c_int64, _i32p] + [_f64p] * 6 + [
        _f64p, _f64p, _f64p, _i32p, C.c_int]
    L.refpin_beam_push.argtypes = [C.POINTER(QsConfig), C.c_int64] + [_i32p] * 3 + [_f64p] * 7 + [
        _f64p, _f64p]
    return L


def reference_lib():
    """The built reference twins (ref_linearized_loop, ref_linearized_iterate_loop)
    or None when they were not built."""
    if not os.path.exists(REF_LIB_PATH):
        return None
    L = C.CDLL(REF_LIB_PATH)
    for name in ("ref_linearized_loop", "ref_linearized_iterate_loop"):
        getattr(L, name).argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.POINTER(C.c_void_p)]
    return L


def predictor_modes(ny, nz, hx, dens, ylen, zlen, P, beam):
    """Oracle per-mode predictor.  P: dict RhoP, JxP, JyP, JzP, ExP, EyP, EzP;
    beam: dict RhoBeam, RhoBeamP, JxBeam (flat float64 arrays of ny*nz).
    Returns dict Rho, Ex, Ey, Ez, Jx, Jy, Jz, Bx, By, Bz."""
    out = {k: np.empty(ny * nz) for k in ("Rho", "Ex", "Ey", "Ez", "Jx", "Jy", "Jz", "Bx",
                                          "By", "Bz")}
    a = [np.ascontiguousarray(P[k], dtype=np.float64) for k in
         ("RhoP", "JxP", "JyP", "JzP", "ExP", "EyP", "EzP")]
    b = [np.ascontiguousarray(beam[k], dtype=np.float64) for k in ("RhoBeam", "RhoBeamP",
                                                                   "JxBeam")]
    lib().qso_predictor_modes(ny, nz, hx, dens, ylen, zlen, *a, *b,
                              *[out[k] for k in ("Rho", "Ex", "Ey", "Ez", "Jx", "Jy", "Jz", "Bx",
                                                 "By", "Bz")])
    return out


def corrector_modes(ny, nz, hx, dens, ylen, zlen, P, beam, J, rho_old):
    """Oracle per-mode corrector.  J: dict Jx, Jy, Jz of the C deposit;
    rho_old: the C-layer rho spectrum before the update.
    Returns dict Rho, Ex, Ey, Ez, Bx, By, Bz."""
    out = {k: np.empty(ny * nz) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")}
    out["Rho"] = np.array(rho_old, dtype=np.float64)
    a = [np.ascontiguousarray(P[k], dtype=np.float64) for k in
         ("RhoP", "JxP", "JyP", "JzP", "EyP", "EzP")]
    b = [np.ascontiguousarray(beam[k], dtype=np.float64) for k in ("RhoBeam", "RhoBeamP",
                                                                   "JxBeam")]
    j = [np.ascontiguousarray(J[k], dtype=np.float64) for k in ("Jx", "Jy", "Jz")]
    lib().qso_corrector_modes(ny, nz, hx, dens, ylen, zlen, *a, *b, *j,
                              *[out[k] for k in ("Rho", "Ex", "Ey", "Ez", "Bx", "By", "Bz")])
    return out


def _stale() -> bool:
    lib_t = os.path.getmtime(_LIB_PATH)
    srcs = [os.path.join(_HERE, "qs_oracle.cpp"), os.path.join(_HERE, "qs_oracle.h"),
            os.path.join(_HERE, "..", "include", "qsb200.h")]
    return any(os.path.getmtime(s) > lib_t for s in srcs if os.path.exists(s))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


def _declare(L):
    from tertia_b200.abi import QsConfig  # the shared config struct layout

    P = C.c_void_p
    L.qso_create.argtypes = [C.POINTER(QsConfig), C.POINTER(P)]
    L.qso_destroy.argtypes = [P]
    L.qso_destroy.restype = None
    L.qso_predictor_modes.argtypes = [C.c_int, C.c_int] + [C.c_double] * 4 + [_f64p] * 20
    L.qso_predictor_modes.restype = None
    L.qso_corrector_modes.argtypes = [C.c_int, C.c_int] + [C.c_double] * 4 + [_f64p] * 19
    L.qso_corrector_modes.restype = None
    L.qso_set_threads.argtypes = [C.c_int]
    L.qso_set_threads.restype = None
    L.qso_get_threads.restype = C.c_int
    L.qso_load_beam.argtypes = [P, C.c_int64] + [_i32p] * 3 + [_f64p] * 7
    L.qso_get_beam.argtypes = [P, C.c_int64] + [_i32p] * 3 + [_f64p] * 7
    L.qso_beam_count.argtypes = [P]
    L.qso_beam_count.restype = C.c_int64
    L.qso_load_front_plasma.argtypes = [P, C.c_int64, _i32p] + [_f64p] * 6
    L.qso_plasma_count.argtypes = [P]
    L.qso_plasma_count.restype = C.c_int64
    L.qso_get_plasma.argtypes = [P, C.c_int64, _i32p] + [_f64p] * 6
    for name in ("qso_set_layer", "qso_get_layer"):
        getattr(L, name).argtypes = [P, C.c_int, C.c_int, _f64p]
    for name in ("qso_get_field3d", "qso_set_beam_currents", "qso_get_beam_currents"):
        getattr(L, name).argtypes = [P, C.c_int, C.c_int, _f64p]
    L.qso_get_onaxis_ex.argtypes = [P, _f64p]
    L.qso_get_psi.argtypes = [P, _f64p]
    L.qso_set_field3d.argtypes = [P, C.c_int, C.c_int, _f64p]
    L.qso_get_charge_sums.argtypes = [P, _f64p, _f64p, _f64p]
    for name in ("qso_step", "qso_move_beam_particles", "qso_move_all_split_layers",
                 "qso_begin_march"):
        getattr(L, name).argtypes = [P]
    for name in ("qso_layer_begin", "qso_move_split_layer", "qso_guess_fields", "qso_layer_end"):
        getattr(L, name).argtypes = [P, C.c_int, C.c_int]
    L.qso_move_particles_layer.argtypes = [P, C.c_int, C.c_int, C.c_int]
    L.qso_iterate_fields.argtypes = [P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    from tertia_b200.abi import QsDensityProfile
    L.qso_density.argtypes = [C.POINTER(QsDensityProfile), C.c_double, C.c_double, C.c_double]
    L.qso_density.restype = C.c_double
    L.qso_set_density_profile.argtypes = [P, C.POINTER(QsDensityProfile)]
    L.qso_set_phase.argtypes = [P, C.c_double]
    L.qso_front_weights.argtypes = [P, _f64p]
    L.qso_layer_pack_size.argtypes = [P]
    L.qso_layer_pack_size.restype = C.c_int64
    L.qso_pack_layer.argtypes = [P, _f64p, C.c_int64]
    L.qso_unpack_layer.argtypes = [P, _f64p, C.c_int64]
    L.qso_dtt1d.argtypes = [C.c_int, C.c_int, _f64p, _f64p, C.c_int]
    L.qso_transform2d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_int]
    L.qso_push_layer_f64.argtypes = [C.POINTER(QsConfig), C.c_int64, _i32p] + [_f64p] * 9 + [
        _i32p, C.c_int, C.c_int]
    L.qso_push_layer_f32.argtypes = [C.POINTER(QsConfig), C.c_int64, _i32p] + [_f32p] * 9 + [
        _i32p, C.c_int, C.c_int]


class OracleError(RuntimeError):
    pass


def _check(st, what):
    if st != 0:
        raise OracleError(f"{what} failed with status {st}")


def set_threads(n: int):
    lib().qso_set_threads(int(n))


def dtt1d(x, kind: int, direct: bool = False):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    _check(lib().qso_dtt1d(x.size, kind, x, out, int(direct)), "qso_dtt1d")
    return out


def transform2d(x, kind_z: int, kind_y: int, direct: bool = False):
    """x: (..., nz, ny) planes; returns the unnormalised 2-D transform."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    nz, ny = x.shape[-2:]
    batch = int(np.prod(x.shape[:-2])) if x.ndim > 2 else 1
    out = np.empty_like(x)
    _check(lib().qso_transform2d(nz, ny, kind_z, kind_y, batch, x, out, int(direct)),
           "qso_transform2d")
    return out


def push_layer(cfg, cell, y, z, px, py, pz, w, P, C_, dep=None, full=False, precise=False,
               dtype=np.float64):
    """Kernel-level oracle of one plasma sub-push on arrays (see qs_oracle.h)."""
    n = len(y)
    conv = lambda a: np.ascontiguousarray(a, dtype=dtype)
    cell = np.ascontiguousarray(cell, dtype=np.int32).copy()
    y, z, px, py, pz = (conv(a).copy() for a in (y, z, px, py, pz))
    w = conv(w)
    P = conv(P)
    C_ = conv(C_)
    plane = cfg.ny * cfg.nz
    if dep is None:
        dep = np.zeros(4 * plane, dtype=dtype)
    else:
        dep = conv(dep).copy().reshape(-1)
    dep_cell = np.zeros(n, dtype=np.int32)
    fn = lib().qso_push_layer_f64 if dtype == np.float64 else lib().qso_push_layer_f32
    _check(fn(C.byref(cfg), n, cell, y, z, px, py, pz, w, P.reshape(-1), C_.reshape(-1), dep,
              dep_cell, int(full), int(precise)), "qso_push_layer")
    return dict(cell=cell, y=y, z=z, px=px, py=py, pz=pz, dep=dep.reshape(4, cfg.nz, cfg.ny),
                dep_cell=dep_cell)


def density(prof, x: float, y: float, z: float) -> float:
    """Oracle Specie::Density of a QsDensityProfile at (x, y, z)."""
    return float(lib().qso_density(C.byref(prof), float(x), float(y), float(z)))


class Oracle:
    """The oracle mesh: same call surface as tertia_b200.Mesh."""

    def __init__(self, cfg):
        self.cfg = cfg
        h = C.c_void_p()
        _check(lib().qso_create(C.byref(cfg), C.byref(h)), "qso_create")
        self._h = h
        self.plane = cfg.ny * cfg.nz

    def close(self):
        if self._h:
            lib().qso_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _plane_out(self):
        return np.empty(self.plane, dtype=np.float64)

    def set_density_profile(self, prof):
        _check(lib().qso_set_density_profile(self._h, C.byref(prof) if prof is not None
                                             else None), "qso_set_density_profile")

    def set_phase(self, phase: float):
        _check(lib().qso_set_phase(self._h, float(phase)), "qso_set_phase")

    def pack_layer(self):
        n = int(lib().qso_layer_pack_size(self._h))
        out = np.empty(n)
        _check(lib().qso_pack_layer(self._h, out, n), "qso_pack_layer")
        return out

    def unpack_layer(self, buf):
        b = np.ascontiguousarray(buf, dtype=np.float64)
        _check(lib().qso_unpack_layer(self._h, b, b.size), "qso_unpack_layer")

    def front_weights(self):
        """Weights SeedParticles gives each cell's front particles (ny*nz)."""
        out = self._plane_out()
        _check(lib().qso_front_weights(self._h, out), "qso_front_weights")
        return out

    def load_beam(self, b):
        n = len(b["x"])
        a = {k: np.ascontiguousarray(b[k], dtype=np.int32 if k in "ijk" else np.float64)
             for k in ("i", "j", "k", "x", "y", "z", "px", "py", "pz", "w")}
        _check(lib().qso_load_beam(self._h, n, a["i"], a["j"], a["k"], a["x"], a["y"], a["z"],
                                   a["px"], a["py"], a["pz"], a["w"]), "qso_load_beam")

    def get_beam(self):
        n = lib().qso_beam_count(self._h)
        out = {k: np.empty(n, dtype=np.int32) for k in "ijk"}
        out.update({k: np.empty(n) for k in ("x", "y", "z", "px", "py", "pz", "w")})
        _check(lib().qso_get_beam(self._h, n, out["i"], out["j"], out["k"], out["x"], out["y"],
                                  out["z"], out["px"], out["py"], out["pz"], out["w"]),
               "qso_get_beam")
        return out

    def load_front_plasma(self, p):
        n = len(p["y"])
        cell = np.ascontiguousarray(p["cell"], dtype=np.int32)
        f = [np.ascontiguousarray(p[k], dtype=np.float64) for k in ("y", "z", "px", "py", "pz", "w")]
        _check(lib().qso_load_front_plasma(self._h, n, cell, *f), "qso_load_front_plasma")

    def get_plasma(self):
        n = lib().qso_plasma_count(self._h)
        out = {"cell": np.empty(n, dtype=np.int32)}
        out.update({k: np.empty(n) for k in ("y", "z", "px", "py", "pz", "w")})
        _check(lib().qso_get_plasma(self._h, n, out["cell"], out["y"], out["z"], out["px"],
                                    out["py"], out["pz"], out["w"]), "qso_get_plasma")
        return out

    def set_layer(self, which, field, data):
        _check(lib().qso_set_layer(self._h, which, field,
                                   np.ascontiguousarray(data, dtype=np.float64).reshape(-1)),
               "qso_set_layer")

    def get_layer(self, which, field):
        out = self._plane_out()
        _check(lib().qso_get_layer(self._h, which, field, out), "qso_get_layer")
        return out.reshape(self.cfg.nz, self.cfg.ny)

    def get_field3d(self, field, layer):
        out = self._plane_out()
        _check(lib().qso_get_field3d(self._h, field, layer, out), "qso_get_field3d")
        return out.reshape(self.cfg.nz, self.cfg.ny)

    def set_beam_currents(self, field, layer, data):
        _check(lib().qso_set_beam_currents(
            self._h, field, layer, np.ascontiguousarray(data, dtype=np.float64).reshape(-1)),
            "qso_set_beam_currents")

    def get_beam_currents(self, field, layer):
        out = self._plane_out()
        _check(lib().qso_get_beam_currents(self._h, field, layer, out), "qso_get_beam_currents")
        return out.reshape(self.cfg.nz, self.cfg.ny)

    def onaxis_ex(self):
        out = np.empty(self.cfg.nx)
        _check(lib().qso_get_onaxis_ex(self._h, out), "qso_get_onaxis_ex")
        return out

    def psi(self):
        out = np.empty(self.cfg.nx)
        _check(lib().qso_get_psi(self._h, out), "qso_get_psi")
        return out

    def charge_sums(self):
        """FP64 per-layer sums: rho (nx), jx (nx), rho_beam (nx + 1)."""
        r, j, b = np.empty(self.cfg.nx), np.empty(self.cfg.nx), np.empty(self.cfg.nx + 1)
        _check(lib().qso_get_charge_sums(self._h, r, j, b), "qso_get_charge_sums")
        return {"rho": r, "jx": j, "rho_beam": b}

    def set_field3d(self, field, layer, data):
        _check(lib().qso_set_field3d(self._h, field, layer,
                                     np.ascontiguousarray(data, dtype=np.float64).reshape(-1)),
               "qso_set_field3d")

    def step(self):
        _check(lib().qso_step(self._h), "qso_step")

    def move_beam_particles(self):
        _check(lib().qso_move_beam_particles(self._h), "qso_move_beam_particles")

    def move_all_split_layers(self):
        _check(lib().qso_move_all_split_layers(self._h), "qso_move_all_split_layers")

    def begin_march(self):
        _check(lib().qso_begin_march(self._h), "qso_begin_march")

    def layer_begin(self, i, s=0):
        _check(lib().qso_layer_begin(self._h, i, s), "qso_layer_begin")

    def move_split_layer(self, i, s=0):
        _check(lib().qso_move_split_layer(self._h, i, s), "qso_move_split_layer")

    def guess_fields(self, i, s=0):
        _check(lib().qso_guess_fields(self._h, i, s), "qso_guess_fields")

    def move_particles_layer(self, i, s, full):
        _check(lib().qso_move_particles_layer(self._h, i, s, int(full)), "qso_move_particles_layer")

    def iterate_fields(self, i, s, it):
        e = C.c_double(0.0)
        _check(lib().qso_iterate_fields(self._h, i, s, it, C.byref(e)), "qso_iterate_fields")
        return e.value

    def layer_end(self, i, s=0):
        _check(lib().qso_layer_end(self._h, i, s), "qso_layer_end")
