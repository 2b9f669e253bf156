"""ctypes mirror of include/qsb200.h: the qs_config struct, enums, and the
loader of the in-tree CUDA library libqsb200.so.

The product path fails loudly when the CUDA library is missing: there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libqsb200.so")

# qs_status
QS_OK = 0
QS_ERR_INVALID = 1
QS_ERR_CUDA = 2
QS_ERR_OOM = 3
QS_ERR_DEVICE = 4
QS_ERR_BEAM_CURRENT = 5
QS_ERR_PARTICLE_RANGE = 6
QS_ERR_UNSUPPORTED = 7
QS_ERR_TIMEOUT = 8
QS_ERR_STATE = 9

# qs_precision
QS_PREC_FP64 = 0
QS_PREC_FP32 = 1
QS_PREC_TF32X3 = 2
QS_PREC_BF16X3 = 3
QS_PREC_BF16X6 = 4
QS_PREC_FP64_FFT = 5
PRECISIONS = {"fp64": QS_PREC_FP64, "fp32": QS_PREC_FP32, "tf32x3": QS_PREC_TF32X3,
              "bf16x3": QS_PREC_BF16X3, "bf16x6": QS_PREC_BF16X6, "fp64fft": QS_PREC_FP64_FFT}

# qs_shape
QS_SHAPE_NGP = 0
QS_SHAPE_CIC = 1

# qs_dtt_kind
QS_REDFT11 = 0
QS_RODFT11 = 1

# qs_field
QS_F_EX, QS_F_EY, QS_F_EZ, QS_F_BX, QS_F_BY, QS_F_BZ = range(6)
QS_F_JX, QS_F_JY, QS_F_JZ, QS_F_DENS = 6, 7, 8, 9
QS_F_RHOBEAM, QS_F_JXBEAM = 10, 11

QS_LAYER_P = 0
QS_LAYER_C = 1


class QsConfig(C.Structure):
    """Layout-identical mirror of struct qs_config."""

    _fields_ = [
        ("ny", C.c_int32), ("nz", C.c_int32), ("nx", C.c_int32),
        ("nx_split", C.c_int32), ("n_iter", C.c_int32), ("ppc", C.c_int32),
        ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double), ("ts", C.c_double),
        ("plasma_density", C.c_double), ("plasma_q2m", C.c_double),
        ("plasma_djx0", C.c_double), ("plasma_djy0", C.c_double),
        ("plasma_djz0", C.c_double), ("plasma_drho0", C.c_double),
        ("plasma_px0", C.c_double), ("plasma_py0", C.c_double), ("plasma_pz0", C.c_double),
        ("pspread_x", C.c_double), ("pspread_y", C.c_double), ("pspread_z", C.c_double),
        ("bx_ext", C.c_double), ("by_ext", C.c_double), ("bz_ext", C.c_double),
        ("beam_q2m", C.c_double), ("beam_polarity", C.c_double),
        ("syn_min", C.c_double), ("wavelength", C.c_double),
        ("synchrotron", C.c_int32), ("precision", C.c_int32), ("shape", C.c_int32),
        ("device", C.c_int32), ("store_sources", C.c_int32), ("use_graph", C.c_int32),
        ("seed", C.c_uint64),
    ]

    def copy(self) -> "QsConfig":
        c = QsConfig()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(QsConfig))
        return c

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def default_config(**overrides) -> QsConfig:
    """Reference namelist defaults for a uniform-plasma deck (Python twin of
    qs_config_default; kept identical by a test)."""
    c = QsConfig()
    c.ny = c.nz = 128
    c.nx = 256
    c.nx_split = 1        # Domain NxSplit default (domain.cpp:43)
    c.n_iter = 1          # Domain nIter default (domain.cpp:44)
    c.ppc = 4
    c.hx = c.hy = c.hz = 0.05
    c.ts = 1.0            # Domain Ts default (domain.cpp:50)
    c.plasma_density = 1.0
    c.plasma_q2m = -1.0   # Specie electrons (elements.cpp:89)
    c.plasma_djx0 = c.plasma_djy0 = c.plasma_djz0 = c.plasma_drho0 = -1.0  # elements.cpp:102-107
    c.plasma_px0 = c.plasma_py0 = c.plasma_pz0 = 0.0
    c.pspread_x = c.pspread_y = c.pspread_z = 0.0
    c.bx_ext = c.by_ext = c.bz_ext = 0.0
    c.beam_q2m = -1.0
    c.beam_polarity = -1.0
    c.syn_min = 100.0     # Synchrotron SynMin default (synchrotron.cpp:13)
    c.wavelength = 0.001  # Domain Wavelength default (domain.cpp:56)
    c.synchrotron = 1
    c.precision = QS_PREC_FP32
    c.shape = QS_SHAPE_NGP
    c.device = 0
    c.store_sources = 0
    c.use_graph = 1
    c.seed = 12345
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


# qs_density_profile distributions (Specie i_Distribution, plasma.cpp)
DIST_TRAPEZOID, DIST_GAUSS_ELLIPSOID, DIST_GAUSS_CHANNEL, DIST_CURVED_CHANNEL = 0, 1, 2, 3
DIST_PARALLELEPIPED, DIST_EXPONENTIAL, DIST_EMPTY_CHANNEL, DIST_COS_GAUSS = 4, 5, 6, 7
DIST_TANH_STEP, DIST_ROD, DIST_LINEAR_STEP, DIST_GRADIENT, DIST_PERIODIC = 8, 9, 10, 11, 12


class QsDensityProfile(C.Structure):
    """Layout-identical mirror of struct qs_density_profile."""

    _fields_ = [("distribution", C.c_int32), ("reserved", C.c_int32)] + [
        (name, C.c_double) for name in (
            "density", "density1", "begin", "end", "plateau_begin", "plateau_end", "scale",
            "delta", "radius", "radius_x", "radius_y", "radius_z", "x0", "y0", "z0", "xperiod",
            "yperiod", "zperiod", "angle_y", "y_curvature", "z_curvature", "curvature_begin",
            "curvature_end")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def density_profile(**values) -> QsDensityProfile:
    """A profile from the uniform default (Python twin of
    qs_density_profile_default; kept identical by a test) with `values` set."""
    p = QsDensityProfile()
    p.density = 1.0
    p.plateau_end = p.end = 1e30
    p.curvature_end = 1e20
    for k, v in values.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


_lib = None


class QsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[qs status {status}] {msg}")
        self.status = status


TRACE_LIB_PATH = os.path.join(_PKG, "libqsb200_trace.so")


def use_trace_library():
    """Make this process load libqsb200_trace.so (the same library with the
    march kernels' device timeline, include/qsb200_trace.h) instead of
    libqsb200.so; must come before the first load_library()."""
    global LIB_PATH
    if _lib is not None and LIB_PATH != TRACE_LIB_PATH:
        raise RuntimeError("libqsb200.so is already loaded in this process")
    LIB_PATH = TRACE_LIB_PATH


def load_library():
    """Load the in-tree libqsb200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python -c 'import __graft_entry__ as g; g.build()')")
    L = C.CDLL(LIB_PATH)
    _declare(L)
    _lib = L
    return L


def _declare(L):
    P = C.c_void_p
    i32p = C.POINTER(C.c_int32)
    f64p = C.POINTER(C.c_double)
    L.qs_config_default.argtypes = [C.POINTER(QsConfig)]
    L.qs_create.argtypes = [C.POINTER(QsConfig), C.POINTER(P)]
    L.qs_destroy.argtypes = [P]
    L.qs_last_error.argtypes = [P]
    L.qs_last_error.restype = C.c_char_p
    L.qs_status_string.argtypes = [C.c_int]
    L.qs_status_string.restype = C.c_char_p
    L.qs_sync.argtypes = [P]
    L.qs_get_stream.argtypes = [P, C.POINTER(P)]
    L.qs_load_beam.argtypes = [P, C.c_int64] + [i32p] * 3 + [f64p] * 7
    L.qs_get_beam.argtypes = [P, C.c_int64] + [i32p] * 3 + [f64p] * 7
    L.qs_beam_count.argtypes = [P]
    L.qs_beam_count.restype = C.c_int64
    L.qs_load_front_plasma.argtypes = [P, C.c_int64, i32p] + [f64p] * 6
    L.qs_seed_front_plasma.argtypes = [P, C.c_uint64]
    L.qs_plasma_count.argtypes = [P]
    L.qs_plasma_count.restype = C.c_int64
    L.qs_get_plasma.argtypes = [P, C.c_int64, i32p] + [f64p] * 6
    L.qs_set_layer.argtypes = [P, C.c_int, C.c_int, f64p]
    L.qs_get_layer.argtypes = [P, C.c_int, C.c_int, f64p]
    L.qs_get_field3d.argtypes = [P, C.c_int, C.c_int, f64p]
    L.qs_set_beam_currents.argtypes = [P, C.c_int, C.c_int, f64p]
    L.qs_get_beam_currents.argtypes = [P, C.c_int, C.c_int, f64p]
    L.qs_get_onaxis_ex.argtypes = [P, f64p]
    L.qs_get_psi.argtypes = [P, f64p]
    L.qs_get_charge_sums.argtypes = [P, f64p, f64p, f64p]
    L.qs_selftest_wait_limit.argtypes = [P, C.c_uint]
    L.qs_save_fields.argtypes = [P, C.c_char_p]
    L.qs_save_movie_frame.argtypes = [P, C.c_char_p]
    for name in ("qs_step", "qs_move_beam_particles", "qs_move_all_split_layers", "qs_begin_march"):
        getattr(L, name).argtypes = [P]
    for name in ("qs_layer_begin", "qs_move_split_layer", "qs_guess_fields", "qs_layer_end"):
        getattr(L, name).argtypes = [P, C.c_int, C.c_int]
    L.qs_move_particles_layer.argtypes = [P, C.c_int, C.c_int, C.c_int]
    L.qs_iterate_fields.argtypes = [P, C.c_int, C.c_int, C.c_int, f64p]
    L.qs_transform2d.argtypes = [P, C.c_int, C.c_int, C.c_int, f64p, f64p]
    L.qs_transform2d_dev.argtypes = [P, C.c_int, C.c_int, C.c_int, P, P]
    L.qs_transform2d_noalloc.argtypes = [C.c_int] * 5 + [P, P, P]
    L.qs_step_host.argtypes = ([P, C.c_int64] + [i32p] * 3 + [f64p] * 7 + [i32p] * 3 +
                               [f64p] * 6 + [f64p])
    L.qs_density_profile_default.argtypes = [C.POINTER(QsDensityProfile)]
    L.qs_set_density_profile.argtypes = [P, C.POINTER(QsDensityProfile)]
    L.qs_plasma_density.argtypes = [P, C.c_double, C.c_double, C.c_double,
                                    C.POINTER(C.c_double)]
    L.qs_set_phase.argtypes = [P, C.c_double]
    L.qs_layer_pack_size.argtypes = [P]
    L.qs_layer_pack_size.restype = C.c_int64
    L.qs_pack_layer.argtypes = [P, f64p, C.c_int64]
    L.qs_unpack_layer.argtypes = [P, f64p, C.c_int64]
    L.qs_clear_front_layer.argtypes = [P]
    L.qs_get_phase.argtypes = [P, C.POINTER(C.c_double)]
    L.qs_adjoint_checkpoints.argtypes = [P, C.c_int]
    L.qs_adjoint.argtypes = [P, f64p, f64p]
    L.qs_kernel_launches.argtypes = [P]
    L.qs_kernel_launches.restype = C.c_int64
    L.qs_profile_enable.argtypes = [P, C.c_int]
    L.qs_profile_read.argtypes = [P, f64p, C.POINTER(C.c_int64), C.c_int]


# Every symbol include/qsb200.h declares (checked against the library by a test).
EXPORTED_SYMBOLS = [
    "qs_config_default", "qs_create", "qs_destroy", "qs_last_error", "qs_status_string",
    "qs_sync", "qs_get_stream", "qs_load_beam", "qs_get_beam", "qs_beam_count",
    "qs_load_front_plasma", "qs_seed_front_plasma", "qs_plasma_count", "qs_get_plasma",
    "qs_density_profile_default", "qs_set_density_profile", "qs_plasma_density",
    "qs_set_phase", "qs_get_phase", "qs_layer_pack_size", "qs_pack_layer", "qs_unpack_layer",
    "qs_clear_front_layer",
    "qs_set_layer", "qs_get_layer", "qs_get_field3d", "qs_set_beam_currents",
    "qs_get_beam_currents", "qs_get_onaxis_ex", "qs_get_psi", "qs_get_charge_sums", "qs_selftest_wait_limit", "qs_save_fields",
    "qs_save_movie_frame", "qs_step",
    "qs_move_beam_particles", "qs_move_all_split_layers", "qs_begin_march", "qs_layer_begin",
    "qs_move_split_layer", "qs_guess_fields", "qs_move_particles_layer", "qs_iterate_fields",
    "qs_layer_end", "qs_transform2d", "qs_transform2d_dev", "qs_transform2d_noalloc",
    "qs_adjoint_checkpoints", "qs_adjoint", "qs_step_host",
    "qs_kernel_launches", "qs_profile_enable", "qs_profile_read",
]

KERNEL_CLASSES = ["push_deposit", "transform_gemm", "transform_split", "spectral_maps",
                  "beam_spectra", "beam_push", "front_seed", "other", "plasma_regroup"]
