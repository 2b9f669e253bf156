"""B200-native quasi-static xi-layer loop (the hot path of snytav/tertia).

The compute path is libqsb200.so (hand-written sm_100a CUDA behind a C ABI,
include/qsb200.h); this package holds its Python mirror of the reference's
Mesh call surface, the config struct and the synthetic workloads.
"""
from .abi import (QsConfig, QsError, default_config, load_library, PRECISIONS,  # noqa: F401
                  QS_SHAPE_NGP, QS_SHAPE_CIC, QS_REDFT11, QS_RODFT11)

__all__ = ["QsConfig", "QsError", "default_config", "load_library", "Mesh", "PRECISIONS"]


def __getattr__(name):
    if name == "Mesh":
        from .mesh import Mesh
        return Mesh
    raise AttributeError(name)
