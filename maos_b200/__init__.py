"""B200-native physical-optics Shack-Hartmann wavefront-sensor frame.

The hot path (ray trace, field, FFT imaging with DTF/ETF, pixel sampling,
noise, CoG / matched-filter gradients) is CUDA for sm_100a behind the C ABI in
include/shwfs_b200.h; :mod:`maos_b200.shwfs` binds it.  The binding (and with
it the native library) loads on first use, so the pure-Python modules
(configs, replicas) import without it.
"""
import importlib

__all__ = ["shwfs", "Context", "ShwfsError"]


def __getattr__(name):
    if name == "shwfs":
        return importlib.import_module(".shwfs", __name__)
    if name in ("Context", "ShwfsError"):
        return getattr(importlib.import_module(".shwfs", __name__), name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
