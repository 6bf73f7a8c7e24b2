"""B200-native physical-optics Shack-Hartmann wavefront-sensor frame.

The hot path (ray trace, field, FFT imaging with DTF/ETF, pixel sampling,
noise, CoG / matched-filter gradients) is CUDA for sm_100a behind the C ABI in
include/shwfs_b200.h; :mod:`maos_b200.shwfs` binds it.
"""
from . import shwfs  # noqa: F401
from .shwfs import Context, ShwfsError  # noqa: F401
