"""mochii_b200: B200-native photon-packet transport and per-cell ionisation
balance for MoCHII-style photoionisation runs (the C ABI lives in
include/mochii_gpu.h; this package holds the CUDA sources, the build and a
Python mirror of the reference's entry points)."""
from ._lib import MochiiError, Params  # noqa: F401
from .host import (Batch, Nebula, default_params, parse_namelist, read_input, run,  # noqa: F401
                   set_param, sobol_uniforms)
