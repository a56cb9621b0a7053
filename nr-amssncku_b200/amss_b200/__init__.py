"""amss_b200 -- B200-native (sm_100a) BSSN evolution hot path of AMSS-NCKU.

`dropin` mirrors the reference's per-block Fortran kernel calls; `engine` is
the batched device-resident level step.  Both run only on a CUDA device.
"""
from ._lib import AmssError, lib, last_error, header_functions  # noqa: F401
from . import dropin, engine  # noqa: F401
from .engine import Engine  # noqa: F401

__all__ = ["AmssError", "lib", "last_error", "header_functions", "dropin", "engine", "Engine"]
