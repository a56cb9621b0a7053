"""amss_b200 -- B200-native (sm_100a) BSSN evolution hot path of AMSS-NCKU.

`dropin` mirrors the reference's per-block Fortran kernel calls; `engine` is
the batched device-resident level step; `adjoint` differentiates a block's
evolution (torch.autograd.Function); `initial` builds puncture initial data
on hierarchies; `monitor` writes the constraint output file.  All compute runs
only on a CUDA device.
"""
from ._lib import AmssError, lib, last_error, header_functions  # noqa: F401
from . import dropin, engine, initial, monitor  # noqa: F401
from .engine import Engine  # noqa: F401

__all__ = ["AmssError", "lib", "last_error", "header_functions", "dropin", "engine", "initial", "monitor",
           "Engine"]


def __getattr__(name):
    # the adjoint wrapper needs torch; import it on first use only
    if name == "adjoint":
        import importlib
        return importlib.import_module(".adjoint", __name__)
    raise AttributeError(name)
