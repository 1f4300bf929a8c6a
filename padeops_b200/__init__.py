"""padeops_b200 -- B200-native (CUDA sm_100a, FP64) compact-difference operators.

A drop-in for the hot path of PadeOps: the cd06 / cd10 Pade derivatives and
the cf90 compact filter along x, y and z, periodic or bounded, and the
staggered cd06 scheme along z (cd06stagg), and fields split over several
GPUs in z-slabs (padeops_b200.slabs), behind the C
ABI of include/pado.h (for the Fortran solver) and the reference-shaped
Python objects below.  The CUDA library (padeops_b200/_lib/libpado.so) is
required: the first operation loads it and raises ImportError if it is
missing.  There is no CPU path.
"""
from . import _lib
from ._lib import CD06, CD10, CF90, D1, D2, FILTER, PadoError
from .operators import Derivatives, Filters, cd06, cd10, cf90
from .stagg import cd06stagg
from . import slabs

__all__ = ["cd06", "cd10", "cf90", "cd06stagg", "Derivatives", "Filters", "PadoError", "CD06", "CD10", "CF90", "D1", "D2",
           "FILTER", "slabs", "launch_count", "version"]

def launch_count() -> int:
    """Kernel launches this process has enqueued through the library."""
    return int(_lib.lib().pado_launch_count())


def version() -> str:
    return _lib.lib().pado_version().decode()
