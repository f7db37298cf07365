"""mumax-plus B200: the effective-field + Runge-Kutta hot path of mumax+ on sm_100a.

Python surface of the reference's `mumaxplus` package for that path (World,
Ferromagnet, Grid, TimeSolver, FieldQuantity, Parameter, Variable, DmiTensor,
StrayField), backed by libmpx.so (include/mpx.h).  There is no CPU path:
creating a World needs a CUDA device and the built library.
"""
from . import _abi
from .ferromagnet import Ferromagnet
from .fieldquantity import FieldQuantity, ScalarQuantity
from .grid import Grid
from .parameter import DmiTensor, InterParameter, Parameter, Variable
from .strayfield import StrayField
from .timesolver import TimeSolver, TimeSolverOutput
from .world import World

GAMMALL = 1.7595e11  # rad/(T s)
MU0 = 1.25663706212e-6  # H/m

__all__ = [
    "Ferromagnet",
    "FieldQuantity",
    "ScalarQuantity",
    "Grid",
    "DmiTensor",
    "InterParameter",
    "Parameter",
    "Variable",
    "StrayField",
    "TimeSolver",
    "TimeSolverOutput",
    "World",
    "GAMMALL",
    "MU0",
]
