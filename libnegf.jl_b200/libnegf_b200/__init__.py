"""libnegf_b200: B200-native block-tridiagonal NEGF kernels behind LibNEGF.jl's API.

Layers:
* ``_lib``        -- ctypes binding of libnegf_b200.so (include/negf_b200.h);
* ``blockmatrix`` -- device-resident BlockMatrix / Block and the be_* backend;
* ``algorithms``  -- the reference's sweep functions (RGF, general RGF, RKD,
                     selected inverse, DDRGF) as single library calls;
* ``negf``        -- batched-energy device solves (G^R, G^<, transmission).
"""

from ._lib import load, NegfError, SingularError, LIB_PATH  # noqa: F401
from .blockmatrix import *  # noqa: F401,F403
from .algorithms import *  # noqa: F401,F403
from .negf import BatchSolver, Device, Solver, make_opts  # noqa: F401

__version__ = "1.0"
