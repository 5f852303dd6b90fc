"""cmmdft_b200: the CmmDFT 3D grid solve (an LJ adsorbate, spherical or rigid
multi-site, in a periodic host) as hand-written FP64 CUDA kernels for B200
(sm_100a), behind the reference's Python API.

Host-side modules import without a GPU; every field operation requires the
CUDA library (libcmmdft_b200.so) and a CUDA device -- there is no CPU path.
"""
from .units import *  # noqa: F401,F403
from .system import (Cell, System, Host, NanoporousHost, EmptyHost, Guest, SphericalLJGuest,  # noqa: F401
                     NonSphericalGuest, DualModelGuest, Grid, Spectrum, read_chk, read_pars_file)
from .eos import (EquationOfState, SumOfEOS, ModifiedBenedictWebbRubinEOS, CarnahanStarlingEOS,  # noqa: F401
                  MFAEOS)
from .functionals import (FreeEnergy, HardSphereFunctional, MFAFunctional, ExternalPotential,  # noqa: F401
                          WDAVFunctional, LDAFunctional)
from .solver import Solver, Picard, Anderson, QuasiNewton, Fire, NoSolutionError  # noqa: F401
from .program import Program  # noqa: F401
from .calculator import Calculator  # noqa: F401
from .tools import get_file_suffix  # noqa: F401
from .log import log  # noqa: F401

__version__ = "0.1.0"
