"""B200-native ETD2 propagation core for ultra-high-energy cosmic-ray transport.

The package keeps PriNCe's propagation-solver / run / result API
(``UHECRPropagationSolverETD2``, ``MultiRHSPropagationSolverETD2``,
``UHECRPropagationResult``, ``PriNCeRun``) and runs the redshift stepping
on hand-written sm_100a CUDA kernels behind a C ABI (``include/prince_b200.h``)
loaded with ctypes.
"""

from . import constants, cosmology, cr_sources, data, photonfields, synth
from .constants import PRINCE_UNITS, BackendConfig
from .data import EnergyGrid, SpeciesManager
from .run import FixedKernelModel, PriNCeRun

__version__ = "0.1.0"
