"""gacelle_b200 -- B200 (sm_100a) engine for GACELLE's voxel-parallel solvers.

Mirrors the reference's askadam / mcmc solvers and the built-in model classes
gpuR2starMapping, gpuJointR1R2starMapping, gpuNEXI and gpuNEXIrice on top of the C-ABI
library libgacelle_b200.so (include/gacelle_b200.h).
"""
from ._lib import Context, GacelleError, lib  # noqa: F401
from .askadam_solver import askadam  # noqa: F401
from .mcmc_solver import mcmc  # noqa: F401
from .models import gpuJointR1R2starMapping, gpuNEXI, gpuNEXIrice, gpuR2starMapping  # noqa: F401
from . import utils  # noqa: F401

__version__ = "0.1.0"
