"""B200-native NICAM-DC dynamical-core time step.

A ``cuda`` backend for pyNICAM-DC's ``Dyn.dynamics_step``
(pynicamdc/nhm/dynamics/mod_dynamics.py:1725): the RK3/HEVI large step runs as
hand-written sm_100a CUDA kernels in ``libnicamcuda.so`` behind a C ABI
(include/nicam_cuda.h), with the reference's prognostic layout, region/halo
conventions and step API kept on the host side.
"""
from .runtime import NicamCuda, NicamError, NonFiniteStateError, load_library, setup_table, LIB_PATH, EXPORTS  # noqa: F401
from .backend import CudaDyn  # noqa: F401
from . import halo, restart  # noqa: F401
