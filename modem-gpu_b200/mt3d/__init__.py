"""mt3d -- host side of the B200-native 3D magnetotelluric forward/adjoint solve.

``mt3d.capi`` binds the CUDA library (libmt3d.so, C ABI in include/mt3d.h);
``mt3d.models`` and ``mt3d.bc`` build the grids, conductivity models and
boundary data a ModEM run would read from its input files.
"""
from . import bc, models  # noqa: F401
