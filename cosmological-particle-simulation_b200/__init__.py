"""B200 (sm_100a) TreePM gravity solve — a drop-in for the reference crate's per-step path.

The compute runs in libcpm_cuda.so (hand-written CUDA behind the C ABI of include/cpm.h);
this package is its ctypes front end with the reference's interface names. Import does not
touch the GPU; the first call loads the library and fails loudly when it is missing.
"""
from ._native import CpmError, Cosmology, exported_symbols, lib  # noqa: F401
from .api import (Context, Ensemble, Fft3, ForceSplit, Mesh, PoissonSolver, Simulation, density_contrast, density_grid,  # noqa: F401
                  interpolate3, ln_a_schedule, octant_keys, power_spectrum, short_range_factor, tree_accelerations,
                  wavenumber, zeldovich)
from .learned import ShortRangeNet  # noqa: F401

__version__ = "0.1.0"
