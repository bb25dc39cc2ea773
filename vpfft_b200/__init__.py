"""vpfft_b200 -- B200-native (sm_100a) implementation of VPFFT's fixed-point
solve on a periodic 3D voxel polycrystal.

The compute runs in the CUDA library vpfft_b200/lib/libvpfft_b200.so behind
the C ABI of include/vpfft_capi.h; this package is its Python host mirror of
the reference's MaterialGrid / Solvers / ConfigFile surface.
"""
from . import capi
from .capi import Material, SolverOptions, Stats, VpfftError, device_count, load, material
from .config import ConfigFile
from .material_grid import MaterialGrid
from .batch import Batch, BatchResult

__all__ = ["capi", "Material", "SolverOptions", "Stats", "VpfftError", "device_count", "load",
           "material", "MaterialGrid", "ConfigFile", "Batch", "BatchResult"]
