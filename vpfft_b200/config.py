"""Utilities::ConfigFile (Config.h:21-85) over vpfft_config_read."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi


class ConfigFile:
    """Keyword configuration file of the reference, with its defects fixed
    (see vpfft_b200/csrc/config.cpp)."""

    eInitTwoGrain = 0
    eInitFile = 1

    def __init__(self):
        self._c = capi.Config()

    def Read(self, Filename: str) -> bool:
        """Returns True on success; the error text is kept in self.error."""
        err = C.create_string_buffer(512)
        st = capi.load().vpfft_config_read(Filename.encode(), C.byref(self._c), err, 512)
        self.error = err.value.decode()
        return st == capi.OK

    @property
    def NumX(self):
        return self._c.num_x

    @property
    def NumY(self):
        return self._c.num_y

    @property
    def NumZ(self):
        return self._c.num_z

    @property
    def InputStrainRate(self) -> np.ndarray:
        return np.array(self._c.input_strain_rate[:]).reshape(3, 3)

    @property
    def MaxNRIter(self):
        return self._c.max_nr_iter

    @property
    def NRTolerence(self):
        return self._c.nr_tolerance

    @property
    def TimeStep(self):
        return self._c.time_step

    @property
    def NumTimeIter(self):
        return self._c.num_time_iter

    @property
    def InitMethod(self):
        return self._c.init_method

    @property
    def InputMicrostructureFilename(self) -> str:
        return self._c.input_microstructure.decode()

    @property
    def CRSS(self):
        return np.array(self._c.material.crss[:])

    @property
    def GammaDotBase(self):
        return np.array(self._c.material.gamma_dot_base[:])

    @property
    def RateSensitivity(self):
        return np.array(self._c.material.rate_sensitivity[:])

    @property
    def material(self) -> capi.Material:
        return self._c.material

    @property
    def VoxelLength(self):
        return np.array(self._c.voxel_length[:])

    @property
    def ConvergenceEpsilon(self):
        return self._c.convergence_epsilon

    @property
    def MaxIter(self):
        return self._c.max_iter

    @property
    def precision(self) -> str:
        return "fp64" if self._c.precision == capi.PREC_FP64 else "mixed"
