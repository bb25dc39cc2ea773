"""Python mirror of VPFFT::DataStructures::MaterialGrid (MaterialGrid.h:59-577)
over the C ABI.  Method names, argument meaning and order follow the
reference; arrays are numpy with the reference's layouts (voxel index
x*Ny*Nz + y*Nz + z, 3x3 row-major orientations, deviatoric 5-vectors).
Errors raise VpfftError instead of exiting the process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import check, dptr, f64


class MaterialGrid:
    """One RVE resident on the current CUDA device."""

    def __init__(self, DimX: int, DimY: int, DimZ: int, material: capi.Material | None = None,
                 precision: str = "fp64", options: capi.SolverOptions | None = None):
        lib = capi.load()
        prec = {"fp64": capi.PREC_FP64, "mixed": capi.PREC_MIXED}[precision]
        h = C.c_void_p()
        st = lib.vpfft_grid_create(DimX, DimY, DimZ, C.byref(material) if material else None,
                                   C.byref(options) if options else None, prec, C.byref(h))
        check(st)
        self._h = h
        self._lib = lib
        self.DimX, self.DimY, self.DimZ = DimX, DimY, DimZ
        self.N = DimX * DimY * DimZ
        self.precision = precision
        self.last_stats: capi.Stats | None = None

    # ---------------------------------------------------------------- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.vpfft_grid_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def NumX(self) -> int:
        return self.DimX

    def NumY(self) -> int:
        return self.DimY

    def NumZ(self) -> int:
        return self.DimZ

    def ToIndex(self, x: int, y: int, z: int) -> int:
        return (x * self.DimY + y) * self.DimZ + z

    # ---------------------------------------------------------------- set-up
    def SendDataAndInitialize(self, Orientations, Stress=None) -> None:
        """MaterialGrid::SendDataAndInitialize (MaterialGrid.cpp:425-534)."""
        R = f64(Orientations, (self.N, 9))
        S = None if Stress is None else f64(Stress, (self.N, 5))
        check(self._lib.vpfft_grid_set_fields(self._h, dptr(R), dptr(S) if S is not None else None),
              self._h)

    def SetVoxelLength(self, x: float, y: float, z: float) -> None:
        check(self._lib.vpfft_grid_set_voxel_length(self._h, x, y, z), self._h)

    def VoxelLength(self) -> np.ndarray:
        h = np.zeros(3)
        check(self._lib.vpfft_grid_get_voxel_length(self._h, dptr(h)), self._h)
        return h

    def SetCRSS(self, crss) -> None:
        """Per-voxel CRSS (N x 12), or None for the material's uniform values."""
        if crss is None:
            check(self._lib.vpfft_grid_set_crss(self._h, None), self._h)
        else:
            a = f64(crss, (self.N, 12))
            check(self._lib.vpfft_grid_set_crss(self._h, dptr(a)), self._h)

    # ---------------------------------------------------------------- solve
    def RunSingleStrainStep(self, MacroscopicStrainRate, NumMaxIterations: int, TimeStep: float,
                            ConvergenceEpsilon: float) -> np.ndarray:
        """MaterialGrid::RunSingleStrainStep (MaterialGrid.cpp:897-1084); returns <sigma>."""
        e = f64(MacroscopicStrainRate, (5,))
        avg = np.zeros(5)
        st = capi.Stats()
        check(self._lib.vpfft_run_single_strain_step(self._h, dptr(e), int(NumMaxIterations),
                                                     float(TimeStep), float(ConvergenceEpsilon),
                                                     dptr(avg), C.byref(st)), self._h)
        self.last_stats = st
        return avg

    def RunVPFFT(self, MacroscopicStrainRate, NumMaxIterations: int, NumTimeSteps: int,
                 TimeStep: float, ConvergenceEpsilon: float,
                 stress_strain_path: str | None = "Stress_Strain.txt") -> list:
        """MaterialGrid::RunVPFFT (MaterialGrid.cpp:1202-1228): returns one
        (step, strain, <sigma>) row per increment and writes the reference's
        Stress_Strain.txt when a path is given."""
        e = f64(MacroscopicStrainRate, (5,))
        rows = []

        @capi.STEP_CALLBACK
        def cb(step, strain, stress, user):
            rows.append((step, np.ctypeslib.as_array(strain, (5,)).copy(),
                         np.ctypeslib.as_array(stress, (5,)).copy()))
            return 0

        path = stress_strain_path.encode() if stress_strain_path else None
        check(self._lib.vpfft_run(self._h, dptr(e), int(NumMaxIterations), int(NumTimeSteps),
                                  float(TimeStep), float(ConvergenceEpsilon), path, cb, None),
              self._h)
        return rows

    # phases of RunSingleStrainStep
    def InitializeComputation(self, MacroscopicStrainRate) -> None:
        e = f64(MacroscopicStrainRate, (5,))
        check(self._lib.vpfft_initialize_computation(self._h, dptr(e)), self._h)

    def BuildLinearRefMediumStiffness(self) -> np.ndarray:
        """Returns L0 as a 5x5 array indexed [i, j]."""
        L = np.zeros(25)
        check(self._lib.vpfft_build_reference_medium(self._h, dptr(L)), self._h)
        return L.reshape(5, 5).T.copy()  # column-major storage -> [i, j]

    def FixedPoint(self, MacroscopicStrainRate, NumMaxIterations: int,
                   ConvergenceEpsilon: float) -> np.ndarray:
        """The fixed-point loop (MaterialGrid.cpp:930-1068); returns the history
        rows (<sigma>(5), <edot>(5), delta_sigma, delta_eps) per iteration."""
        e = f64(MacroscopicStrainRate, (5,))
        hist = np.zeros((max(int(NumMaxIterations), 1), 12))
        st = capi.Stats()
        check(self._lib.vpfft_fixed_point(self._h, dptr(e), int(NumMaxIterations),
                                          float(ConvergenceEpsilon), dptr(hist), C.byref(st)),
              self._h)
        self.last_stats = st
        return hist[: st.iterations].copy()

    def PostIncrement(self, MacroscopicStrainRate, TimeStep: float) -> None:
        e = f64(MacroscopicStrainRate, (5,))
        check(self._lib.vpfft_post_increment(self._h, dptr(e), float(TimeStep)), self._h)

    # ---------------------------------------------------------------- fields
    def field(self, which: int) -> np.ndarray:
        w = capi.FIELD_WIDTH[which]
        out = np.zeros(self.N * w)
        check(self._lib.vpfft_grid_get_field(self._h, which, dptr(out)), self._h)
        return out.reshape(self.N, w) if w > 1 else out

    def set_field(self, which: int, values) -> None:
        w = capi.FIELD_WIDTH[which]
        a = f64(values, (self.N * w,))
        check(self._lib.vpfft_grid_set_field(self._h, which, dptr(a)), self._h)

    # ---------------------------------------------------------------- checkpoint
    def snapshot(self) -> bytes:
        """The grid's whole state (vpfft_grid_snapshot) as bytes."""
        n = C.c_size_t(0)
        check(self._lib.vpfft_grid_snapshot_size(self._h, C.byref(n)), self._h)
        buf = C.create_string_buffer(n.value)
        check(self._lib.vpfft_grid_snapshot(self._h, buf, n.value), self._h)
        return buf.raw

    def restore(self, data: bytes) -> None:
        """Continue from a snapshot of a grid of the same dimensions and
        precision (vpfft_grid_restore)."""
        check(self._lib.vpfft_grid_restore(self._h, data, len(data)), self._h)

    def Stress(self) -> np.ndarray:
        return self.field(capi.FIELD_STRESS)

    def LagrangeMultiplier(self) -> np.ndarray:
        return self.field(capi.FIELD_LAGRANGE)

    def Orientation(self) -> np.ndarray:
        return self.field(capi.FIELD_ORIENTATION)

    def CRSS(self) -> np.ndarray:
        return self.field(capi.FIELD_CRSS)

    def AccumulatedShear(self) -> np.ndarray:
        return self.field(capi.FIELD_ACCUMULATED_SHEAR)

    def PolarizationField(self) -> np.ndarray:
        return self.field(capi.FIELD_POLARIZATION)

    def DisplacementVariation(self) -> np.ndarray:
        """Re of the strain-rate variation d~ of the last iteration."""
        return self.field(capi.FIELD_STRAIN_RATE_VARIATION)

    def StrainRate(self) -> np.ndarray:
        return self.field(capi.FIELD_STRAIN_RATE)

    def SchmidtTensorList(self) -> np.ndarray:
        return self.field(capi.FIELD_SCHMID).reshape(self.N, 12, 5)

    # ---------------------------------------------------------------- text dumps
    def _print(self, kind: int, filename: str) -> None:
        check(self._lib.vpfft_grid_print(self._h, kind, str(filename).encode()), self._h)

    def PrintStrain(self, filename: str) -> None:
        """MaterialGrid::PrintStrain (MaterialGrid.cpp:15-35)."""
        self._print(capi.PRINT_STRAIN, filename)

    def PrintStress(self, filename: str) -> None:
        """MaterialGrid::PrintStress (MaterialGrid.cpp:40-55)."""
        self._print(capi.PRINT_STRESS, filename)

    def PrintLagrangeMultiplier(self, filename: str) -> None:
        """MaterialGrid::PrintLagrangeMultiplier (MaterialGrid.cpp:60-75)."""
        self._print(capi.PRINT_LAGRANGE, filename)

    def PrintPolarization(self, filename: str) -> None:
        """MaterialGrid::PrintPolarization (MaterialGrid.cpp:80-100)."""
        self._print(capi.PRINT_POLARIZATION, filename)

    def green_operator(self) -> dict:
        """The x pass's Green operator (vpfft_grid_green_operator): mode 1
        computed per wave vector, 2 stored table, 0 not chosen yet, with the x
        pass times (ms) measured when it was chosen."""
        mode = C.c_int()
        a, b = C.c_double(), C.c_double()
        check(self._lib.vpfft_grid_green_operator(self._h, C.byref(mode), C.byref(a), C.byref(b)),
              self._h)
        return {"mode": int(mode.value), "ms_compute": a.value, "ms_table": b.value}

    def launch_count(self) -> int:
        return int(self._lib.vpfft_grid_launch_count(self._h))

    def set_profiling(self, enabled: bool) -> None:
        check(self._lib.vpfft_grid_set_profiling(self._h, int(bool(enabled))), self._h)

    def phase_times(self) -> dict:
        """{phase name: (total device ms, launches)} of the fixed-point loop."""
        ms = np.zeros(capi.NUM_PHASES)
        cnt = np.zeros(capi.NUM_PHASES, np.int64)
        check(self._lib.vpfft_grid_phase_times(self._h, dptr(ms),
                                               cnt.ctypes.data_as(C.POINTER(C.c_int64))), self._h)
        return {self._lib.vpfft_phase_name(k).decode(): (float(ms[k]), int(cnt[k]))
                for k in range(capi.NUM_PHASES)}

    def synchronize(self) -> None:
        check(self._lib.vpfft_grid_synchronize(self._h), self._h)

    def stream(self) -> int:
        return int(self._lib.vpfft_grid_stream(self._h) or 0)
