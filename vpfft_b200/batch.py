"""Batches of RVEs over the C ABI (vpfft_batch_*): many MaterialGrids of
different sizes advanced together, one kernel launch per phase, with requests
admitted between ticks (continuous batching).  Each request is one
RunSingleStrainStep (MaterialGrid.cpp:897-1084) on a caller-owned grid whose
fields and texture persist across requests.  The reference has no batch API;
it solves one RVE per MPI job.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .capi import f64
from .material_grid import MaterialGrid


@dataclass
class BatchResult:
    request_id: int
    status: int
    iterations: int
    converged: bool
    avg_stress: np.ndarray
    stress_error: float
    strain_rate_error: float
    nr_not_converged: int
    status_bits: int
    seconds_queued: float
    seconds_total: float


class Batch:
    """A batch engine bound to the current CUDA device."""

    def __init__(self, precision: str = "mixed", material: capi.Material | None = None,
                 options: capi.SolverOptions | None = None, max_slots: int = 256,
                 iterations_per_tick: int = 8, hbm_budget_bytes: int = 8 << 30,
                 use_graphs: bool = True, fft_tiles: int = -1):
        lib = capi.load()
        bo = capi.BatchOptions()
        lib.vpfft_batch_options_default(C.byref(bo))
        bo.max_slots = max_slots
        bo.iterations_per_tick = iterations_per_tick
        bo.hbm_budget_bytes = hbm_budget_bytes
        bo.use_graphs = int(bool(use_graphs))
        bo.fft_tiles = int(fft_tiles)
        prec = {"fp64": capi.PREC_FP64, "mixed": capi.PREC_MIXED}[precision]
        h = C.c_void_p()
        self._lib = lib
        self._check(lib.vpfft_batch_create(prec, C.byref(material) if material else None,
                                           C.byref(options) if options else None, C.byref(bo),
                                           C.byref(h)), None)
        self._h = h
        self.precision = precision
        self.material = material
        self.options = options

    def _check(self, st: int, h) -> None:
        if st != capi.OK:
            msg = self._lib.vpfft_batch_last_error(h).decode(errors="replace")
            base = self._lib.vpfft_status_string(st).decode()
            raise capi.VpfftError(st, f"{base}: {msg}" if msg else base)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.vpfft_batch_destroy(self._h)
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

    def new_grid(self, DimX: int, DimY: int, DimZ: int) -> MaterialGrid:
        """A MaterialGrid with the batch's precision, material and options."""
        return MaterialGrid(DimX, DimY, DimZ, material=self.material, precision=self.precision,
                            options=self.options)

    def submit(self, grid: MaterialGrid, MacroscopicStrainRate, NumMaxIterations: int = 100,
               TimeStep: float = 0.005, ConvergenceEpsilon: float = 1e-5) -> int:
        e = f64(MacroscopicStrainRate, (5,))
        rid = C.c_int64()
        self._check(self._lib.vpfft_batch_submit(self._h, grid._h, capi.dptr(e),
                                                 int(NumMaxIterations), float(TimeStep),
                                                 float(ConvergenceEpsilon), C.byref(rid)),
                    self._h)
        return int(rid.value)

    def step(self) -> int:
        """One tick; returns the number of requests still queued or active."""
        pending = C.c_int()
        self._check(self._lib.vpfft_batch_step(self._h, C.byref(pending)), self._h)
        return int(pending.value)

    def run(self) -> None:
        self._check(self._lib.vpfft_batch_run(self._h), self._h)

    def poll(self, cap: int = 1024) -> list[BatchResult]:
        buf = (capi.BatchResult * cap)()
        n = C.c_int()
        self._check(self._lib.vpfft_batch_poll(self._h, buf, cap, C.byref(n)), self._h)
        out = []
        for r in buf[: n.value]:
            out.append(BatchResult(int(r.request_id), int(r.status), int(r.iterations),
                                   bool(r.converged), np.array(r.avg_stress[:]),
                                   float(r.stress_error), float(r.strain_rate_error),
                                   int(r.nr_not_converged), int(r.status_bits),
                                   float(r.seconds_queued),
                                   float(r.seconds_total)))
        return out

    def cancel(self, request_id: int) -> None:
        self._check(self._lib.vpfft_batch_cancel(self._h, int(request_id)), self._h)

    def info(self) -> dict:
        i = capi.BatchInfo()
        self._check(self._lib.vpfft_batch_get_info(self._h, C.byref(i)), self._h)
        return {name: int(getattr(i, name)) for name, _ in capi.BatchInfo._fields_}

    def tunings(self) -> list[dict]:
        """Tile family of the batched FFT passes per RVE size admitted so far
        (vpfft_batch_get_tunings): the family used, how many the size offers,
        how it was chosen and the timed five-pass chain per family (ms)."""
        n = C.c_int()
        self._check(self._lib.vpfft_batch_get_tunings(self._h, None, 0, C.byref(n)), self._h)
        buf = (capi.TileTuning * max(1, n.value))()
        self._check(self._lib.vpfft_batch_get_tunings(self._h, buf, n.value, C.byref(n)),
                    self._h)
        src = {0: "options", 1: "single family", 2: "cached", 3: "timed"}
        return [{"dims": (int(t.nx), int(t.ny), int(t.nz)), "fft_tiles": int(t.fft_tiles),
                 "families": int(t.families), "source": src.get(int(t.source), "?"),
                 "ms_per_chain": [float(v) for v in t.ms_per_chain[: int(t.families)]]}
                for t in buf[: n.value]]
