"""Benchmark of the VPFFT fixed-point solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the headline configuration): a 256^3 periodic Voronoi polycrystal
with 1000 grains and uniform random orientations, FCC 12 {111}<110> systems,
power law n = 20, gdot0 = 1, uniform CRSS 1, plane-strain compression
velocity gradient diag(1, 0, -1); mixed precision (FP32 fields, FFTs and
Green operator; FP64 Newton-Raphson and compensated FP64 reductions).
Synthetic data from the seeded fixture generator.

A step is one fixed-point iteration over the whole grid (MaterialGrid.cpp:
930-1068): forward R2C FFT of the polarization, Green operator, inverse FFT,
per-voxel NR solve, constitutive update, reductions and convergence test.
The metric is voxel-iterations per second (voxels x iterations / time).

  value  -- K iterations timed with CUDA events on the grid's stream, state
            resident in HBM (inputs ~2.3 GB, far larger than the 126 MB L2);
  e2e    -- the same metric through the C ABI call a user makes,
            vpfft_run_single_strain_step, one full increment per step
            (initialisation, reference medium, up to 100 iterations to
            eps = 1e-5, texture and hardening update), with the orientation and
            stress arrays copied from pinned host memory and the stress field
            copied back inside the timed region;
  fp64   -- the all-FP64 GPU path on the same workload;
  cpu_baseline -- the reference's own code (oracle/_ref, else the C
            restatement) on a bounded sample of the same workload on the host;
  batched / serving -- 256 RVEs of 16-64^3 in one batch, and a Poisson
            request stream served by continuous batching (host wall clock:
            the batch synchronises every tick), each with a cpu_baseline of
            the reference on every host core, modelled from its measured
            per-edge increment costs (full CPU solves would take hours).

Multi-GPU: one process per GPU (torchrun); every rank solves its own replica
RVE (weak scaling, no collective in the data path); the elapsed time is the
maximum over ranks.  --impl reference times the reference's CPU solve with
every host core running its own sample (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

# One visible GPU per rank, set before any CUDA runtime initialises.
if "LOCAL_RANK" in os.environ and int(os.environ.get("WORLD_SIZE", "1")) > 1:
    os.environ["CUDA_VISIBLE_DEVICES"] = os.environ["LOCAL_RANK"]

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "voxel-iters/s at 256^3 mixed precision (FP64 path reported beside)"
UNIT = "voxel-iter/s"

N_GRID = 256
N_GRAINS = 1000
SEED = 2024
RATE_SENS = 20
VEL_GRAD = np.diag([1.0, 0.0, -1.0])

def workload(n: int) -> str:
    return (f"{n}^3 periodic Voronoi polycrystal, 1000 grains, uniform SO(3) orientations, "
            "FCC 12 {111}<110>, n=20, gdot0=1, CRSS=1, plane-strain diag(1,0,-1), one "
            "fixed-point iteration per step")


WORKLOAD = workload(256)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and throttle reasons of the GPU this process uses, sampled
    every ~5 ms through NVML while the timed region runs (the GPU is found by
    the PCI bus id of CUDA device 0, so the index nvidia-smi gives it does not
    matter)."""

    # NVML clocks-event-reason bits (nvml.h)
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}

    def __init__(self, period_s: float = 0.005):
        self.period = period_s
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._h = None

    def _handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        self._nvml = pynvml
        p = torch.cuda.get_device_properties(0)
        bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        return pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def __enter__(self):
        try:
            self._h = self._handle()
            self.max_mhz = float(self._nvml.nvmlDeviceGetMaxClockInfo(self._h,
                                                                       self._nvml.NVML_CLOCK_SM))
        except Exception:  # no NVML: the line then records no samples
            self._h = None
            return self
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _run(self):
        nv = self._nvml
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                self.samples.append((float(mhz), int(bits)))
            except Exception:
                return
            self._stop.wait(self.period)

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)

    def summary(self, gpu_index: int = 0):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        reasons = sorted(nm for nm, bit in self.REASONS.items()
                         if any(b & bit for _, b in self.samples))
        return {"sm_mhz": statistics.median(m for m, _ in self.samples),
                "sm_max_mhz": self.max_mhz, "reasons": reasons, "samples": len(self.samples),
                "source": "NVML every 5 ms during the timed region"}


# ------------------------------------------------------------------ inputs
def make_inputs(n=N_GRID, grains=N_GRAINS, seed=SEED):
    from vpfft_b200 import fixtures

    R = fixtures.polycrystal(n, n, n, grains, seed)
    edot = fixtures.edot_from_matrix(VEL_GRAD)
    return R, edot


def material():
    import vpfft_b200 as vp

    return vp.material(gamma_dot_base=1.0, rate_sensitivity=RATE_SENS, crss=1.0, tau0=1.0,
                       tau1=0.5, theta0=20.0, theta1=1.0)


def alg_bytes_per_voxel(s: int, nz: int, keep_d: bool = False) -> dict:
    """Compulsory HBM bytes per voxel of each kernel of one iteration, for
    field storage size s (4 mixed, 8 FP64): complex values are 2s, the half
    spectrum has nz/2+1 of nz points along z, 5 components everywhere."""
    h = (nz // 2 + 1) / nz
    spec = 5 * 2 * s * h
    return {
        "fft_z_r2c": 5 * s + spec,
        "fft_y_forward": 2 * spec,
        "fft_x_green": 2 * spec,
        "fft_y_inverse": 2 * spec,
        "fft_z_c2r": spec + 5 * s,
        # R (9), sigma, lambda, d~ (5 each) read; sigma, lambda, P written
        "nr_update": (9 + 5 + 5 + 5) * s + 15 * s + (5 * s if keep_d else 0),
        "iter_finish": 0.0,
    }


# ------------------------------------------------------------------ our arm
def device_arm(args, R, edot, precision):
    import torch

    import vpfft_b200 as vp

    n = args.grid
    N = n ** 3
    grid = vp.MaterialGrid(n, n, n, material=material(), precision=precision)
    grid.SendDataAndInitialize(R, None)
    grid.InitializeComputation(edot)
    grid.BuildLinearRefMediumStiffness()
    stream = torch.cuda.ExternalStream(grid.stream())
    # warm-up iterations (eps = 0: the loop runs exactly the requested count)
    grid.FixedPoint(edot, args.warmup, 0.0)
    grid.set_profiling(True)
    launches0 = grid.launch_count()
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with ClockSampler() as clk:
        start.record(stream)
        hist = grid.FixedPoint(edot, args.steps, 0.0)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(end)
    launches = grid.launch_count() - launches0
    phases = grid.phase_times()
    avg = hist[-1, :5].copy()
    st = grid.last_stats
    res = dict(ms=ms, N=N, phases=phases, launches=launches, clocks=clk.summary(0), avg=avg,
               iters=int(st.iterations), grid=grid, nr_capped=int(st.nr_not_converged))
    return res


def e2e_arm(args, R, edot):
    """Full increments through vpfft_run_single_strain_step with pinned host I/O."""
    import torch

    import vpfft_b200 as vp
    from vpfft_b200 import capi

    n = args.grid
    N = n ** 3
    Rp = torch.empty((N, 9), dtype=torch.float64, pin_memory=True)
    Rp.numpy()[:] = R
    Sp = torch.zeros((N, 5), dtype=torch.float64, pin_memory=True)
    Op = torch.empty((N, 5), dtype=torch.float64, pin_memory=True)
    lib = capi.load()
    grid = vp.MaterialGrid(n, n, n, material=material(), precision=args.precision)
    import ctypes as C

    e = np.ascontiguousarray(edot)
    avg = np.zeros(5)
    st = capi.Stats()
    P = C.POINTER(C.c_double)

    def one():
        capi.check(lib.vpfft_grid_set_fields(grid._h, C.cast(Rp.data_ptr(), P),
                                             C.cast(Sp.data_ptr(), P)), grid._h)
        capi.check(lib.vpfft_run_single_strain_step(grid._h, e.ctypes.data_as(P), 100, 0.005,
                                                    1e-5, avg.ctypes.data_as(P), C.byref(st)),
                   grid._h)
        capi.check(lib.vpfft_grid_get_field(grid._h, capi.FIELD_STRESS, C.cast(Op.data_ptr(), P)),
                   grid._h)
        return int(st.iterations)

    one()  # warm-up increment
    # Device-side timing on the grid's stream: every call above returns after
    # its work and copies are done, so the stream is idle between calls and
    # the two events bracket the whole host-to-host sequence.
    stream = torch.cuda.ExternalStream(grid.stream())
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    start.record(stream)
    iters = 0
    for _ in range(args.e2e_steps):
        iters += one()
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    dt = max_over_ranks(start.elapsed_time(end) / 1e3)
    grid.close()
    return dict(seconds=dt, iters=iters, N=N, h2d=N * 14 * 8, d2h=N * 5 * 8 + 40)


# ------------------------------------------------------------------ batched and serving
def material_n10():
    import vpfft_b200 as vp

    return vp.material(gamma_dot_base=1.0, rate_sensitivity=10, crss=1.0, tau0=1.0, tau1=0.5,
                       theta0=20.0, theta1=1.0)


def green_operator_arm(edges=(64, 128, 256)) -> dict:
    """The x pass's Green operator per grid size (mixed, the headline material):
    computed per wave vector or read from a stored table, as the library
    chooses it on a grid's first solve (the table is timed against the
    computed operator where it would take at most 512 MiB)."""
    import vpfft_b200 as vp
    from vpfft_b200 import fixtures

    out = {}
    e = fixtures.edot_from_matrix(VEL_GRAD)
    for n in edges:
        grains = max(1, round(N_GRAINS * (n / N_GRID) ** 3))
        g = vp.MaterialGrid(n, n, n, material=material(), precision="mixed")
        g.SendDataAndInitialize(fixtures.polycrystal(n, n, n, grains, SEED))
        g.RunSingleStrainStep(e, 2, 0.005, 0.0)
        info = g.green_operator()
        g.close()
        out[str(n)] = {"operator": {1: "computed", 2: "stored table"}.get(info["mode"], "?"),
                       "x_pass_ms_computed": info["ms_compute"] or None,
                       "x_pass_ms_table": info["ms_table"] or None,
                       "table_mib": 10 * 4 * n * n * (n // 2 + 1) / 2 ** 20}
    return out


def batched_arm(n_rves: int, iterations_per_tick: int = 8) -> dict:
    """Batched RVE solves: n_rves RVEs with edges uniform in {16, 32, 48, 64},
    8-200 Voronoi grains, random traceless velocity gradients (equivalent
    strain rate 1), n = 10, one increment each (max 100 iterations, eps 1e-5),
    all in one mixed-precision batch; against the same solves one at a time on
    the FP64 single-grid path."""
    import vpfft_b200 as vp
    from vpfft_b200 import fixtures

    rng = np.random.default_rng(SEED + 4)
    specs = [(int(rng.choice([16, 32, 48, 64])), int(rng.integers(8, 201))) for _ in range(n_rves)]
    edots = [fixtures.edot_from_matrix(fixtures.random_traceless_velocity_gradient(rng))
             for _ in specs]
    Rs = [fixtures.polycrystal(e, e, e, ng, SEED * 7 + k) for k, (e, ng) in enumerate(specs)]
    mat = material_n10()
    voxels = sum(e ** 3 for e, _ in specs)

    def run_batch(precision, grids):
        b = vp.Batch(precision, material=mat, max_slots=len(grids),
                     iterations_per_tick=iterations_per_tick)
        gs = [b.new_grid(e, e, e) for e, _ in grids]
        return b, gs

    # warm-up batch (module loading, shared-memory attributes, graph capture,
    # and the tile autotuner's one timing per RVE size): one RVE of each edge
    warm = sorted({e: k for k, (e, _) in reversed(list(enumerate(specs)))}.values())
    b, gs = run_batch("mixed", [specs[k] for k in warm])
    for g, R, e in zip(gs, [Rs[k] for k in warm], [edots[k] for k in warm]):
        g.SendDataAndInitialize(R)
        b.submit(g, e)
    b.run()
    b.poll()
    for g in gs:
        g.close()
    b.close()

    b, gs = run_batch("mixed", specs)
    for g, R in zip(gs, Rs):
        g.SendDataAndInitialize(R)
    t0 = time.perf_counter()
    ids = [b.submit(g, e) for g, e in zip(gs, edots)]
    b.run()
    t_batch = time.perf_counter() - t0
    res = {r.request_id: r for r in b.poll()}
    info = b.info()
    tunings = b.tunings()
    avg_mixed = [res[i].avg_stress for i in ids]
    iters = [res[i].iterations for i in ids]
    for g in gs:
        g.close()
    b.close()

    # one at a time, FP64 single-grid path
    t_seq = 0.0
    err = []
    for k, ((e, _), R, ed) in enumerate(zip(specs, Rs, edots)):
        if k == 0:  # warm-up of the FP64 kernels, on a grid of its own (an increment
            # also updates the voxel lengths, which SendDataAndInitialize keeps)
            w = vp.MaterialGrid(e, e, e, material=mat, precision="fp64")
            w.SendDataAndInitialize(R)
            w.RunSingleStrainStep(ed, 100, 0.005, 1e-5)
            w.close()
        g = vp.MaterialGrid(e, e, e, material=mat, precision="fp64")
        g.SendDataAndInitialize(R)
        t0 = time.perf_counter()
        avg = g.RunSingleStrainStep(ed, 100, 0.005, 1e-5)
        t_seq += time.perf_counter() - t0
        err.append(float(np.linalg.norm(avg_mixed[k] - avg) / np.linalg.norm(avg)))
        g.close()
    return {
        "metric": "RVE solves/s (one increment each), batched mixed vs one-at-a-time FP64",
        "value": n_rves / t_batch, "unit": "solves/s",
        "one_at_a_time_fp64": n_rves / t_seq,
        "speedup_vs_one_at_a_time_fp64": t_seq / t_batch,
        "rves": n_rves, "voxels": voxels, "iterations_mean": float(np.mean(iters)),
        "voxel_iters_per_s": float(sum(e ** 3 * it for (e, _), it in zip(specs, iters)) / t_batch),
        "avg_stress_rel_err_vs_fp64_max": float(max(err)),
        "graph_replays": info["graph_replays"], "kernel_launches": info["kernel_launches"],
        "ticks": info["ticks"],
        "fft_tiles_autotuned": [{"edge": t["dims"][0], "family": t["fft_tiles"],
                                 "source": t["source"],
                                 "ms_per_chain": [round(v, 4) for v in t["ms_per_chain"]]}
                                for t in tunings],
        "timing": "host wall clock around submit + run (the batch synchronises every tick)",
        "config": ("edges uniform {16,32,48,64}, grains uniform [8,200], random traceless L, "
                   "n=10, gdot0=1, CRSS=1, max 100 iterations, eps 1e-5, dt 0.005"),
        # for the CPU comparison (removed before printing)
        "_cpu_model": {"edges": [e for e, _ in specs], "iters": [int(i) for i in iters]},
    }


def serving_arm(n_requests: int, budget: int = 256 << 20) -> dict:
    """Serving: Poisson arrivals (mean 500/s) of one-increment requests on a
    pool of 64 persistent RVEs with edges {32, 48, 64, 96} (weights
    0.4/0.3/0.2/0.1), each request with its own random traceless velocity
    gradient; continuous batching through one mixed-precision batch.  The HBM
    budget for the requests' spectra (256 MiB) is about half of what all 64
    RVEs in flight would hold, so admission waits for memory as well as for
    slots (the line counts those waits)."""
    import vpfft_b200 as vp
    from vpfft_b200 import serving

    sizes, weights = [32, 48, 64, 96], [0.4, 0.3, 0.2, 0.1]
    b = vp.Batch("mixed", material=material_n10(), max_slots=64, iterations_per_tick=4,
                 hbm_budget_bytes=budget)
    pool = serving.rve_pool(b, sizes, weights, 64, SEED)
    serving.serve(b, pool, serving.poisson_trace(32, 500.0, len(pool), SEED + 1))  # warm-up
    trace = serving.poisson_trace(n_requests, 500.0, len(pool), SEED + 2)
    r = serving.serve(b, pool, trace)
    info = b.info()
    for g in pool:
        g.close()
    b.close()
    return {
        "metric": "served RVE solves/s with p50/p99 latency (arrival -> result)",
        "value": r["throughput"], "unit": "solves/s",
        "offered_rate": r["offered_rate"], "requests": r["requests"],
        "completed_ok": r["completed_ok"],
        "latency_p50_s": r["latency_p50_s"], "latency_p99_s": r["latency_p99_s"],
        "latency_max_s": r["latency_max_s"], "iterations_mean": r["iterations_mean"],
        "pool_rves": len(pool), "max_slots": 64, "iterations_per_tick": 4,
        "hbm_budget_bytes": budget,
        "admissions_deferred_for_memory": info["admissions_deferred_for_memory"],
        "config": ("Poisson arrivals mean 500/s, pool of 64 RVEs, edges {32,48,64,96} weights "
                   "0.4/0.3/0.2/0.1, grains uniform [8,200], random traceless L per request, "
                   "n=10, mixed, max 100 iterations, eps 1e-5, dt 0.005"),
        # for the CPU comparison (removed before printing)
        "_cpu_model": {"trace": trace,
                       "edges": [e for e, _ in serving.pool_specs(sizes, weights, 64, SEED)],
                       "iters": [res.iterations if res is not None else 100
                                 for res in r["results"]]},
    }


# ------------------------------------------------------------------ CPU side
def ref_binary(timing: bool = False):
    """The reference build (oracle/_ref): for timed runs its speed build
    (vpfft_ref_native, release flags + -march=x86-64-v4) when present, else the
    parity build; the C restatement when neither exists."""
    from oracle import refio

    native = os.path.join(os.path.dirname(refio.REF_BIN), "vpfft_ref_native")
    if timing and os.path.exists(native):
        return native, "reference"
    if os.path.exists(refio.REF_BIN):
        return refio.REF_BIN, "reference"
    from oracle import portlib

    portlib.build()
    return refio.PORT_BIN, "port"


def mem_available_bytes() -> int:
    try:
        with open("/proc/meminfo") as fh:
            for line in fh:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


# Host memory of the reference per voxel: its fields (orientation, stress,
# Lagrange multiplier, per-system Schmid tensors and CRSS in nested vectors,
# accumulated shear; MaterialGrid.cpp:312-394), its ten complex FFT buffers,
# and the send buffers of the input distribution (orientation + stress).
REF_BYTES_PER_VOXEL = 1300


def reference_solve(n_side, grains, seed, warm, timed, ranks):
    """The reference's own solve of the workload (n_side^3, `grains` grains,
    the fixture seed, n = 20, plane strain) on the host: the reference build
    (oracle/_ref/vpfft_ref) run as `ranks` MPI ranks over the multi-process
    stand-ins (its FFTW-MPI slab decomposition, one single-threaded process
    per core), which generates the polycrystal itself (oracle/common/
    polycrystal.c, bit-identical to the product's fixture); one increment of
    warm + timed fixed-point iterations with eps = 0.  Returns the rate over
    the timed iterations (from rank 0's timestamps at each iteration's forward
    FFT) and the share of that time inside the FFT stand-in."""
    from oracle import portlib, refio

    binary, kind = ref_binary(timing=True)
    edot = refio.edot_from_matrix(VEL_GRAD)
    m = refio.Material.uniform(1.0, RATE_SENS, 1.0, 0.5, 20.0, 1.0)
    tmp = tempfile.mkdtemp(prefix="vpfft_ref_")
    n = n_side ** 3
    try:
        if kind == "reference":
            case = refio.Case((n_side,) * 3, None, None, np.ones(12), m, edot, nsteps=1,
                              max_iter=warm + timed, dt=0.005, eps=0.0)
            extra = ["--generate", grains, seed, "--ranks", ranks, "--timing-only"]
        else:  # the C restatement has no MPI: one process
            ranks = 1
            case = refio.Case((n_side,) * 3, portlib.polycrystal(n_side, n_side, n_side, grains,
                                                                 seed, threads=host_cores()),
                              np.zeros((n, 5)), np.ones(12), m, edot, nsteps=1,
                              max_iter=warm + timed, dt=0.005, eps=0.0)
            extra = []
        t0 = time.time()
        try:
            out = refio.run(binary, case, tmp, extra_args=extra)
        except RuntimeError:
            if not binary.endswith("_native"):
                raise
            # the speed build does not run on this host's CPU: the parity build
            binary = refio.REF_BIN
            t0 = time.time()
            out = refio.run(binary, case, tmp, extra_args=extra)
        wall = time.time() - t0
    finally:
        import shutil

        shutil.rmtree(tmp, ignore_errors=True)
    ft, fs = out["fwd_times"], out["fwd_fft_seconds"]
    # ft[k]: start of iteration k's forward FFT; ft[warm + timed] starts the
    # post-loop orientation update
    span = float(ft[warm + timed] - ft[warm])
    fft_share = (float(fs[warm + timed] - fs[warm]) / span) if fs is not None else None
    return {"rate": n * timed / span, "iter_s": span / timed, "fft_share": fft_share,
            "setup_s": wall - float(ft[-1] - ft[0]),
            "wall_s": wall, "ranks": ranks, "kind": kind, "binary": binary}


def reference_sample_text(r, n_side, grains, warm, timed) -> str:
    flags = ("release flags -O3 -DNDEBUG plus -march=x86-64-v4" if r["binary"].endswith("_native")
             else "release flags -O3 -DNDEBUG")
    return (f"the reference's own code ({os.path.relpath(r['binary'], ROOT)}: Src/*.cpp "
            f"compiled unmodified, {flags}, against the project's MPI/FFTW/Eigen stand-ins) "
            f"on the full "
            f"{n_side}^3 workload ({grains} grains, same seed, material and strain rate), run as "
            f"{r['ranks']} MPI ranks (FFTW-MPI slab decomposition, one single-threaded process "
            f"per core); {warm} warm-up + {timed} timed fixed-point iterations of one increment; "
            f"{r['fft_share'] * 100:.1f} % of the timed time inside the FFT stand-in"
            if r.get("fft_share") is not None else "")


def cpu_baseline_ours(n_side=N_GRID):
    warm, timed = 1, 2
    cores = host_cores()
    need = REF_BYTES_PER_VOXEL * n_side ** 3
    if mem_available_bytes() < 1.2 * need:
        return {"unavailable": f"the reference needs ~{need / 2**30:.0f} GiB of host memory at "
                               f"{n_side}^3; {mem_available_bytes() / 2**30:.0f} GiB available"}
    r = reference_solve(n_side, N_GRAINS, SEED, warm, timed, cores)
    return {"value": r["rate"], "unit": UNIT, "cores": r["ranks"], "kind": r["kind"],
            "seconds_per_iteration": r["iter_s"], "fft_share": r["fft_share"],
            "sample": reference_sample_text(r, n_side, N_GRAINS, warm, timed)}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_increment_costs(edges, k_iters: int = 2):
    """The reference's cost of one increment (RunSingleStrainStep) of one RVE
    per edge length on the host: one single-threaded process per edge, run
    concurrently, each with eps = 0 so that it takes exactly k_iters
    fixed-point iterations (the batched/serving material, n = 10, and a
    random traceless velocity gradient).  Returns {edge: (fixed_s, iter_s)}:
    iter_s = the last iteration's time (from the harness's timestamps at each
    iteration's forward FFT), fixed_s = the increment's time outside its
    iterations (initialisation, reference medium, texture and hardening)."""
    import shutil

    from oracle import portlib, refio
    from vpfft_b200 import fixtures

    binary, kind = ref_binary()
    m = refio.Material.uniform(1.0, 10, 1.0, 0.5, 20.0, 1.0)
    rng = np.random.default_rng(SEED + 9)
    tmp = tempfile.mkdtemp(prefix="vpfft_cpu_rve_")
    runs = []
    try:
        for e in edges:
            R = portlib.polycrystal(e, e, e, 104, SEED + 11 * e)
            ed = fixtures.edot_from_matrix(fixtures.random_traceless_velocity_gradient(rng))
            case = refio.Case((e,) * 3, R, np.zeros((e ** 3, 5)), np.ones(12), m, ed, nsteps=1,
                              max_iter=k_iters, dt=0.005, eps=0.0)
            d = os.path.join(tmp, str(e))
            os.makedirs(d)
            refio.write_input(os.path.join(d, "input.bin"), case)
            runs.append((e, d, subprocess.Popen([binary, os.path.join(d, "input.bin"), d,
                                                 "--quiet"], stdout=subprocess.DEVNULL,
                                                stderr=subprocess.PIPE)))
        costs = {}
        for e, d, pr in runs:
            _, err = pr.communicate()
            if pr.returncode != 0:
                raise RuntimeError(f"reference failed at {e}^3: {err.decode()[-300:]}")
            t_inc = float(np.fromfile(os.path.join(d, "step_seconds.bin"))[0])
            ft = np.fromfile(os.path.join(d, "fwd_times.bin"))
            t_it = float(ft[k_iters] - ft[k_iters - 1])
            costs[e] = (max(0.0, t_inc - k_iters * t_it), t_it)
    finally:
        for _, _, pr in runs:
            if pr.poll() is None:
                pr.kill()
        shutil.rmtree(tmp, ignore_errors=True)
    return costs, kind, binary


def lpt_makespan(times, workers: int) -> float:
    """Makespan of independent jobs on `workers` identical workers, longest
    job first onto the least-loaded worker."""
    import heapq

    loads = [0.0] * max(1, int(workers))
    for t in sorted(times, reverse=True):
        heapq.heapreplace(loads, loads[0] + t)
    return max(loads)


def cpu_rve_baselines(models: dict) -> dict:
    """The reference on the host cores beside the batched and serving arms.
    Full solves of every RVE would take hours of CPU time (a 96^3 increment of
    100 iterations takes ~10 min on one core), so each solve's time is formed
    from measured per-edge costs: fixed_s + iterations x iter_s, with the
    iteration count of the same solve on the GPU.  Batched: the solves as
    independent single-threaded processes on every host core (longest first,
    makespan).  Serving: the same Poisson trace replayed through a FIFO pool of
    one single-threaded solver per core (serving.fifo_replay)."""
    from vpfft_b200 import serving

    edges = sorted({int(e) for mdl in models.values() for e in mdl["edges"]})
    k_iters = 2
    costs, kind, binary = cpu_increment_costs(edges, k_iters)
    cores = host_cores()

    def solve_s(e, iters):
        fixed, it = costs[int(e)]
        return fixed + iters * it

    how = (f"the reference ({os.path.relpath(binary, ROOT)}) timed per RVE edge: one increment "
           f"of one RVE per edge {edges} with {k_iters} fixed-point iterations (eps 0), one "
           "single-threaded process per edge, run concurrently; a solve's time = the measured "
           "cost outside the iterations + its iteration count (that of the same solve on the "
           "GPU) x the measured iteration time")
    per_edge = {str(e): {"fixed_s": c[0], "iteration_s": c[1]} for e, c in costs.items()}
    out = {}
    if "batched" in models:
        bm = models["batched"]
        times = [solve_s(e, it) for e, it in zip(bm["edges"], bm["iters"])]
        mk = lpt_makespan(times, cores)
        out["batched"] = {
            "value": len(times) / mk, "unit": "solves/s", "cores": cores, "kind": kind,
            "method": "modelled from measured per-edge costs",
            "sample": how + f"; {len(times)} solves on {cores} cores, longest first (makespan "
                            f"{mk:.1f} s)",
            "per_edge": per_edge}
    if "serving" in models:
        sm = models["serving"]
        trace = sm["trace"]
        svc = [solve_s(sm["edges"][req.rve], it) for req, it in zip(trace, sm["iters"])]
        rep = serving.fifo_replay(trace, svc, cores)
        out["serving"] = {
            "value": rep["throughput"], "unit": "solves/s", "cores": cores, "kind": kind,
            "latency_p50_s": rep["latency_p50_s"], "latency_p99_s": rep["latency_p99_s"],
            "method": "modelled from measured per-edge costs",
            "sample": how + f"; the same {len(trace)}-request trace through a FIFO pool of "
                            f"{cores} single-threaded solvers",
            "per_edge": per_edge}
    return out


# ------------------------------------------------------------------ distributed helpers
_dist = None


def setup_dist(n_gpus, backend: str = "nccl"):
    """One process per GPU under torchrun (RANK/WORLD_SIZE/MASTER_* from the
    environment); the process group only carries the barrier and the
    max-over-ranks of the timings (replicas: no collective in the data path).
    backend "gloo" runs the same logic on CPU."""
    global _dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        _dist = dist
    return int(os.environ.get("RANK", "0")), ws


def _coll_device():
    return "cuda" if _dist is not None and _dist.get_backend() == "nccl" else "cpu"


def barrier():
    if _dist is not None:
        if _coll_device() == "cuda":
            import torch

            _dist.barrier(device_ids=[torch.cuda.current_device()])
        else:
            _dist.barrier()


def max_over_ranks(x: float) -> float:
    if _dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=_coll_device())
    _dist.all_reduce(t, op=_dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world_size: int, seconds_max: float) -> float:
    """Aggregate rate of a replica run: every rank processed units_per_rank in
    at most seconds_max (the maximum over ranks)."""
    return units_per_rank * world_size / seconds_max


# ------------------------------------------------------------------ main
def run_reference_arm(args, rank, ws):
    """The reference's CPU solve of the headline workload on the host cores
    (rank 0 only), printed as the reference arm's JSON line."""
    if rank != 0:
        return 0
    n_side = args.grid
    grains = N_GRAINS if n_side == N_GRID else max(1, round(N_GRAINS * (n_side / N_GRID) ** 3))
    cores = host_cores()
    need = REF_BYTES_PER_VOXEL * n_side ** 3
    base = {"metric": METRIC, "impl": "reference", "unit": UNIT}
    if mem_available_bytes() < 1.2 * need:
        base["unavailable"] = (f"the reference needs ~{need / 2**30:.0f} GiB of host memory at "
                               f"{n_side}^3 and {mem_available_bytes() / 2**30:.0f} GiB are "
                               "available")
        print(json.dumps(base), flush=True)
        return 0
    r = reference_solve(n_side, grains, SEED, args.warmup, args.steps, cores)
    line = dict(base)
    line.update({
        "value": r["rate"], "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * r["iter_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload(n_side), "grid": [n_side] * 3, "grains": grains,
                   "seed": SEED, "precision": "fp64 (the reference's Float is double)",
                   "step": "one fixed-point iteration of the whole grid",
                   "mpi_ranks": r["ranks"]},
        "cpu_baseline": {"value": r["rate"], "unit": UNIT, "cores": r["ranks"], "kind": r["kind"],
                         "seconds_per_iteration": r["iter_s"], "fft_share": r["fft_share"],
                         "sample": reference_sample_text(r, n_side, grains, args.warmup,
                                                         args.steps)},
        "e2e": {"value": r["rate"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "wall_s": r["wall_s"],
    })
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", type=int, default=N_GRID)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-green", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--batch-rves", type=int, default=256)
    ap.add_argument("--serve-requests", type=int, default=1000)
    args = ap.parse_args(argv)
    rank, ws = setup_dist(args.gpus)
    if args.impl == "reference":
        rc = run_reference_arm(args, rank, ws)
        if _dist is not None:
            _dist.destroy_process_group()
        return rc

    import torch

    import vpfft_b200 as vp
    from vpfft_b200 import build as vbuild

    if not os.path.exists(vp.capi.LIB_PATH):
        vbuild.build()
    torch.cuda.init()
    R, edot = make_inputs(args.grid, N_GRAINS if args.grid == N_GRID else
                          max(1, round(N_GRAINS * (args.grid / N_GRID) ** 3)))
    hbm, peak_kind = peaks()

    main_res = device_arm(args, R, edot, args.precision)
    ms = max_over_ranks(main_res["ms"])
    N = main_res["N"]
    value = whole_job_rate(N * args.steps, ws, ms / 1e3)

    # per-kernel device times and the roofline of the dominant kernel
    s = 4 if args.precision == "mixed" else 8
    alg = alg_bytes_per_voxel(s, args.grid)
    kernels = {}
    for name, (tot_ms, cnt) in main_res["phases"].items():
        if cnt == 0:
            continue
        avg_ms = tot_ms / cnt
        kernels[name] = {"avg_ms": avg_ms, "launches": cnt,
                         "alg_bytes": alg[name] * N,
                         "achieved_gbs": alg[name] * N / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0}
    total_k = sum(k["avg_ms"] for k in kernels.values())
    for k in kernels.values():
        k["share"] = k["avg_ms"] / total_k if total_k else 0
    dom = max(kernels, key=lambda k: kernels[k]["avg_ms"])
    it_bytes = sum(alg.values()) * N
    roofline = {
        "bound": "hbm", "kernel": dom,
        "achieved": kernels[dom]["achieved_gbs"], "peak": hbm, "unit": "GB/s",
        "frac": kernels[dom]["achieved_gbs"] / hbm, "peak_kind": peak_kind,
        "traffic": (TRAFFIC_PER_VOXEL[(args.precision, dom)] * N
                    if (args.precision, dom) in TRAFFIC_PER_VOXEL else None),
        "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at "
                           "192^3, scaled by the voxel count"
                           if (args.precision, dom) in TRAFFIC_PER_VOXEL else None),
        "alg_bytes_per_voxel": alg[dom],
        "iteration": {"alg_bytes_per_voxel": sum(alg.values()),
                      "achieved_gbs": it_bytes / (ms / args.steps * 1e-3) / 1e9,
                      "frac": it_bytes / (ms / args.steps * 1e-3) / 1e9 / hbm},
    }
    if (args.precision, dom) in WARP_INST_PER_VOXEL:
        # the bound the NR sweep actually meets: instruction issue (four
        # schedulers per SM, one warp instruction per cycle each)
        import torch

        sms = torch.cuda.get_device_properties(0).multi_processor_count
        clk = main_res["clocks"].get("sm_mhz") or main_res["clocks"].get("sm_max_mhz") or 1965.0
        wpv = WARP_INST_PER_VOXEL[(args.precision, dom)]
        achieved_i = wpv * N / (kernels[dom]["avg_ms"] * 1e-3)
        peak_i = sms * 4 * clk * 1e6
        roofline["issue"] = {
            "bound": "instruction issue", "achieved": achieved_i / 1e9, "peak": peak_i / 1e9,
            "unit": "G warp-instructions/s", "frac": achieved_i / peak_i,
            "warp_instructions_per_voxel": wpv, "sm_mhz": clk, "sms": sms,
            "source": ("smsp__inst_executed.sum of one launch at 192^3 per voxel (ncu), x the "
                       "voxel count, / the kernel's CUDA-event duration; peak = SMs x 4 "
                       "schedulers x the sampled SM clock")}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 fields/FFT + f64 NR" if args.precision == "mixed" else "f64",
        "data": "synthetic",
        "config": {"workload": workload(args.grid), "grid": [args.grid] * 3, "grains": N_GRAINS,
                   "seed": SEED, "precision": args.precision,
                   "l2": (f"inputs larger than L2 (resident fields of the {args.grid}^3 grid)"
                          if args.grid >= 128 else
                          f"resident fields of the {args.grid}^3 grid (smaller than L2)"),
                   "parallelism": f"replicas x{ws}"},
        "roofline": roofline,
        "kernels": kernels,
        "gpu_launches": main_res["launches"],
        "clocks": main_res["clocks"],
    }
    main_grid = main_res.pop("grid")

    if not args.no_fp64 and args.precision == "mixed":
        f = device_arm(args, R, edot, "fp64")
        ms64 = max_over_ranks(f["ms"])
        v64 = N * args.steps * ws / (ms64 / 1e3)
        # error of the mixed path against the FP64 GPU path after the same
        # number of iterations from the same state
        s_m = main_grid.Stress()
        s_d = f["grid"].Stress()
        e_m = main_grid.StrainRate()
        e_d = f["grid"].StrainRate()
        rel_s = np.linalg.norm(s_m - s_d, axis=1) / np.linalg.norm(s_d, axis=1)
        line["fp64"] = {
            "value": v64, "unit": UNIT, "ms_per_step": ms64 / args.steps,
            "mixed_over_fp64": value / v64,
            "error_vs_fp64": {
                "avg_stress_rel": float(np.linalg.norm(main_res["avg"] - f["avg"]) /
                                        np.linalg.norm(f["avg"])),
                "stress_field_max_rel": float(rel_s.max()),
                "stress_field_rel_p99": float(np.quantile(rel_s, 0.99)),
                "stress_field_rel_p99_99": float(np.quantile(rel_s, 0.9999)),
                "voxels_stress_rel_above_1e-3": int(np.count_nonzero(rel_s > 1e-3)),
                "nr_not_converged_voxel_iters": {"mixed": int(main_res["nr_capped"]),
                                               "fp64": int(f["nr_capped"])},
                "strain_rate_field_rms_rel": float(np.sqrt(np.mean((e_m - e_d) ** 2)) /
                                                   np.sqrt(np.mean(e_d ** 2))),
                "iterations": args.warmup + args.steps},
        }
        f["grid"].close()
    main_grid.close()

    if not args.no_e2e:
        e = e2e_arm(args, R, edot)
        line["e2e"] = {"value": e["N"] * e["iters"] * ws / e["seconds"], "unit": UNIT,
                       "h2d_bytes_per_step": e["h2d"], "d2h_bytes_per_step": e["d2h"],
                       "steps": args.e2e_steps, "iterations": e["iters"],
                       "step": ("one increment via vpfft_run_single_strain_step (max_iter 100, "
                                "eps 1e-5) with pinned host orientation/stress in and the "
                                "stress field out")}
    if ws == 1 and not args.no_green:
        line["green_operator"] = green_operator_arm()
    if ws == 1 and not args.no_batched:
        line["batched"] = batched_arm(args.batch_rves)
    if ws == 1 and not args.no_serving:
        line["serving"] = serving_arm(args.serve_requests)
    models = {k: line[k].pop("_cpu_model") for k in ("batched", "serving") if k in line}
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_ours()
        if models:
            try:
                for k, v in cpu_rve_baselines(models).items():
                    line[k]["cpu_baseline"] = v
            except (RuntimeError, OSError, ValueError) as exc:
                for k in models:
                    line[k]["cpu_baseline"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if _dist is not None:
        _dist.destroy_process_group()
    return 0


# DRAM bytes per voxel of one launch (dram__bytes_read.sum + dram__bytes_write.sum
# divided by the voxel count) from the ncu capture at 192^3 summarised in
# profiles/k_nr_update_192cubed_mixed.md; the kernel's traffic is proportional to
# the voxel count (it streams each voxel's fields once), so it scales to 256^3.
TRAFFIC_PER_VOXEL: dict = {("mixed", "nr_update"): 1055.5e6 / 192 ** 3}
# Warp instructions per voxel of one launch (smsp__inst_executed.sum divided by
# the voxel count) from the same capture; the per-voxel instruction count does
# not depend on the grid size (each voxel's solve is independent of it).
WARP_INST_PER_VOXEL: dict = {("mixed", "nr_update"): 0.6927e9 / 192 ** 3}


if __name__ == "__main__":
    sys.exit(main())
