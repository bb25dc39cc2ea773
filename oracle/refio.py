"""I/O for the test oracles (oracle/_ref/vpfft_ref and oracle/_build/vpfft_port).

Test-oracle infrastructure: imported only by tests/, tests/golden/ scripts,
``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py.

Input file ("VPFFTIN1") layout, little-endian:
    char[8]  magic
    int32[8] nx, ny, nz, nsteps, max_iter, crss_per_voxel, edot_per_increment, generated
    f64      dt, eps, edot[5], h[3]
    f64[12]  gamma_dot_base          int32[12] rate_sensitivity
    f64[12]  tau0, tau1, theta0, theta1
    f64[144] hardening matrix (row-major h[s][t])
    f64[N*9] R   (row-major 3x3 per voxel, voxel index x*Ny*Nz + y*Nz + z)
    f64[N*5] sigma (deviatoric 5-vector per voxel)
                 (R and sigma are absent when `generated`: the reference
                 harness then makes the synthetic polycrystal itself from
                 --generate GRAINS SEED, with sigma = 0)
    f64[N*12 or 12] CRSS
    f64[nsteps*5] strain rate of each increment (only when edot_per_increment;
                  otherwise every increment uses `edot`)

The per-voxel order and the 3x3 / 5-vector layouts are the reference's
(MaterialGrid.h:121-124 ToIndex; SMatrix3x3 m[3][3], LinearAlgebra.h:114;
EigenRep m[5], LinearAlgebra.h:300).
"""
from __future__ import annotations

import json
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "vpfft_ref")
PORT_BIN = os.path.join(HERE, "_build", "vpfft_port")


@dataclass
class Material:
    """Per-slip-system material constants (12 FCC systems)."""

    gamma_dot_base: np.ndarray = field(default_factory=lambda: np.full(12, 15.5))
    rate_sensitivity: np.ndarray = field(default_factory=lambda: np.full(12, 10, np.int32))
    tau0: np.ndarray = field(default_factory=lambda: np.full(12, 11.0))
    tau1: np.ndarray = field(default_factory=lambda: np.full(12, 11.0))
    theta0: np.ndarray = field(default_factory=lambda: np.full(12, 430.0))
    theta1: np.ndarray = field(default_factory=lambda: np.full(12, 110.0))
    hardening: np.ndarray = field(default_factory=lambda: np.ones((12, 12)))

    @staticmethod
    def uniform(gdot, n, tau0=11.0, tau1=11.0, theta0=430.0, theta1=110.0, h=1.0):
        return Material(
            np.full(12, float(gdot)),
            np.full(12, int(n), np.int32),
            np.full(12, float(tau0)),
            np.full(12, float(tau1)),
            np.full(12, float(theta0)),
            np.full(12, float(theta1)),
            np.full((12, 12), float(h)),
        )


@dataclass
class Case:
    dims: tuple
    R: np.ndarray  # (N, 9), or None: the harness generates the orientations
    sigma: np.ndarray  # (N, 5)
    crss: np.ndarray  # (12,) or (N, 12)
    material: Material
    edot: np.ndarray  # (5,)
    nsteps: int = 1
    max_iter: int = 100
    dt: float = 0.005
    eps: float = 1e-5
    h: tuple = (1.0, 1.0, 1.0)
    edot_steps: np.ndarray = None  # (nsteps, 5): a strain rate per increment


def edot_from_matrix(L) -> np.ndarray:
    """EigenRep(SMatrix3x3) (LinearAlgebra.h:307-312): the projection of a 3x3
    velocity gradient on the deviatoric basis (LinearAlgebra.h:207-247), summed
    over the nine entries in row-major order."""
    a, b = 1.0 / np.sqrt(2.0), 1.0 / np.sqrt(6.0)
    B = np.zeros((5, 3, 3))
    B[0, 0, 0], B[0, 1, 1] = -1 * a, 1 * a
    B[1, 0, 0], B[1, 1, 1], B[1, 2, 2] = -1 * b, -1 * b, 2 * b
    B[2, 1, 2] = B[2, 2, 1] = 1 * a
    B[3, 0, 2] = B[3, 2, 0] = 1 * a
    B[4, 0, 1] = B[4, 1, 0] = 1 * a
    L = np.asarray(L, np.float64).reshape(3, 3)
    out = np.zeros(5)
    for k in range(5):
        r = 0.0
        for i in range(3):
            for j in range(3):
                r += float(L[i, j]) * float(B[k, i, j])
        out[k] = r
    return out


def write_input(path: str, c: Case) -> None:
    nx, ny, nz = c.dims
    n = nx * ny * nz
    per_voxel = 1 if np.asarray(c.crss).ndim == 2 else 0
    per_inc = 0 if c.edot_steps is None else 1
    generated = 1 if c.R is None else 0
    m = c.material
    with open(path, "wb") as f:
        f.write(b"VPFFTIN1")
        f.write(np.array([nx, ny, nz, c.nsteps, c.max_iter, per_voxel, per_inc, generated],
                         "<i4").tobytes())
        f.write(np.array([c.dt, c.eps], "<f8").tobytes())
        f.write(np.asarray(c.edot, "<f8").reshape(5).tobytes())
        f.write(np.asarray(c.h, "<f8").reshape(3).tobytes())
        f.write(np.asarray(m.gamma_dot_base, "<f8").reshape(12).tobytes())
        f.write(np.asarray(m.rate_sensitivity, "<i4").reshape(12).tobytes())
        for a in (m.tau0, m.tau1, m.theta0, m.theta1):
            f.write(np.asarray(a, "<f8").reshape(12).tobytes())
        f.write(np.asarray(m.hardening, "<f8").reshape(144).tobytes())
        if not generated:
            f.write(np.ascontiguousarray(c.R, "<f8").reshape(n * 9).tobytes())
            f.write(np.ascontiguousarray(c.sigma, "<f8").reshape(n * 5).tobytes())
        f.write(np.ascontiguousarray(c.crss, "<f8").reshape(-1).tobytes())
        if per_inc:
            f.write(np.ascontiguousarray(c.edot_steps, "<f8").reshape(c.nsteps * 5).tobytes())


def _rd(outdir, name, shape=None):
    p = os.path.join(outdir, name)
    if not os.path.exists(p):
        return None
    a = np.fromfile(p, "<f8")
    if shape is not None and a.size == 0:
        return None  # not recorded (--timing-only)
    return a.reshape(shape) if shape is not None else a


def read_output(outdir: str, n: int) -> dict:
    """Read what the oracle CLI wrote (see ref_harness.cpp)."""
    out = {}
    steps = _rd(outdir, "steps.bin", (-1, 6))
    out["iters"] = steps[:, 0].astype(int)
    out["avg_stress"] = steps[:, 1:]
    out["allreduce"] = _rd(outdir, "allreduce.bin")
    out["allreduce_counts"] = _rd(outdir, "allreduce_counts.bin").astype(int)
    out["step_seconds"] = _rd(outdir, "step_seconds.bin")
    out["fwd_times"] = _rd(outdir, "fwd_times.bin")
    out["fwd_increment"] = _rd(outdir, "fwd_increment.bin")
    out["fwd_fft_seconds"] = _rd(outdir, "fwd_fft_seconds.bin")
    for name, w in (("sigma", 5), ("lambda", 5), ("R", 9), ("crss", 12), ("P_last", 5),
                    ("dtilde_last", 5), ("schmid", 60)):
        out[name] = _rd(outdir, name + ".bin", (n, w))
    out["accshear"] = _rd(outdir, "accshear.bin")
    out["voxlen"] = _rd(outdir, "voxlen.bin")
    widths = {"sigma": 5, "lambda": 5, "R": 9, "crss": 12, "P": 5, "dtilde": 5}
    for fn in os.listdir(outdir):
        if (fn.startswith("it") or fn.startswith("inc")) and fn.endswith(".bin"):
            key = fn[:-4]
            out[key] = _rd(outdir, fn, (n, widths[key.split("_", 1)[1]]))
    return out


def l0_per_increment(out: dict, nx: int) -> list:
    """Reference medium L0 of each increment, from the 25 allreduce values that
    open it (MaterialGrid.cpp:257-271: value = M(i,j)*DimXLocal, then
    M(i,j) = value/DimX, then NormalizeValues zeroes |M_ij| < 1e-10,
    LinearAlgebra.h:605-613).  Returned as 5x5 arrays indexed [i, j]."""
    ar = out["allreduce"]
    res, off = [], 0
    for cnt in out["allreduce_counts"]:
        vals = ar[off:off + 25]
        m = np.zeros((5, 5))
        k = 0
        for i in range(5):
            for j in range(5):
                v = vals[k] / float(nx)
                m[i, j] = 0.0 if abs(v) < 1e-10 else v
                k += 1
        res.append(m)
        off += cnt
    return res


def _inner(a, b) -> float:
    r = 0.0
    for x, y in zip(a, b):
        r += float(x) * float(y)
    return r


def iteration_history(out: dict, dims, edot) -> list:
    """Per increment, per fixed-point iteration: (<sigma>, <edot>, delta_sigma,
    delta_eps) formed from the reduced sums exactly as the reference does
    (MaterialGrid.cpp:1009-1053): sums / N, then the error norms divided by
    |<sigma>| and |Edot|.  `edot` is one strain rate (5,) or one per
    increment (nsteps, 5)."""
    nx, ny, nz = dims
    n = float(nx * ny * nz)
    edots = np.asarray(edot, np.float64).reshape(-1, 5)
    ar = out["allreduce"]
    hist, off = [], 0
    for k, cnt in enumerate(out["allreduce_counts"]):
        e_k = edots[k if len(edots) > 1 else 0]
        en = np.sqrt(_inner(e_k, e_k))
        its = []
        vals = ar[off + 25: off + cnt].reshape(-1, 12)
        for row in vals:
            s = row[0:10:2] / n
            e = row[1:10:2] / n
            ds = (row[10] / n) / np.sqrt(_inner(s, s))
            de = (row[11] / n) / en
            its.append((s, e, ds, de))
        hist.append(its)
        off += cnt
    return hist


def run(binary: str, case: Case, workdir: str, dump_iters=(), dump_increments=False,
        timeout=None, run_vpfft=False, extra_args=()) -> dict:
    """Run an oracle CLI on `case` in `workdir` and read its outputs.
    run_vpfft: drive the increments through the reference's own RunVPFFT
    (reference build only), which also writes workdir/Stress_Strain.txt."""
    os.makedirs(workdir, exist_ok=True)
    inp = os.path.join(workdir, "input.bin")
    write_input(inp, case)
    cmd = [binary, inp, workdir, "--quiet"]
    for k in dump_iters:
        cmd += ["--dump-iter", str(int(k))]
    if dump_increments:
        cmd += ["--dump-increments"]
    if run_vpfft:
        cmd += ["--run-vpfft"]
    cmd += [str(a) for a in extra_args]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{binary} failed ({r.returncode}): {r.stderr[-2000:]}")
    summary = json.loads(r.stdout.strip().splitlines()[-1])
    nx, ny, nz = case.dims
    out = read_output(workdir, nx * ny * nz)
    out["summary"] = summary
    return out
