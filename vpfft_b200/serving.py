"""A request loop standing in for a multiscale macro driver: RVE solve
requests arrive as a Poisson stream, each one increment on a persistent
device-resident RVE of a pool (fields, texture and CRSS kept across requests)
with its own velocity gradient.  Requests are submitted to a Batch as they
arrive and admitted by the engine as slots and HBM budget free up, so their
work overlaps on the device with the requests already running (continuous
batching).  Latency is measured from the scheduled arrival time to the end of
the tick that completed the request.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import capi, fixtures
from .batch import Batch


@dataclass
class Request:
    t_arrival: float        # seconds after the start of the trace
    rve: int                # index into the pool
    L: np.ndarray           # 3x3 velocity gradient
    edot: np.ndarray = field(default=None)


def poisson_trace(n: int, rate: float, n_rves: int, seed: int) -> list[Request]:
    """n arrivals with exponential inter-arrival times (mean 1/rate), each
    targeting a uniformly chosen RVE of the pool, with a random traceless
    velocity gradient normalised to equivalent strain rate 1."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for k in range(n):
        L = fixtures.random_traceless_velocity_gradient(rng)
        out.append(Request(float(t[k]), int(rng.integers(n_rves)), L, fixtures.edot_from_matrix(L)))
    return out


def pool_specs(sizes, weights, n: int, seed: int, grains=(8, 200)) -> list[tuple[int, int]]:
    """(edge, grain count) of the n RVEs of a pool: edges drawn from `sizes`
    with `weights`, grain counts uniform in `grains` (seeded)."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        s = int(rng.choice(sizes, p=np.asarray(weights) / np.sum(weights)))
        ng = int(rng.integers(grains[0], grains[1] + 1))
        specs.append((s, ng))
    return specs


def rve_pool(batch: Batch, sizes, weights, n: int, seed: int, grains=(8, 200)):
    """n grids with sizes drawn from `sizes` (edge lengths) with `weights`,
    seeded Voronoi microstructures with a grain count uniform in `grains`."""
    pool = []
    for k, (s, ng) in enumerate(pool_specs(sizes, weights, n, seed, grains)):
        g = batch.new_grid(s, s, s)
        g.SendDataAndInitialize(fixtures.polycrystal(s, s, s, ng, seed * 1000 + k))
        pool.append(g)
    return pool


def fifo_replay(trace: list[Request], service_s, workers: int) -> dict:
    """Latency and throughput of a trace served by `workers` single-threaded
    solvers taking requests in arrival order, each request on the earliest
    free worker but not before the previous request on its RVE has finished
    (an RVE's state carries from one increment to the next).  service_s[k]
    is request k's solve time in seconds."""
    import heapq

    free = [0.0] * max(1, int(workers))
    rve_free: dict[int, float] = {}
    latency = np.zeros(len(trace))
    last = 0.0
    for k, r in enumerate(trace):
        w = heapq.heappop(free)
        start = max(r.t_arrival, w, rve_free.get(r.rve, 0.0))
        done = start + float(service_s[k])
        heapq.heappush(free, done)
        rve_free[r.rve] = done
        latency[k] = done - r.t_arrival
        last = max(last, done)
    span = last - trace[0].t_arrival
    return {
        "throughput": len(trace) / span if span > 0 else float("inf"),
        "latency_p50_s": float(np.quantile(latency, 0.5)),
        "latency_p99_s": float(np.quantile(latency, 0.99)),
        "latency_max_s": float(latency.max()),
    }


def serve(batch: Batch, pool, trace: list[Request], max_iter: int = 100, dt: float = 0.005,
          eps: float = 1e-5) -> dict:
    """Replays the trace in real time through the batch.  Returns throughput,
    latency percentiles and the per-request results (in trace order)."""
    pending = list(range(len(trace)))
    pending.reverse()  # pop() gives arrival order
    id_to_req: dict[int, int] = {}
    results: list = [None] * len(trace)
    latency = np.zeros(len(trace))
    t0 = time.perf_counter()
    in_flight = 0
    while pending or in_flight:
        now = time.perf_counter() - t0
        while pending and trace[pending[-1]].t_arrival <= now:
            k = pending.pop()
            r = trace[k]
            rid = batch.submit(pool[r.rve], r.edot, max_iter, dt, eps)
            id_to_req[rid] = k
            in_flight += 1
        if in_flight == 0:
            time.sleep(max(0.0, trace[pending[-1]].t_arrival - now))
            continue
        batch.step()
        t_done = time.perf_counter() - t0
        for res in batch.poll():
            k = id_to_req.pop(res.request_id)
            results[k] = res
            latency[k] = t_done - trace[k].t_arrival
            in_flight -= 1
    elapsed = time.perf_counter() - t0
    ok = [r for r in results if r is not None and r.status == capi.OK]
    span = elapsed - trace[0].t_arrival
    return {
        "requests": len(trace),
        "completed_ok": len(ok),
        "seconds": elapsed,
        "throughput": len(trace) / span,
        "offered_rate": len(trace) / trace[-1].t_arrival,
        "latency_p50_s": float(np.quantile(latency, 0.5)),
        "latency_p99_s": float(np.quantile(latency, 0.99)),
        "latency_max_s": float(latency.max()),
        "iterations_mean": float(np.mean([r.iterations for r in ok])) if ok else 0.0,
        "results": results,
        "latency": latency,
    }
