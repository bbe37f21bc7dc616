"""Serving loop: many independent lattices resident on one GPU.

A thin wrapper of the ``m3lb_serve_*`` C ABI (include/m3lb.h) plus the
seeded request stream of the serving workload and its latency summary.  The
reference runs one solver per process and has no serving loop; the request
mix below is the serving workload of the benchmark: Poisson arrivals at a
mean rate, cubic periodic Taylor-Green boxes of N in {32, 48, ..., 160},
operator uniform over BGK / TRT / CM, amplitude u0 uniform in [0.02, 0.08],
step count uniform in [200, 2000], FP16 storage.  The workload states no
relaxation time; requests use tau = 0.6 (TRT: omega_minus from the magic
parameter 3/16), a choice stable for all three operators at these amplitudes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi

OP_CODES = {"bgk": capi.OP_BGK, "trt": capi.OP_TRT, "mrt": capi.OP_MRT, "cm": capi.OP_CM}
SIZES = tuple(range(32, 161, 16))
TAU = 0.6
LAMBDA_TRT = 3.0 / 16.0


def rates(op: int, tau: float = TAU):
    """(omega, omega2) of a request: BGK/CM at 1/tau; TRT omega_minus from
    the magic parameter (TRT.hpp:92-127); the moment operators' bulk rate
    follows omega (omega2 < 0)."""
    w = 1.0 / tau
    if op == capi.OP_TRT:
        return w, 1.0 / (LAMBDA_TRT / (1.0 / w - 0.5) + 0.5)
    return w, -1.0


@dataclass
class Request:
    id: int
    arrival: float
    n: int
    op: int
    steps: int
    u0: float

    def nodes(self) -> int:
        return self.n ** 3


def request_stream(count: int = 500, rate: float = 50.0, seed: int = 0, sizes=SIZES,
                   ops=("bgk", "trt", "cm"), u0=(0.02, 0.08), steps=(200, 2000)):
    """The seeded serving workload: `count` requests, Poisson arrivals at
    `rate` per second starting at t = 0."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    t = np.concatenate([[0.0], np.cumsum(gaps[:-1])])
    ns = rng.choice(np.asarray(sizes), size=count)
    op = rng.choice(np.asarray([OP_CODES[o] for o in ops]), size=count)
    amp = rng.uniform(u0[0], u0[1], size=count)
    st = rng.integers(steps[0], steps[1] + 1, size=count)
    return [Request(i, float(t[i]), int(ns[i]), int(op[i]), int(st[i]), float(amp[i]))
            for i in range(count)]


def offered_lups(reqs) -> float:
    """Lattice updates per second the stream asks for (sum of N^3 * steps
    over the arrival window)."""
    if len(reqs) < 2:
        return 0.0
    span = max(r.arrival for r in reqs) - min(r.arrival for r in reqs)
    return sum(r.nodes() * r.steps for r in reqs) / max(span, 1e-9)


class Server:
    """One serving loop on the current CUDA device."""

    MAPPINGS = {"auto": capi.MAP_AUTO, "chunks": capi.MAP_CHUNKS, "dense": capi.MAP_DENSE,
                "tune": capi.MAP_TUNE, "rows": capi.MAP_ROWS}

    def __init__(self, hbm_budget: int = 4 << 30, max_resident: int = 32, round_steps: int = 50,
                 storage: str = "f16", keep_fields: bool = False, mapping: str = "auto"):
        self.storage = capi.STORAGE_NAMES[storage]
        cfg = capi.ServeConfig(hbm_budget, max_resident, round_steps, self.storage,
                               int(keep_fields), self.MAPPINGS[mapping])
        h = C.c_void_p()
        capi.check(capi.lib().m3lb_serve_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._n = {}

    def submit(self, r: Request, tau: float = TAU):
        w, w2 = rates(r.op, tau)
        req = capi.Request(r.id, r.arrival, r.n, r.op, r.steps, r.u0, w, w2)
        capi.check(capi.lib().m3lb_serve_submit(self._h, C.byref(req)))
        self._n[r.id] = r.n

    def run(self, time_limit: float = 0.0):
        capi.check(capi.lib().m3lb_serve_run(self._h, float(time_limit)))

    def results(self):
        cnt = C.c_int(0)
        capi.check(capi.lib().m3lb_serve_results(self._h, None, 0, C.byref(cnt)))
        arr = (capi.Result * max(cnt.value, 1))()
        capi.check(capi.lib().m3lb_serve_results(self._h, arr, cnt.value, C.byref(cnt)))
        return [arr[i] for i in range(cnt.value)]

    def fields(self, rid: int):
        n = self._n[rid]
        out = [np.empty((n, n, n), np.float32) for _ in range(4)]
        capi.check(capi.lib().m3lb_serve_fields(self._h, rid, *[a.ctypes.data for a in out]))
        return out

    def stats(self):
        st = capi.ServeStats()
        capi.check(capi.lib().m3lb_serve_get_stats(self._h, C.byref(st)))
        return st

    def close(self):
        if self._h:
            capi.lib().m3lb_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def summary(results, reqs=None) -> dict:
    """Latency (queue + run, per request) percentiles, served rate and the
    aggregate lattice-update rate over the makespan."""
    lat = np.array([r.finished - r.arrival for r in results])
    end = max(r.finished for r in results)
    start = min(r.arrival for r in results)
    lups = sum(r.node_steps for r in results)
    out = {
        "requests": len(results),
        "latency_p50_s": float(np.percentile(lat, 50)),
        "latency_p99_s": float(np.percentile(lat, 99)),
        "latency_max_s": float(lat.max()),
        "makespan_s": float(end - start),
        "served_rate_per_s": len(results) / float(end - start),
        "aggregate_mlups": lups / float(end - start) / 1e6,
    }
    if reqs:
        span = max(r.arrival for r in reqs) - min(r.arrival for r in reqs)
        out["offered_rate_per_s"] = (len(reqs) - 1) / max(span, 1e-9)
        out["offered_mlups"] = offered_lups(reqs) / 1e6
    return out
