#!/usr/bin/env python
"""Benchmark of the M3LB lattice-Boltzmann step on B200.

Workload (one "step" = one fused stream-collide time step over the whole
lattice): D3Q27 central-moment Taylor-Green vortex on a periodic 256^3
lattice (u0 = 0.05, Re = 1600 on L = N / 2 pi, tau = 0.5 + 3 u0 N / (2 pi Re)),
populations stored shifted in FP16 with FP32 arithmetic.  The same workload
with FP32 storage is timed alongside for the FP16/FP32 ratio.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl m3lb|reference]

One process per GPU; under torchrun each rank advances its own replica
lattice (no data exchange: "replicas only"), time is the max over ranks.
Prints one JSON line on rank 0.  --impl reference times the reference's own
CPU implementation of the step (its src/ headers built against a host stand-in
for Kokkos, oracle/_ref) on this machine's host cores.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import math
import os
import subprocess
import sys
import time
from datetime import timedelta
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

N_DEFAULT = 256
KERNELS = {"auto": 0, "nodes": 1, "pairs": 2, "stream": 3, "rows": 4}
# what auto runs for the 256^3 FP16 workload (FP32 storage runs step_pairs)
KERNEL_NAMES = {"auto": "step_rows", "pairs": "step_pairs", "stream": "step_stream",
                "nodes": "step_nodes", "rows": "step_rows"}
U0 = 0.05
RE = 1600.0
Q = 27
L2_BYTES = 126 * 2 ** 20
STORAGE_BYTES = {"f16": 2, "f16c": 2, "bf16": 2, "f32": 4, "f64": 8}
STORAGE_NOTE = {
    "f16": "IEEE binary16 shifted populations",
    "f16c": ("FP16C shifted populations: a 16-bit float with 1 sign, 4 exponent and 11 mantissa "
             "bits (IEEE binary16's top exponent bit given to the mantissa), FP32 arithmetic"),
    "bf16": "bfloat16 shifted populations", "f32": "FP32 populations"}
METRIC = "D3Q27 CM MLUPS & HBM GB/s (FP16 vs FP32 store) at 256^3; p99 request latency"
WORKLOAD = ("D3Q27 central-moment Taylor-Green vortex, periodic 256^3, "
            "shifted populations stored in 16 bits, FP32 arithmetic")


def tgv_params(n):
    L = n / (2 * math.pi)
    nu = U0 * L / RE
    tau = 3 * nu + 0.5
    return nu, tau, 1.0 / tau


def tgv_fields(n, xp=np):
    """Taylor-Green benchmark initial field (validation/tgv3d_bench.cpp IC):
    u = u0 sin x cos y cos z, v = -u0 cos x sin y cos z, w = 0, analytic
    pressure in the density."""
    k = 2 * math.pi / n
    i = xp.arange(n, dtype=xp.float64) * k
    z, y, x = xp.meshgrid(i, i, i, indexing="ij")
    dr = 3.0 * U0 * U0 / 16.0
    rho = 1 + dr * (xp.cos(2 * x) + xp.cos(2 * y)) * (xp.cos(2 * z) + 2)
    ux = U0 * xp.sin(x) * xp.cos(y) * xp.cos(z)
    uy = -U0 * xp.cos(x) * xp.sin(y) * xp.cos(z)
    uz = xp.zeros_like(ux)
    return rho, ux, uy, uz


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_record(key):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get(key)
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled in the background."""

    FIELDS = ("timestamp,index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, interval_ms=50):
        self.proc = None
        self.t0 = self.t1 = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 f"-lms={interval_ms}"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except Exception:
            self.proc = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def stop(self, bus_id=None):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        rows = []
        for r in csv.reader(io.StringIO(out)):
            if len(r) < 11:
                continue
            r = [c.strip() for c in r]
            if bus_id and bus_id.lower() not in r[2].lower():
                continue
            try:
                ts = time.mktime(time.strptime(r[0].split(".")[0], "%Y/%m/%d %H:%M:%S"))
                ts += float("0." + r[0].split(".")[1]) if "." in r[0] else 0.0
            except Exception:
                ts = None
            rows.append((ts, float(r[3]), float(r[4]), r[7:11]))
        inside = [x for x in rows if x[0] is not None and self.t0 and
                  self.t0 - 0.06 <= x[0] <= (self.t1 or 1e30) + 0.06]
        use = inside or rows
        if not use:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for x in use for k, v in enumerate(x[3]) if v == "Active"})
        return {"sm_mhz": float(np.median([x[1] for x in use])),
                "sm_max_mhz": float(max(x[2] for x in use)),
                "reasons": reasons, "samples": len(use),
                "window": "timed region" if inside else "whole run (timed region shorter than the sampling interval)"}


# ------------------------------------------------------------------ GPU arm
def gpu_arm(args, rank, world, dist):
    import torch
    from m3lb_b200 import capi
    from m3lb_b200 import solver as S

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    props = torch.cuda.get_device_properties(dev)
    bus = None
    try:
        bus = "%08x:%02x:%02x" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
    except Exception:
        bus = None
    n = args.size
    nodes = n ** 3
    nu, tau, omega = tgv_params(n)
    stream = torch.cuda.current_stream(dev)

    def make(storage):
        dom = S.Domain(n, n, n, True, True, True)
        coll = S.CentralMoments(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=omega)
        s = S.FluidSolver(dom, coll, storage=storage)
        s.set_stream(stream)
        s.set_option(capi.OPT_KERNEL, KERNELS[args.kernel])
        rho, ux, uy, uz = [t.to(torch.float32).contiguous()
                           for t in tgv_fields(n, _TorchNp(dev))]
        s.initialize_field_device(rho, ux, uy, uz)
        del rho, ux, uy, uz
        return s

    def timed(s, K, W):
        for _ in range(W):
            s.step()
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
        c0 = s.launch_count()
        sampler.mark_start()
        ev[0].record(stream)
        for k in range(K):
            s.step()
            ev[k + 1].record(stream)
        torch.cuda.synchronize(dev)
        sampler.mark_end()
        launches = s.launch_count() - c0
        if dist:
            dist.barrier()
        total = ev[0].elapsed_time(ev[K]) / 1e3
        per = [ev[k].elapsed_time(ev[k + 1]) / 1e3 for k in range(K)]
        t = torch.tensor([total], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), float(np.mean(per)), launches

    sampler = ClockSampler()
    s16 = make(args.storage)
    t16, per16, launches = timed(s16, args.steps, args.warmup)
    red = s16.reduce()
    finite = bool(np.isfinite(red).all())
    mass_drift = None
    s16.close()
    clocks = sampler.stop(bus)

    # FP32 storage on the same workload, for the FP16/FP32 ratio
    s32 = make("f32")
    t32, per32, _ = timed(s32, args.steps, args.warmup)
    s32.close()
    # the other 16-bit float (IEEE FP16 beside FP16C, or FP16C beside FP16)
    other16 = {"f16": "f16c", "f16c": "f16"}.get(args.storage)
    if other16:
        so = make(other16)
        to, pero, _ = timed(so, args.steps, args.warmup)
        so.close()

    eb = STORAGE_BYTES[args.storage]
    bytes_per_launch = nodes * 2 * Q * eb
    achieved = bytes_per_launch / per16 / 1e9
    peak, peak_kind = measured_peaks()
    value = world * nodes * args.steps / t16 / 1e6
    value32 = world * nodes * args.steps / t32 / 1e6

    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t16 / args.steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "storage": args.storage,
        "data": "synthetic (analytic Taylor-Green initial field, generated on the device)",
        "config": {"workload": WORKLOAD, "lattice": "D3Q27", "operator": "central moments",
                   "nx": n, "ny": n, "nz": n, "nodes_per_gpu": nodes, "tau": round(tau, 6),
                   "u0": U0, "Re": RE, "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2 ({nodes * Q * eb / 1e6:.0f} MB of populations "
                         f"per step vs {L2_BYTES / 1e6:.0f} MB L2)"},
        "hbm_gbs": round(achieved, 1),
        "fp32_storage": {"value": round(value32, 1), "unit": "MLUPS",
                         "ms_per_step": round(t32 / args.steps * 1e3, 4),
                         "hbm_gbs": round(nodes * 2 * Q * 4 / per32 / 1e9, 1)},
        "fp16_over_fp32": round(value / value32, 3),
        "storage_note": STORAGE_NOTE.get(args.storage, ""),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "peak_kind": f"{peak_kind} (copy bandwidth)",
                     "kernel": f"{KERNEL_NAMES[args.kernel]}<D3Q27, {args.storage.upper()}, CM>",
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "traffic": traffic_record(f"D3Q27_CM_{args.storage}_{n}")},
        "gpu_launches": launches,
        "clocks": clocks,
        "state_finite": finite,
    }
    if isinstance(clocks, dict) and clocks.get("sm_mhz"):
        # the step time in clock cycles (ms x MHz): constant across boxes
        # and power states when the kernel is bound by instruction issue
        clocks["ms_x_sm_mhz"] = round(t16 / args.steps * 1e3 * clocks["sm_mhz"], 1)
    if mass_drift is not None:
        out["mass_drift"] = mass_drift
    if other16:
        out[f"{other16}_storage"] = {
            "value": round(world * nodes * args.steps / to / 1e6, 1), "unit": "MLUPS",
            "ms_per_step": round(to / args.steps * 1e3, 4),
            "hbm_gbs": round(nodes * 2 * Q * 2 / pero / 1e9, 1),
            "frac": round(nodes * 2 * Q * 2 / pero / 1e9 / peak, 4)}

    if rank == 0 and not args.no_e2e:
        out["e2e"] = e2e_arm(args, dev, stream, omega)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args)
    if rank == 0 and world == 1 and args.acc_steps > 0:
        out["accuracy"] = accuracy_arm(args, dev, stream, omega)
    if rank == 0 and world == 1 and args.serve_requests > 0:
        out["serving"] = serving_arm(args)
        # the serving target: aggregate within 25 % of the single large lattice
        out["serving"]["aggregate_over_single"] = round(
            out["serving"]["aggregate_mlups"] / out["value"], 3)
    if rank == 0 and world == 1 and args.walls_steps > 0:
        out["walls"] = walls_arm(args, stream, omega)
    if rank == 0 and world == 1 and args.thermal_steps > 0:
        out["thermal"] = thermal_arm(args, stream, omega)
    # the storage gates last, so they sit in the tail of the printed line:
    # the 16-bit storage's velocity error (north-star bound 1e-3), roofline
    # fraction and its MLUPS over FP32 storage's
    if "accuracy" in out:
        out["f16_u_rel_l2"] = {st: out["accuracy"][st]["u_rel_l2"]
                               for st in ("f16", "f16c") if st in out["accuracy"]}
    out["frac"] = out["roofline"]["frac"]
    for key in ("storage_note", "fp32_storage", "fp16_over_fp32"):
        out[key] = out.pop(key)
    return out


def thermal_arm(args, stream, omega):
    """The coupled thermal step on the headline lattice: the D3Q27 CM fluid
    with a Boussinesq force read from a D3Q7 BGK temperature lattice (FP32),
    which is advected by the fluid's stored velocity (m3lb_couple_thermal;
    the reference's validation/rayleigh_benard.cpp loop: fluid.step(true);
    scalar.step()).  Periodic box, temperature seeded with a random field.
    Timed: the coupled pair, and the scalar step alone; the scalar kernel's
    algorithmic bytes per node are 7 x 4 x 2 (populations) + 12 (velocity)
    + 4 (field) + 1 (cell type)."""
    import torch
    from m3lb_b200 import capi
    from m3lb_b200 import solver as S

    n = args.size
    K = args.thermal_steps
    dom = S.Domain(n, n, n, True, True, True)
    coll = S.CentralMoments(S.D3Q27, S.Guo(0.0, 0.0, 0.0), S.ShiftedPopulations, omega=omega)
    fl = S.FluidSolver(dom, coll, storage=args.storage)
    fl.set_stream(stream)
    fl.set_option(capi.OPT_KERNEL, KERNELS[args.kernel])
    th = S.ScalarSolver(dom, S.ScalarBGK(S.D3Q7, omega=1.2), storage="f32")
    rng = np.random.default_rng(0)
    th.initialize_field(0.5 + 0.01 * rng.standard_normal(dom.n_padded))
    fl.initialize(1.0)
    S.couple_thermal(fl, th, g=(0.0, 1.0, 0.0), rho0=1.0, beta=1e-3, T0=0.5)
    for _ in range(3):
        fl.step(True)
        th.step()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(K):
        fl.step(True)
        th.step()
    e1.record(stream)
    th.steps(K)
    e2.record(stream)
    torch.cuda.synchronize()
    pair_ms = e0.elapsed_time(e1) / K
    scalar_ms = e1.elapsed_time(e2) / K
    th.compute_field()
    finite = bool(np.isfinite(th.temperature()).all())
    th.close()
    fl.close()
    nodes = n ** 3
    sbytes = 7 * 4 * 2 + 12 + 4 + 1
    return {"workload": f"D3Q27 CM {n}^3 {args.storage} + D3Q7 BGK FP32 temperature, Boussinesq "
                        f"coupling both ways, {K} steps",
            "coupled_ms_per_step": pair_ms, "coupled_glups": nodes / pair_ms / 1e6,
            "scalar_ms_per_step": scalar_ms, "scalar_glups": nodes / scalar_ms / 1e6,
            "scalar_bytes_per_node": sbytes,
            "scalar_hbm_gbs": nodes * sbytes / scalar_ms / 1e6, "finite": finite}


def walls_arm(args, stream, omega):
    """Cost of wall nodes on the headline lattice: the periodic box against
    a channel (periodic x and z) closed by regularised velocity walls, a
    resting floor at y = 0 and a lid moving at u0 at y = N-1, both driven
    through the boundary-node pass after the bulk kernel; and the same
    channel with free-slip ghost walls (SpecWall).  Same operator, storage
    and kernel choice as the headline; CUDA events over args.walls_steps
    steps each."""
    import torch
    from m3lb_b200 import capi
    from m3lb_b200 import solver as S

    n = args.size
    out = {"workload": f"D3Q27 CM {n}^3 {args.storage}: periodic box vs channel walls at y = 0, {n - 1}",
           "steps": args.walls_steps, "wall_nodes": 2 * n * n}

    def timed(kind):
        dom = S.Domain(n, n, n, True, kind == "periodic", True)
        coll = S.CentralMoments(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=omega)
        s = S.FluidSolver(dom, coll, storage=args.storage)
        s.set_stream(stream)
        s.set_option(capi.OPT_KERNEL, KERNELS[args.kernel])
        codes = np.zeros((n, n, n), np.uint8)
        if kind == "regwall":
            st = np.zeros((n, n, n, 4))
            st[..., 3] = 1.0
            st[:, -1, :, 0] = U0
            codes[:, 0, :] = 4
            codes[:, -1, :] = 3
            s.set_regularized_walls(codes, st)
        elif kind == "specwall":
            codes[:, 0, :] = 4
            codes[:, -1, :] = 3
            s.set_specular_walls(codes)
        del codes
        s.initialize(1.0)
        s.steps(5)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.steps(args.walls_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.walls_steps
        launches = s.launch_count()
        s.close()
        return {"ms_per_step": ms, "glups": n ** 3 / ms / 1e6, "launches_total": launches}

    for kind in ("periodic", "regwall", "specwall"):
        out[kind] = timed(kind)
    for kind in ("regwall", "specwall"):
        out[kind]["vs_periodic"] = out["periodic"]["ms_per_step"] / out[kind]["ms_per_step"]
    return out


def serving_arm(args):
    """The serving stream: seeded Poisson arrivals (mean 50/s) of periodic
    Taylor-Green boxes, N in {32, 48, ..., 160}, BGK / TRT / CM, u0 in
    [0.02, 0.08], 200-2000 steps, FP16 storage, tau = 0.6.  The offered load
    is above one GPU's capacity, so a finite stream is served and the latency
    (arrival to result) includes the queueing."""
    from m3lb_b200 import serve as SV

    reqs = SV.request_stream(count=args.serve_requests, rate=50.0, seed=0)
    srv = SV.Server(hbm_budget=args.serve_budget_gb << 30, max_resident=args.serve_resident,
                    round_steps=args.serve_round, storage="f16", mapping="tune")
    for r in reqs:
        srv.submit(r)
    srv.run(time_limit=900)
    res = srv.results()
    st = srv.stats()
    srv.close()
    s = SV.summary(res, reqs)
    return {
        "metric": "p50 / p99 request latency (arrival to result, queueing included)",
        "p50_ms": round(s["latency_p50_s"] * 1e3, 1),
        "p99_ms": round(s["latency_p99_s"] * 1e3, 1),
        "max_ms": round(s["latency_max_s"] * 1e3, 1),
        "requests": s["requests"],
        "offered_rate_per_s": round(s["offered_rate_per_s"], 2),
        "served_rate_per_s": round(s["served_rate_per_s"], 2),
        "offered_mlups": round(s["offered_mlups"], 1),
        "aggregate_mlups": round(s["aggregate_mlups"], 1),
        "makespan_s": round(s["makespan_s"], 2),
        "all_finite": bool(all(np.isfinite(r.mass) for r in res)),
        "loop": {"rounds": st.rounds, "launches": st.launches,
                 "graph_captures": st.graph_captures, "graph_launches": st.graph_launches,
                 "hbm_budget_gib": args.serve_budget_gb, "max_resident": args.serve_resident,
                 "round_steps": args.serve_round},
        "mapping_tuner": {"chosen": {1: "chunks", 2: "dense", 4: "rows"}.get(st.tuned_mapping,
                                                                              "none"),
                          "chunks_mlups": round(st.tuned_chunks_mlups, 1),
                          "dense_mlups": round(st.tuned_dense_mlups, 1),
                          "rows_mlups": round(st.tuned_rows_mlups, 1),
                          "dense_launches": st.dense_launches,
                          "rows_launches": st.rows_launches},
        "workload": "seed 0, Poisson 50/s, N in {32..160 step 16}, op in {BGK, TRT, CM}, "
                    "u0 ~ U[0.02, 0.08], steps ~ U[200, 2000], FP16, tau 0.6",
    }


class _TorchNp:
    """The few numpy names tgv_fields uses, on a torch device."""

    def __init__(self, dev):
        import torch
        self.t, self.dev = torch, dev
        self.float64 = torch.float64

    def arange(self, n, dtype=None):
        return self.t.arange(n, dtype=dtype, device=self.dev)

    def meshgrid(self, *a, indexing="ij"):
        return self.t.meshgrid(*a, indexing=indexing)

    def cos(self, x):
        return self.t.cos(x)

    def sin(self, x):
        return self.t.sin(x)

    def zeros_like(self, x):
        return self.t.zeros_like(x)


def e2e_arm(args, dev, stream, omega):
    """Same metric through the public API with host buffers: each e2e step
    copies the initial field from pinned host memory, advances
    args.e2e_lbm_steps time steps and reads rho, u back to pinned memory."""
    import torch
    from m3lb_b200 import capi
    from m3lb_b200 import solver as S

    n = args.size
    nodes = n ** 3
    dom = S.Domain(n, n, n, True, True, True)
    coll = S.CentralMoments(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=omega)
    s = S.FluidSolver(dom, coll, storage=args.storage)
    s.set_stream(stream)
    s.set_option(capi.OPT_KERNEL, KERNELS[args.kernel])
    host_in = [torch.from_numpy(a.astype(np.float32)).pin_memory() for a in tgv_fields(n)]
    host_out = [torch.empty((n, n, n), dtype=torch.float32).pin_memory() for _ in range(4)]
    S_lbm = args.e2e_lbm_steps

    def one():
        s.initialize_field_f32(*host_in)
        s.steps(S_lbm)
        s.compute_macroscopic_f32(*host_out)

    one()
    torch.cuda.synchronize(dev)
    reps = args.e2e_reps
    t0 = time.perf_counter()
    for _ in range(reps):
        one()
    torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    ok = bool(torch.isfinite(host_out[1]).all())
    s.close()
    return {"value": round(nodes * S_lbm * reps / dt / 1e6, 1), "unit": "MLUPS",
            "h2d_bytes_per_step": 4 * nodes * 4, "d2h_bytes_per_step": 4 * nodes * 4,
            "lbm_steps_per_e2e_step": S_lbm, "e2e_steps": reps,
            "ms_per_e2e_step": round(dt / reps * 1e3, 3), "finite": ok,
            "api": "m3lb_b200.FluidSolver (C ABI: m3lb_init_field_f32, m3lb_step, m3lb_macro_f32)"}


# ------------------------------------------------------------------ CPU legs
def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _ref_rate(n, steps, threads, warm=1):
    """MLUPS of the reference's own CPU path (oracle/_ref, FP32) on an n^3
    periodic central-moment lattice."""
    import oracle as O
    O.set_ref_threads(threads, "f32")
    _, _, omega = tgv_params(N_DEFAULT)
    s = O.CpuSolver("ref", lattice=27, op="cm", shifted=True, nx=n, ny=n, nz=n,
                    omega=omega, precision="f32")
    s.initialize(1.0, U0, 0.0, 0.0)
    s.step(warm)
    t0 = time.perf_counter()
    s.step(steps)
    dt = time.perf_counter() - t0
    s.close()
    return n ** 3 * steps / dt / 1e6, dt


def accuracy_arm(args, dev, stream, omega):
    """Storage precision against FP64 storage on the same workload: the
    Taylor-Green vortex at args.size^3 after args.acc_steps steps, seeded from
    the same FP64 field.  Velocity: relative L2 over all components and max
    |error| / u0; density: relative L2 and max of rho - 1; mass drift from
    the FP64 device reduction."""
    import torch
    from m3lb_b200 import capi
    from m3lb_b200 import solver as S

    n = args.size

    def run(storage):
        dom = S.Domain(n, n, n, True, True, True)
        coll = S.CentralMoments(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=omega)
        s = S.FluidSolver(dom, coll, storage=storage)
        s.set_stream(stream)
        s.set_option(capi.OPT_KERNEL, KERNELS[args.kernel])
        dt = torch.float64 if storage == "f64" else torch.float32
        f = [t.to(dt).contiguous() for t in tgv_fields(n, _TorchNp(dev))]
        s.initialize_field_device(*f)
        del f
        m0 = s.reduce()[0]
        s.steps(args.acc_steps)
        m1 = s.reduce()[0]
        rho, ux, uy, uz = s.compute_macroscopic()
        s.close()
        return rho, np.stack([ux, uy, uz]), (m1 - m0) / m0

    rho_r, u_r, drift_r = run("f64")
    out = {"workload": f"D3Q27 CM Taylor-Green {n}^3, {args.acc_steps} steps, u0 {U0}, Re {RE}",
           "reference": "FP64 storage (FP64 arithmetic), same seed field",
           "f64": {"mass_drift": float(drift_r)}}
    du = float(np.sqrt(np.sum(u_r * u_r)))
    dr = float(np.sqrt(np.sum((rho_r - 1) ** 2)))
    for st in ("f32", "bf16", "f16", "f16c"):
        rho, u, drift = run(st)
        eu = u - u_r
        er = rho - rho_r
        out[st] = {"u_rel_l2": float(np.sqrt(np.sum(eu * eu)) / du),
                   "u_max_over_u0": float(np.max(np.abs(eu)) / U0),
                   "rho_rel_l2": float(np.sqrt(np.sum(er * er)) / dr),
                   "rho_max": float(np.max(np.abs(er))),
                   "mass_drift": float(drift)}
        del rho, u, eu, er
    return out


def cpu_baseline(args):
    import oracle as O
    if not O.ref_available("f32"):
        return {"value": None, "unit": "MLUPS", "cores": 0, "kind": "reference",
                "sample": "reference build (oracle/_ref) not present"}
    th = _host_threads()
    # calibrate on a small lattice, then a bounded sample of ~10-20 s
    rate, _ = _ref_rate(64, 2, th)
    n = args.cpu_size
    steps = max(1, int(min(12.0 * rate * 1e6 / n ** 3, 50)))
    rate, dt = _ref_rate(n, steps, th)
    return {"value": round(rate, 2), "unit": "MLUPS", "cores": th, "kind": "reference",
            "sample": f"{steps} time steps of the reference src/ FluidSolver (FP32, "
                      f"EsotericPull, CentralMoments, shifted) on a periodic {n}^3 lattice, "
                      f"{dt:.1f} s, OpenMP {th} threads"}


def reference_arm(args):
    import oracle as O
    th = _host_threads()
    base = {"metric": METRIC, "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "impl": "reference",
            "data": "synthetic (uniform flow initial state)"}
    if not O.ref_available("f32"):
        base.update({"unavailable": "reference build oracle/_ref not present"})
        return base
    # each step: one time step of a bounded sample lattice; the whole run
    # (warm-up + steps) is sized to about two minutes of host time
    rate, _ = _ref_rate(64, 2, th)
    per_step_budget = 100.0 / max(args.steps + args.warmup, 1)
    n = int(min(N_DEFAULT, max(32, (per_step_budget * rate * 1e6) ** (1 / 3))))
    n -= n % 2
    r, dt = _ref_rate(n, args.steps, th, warm=args.warmup)
    base.update({
        "value": round(r, 2), "ms_per_step": round(dt / args.steps * 1e3, 3),
        "config": {"workload": f"D3Q27 central moments, FP32, periodic {n}^3 sample of the "
                               f"256^3 workload", "nodes_per_step": n ** 3,
                   "parallelism": f"{th} OpenMP threads"},
        "cpu_baseline": {"value": round(r, 2), "unit": "MLUPS", "cores": th,
                         "kind": "reference",
                         "sample": f"{args.steps} time steps on a periodic {n}^3 lattice"},
        "e2e": {"value": round(r, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    })
    return base


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="m3lb", choices=["m3lb", "reference"])
    ap.add_argument("--storage", default="f16c", choices=["f16", "f16c", "bf16", "f32"])
    ap.add_argument("--size", type=int, default=N_DEFAULT)
    ap.add_argument("--kernel", default="auto", choices=list(KERNELS))
    ap.add_argument("--cpu-size", type=int, default=128)
    ap.add_argument("--e2e-lbm-steps", type=int, default=100)
    ap.add_argument("--e2e-reps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--acc-steps", type=int, default=500,
                    help="steps of the storage-precision comparison (0: skip it)")
    ap.add_argument("--serve-requests", type=int, default=500,
                    help="requests of the serving stream (0: skip it)")
    ap.add_argument("--serve-budget-gb", type=int, default=4)
    ap.add_argument("--serve-resident", type=int, default=16)
    ap.add_argument("--serve-round", type=int, default=100)
    ap.add_argument("--walls-steps", type=int, default=100,
                    help="steps of each wall-cost measurement (0: skip it)")
    ap.add_argument("--thermal-steps", type=int, default=100,
                    help="steps of the coupled thermal measurement (0: skip it)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(args)), flush=True)
        return 0

    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=timedelta(seconds=120))
        dist = tdist
    out = gpu_arm(args, rank, world, dist)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
