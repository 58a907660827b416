#!/usr/bin/env python
"""Benchmark of the SEREN force hot path on B200: particle force evaluations/s.

Workload: the turbulent molecular-cloud core (N = 4,194,304 particles uniform
in a unit sphere, M = 1, G = 1, isothermal c_s = 0.2, divergence-free P(k) ~
k^-4 velocity field at rms Mach 2), seeded synthetic data.  One step = one full
force evaluation (tree build + reorder + stock, grad-h h/rho/Omega solve,
hmax update, neighbour lists, isothermal thermal, hydro forces with MON97
viscosity, Barnes-Hut gravity) followed by a drift r += v dt.  `value` is the
mixed-precision (FP32 pair arithmetic) path with inputs resident in HBM; the
FP64 path is timed on the same state for the speed-up and accuracy figures.
`e2e` is the same metric from pinned host buffers to pinned host buffers
through seren_gpu_force_step_io (inputs copied in and every result copied
back each step, the copies overlapped with the force step on a second
stream; the host's drift between calls is not timed); `e2e_reference_calls` is the same through the host-buffer calls a
Fortran caller of the reference's interface makes (tree_update -> sph_update
-> thermal on the host -> hydro_forces -> grav_forces), copies included.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = ("particle force evals/sec (grav+hydro) at 4M, FP32-comp vs FP64 on B200 at rms "
          "err≤1e-3")
UNIT = "particle evals/s"
N_FULL = 4194304
DT = 1.0e-3
# algorithmic flops per interaction, counted from the reference expressions
# (BHtree/BHgrav_accel.F90:146-226 quadrupole cell term; gravity/gravity_gradh.F90 pair)
FLOPS_CELL = 75
FLOPS_PAIR = 41


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=0,
                    help="particle count (default: 4,194,304 for core, 1,048,576 for plummer, "
                         "8,388,608 for disc)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuning", default="auto",
                    help="kernel knobs: auto (the autotuner, default), default (the library's "
                         "defaults) or k=v pairs, e.g. hydro_sub=4,grav_cap=96,grav_bps=0,"
                         "gradh_bps=0,neib_bps=0 (fixed knobs make ncu captures reproducible)")
    ap.add_argument("--workload", choices=("core", "plummer", "disc", "batched"), default="core",
                    help="core: the turbulent core (default, the headline); plummer: Plummer "
                         "sphere, gravity accuracy over theta^2 in {0.09, 0.25, 0.49}; disc: "
                         "protostellar disc around a sink; batched: 256 independent clouds "
                         "shared out across the ranks")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def dist_init(n_gpus):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, x):
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clock/throttle sampling in the background during a timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
WORKLOAD_N = {"core": N_FULL, "plummer": 1048576, "disc": 8388608}


def workload(n, kind="core"):
    """Seeded synthetic inputs with the configs' shapes and distributions."""
    from seren_b200 import ics
    t0 = time.time()
    if kind == "plummer":
        ic = ics.plummer(n=n, seed=2, thetamaxsqd=0.25)
    elif kind == "disc":
        ic = ics.protostellar_disc(n=n, seed=5)
    else:
        ic = ics.turbulent_core(n=n, seed=4, sound=0.2, mach=2.0, h_fac=1.2, thetamaxsqd=0.25)
    log(f"[bench] workload {ic['name']} generated in {time.time() - t0:.1f}s")
    return ic


def workload_info(kind, n):
    """(metric, data, config workload text) of a workload."""
    if kind == "plummer":
        return ("particle force evals/sec (grav+hydro), Plummer sphere N=1M",
                "synthetic (seeded Plummer sphere, numpy PCG64)",
                f"Plummer sphere a=1 M=1, N={n} per GPU, radii redrawn beyond 20a, AHW velocities, "
                "h_fac for 50 neighbours, c_s=0 (gravity only), theta^2=0.25 (sweep 0.09/0.25/0.49 "
                "in theta_sweep); step = full force evaluation + drift")
    if kind == "disc":
        return ("particle force evals/sec (grav+hydro), protostellar disc N=8M with a sink",
                "synthetic (seeded protostellar disc, numpy PCG64)",
                f"protostellar disc, N={n} per GPU, M_disc=0.1 on R in [0.1, 10] (R uniform), "
                "H=0.05R, c_s=0.05 R^-0.25, Keplerian + pressure correction, one sink M=1 "
                "h=0.05 at the origin (sink-gas forces FP64 direct), h_fac=1.2, theta^2=0.25; "
                "step = full force evaluation + drift")
    return (METRIC, "synthetic (seeded turbulent uniform-sphere core, numpy PCG64)",
            f"turbulent molecular-cloud core, N={n} per GPU, uniform sphere R=1 M=1 G=1, "
            "isothermal c_s=0.2, P(k)~k^-4 Mach 2, h_fac=1.2 (pp_gather 57), theta^2=0.25 "
            "quadrupole geometric MAC, MON97 alpha=1; step = full force evaluation + drift")


def line_config(wdesc, n):
    """The `config` object of the JSON line, the same in both arms."""
    return {"workload": wdesc, "particles": n,
            "l2": "inputs larger than L2 (particles + tree ~1 GB resident)"}


def params_for(ic, precision):
    from seren_b200.cabi import Params
    return Params.make(h_fac=ic["h_fac"], thetamaxsqd=ic["thetamaxsqd"], alpha=ic["alpha"],
                       precision=precision)


TUNING = "auto"


def apply_tuning(g, precision):
    """The kernel knobs of context g for --tuning: the autotuner's choice (two
    force steps per configuration on the live state), the defaults, or the
    given values.  Returns the knobs in use."""
    if TUNING == "auto":
        t = g.autotune(trials=2)
        log(f"[bench] autotune (precision {precision}): {t}")
        return t
    knobs = dict(hydro_sub=4, grav_cap=64, grav_bps=0, gradh_bps=0, neib_bps=0)
    if TUNING != "default":
        for kv in TUNING.split(","):
            k, v = kv.split("=")
            knobs[k.strip()] = int(v)
    g.set_tuning(**knobs)
    return dict(knobs, ms_per_step=None)


def run_resident(ic, precision, steps, warmup, ws):
    """Device-resident steps; returns timing/stat dict and the final state."""
    import torch

    from seren_b200.gpu import GpuHotPath
    n = ic["parray"].shape[0]
    g = GpuHotPath(n, params_for(ic, precision))
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    if ic.get("sink") is not None:
        g.set_sinks(ic["sink"])
    stream = torch.cuda.ExternalStream(g.stream())
    g.force_step(first_call=True)
    # the project's autotuner picks the kernel knobs for this size on the live
    # state (four configurations, two force steps each), then the warm-up runs
    tuning = apply_tuning(g, precision)
    for _ in range(max(warmup, 1) - 1):
        g.drift(DT)
        g.force_step(first_call=False)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stage = np.zeros(8)
    launches = 0
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(steps):
        g.drift(DT)
        launches += 1
        g.force_step(first_call=False)
        ms, nl, counts = g.last_step_stats()
        stage += np.array(ms)
        launches += nl
    end.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    total_ms = start.elapsed_time(end)
    state = g.download()
    res = dict(total_ms=total_ms, stage_ms=(stage / steps).tolist(), launches=launches,
               counts=counts, ctx=g, tuning=tuning)
    return res, state


def run_rk2(ic, precision, steps, warmup, ws, nbuildstep=1):
    """Device-resident integration: seren_gpu_timestep then seren_gpu_rk2_step
    (two force evaluations) per step, from the state after one force step;
    with nbuildstep > 1 the tree is built every nbuildstep evaluations and
    restocked in between (the reference's schedule); timed with CUDA events
    on the library's stream, max over ranks."""
    import torch

    from seren_b200.gpu import GpuHotPath
    n = ic["parray"].shape[0]
    g = GpuHotPath(n, params_for(ic, precision))
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    stream = torch.cuda.ExternalStream(g.stream())
    g.set_build_step(nbuildstep)
    g.force_step(first_call=True)
    dts = []
    for _ in range(max(warmup, 1)):
        g.rk2_step(g.timestep())
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(ws)
    start.record(stream)
    for _ in range(steps):
        dt = g.timestep()
        dts.append(dt)
        g.rk2_step(dt)
    end.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    total_ms = max_over_ranks(ws, start.elapsed_time(end))
    g.close()
    return dict(ms_per_step=total_ms / steps, force_evals_per_step=2,
                value=ws * 2 * n * steps / (total_ms * 1e-3), unit=UNIT,
                dt=[float(x) for x in dts], nbuildstep=nbuildstep,
                api="seren_gpu_timestep + seren_gpu_rk2_step (courant 0.2, accel 0.5)")


def run_block(ic, precision, steps, warmup, ws, nlevels=3, nbuildstep=1):
    """Device-resident block timesteps (seren_gpu_block_step: the forces of
    the accdo particles only, then the reference's level bookkeeping and the
    Runge-Kutta advance of every particle), nlevels levels with the
    reference's default options (RESTRICTED levels, CHECK_NEIB_TIMESTEP = 1);
    integer steps timed with CUDA events on the library's stream after one
    resynchronisation cycle of warm-up."""
    import torch

    from seren_b200.gpu import GpuHotPath
    n = ic["parray"].shape[0]
    g = GpuHotPath(n, params_for(ic, precision))
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    stream = torch.cuda.ExternalStream(g.stream())
    g.set_build_step(nbuildstep)
    g.force_step(first_call=True)
    g.block_start(nlevels=nlevels)
    cycle = 2 ** nlevels                      # integer steps between resynchronisations
    for _ in range(max(warmup, 1) * cycle):
        g.block_step()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(ws)
    start.record(stream)
    active = 0
    nsteps = max(steps, 1) * cycle
    for _ in range(nsteps):
        active += g.block_step()["nactive"]
    end.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    total_ms = max_over_ranks(ws, start.elapsed_time(end))
    g.close()
    return dict(ms_per_integer_step=total_ms / nsteps, integer_steps=nsteps, nlevels=nlevels,
                mean_active_fraction=active / (nsteps * n),
                value=ws * active / (total_ms * 1e-3), unit="active particle force evals/s",
                api="seren_gpu_block_step (RESTRICTED levels, CHECK_NEIB_TIMESTEP=1)")


def run_e2e_io(ic, precision, steps, warmup, ws):
    """Steps through seren_gpu_force_step_io with pinned host buffers: each
    call copies parray, v and c_s^2 in from the host and parray, v, c_s^2,
    rho, omega, a, gpot and the permutation (tree order) back over them; the
    host then drifts its positions (torch CPU ops, all cores, not timed), so
    every call starts from the host's arrays.  The time is the sum over the
    timed calls of CUDA events recorded around each call."""
    import ctypes as C

    import torch

    from seren_b200.gpu import GpuHotPath
    torch.set_num_threads(os.cpu_count() or 1)
    n = ic["parray"].shape[0]
    g = GpuHotPath(n, params_for(ic, precision))

    def pinned(shape, dtype=torch.float64):
        return torch.empty(shape, dtype=dtype, pin_memory=True)

    parray = pinned((n, 6)); parray.copy_(torch.from_numpy(ic["parray"]))
    v = pinned((n, 3)); v.copy_(torch.from_numpy(ic["v"]))
    csq = pinned((n,)); csq.copy_(torch.from_numpy(ic["sound"] ** 2))
    rho, omega, gpot = (pinned((n,)) for _ in range(3))
    a = pinned((n, 3))
    perm = pinned((n,), torch.int32)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    P = lambda x: C.cast(x.data_ptr(), dp)  # noqa: E731
    ctx = g._ctx
    host_s = np.zeros(2)

    stream = torch.cuda.ExternalStream(g.stream())
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(max(steps, 1))]

    def step(first, k=None):
        # the call is timed with events on the library's stream around it (it
        # returns with every copy done); the host's drift between calls is not
        t0 = time.perf_counter()
        if k is not None:
            ev[k][0].record(stream)
        g._call("force_step_io", ctx, n, P(parray), P(v), P(csq), int(first), P(parray), P(v),
                P(csq), P(rho), P(omega), P(a), P(gpot), C.cast(perm.data_ptr(), ip))
        if k is not None:
            ev[k][1].record(stream)
        t1 = time.perf_counter()
        parray[:, 0:3].add_(v, alpha=DT)
        t2 = time.perf_counter()
        host_s[:] += np.diff([t0, t1, t2])

    for w in range(max(warmup, 1)):
        step(w == 0)
    torch.cuda.synchronize()
    barrier(ws)
    host_s[:] = 0.0
    for k in range(steps):
        step(False, k)
    torch.cuda.synchronize()
    barrier(ws)
    total_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev[:steps])
    stages = g.last_step_stats()[0][:6]
    log(f"[bench] e2e (force_step_io) ms/step: call {total_ms / steps:.1f} by events, "
        f"{1e3 * host_s[0] / steps:.1f} by host clock (device stages "
        f"{[round(x, 2) for x in stages]}); host drift between calls {1e3 * host_s[1] / steps:.1f}")
    h2d = n * (48 + 24 + 8)                          # parray, v, c_s^2
    d2h = n * (48 + 24 + 8 + 8 + 8 + 24 + 8 + 4)     # parray, v, c_s^2, rho, omega, a, gpot, perm
    g.close()
    return dict(total_ms=total_ms, h2d=h2d, d2h=d2h)


def run_e2e(ic, precision, steps, warmup, ws):
    """Steps through the host-buffer C ABI, as the Fortran drivers call it, with
    pinned host buffers.  The host does what the Fortran host does between the
    calls, with all its cores (torch CPU ops): applies the tree permutation to
    its own arrays (v, c_s), computes the isothermal thermal state and drifts."""
    import ctypes as C

    import torch

    from seren_b200.gpu import GpuHotPath
    torch.set_num_threads(os.cpu_count() or 1)
    n = ic["parray"].shape[0]
    g = GpuHotPath(n, params_for(ic, precision))

    def pinned(shape, dtype=torch.float64):
        return torch.empty(shape, dtype=dtype, pin_memory=True)

    parray = pinned((n, 6)); parray.copy_(torch.from_numpy(ic["parray"]))
    v = pinned((n, 3)); v.copy_(torch.from_numpy(ic["v"]))
    v2 = pinned((n, 3))
    sound = pinned((n,)); sound.copy_(torch.from_numpy(ic["sound"]))
    sound2 = pinned((n,))
    press = pinned((n,))
    rho, omega, div_v, drhodt, gpot = (pinned((n,)) for _ in range(5))
    a = pinned((n, 3))
    perm = pinned((n,), torch.int32)
    perm64 = torch.empty(n, dtype=torch.int64)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    P = lambda x: C.cast(x.data_ptr(), dp)  # noqa: E731
    ctx = g._ctx
    host_s = np.zeros(6)

    def step(first):
        nonlocal v, v2, sound, sound2
        t0 = time.perf_counter()
        g._call("tree_update", ctx, n, P(parray), 1, 1, C.cast(perm.data_ptr(), ip))
        t1 = time.perf_counter()
        perm64.copy_(perm)
        torch.index_select(v, 0, perm64, out=v2); v, v2 = v2, v
        torch.index_select(sound, 0, perm64, out=sound2); sound, sound2 = sound2, sound
        t2 = time.perf_counter()
        g._call("sph_update", ctx, n, None, 0, P(parray), P(v), P(rho), P(omega), P(div_v),
                P(drhodt), None, None, int(first))
        t3 = time.perf_counter()
        torch.mul(sound, sound, out=press)
        press.mul_(rho)
        g._call("hydro_forces", ctx, None, 0, P(press), P(sound), P(a))
        t4 = time.perf_counter()
        g._call("grav_forces", ctx, None, 0, P(a), P(gpot), 0, None)
        t5 = time.perf_counter()
        parray[:, 0:3].add_(v, alpha=DT)
        t6 = time.perf_counter()
        host_s[:] += np.diff([t0, t1, t2, t3, t4, t5, t6])

    stream = torch.cuda.ExternalStream(g.stream())
    for w in range(max(warmup, 1)):
        step(w == 0)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(ws)
    start.record(stream)
    host_s[:] = 0.0
    for _ in range(steps):
        step(False)
    end.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    total_ms = start.elapsed_time(end)
    log("[bench] e2e host ms/step: " + ", ".join(
        f"{k} {1e3 * x / steps:.1f}" for k, x in zip(
            ("tree_update", "host reorder", "sph_update", "thermal+hydro", "grav", "host drift"),
            host_s)))
    h2d = n * (48 + 24 + 8 + 8 + 24)            # parray, v, press, sound, a (grav adds to it)
    d2h = n * (48 + 4 + 48 + 32 + 24 + 24 + 8)  # parray+perm, parray rows, rho..drhodt, a, a+gpot
    g.close()
    return dict(total_ms=total_ms, h2d=h2d, d2h=d2h)


def traffic_per_launch(n):
    """DRAM bytes of one gravity launch from the committed ncu summary, scaled
    to n particles (profiles/gravity_mixed_ncu.txt, key dram_bytes_per_particle)."""
    path = os.path.join(HERE, "profiles", "gravity_mixed_ncu.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_particle"):
                    return float(line.split("=")[1].split()[0]) * n
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
def cpu_eval(ic_tree, first_call=False):
    """One full force evaluation of the CPU oracle (the C++ FP64 restatement of
    the reference) for every particle on all host cores, as the reference's
    sph_setup.F90:42-66 sequence runs it: tree build + reorder + stock, grad-h
    h/rho/Omega solve, hmax update, neighbour lists, isothermal thermal, hydro
    forces, gravity.  No sampling and no scaling.  Returns the wall seconds of
    the evaluation, the per-stage seconds (the reference's BH_TREE,
    ALL_SPH_GRADH, BHHYDRO_UPDATE, GET_NEIB, THERMAL, HYDRO_FORCES and
    GRAVITY_FORCES markers) and the state in the oracle's tree order."""
    from oracle.oracle import Oracle, set_threads
    cores = set_threads(os.cpu_count() or 1)
    parray = ic_tree["parray"]
    n = parray.shape[0]
    o = Oracle(n, params_for(ic_tree, 0))
    t0 = time.perf_counter()
    po, perm = o.tree_update(parray)
    t1 = time.perf_counter()
    v = ic_tree["v"][perm]
    sound = ic_tree["sound"][perm]
    t2 = time.perf_counter()
    out = o.sph_update(po, v, first_call=first_call, lists=False)
    t3 = time.perf_counter()
    press = sound * sound * out["rho"]
    t4 = time.perf_counter()
    a = o.hydro_forces(press, sound)
    t5 = time.perf_counter()
    a, gpot = o.grav_forces(a)
    t6 = time.perf_counter()
    st = o.stage_seconds()          # tree, grad-h, hmax, neib, hydro, gravity (oracle clocks)
    stages = {"BH_TREE": t1 - t0, "ALL_SPH_GRADH": st[1], "BHHYDRO_UPDATE": st[2],
              "GET_NEIB": st[3], "SPH_UPDATE_OTHER": max(0.0, (t3 - t2) - sum(st[1:4])),
              "THERMAL": t4 - t3, "HYDRO_FORCES": t5 - t4, "GRAVITY_FORCES": t6 - t5}
    sec = (t1 - t0) + (t3 - t2) + (t6 - t3)   # the host-side gathers of v and c_s are excluded
    return dict(sec=sec, cores=cores, oracle=o, parray=out["parray"], perm=perm, a=a, gpot=gpot,
                rho=out["rho"], stages={k: round(x, 3) for k, x in stages.items()})


def cpu_host():
    """CPU model of this host (for the CPU-baseline lines)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def gravity_accuracy(ic, parray, nsub=256):
    """Gravity-only accelerations of the GPU (mixed and FP64 walks) and of the
    oracle's tree walk on one state (parray: positions, masses, h, zeta), each
    against the FP64 direct sum (sph/direct_sph_gravity.F90) of the oracle for
    nsub particles: rms and max |da|/|a|."""
    from oracle.oracle import Oracle
    from seren_b200.gpu import GpuHotPath
    n = parray.shape[0]
    ids = np.arange(0, n, max(1, n // nsub), dtype=np.int32)[:nsub]
    o = Oracle(n, params_for(ic, 0))
    po, permo = o.tree_update(parray)
    ad, _ = o.direct_gravity(ids)
    at, _ = o.grav_forces(np.zeros((n, 3)), acclist=ids)

    def stats(a):
        err = np.linalg.norm(a - ad, axis=1) / np.linalg.norm(ad, axis=1)
        return float(np.sqrt(np.mean(err ** 2))), float(err.max())
    out = {"direct_subset": int(ids.size)}
    out["oracle_tree_rms_vs_direct"], out["oracle_tree_max_vs_direct"] = stats(at[ids])
    for prec, key in ((1, "mixed"), (0, "fp64")):
        g = GpuHotPath(n, params_for(ic, prec))
        pg, permg = g.tree_update(parray)
        assert np.array_equal(permg, permo)
        ag, _ = g.grav_forces(np.zeros((n, 3)))
        g.close()
        out[f"{key}_rms_vs_direct"], out[f"{key}_max_vs_direct"] = stats(ag[ids])
    o.close()
    return out


# ---------------------------------------------------------------------------
def batched_main(args, ws, rank, local):
    """256 independent clouds (N_i log-uniform in [8192, 262144], seeds
    1000+i): each rank takes its longest-processing-time share of them.  The
    headline is the forest path: one context holds the rank's clouds
    (seren_gpu_set_clouds), so a step - a drift and a force evaluation of
    every cloud - is one tree build for all of them and one launch per stage.
    The comparison leg is the per-cloud loop of plain launches (one context
    and stream per cloud, issued from host threads).  Total work is fixed, so
    scaling is strong."""
    import torch

    from seren_b200 import ics
    from seren_b200.batch import CloudBatch, CloudForest, lpt_partition
    torch.cuda.set_device(local)
    clouds = ics.batched_clouds()
    ns = [c["parray"].shape[0] for c in clouds]
    mine = lpt_partition(ns, ws)[rank]
    sub = [clouds[i] for i in mine]
    del clouds

    def timed(b, sample_clocks):
        b.step(first_call=True)
        if hasattr(b, "g"):                  # the forest context: the autotuner's knobs
            apply_tuning(b.g, 1)
        for _ in range(max(args.warmup, 1) - 1):
            b.step(dt=DT)
        sampler = ClockSampler(local) if sample_clocks else None
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = 0
        torch.cuda.synchronize()
        barrier(ws)
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        start.record()
        for _ in range(args.steps):
            launches += b.step(dt=DT)      # every call synchronises its stream(s)
        end.record()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier(ws)
        t = max_over_ranks(ws, start.elapsed_time(end))
        b.close()
        return t, launches, clocks

    t_forest, launches, clocks = timed(CloudForest(sub, precision=1), True)
    t_loop, launches_loop, _ = timed(CloudBatch(sub, precision=1), False)
    total = sum(ns)
    value = total * args.steps / (t_forest * 1e-3)
    log(f"[bench] batched: rank {rank} {len(mine)} clouds, {sum(ns[i] for i in mine)} particles; "
        f"forest {t_forest / args.steps:.2f} ms/step, per-cloud loop {t_loop / args.steps:.2f} "
        f"ms/step (max over ranks)")
    if rank != 0:
        return
    print(json.dumps({
        "metric": "particle force evals/sec (grav+hydro), 256 independent clouds",
        "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_forest / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "fp32+fp64",
        "data": "synthetic (256 seeded uniform-sphere clouds, numpy PCG64, seeds 1000+i)",
        "config": {"workload": f"batched clouds: 256 uniform spheres, N_i log-uniform in "
                               f"[8192, 262144] (total {total}), c_s ~ U[0.05, 0.3], "
                               "h_fac=1.2, theta^2=0.25, MON97 alpha=1; each cloud its own tree; "
                               "step = drift + full force evaluation of every cloud",
                   "particles": total, "l2": "inputs larger than L2"},
        "precision": "mixed (FP32 pair arithmetic, FP64 walk/MAC/grad-h)",
        "parallelism": f"clouds sharded over {ws} ranks (longest-processing-time on N log N), "
                       "no exchange; on each rank one forest context, one launch per stage",
        "per_cloud_loop": {"ms_per_step": t_loop / args.steps,
                           "value": total * args.steps / (t_loop * 1e-3), "unit": UNIT,
                           "gpu_launches": launches_loop,
                           "api": "one context and stream per cloud, host threads"},
        "e2e": None, "cpu_baseline": None, "roofline": None,
        "gpu_launches": launches, "clocks": clocks}), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    global TUNING
    args = parse()
    TUNING = args.tuning
    ws, rank, local = dist_init(args.gpus)
    if args.workload == "batched":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference arm times "
                                  "the core workload only"}), flush=True)
            return
        return batched_main(args, ws, rank, local)
    n = args.n or WORKLOAD_N[args.workload]
    if args.impl == "reference":
        return reference_arm(args, ws, rank, n)
    import torch
    torch.cuda.set_device(local)
    ic = workload(n, args.workload)
    metric, data, wdesc = workload_info(args.workload, n)
    if args.workload != "core":        # the e2e and CPU legs belong to the headline workload
        args.no_e2e = True
        args.no_cpu_baseline = True
    sampler = ClockSampler(local)
    # mixed precision: the headline
    sampler.start()
    mixed, state_m = run_resident(ic, 1, args.steps, args.warmup, ws)
    clocks = sampler.stop()
    t_mixed = max_over_ranks(ws, mixed["total_ms"])
    value = ws * n * args.steps / (t_mixed * 1e-3)
    log(f"[bench] mixed: {t_mixed / args.steps:.2f} ms/step, stages {mixed['stage_ms'][:6]}, "
        f"launches {mixed['launches']}, counts {mixed['counts']}, clocks {clocks}")
    g = mixed["ctx"]
    fp32_peak = g.fma_peak(1)
    fp64_peak = g.fma_peak(0)
    ncell, npair = mixed["counts"][0], mixed["counts"][1]
    flops = FLOPS_CELL * ncell + FLOPS_PAIR * npair
    grav_ms = mixed["stage_ms"][4]
    achieved = flops / (grav_ms * 1e-3) / 1e12
    g.close()
    fp64 = None
    acc = {}
    if not args.no_fp64:
        f64, state_d = run_resident(ic, 0, args.steps, args.warmup, ws)
        f64["ctx"].close()
        fp64 = dict(value=ws * n * args.steps / (max_over_ranks(ws, f64["total_ms"]) * 1e-3),
                    ms_per_step=f64["total_ms"] / args.steps, tuning=f64["tuning"],
                    stage_ms=[round(x, 3) for x in f64["stage_ms"][:6]])
        am, ad = state_m["a"], state_d["a"]
        # both runs start from the same state and drift identically, so the trees,
        # the particle order and h agree; compare accelerations row by row
        same = np.array_equal(state_m["perm"], state_d["perm"])
        err = np.linalg.norm(am - ad, axis=1) / np.maximum(np.linalg.norm(ad, axis=1), 1e-300)
        drho = np.abs(state_m["rho"] - state_d["rho"]) / state_d["rho"]
        acc = dict(rms_vs_fp64=float(np.sqrt(np.mean(err ** 2))), max_vs_fp64=float(err.max()),
                   rho_rms_vs_fp64=float(np.sqrt(np.mean(drho ** 2))),
                   rho_max_vs_fp64=float(drho.max()), same_order=bool(same))
        log(f"[bench] fp64: {fp64['ms_per_step']:.2f} ms/step, stages {fp64['stage_ms']}, {acc}")
    rk2 = rk2_8 = blk = None
    if args.workload == "core":
        rk2 = run_rk2(ic, 1, args.steps, args.warmup, ws)
        log(f"[bench] rk2 step: {rk2['ms_per_step']:.2f} ms (two force evaluations), dt {rk2['dt']}")
        rk2_8 = run_rk2(ic, 1, args.steps, args.warmup, ws, nbuildstep=8)
        log(f"[bench] rk2 step, build every 8 evaluations: {rk2_8['ms_per_step']:.2f} ms")
        blk = run_block(ic, 1, 1, 1, ws)
        log(f"[bench] block timesteps: {blk}")
    e2e = e2e_calls = None
    if not args.no_e2e:
        r = run_e2e_io(ic, 1, args.steps, args.warmup, ws)
        e2e = dict(value=ws * n * args.steps / (max_over_ranks(ws, r["total_ms"]) * 1e-3),
                   unit=UNIT, h2d_bytes_per_step=r["h2d"], d2h_bytes_per_step=r["d2h"],
                   ms_per_step=r["total_ms"] / args.steps,
                   api="seren_gpu_force_step_io (pinned host buffers in and out every step)")
        r = run_e2e(ic, 1, args.steps, args.warmup, ws)
        e2e_calls = dict(value=ws * n * args.steps / (max_over_ranks(ws, r["total_ms"]) * 1e-3),
                         unit=UNIT, h2d_bytes_per_step=r["h2d"], d2h_bytes_per_step=r["d2h"],
                         ms_per_step=r["total_ms"] / args.steps,
                         api="tree_update, sph_update, hydro_forces, grav_forces")
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        st = dict(state_m)
        assert np.all(ic["sound"] == ic["sound"][0]), "the core is isothermal at one c_s"
        ic_cpu = dict(parray=st["parray"], v=st["v"], sound=np.full(n, float(ic["sound"][0])),
                      h_fac=ic["h_fac"], thetamaxsqd=ic["thetamaxsqd"], alpha=ic["alpha"])
        r = cpu_eval(ic_cpu)
        log(f"[bench] CPU baseline: {r['sec']:.2f} s per evaluation on {r['cores']} threads, "
            f"stages {r['stages']}")
        cpu = dict(value=n / r["sec"], unit=UNIT, cores=r["cores"], kind="port",
                   cpu=cpu_host(), seconds_per_evaluation=round(r["sec"], 3),
                   stage_seconds=r["stages"],
                   sample=(f"one full force evaluation of all {n} particles (no sampling) by the "
                           f"C++ FP64 restatement of the reference (oracle/) on the converged "
                           f"state after the GPU run: tree build+reorder+stock, grad-h, hmax, "
                           f"neighbour lists, thermal, hydro, gravity; {r['sec']:.2f} s"))
        r["oracle"].close()
    if rank == 0 and ws == 1:
        acc.update(gravity_accuracy(ic, state_m["parray"],
                                    nsub=4096 if args.workload == "plummer" else 256))
    sweep = None
    if args.workload == "plummer" and rank == 0 and ws == 1:
        sweep = {}
        for th in (0.09, 0.25, 0.49):
            ic_th = dict(ic, thetamaxsqd=th)
            r_th, st_th = run_resident(ic_th, 1, 2, 2, ws)
            r_th["ctx"].close()
            a_th = gravity_accuracy(ic_th, st_th["parray"], nsub=4096)
            sweep[str(th)] = dict(gravity_ms=round(r_th["stage_ms"][4], 3),
                                  step_ms=round(r_th["total_ms"] / 2, 3),
                                  cells=r_th["counts"][0], pairs=r_th["counts"][1], **a_th)
            log(f"[bench] theta^2={th}: {sweep[str(th)]}")
    if rank != 0:
        return
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_mixed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64",
        "data": data,
        "config": line_config(wdesc, n),
        "precision": "mixed (FP32 pair arithmetic, FP64 walk/MAC/grad-h)",
        "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
        "stage_ms": {k: round(x, 3) for k, x in zip(
            ("tree", "gradh", "neib", "hydro", "gravity", "total"), mixed["stage_ms"][:6])},
        "tuning": mixed["tuning"],
        "fp64": fp64,
        "mixed_speedup_vs_fp64": (value / fp64["value"]) if fp64 else None,
        "accuracy": acc,
        "theta_sweep": sweep,
        "roofline": {"bound": "fp32", "kernel": "gravity walk (k_grav_walk<true>)",
                     "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak, "traffic": traffic_per_launch(n),
                     "flops_per_launch": flops, "cells": ncell, "pairs": npair,
                     "launch_ms": grav_ms,
                     "peak_source": "measured FP32 FMA throughput (seren_gpu_fma_peak); "
                                    "MEASURED_PEAKS.json has no non-tensor FP32 figure",
                     "fp64_peak": fp64_peak},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "e2e_reference_calls": e2e_calls,
        "rk2_step": rk2,
        "rk2_step_nbuildstep8": rk2_8,
        "block_timesteps": blk,
        "gpu_launches": mixed["launches"],
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def reference_arm(args, ws, rank, n):
    """The reference's CPU path on the host cores, rank 0 only: its C++ FP64
    restatement in oracle/ (the Fortran reference cannot be compiled here: no
    Fortran compiler), on all host threads.  Every step is one full force
    evaluation of all N particles (no sampling), from the state the previous
    step left: the first warm-up step starts from the h guess (first call),
    later ones carry every particle's converged h and drift r += v dt, as the
    repository's arm does on the GPU."""
    if rank != 0:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    ic = workload(n, args.workload)
    metric, data, wdesc = workload_info(args.workload, n)
    state = dict(parray=ic["parray"].copy(), v=ic["v"], sound=ic["sound"], h_fac=ic["h_fac"],
                 thetamaxsqd=ic["thetamaxsqd"], alpha=ic["alpha"])
    total = 0.0
    cores = 1
    stages = {}
    for k in range(args.warmup + args.steps):
        r = cpu_eval(state, first_call=(k == 0))
        cores = r["cores"]
        log(f"[bench] reference step {k}: {r['sec']:.2f} s, stages {r['stages']}")
        # carry h and zeta of every particle forward in the oracle's tree order, then drift
        state["parray"] = r["parray"]
        state["v"] = state["v"][r["perm"]]
        state["sound"] = state["sound"][r["perm"]]
        state["parray"][:, 0:3] += state["v"] * DT
        r["oracle"].close()
        if k >= args.warmup:
            total += r["sec"]
            for key, x in r["stages"].items():
                stages[key] = stages.get(key, 0.0) + x / args.steps
    value = n * args.steps / total
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
        "data": data, "config": line_config(wdesc, n),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "cpu": cpu_host(),
                         "stage_seconds": {key: round(x, 3) for key, x in stages.items()},
                         "sample": (f"C++ FP64 restatement of the reference (oracle/; the Fortran "
                                    f"reference has no compiler here) on {cores} threads: every "
                                    f"step one full force evaluation of all {n} particles, no "
                                    f"sampling, from the previous step's converged h")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
