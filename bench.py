#!/usr/bin/env python
"""Benchmark: SPH fluid particle-steps/s of the plain f64 WCSPH step on B200.

Workload (default, `dam_break_1m`): the synthetic 3-D dam break at 1M fluid
particles — a 100^3 lattice at dx = 0.01 m with seeded +-1e-4 m jitter in a
4.0 x 1.6 x 2.4 m tank walled by a 1-layer Akinci shell (396,802 boundary
samples); cubic spline h = 2 dx, rho0 = 1000, Tait gamma = 7 with a fixed
c0 = 20 m/s, alpha = 0.01, XSPH 0.25, g = -9.81 z, dt = 1e-4 s. One "step" is
one `WcsphWorld::step` (crates/pe-fluid/src/wcsph.rs:326) of the whole tank.
Counted units are fluid particles x steps.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
N > 1 runs under torch.distributed (one process per GPU); each rank advances
its own independent tank (weak scaling, no data-path collective) and the
job's value is the sum over ranks with the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "physics-engine_b200"))

METRIC = "SPH fluid particle-steps/s @1M (plain f64 WCSPH step)"
UNIT = "particle-steps/s"

WORKLOADS = {
    # name: (fluid lattice nx, ny, nz), tank extent
    "dam_break_1m": ((100, 100, 100), (4.0, 1.6, 2.4)),
    # 160 x 0.01 from origin dx puts the top fluid row on the y = 1.60 wall; the
    # tank grows to 1.62 m in y.
    "dam_break_4m": ((160, 160, 160), (4.0, 1.62, 2.4)),
    "dam_break_32k": ((32, 32, 32), (1.0, 0.4, 0.6)),
    # mid-size case for profiler captures (~1.5 GB on the device)
    "dam_break_262k": ((64, 64, 64), (2.56, 1.0, 1.5)),
}
DX, DT, SEED, JITTER = 0.01, 1e-4, 0x5EED5EED, 1e-4

# Algorithmic HBM bytes per fluid particle of the fused force + kick + drift
# pass: read x, v, rho (56 B), write x, v (48 B).
FORCE_BYTES_PER_FLUID = 104.0
# Algorithmic FP64 operations per visited in-support pair (add, mul, div, sqrt
# counted as one each): force pass 65, density 18, XSPH 31.
FORCE_OPS_PER_PAIR = 65.0
# DRAM bytes (read + write) of one force-pass launch per fluid particle, from
# the ncu capture of the 262,144-particle dam break (the neighbour lists
# dominate; traffic grows with the particle count).
FORCE_TRAFFIC_PER_FLUID = (429.341184e6 + 22.202624e6) / 262144
# sm__pipe_fp64_cycles_active of the force pass in the same capture
FORCE_FP64_PIPE_ACTIVE = 0.507
# smsp__issue_active of the list build (k_nlist_both) in the same capture
LISTS_ISSUE_ACTIVE = 0.592
# Whole step, per fluid / per boundary particle (cell key 28 + sort 8 +
# density 32 + XSPH 80 + forces 104; boundary 28 + 8 + 3 x 24).
STEP_BYTES_FLUID, STEP_BYTES_BOUNDARY = 252.0, 108.0
# Single-precision force pass: read cell-local x, v, rho (28 B), write x, v (24 B).
FORCE_BYTES_F32 = 52.0


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="dam_break_1m")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--train-tanks", type=int, default=16,
                    help="learned form: seeded 64k-particle tanks rolled out for training")
    ap.add_argument("--train-steps", type=int, default=300, help="learned form: plain steps trained on")
    ap.add_argument("--rollout-steps", type=int, default=200, help="learned form: steps of the 1M rollout")
    ap.add_argument("--form", choices=("plain", "f32", "batched", "learned", "pbf", "dfsph"), default="plain",
                    help="plain: the f64 step (reference bits); f32: the single-precision "
                         "form, timed and compared with the f64 step after the same steps; "
                         "batched: 512 seeded tanks in one world against a loop of "
                         "single-tank worlds; learned: the surrogate trained on plain "
                         "rollouts, judged every 10 steps, against the plain step")
    ap.add_argument("--precision", choices=("f64", "f32"), default="f64",
                    help="arithmetic of the batched form")
    ap.add_argument("--tanks", type=int, default=512)
    ap.add_argument("--loop-sample", type=int, default=32,
                    help="tanks of the batch timed one by one for the per-tank loop")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="plain form: skip the FP32 and learned legs of the default line")
    ap.add_argument("--f32-steps", type=int, default=200,
                    help="plain form's FP32 leg: steps both forms advance before the error comparison")
    ap.add_argument("--f32-timed-steps", type=int, default=20)
    ap.add_argument("--leg-train-tanks", type=int, default=4,
                    help="plain form's learned leg: seeded 64k-particle training tanks")
    ap.add_argument("--leg-train-steps", type=int, default=150)
    ap.add_argument("--leg-warm-steps", type=int, default=100,
                    help="learned form: untimed plain steps of the bench tank before the rollout")
    ap.add_argument("--leg-rollout-steps", type=int, default=50)
    return ap.parse_args()


def fp64_rate(pe, device):
    """The device's measured FP64 issue rate (Gop/s) of non-fused DMUL/DADD."""
    import ctypes as C

    g = C.c_double(0.0)
    rc = pe.load_library().pe_fluid_probe_fp64_rate(int(device), C.byref(g))
    return g.value if rc == 0 else None


def phase_overhead(pe, device, phases=64):
    """Measured cost of one phase boundary: a kernel node of a replayed CUDA
    graph against a grid-wide barrier inside one cooperative kernel (us)."""
    import ctypes as C

    a, b = C.c_double(0.0), C.c_double(0.0)
    f = pe.load_library().pe_fluid_probe_phase_overhead
    f.argtypes = [C.c_int32, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    rc = f(int(device), int(phases), C.byref(a), C.byref(b))
    return {"graph_node_us": a.value, "grid_barrier_us": b.value, "phases": phases} if rc == 0 else None


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, torch) -> float:
    """The maximum of x over all ranks (device timings are reported as the
    slowest rank's); x itself on one rank."""
    dist = torch.distributed
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, steps, slowest_ms, ranks):
    """Whole-job particle-steps/s: every rank advances its own tank(s) of
    `units_per_rank` fluid particles for `steps` steps; the job's time is the
    slowest rank's (max over ranks)."""
    return ranks * units_per_rank * steps / (slowest_ms / 1e3)


def build_scene(pe, workload):
    (nx, ny, nz), box = WORKLOADS[workload]
    mass = pe.mass_from_spacing(1000.0, DX, 3)
    p = pe.Particles(3, 1000.0, mass, 2.0 * DX)
    p.fill_box((DX, DX, DX), nx, ny, nz, DX)
    p.jitter_fluid(SEED, JITTER)
    p.fill_box_boundary((0.0, 0.0, 0.0), box, DX, 1)
    prm = pe.WcsphParams.water(1000.0, 20.0, (0.0, 0.0, -9.81))
    prm.adapt_sound_speed = False
    return p, prm, nx * ny * nz


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        try:
            for line in open(self.path):
                parts = [t.strip() for t in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
            os.unlink(self.path)
        except Exception:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def _oracle_world_1m(O, workload, threads):
    """The bench workload built by the oracle's builders (the reference's
    fill_box / fill_box_boundary / jitter), stepped by the oracle with
    `threads` host threads (the parallel oracle gives the sequential one's
    bits). Neighbour lists are materialised as the reference does
    (wcsph.rs:102-114) when the host has the memory for them (~1,700 entries
    of 8 bytes per fluid particle)."""
    import psutil

    (nx, ny, nz), box = WORKLOADS[workload]
    s = O.dam_break_scene(None, dx=DX, box=box, jitter=JITTER, seed=SEED, nxyz=(nx, ny, nz))
    need = nx * ny * nz * 1800 * 8 * 1.5
    materialize = psutil.virtual_memory().available > need
    w = O.World(s, O.dam_break_params(materialize=materialize))
    w.set_threads(threads)
    return w, nx * ny * nz, materialize


def cpu_baseline(workload, steps=2, single_steps=5):
    """The oracle (CPU port of the reference step) on the bench workload with
    all host threads for `steps` steps, and the single-threaded sequential
    oracle on the 32^3 dam break for `single_steps` steps (the reference path
    is single-threaded, docs/FLUID.md:104)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = os.cpu_count() or 1
    w, nf, mat = _oracle_world_1m(O, workload, threads)
    w.step(DT)  # first step outside the timing (neighbour-list allocation)
    t0 = time.perf_counter()
    w.run(DT, steps)
    sec = time.perf_counter() - t0
    del w
    s1 = O.dam_break_scene(32)
    w1 = O.World(s1, O.dam_break_params(materialize=True))
    w1.step(DT)
    t1 = time.perf_counter()
    w1.run(DT, single_steps)
    sec1 = time.perf_counter() - t1
    return {"value": nf * steps / sec, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{workload}: {steps} steps of the oracle's restatement of WcsphWorld::step "
                      f"(-O2 -ffp-contract=off) on {threads} host threads, the parallel form whose "
                      f"results are the sequential oracle's bits; neighbour lists "
                      f"{'materialised as the reference' if mat else 'not materialised (host memory)'}; "
                      f"{sec:.1f} s",
            "cpu_model": _cpu_model(), "host_cpus": os.cpu_count(),
            "single_thread": {"value": 32 ** 3 * single_steps / sec1, "unit": UNIT, "cores": 1,
                              "sample": f"32^3 dam break (32,768 fluid + 24,802 boundary), {single_steps} "
                                        f"steps of the sequential oracle, 1 thread used, neighbour lists "
                                        f"materialised; {sec1:.1f} s"}}


def run_reference(args, ws, rank):
    """The reference arm: the oracle's restatement of WcsphWorld::step on the
    same workload, one whole step of the tank per bench step, with every host
    thread (the parallel oracle; same bits as the sequential one). Rank 0 only."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = os.cpu_count() or 1
    w, nf, mat = _oracle_world_1m(O, args.workload, threads)
    for _ in range(args.warmup):
        w.step(DT)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        w.step(DT)
    sec = time.perf_counter() - t0
    value = nf * args.steps / sec
    sample = (f"one whole step of the {args.workload} tank per bench step; oracle port of "
              f"WcsphWorld::step on {threads} host threads (the parallel form reproduces the "
              f"sequential restatement bit for bit; the reference itself is single-threaded, "
              f"docs/FLUID.md:104); neighbour lists "
              f"{'materialised as the reference' if mat else 'not materialised (host memory)'}")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": _config(args.workload, nf, w.n - nf, ws),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample, "cpu_model": _cpu_model()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _config(workload, nf, nb, ws):
    return {"workload": workload, "fluid_particles": nf, "boundary_particles": nb,
            "dx": DX, "dt": DT, "h_over_dx": 2.0, "sound_speed": 20.0,
            "adapt_sound_speed": False, "xsph": 0.25, "visc_alpha": 0.01,
            "parallelism": f"{ws} independent tank(s), one per GPU",
            "l2": "state + neighbour lists (> 2 GB) exceed the 126 MB L2; no flush needed"}


def _device_summary(world):
    """Fluid centre of mass and total energy (kinetic + m g z) from the device
    FP64 reductions in original index order (diagnostics.rs:52-71)."""
    d = world.diagnostics()
    return world.fluid_center_of_mass(), d["kinetic_energy"] + d["gravitational_potential"], d


def f32_leg(workload, local, torch, pe, timed_steps, warm, total_steps):
    """The single-precision form next to the f64 step on the same tank, both
    from the same start: `warm` untimed steps, `timed_steps` steps timed with
    CUDA events on each world's stream, then steps up to `total_steps`; then
    densities (per particle, host), the centre of mass and the total energy
    (FP64 device reductions) of the f32 world against the f64 world's."""
    import numpy as np

    ps, prm, nf = build_scene(pe, workload)
    nb = len(ps) - nf
    fluid = ps.arrays()["kind"] == 0
    w64 = pe.WcsphWorld(ps, prm, pe.WcsphConfig(device=local))
    w32 = pe.WcsphWorld(ps, prm, pe.WcsphConfig(device=local, precision=pe.PRECISION_F32))
    del ps
    timings = {}
    for name, w in (("f32", w32), ("f64", w64)):
        stream = torch.cuda.ExternalStream(w.stream_handle(), device=local)
        w.run(DT, warm)
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if name == "f32" else None
        if sampler:
            sampler.start()
        w.set_profiling(True)
        w.profile(reset=True)
        w.kernel_launches(reset=True)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        w.run(DT, timed_steps)
        b.record(stream)
        b.synchronize()
        timings[name] = (a.elapsed_time(b), w.profile(reset=True), w.kernel_launches(),
                         sampler.stop() if sampler else None, w.status())
        w.set_profiling(False)
        rest = total_steps - warm - timed_steps
        if rest > 0:
            w.run(DT, rest)
    com32, e32, _ = _device_summary(w32)
    com64, e64, _ = _device_summary(w64)
    rho32, rho64 = w32.densities()[fluid], w64.densities()[fluid]
    rel = np.abs(rho32 - rho64) / rho64
    ms32, prof32, launches, clocks, status = timings["f32"]
    ms64 = timings["f64"][0]
    hbm_peak, peak_kind = _peaks()
    f_ms, f_n = prof32["forces"]
    achieved = FORCE_BYTES_F32 * nf * f_n / (f_ms / 1e3) / 1e9 if f_ms > 0 else 0.0
    leg = {
        "value": nf * timed_steps / (ms32 / 1e3), "unit": UNIT, "ms_per_step": ms32 / timed_steps,
        "timed_steps": timed_steps, "warmup": warm, "dtype": "f32 pair arithmetic (Kahan sums), f64 grid/CFL/reductions",
        "f64_ms_per_step": ms64 / timed_steps, "speedup_vs_f64_step": ms64 / ms32,
        "gpu_launches": int(launches), "status": int(status),
        "pair_weights": {"f32": w32.pair_weights(), "f64": w64.pair_weights()},
        "phases_ms_per_step": {k: v[0] / max(1, timed_steps) for k, v in prof32.items()},
        "error_vs_f64": {
            "after_steps": max(total_steps, warm + timed_steps),
            "density_rel_max": float(rel.max()), "density_rel_mean": float(rel.mean()),
            "com_drift_m": float(np.linalg.norm(com32 - com64)),
            "energy_rel_drift": float((e32 - e64) / abs(e64)),
            "reductions": "centre of mass and energy: FP64 device sums in original index order",
        },
        "roofline": {"bound": "hbm", "kernel": "k_forces_f32 (force + kick + drift)",
                     "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "peak_kind": peak_kind, "traffic": None,
                     "bytes_per_unit": FORCE_BYTES_F32, "units_per_launch": nf,
                     "launch_ms": f_ms / max(1, f_n)},
        "clocks": clocks,
    }
    w32.close()
    w64.close()
    return leg, nf, nb


def run_f32(args, ws, rank, local, torch, pe):
    """Single-precision form next to the f64 step on the same tank."""
    warm = max(args.warmup, 3)
    leg, nf, nb = f32_leg(args.workload, local, torch, pe, args.steps, warm, warm + args.steps)
    line = {
        "metric": "SPH fluid particle-steps/s @1M (FP32 form)", "value": leg["value"], "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "warmup": warm, "ms_per_step": leg["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "form": "f32",
        "config": {"workload": args.workload, "fluid_particles": nf, "boundary_particles": nb,
                   "dx": DX, "dt": DT, "sound_speed": 20.0, "adapt_sound_speed": False},
    }
    line.update({k: v for k, v in leg.items() if k not in ("value", "unit", "ms_per_step")})
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batched(args, ws, rank, local, torch, pe):
    """512 seeded dam-break tanks (2,048..65,536 particles, 0.3..1.2 m per axis)
    advanced by one world: each phase is one launch over all tanks, the steps are
    replayed as a captured CUDA graph, launch shapes come from the autotuner.
    Compared with looping the plain single-tank step over a sample of the same
    tanks (same steps, per-tank worlds, CUDA-event timed)."""
    import numpy as np
    from physics_engine_rs import scenes

    seed = SEED + rank  # each rank its own batch (independent tanks, no exchange)
    t_build = time.perf_counter()
    tanks, spec = scenes.batch_dam_break(args.tanks, seed)
    nf_t = [int(np.prod(s_["block"])) for s_ in spec]
    nf = sum(nf_t)
    prm = pe.WcsphParams.water(1000.0, 20.0, (0.0, 0.0, -9.81))
    prm.adapt_sound_speed = False
    prec = pe.PRECISION_F32 if args.precision == "f32" else pe.PRECISION_F64
    cfg = pe.WcsphConfig(device=local, precision=prec, use_graph=True)
    w = pe.WcsphWorld.from_tanks(prm, tanks, cfg)
    build_s = time.perf_counter() - t_build
    stream = torch.cuda.ExternalStream(w.stream_handle(), device=local)
    warm = max(args.warmup, 3)
    w.run(DT, warm)
    shapes = w.autotune()
    w.run(DT, 6)  # settle and capture the graph with the tuned shapes
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    w.kernel_launches(reset=True)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    w.run(DT, args.steps)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    clocks = sampler.stop()
    launches = w.kernel_launches()
    status = w.status()
    cap = w.capacity_info()
    pair_weights = w.pair_weights()
    ms = max_over_ranks(ms, torch)
    value = job_throughput(nf, args.steps, ms, ws)
    w.close()
    del w

    # per-tank loop: the plain step of single-tank worlds, a sample of the tanks
    loop_ms, loop_nf = 0.0, 0
    sample = list(range(0, len(tanks), max(1, len(tanks) // max(1, args.loop_sample))))[: args.loop_sample]
    for t in sample:
        wt = pe.WcsphWorld(tanks[t], prm, pe.WcsphConfig(device=local, precision=prec))
        st = torch.cuda.ExternalStream(wt.stream_handle(), device=local)
        wt.run(DT, warm)
        torch.cuda.synchronize()
        a.record(st)
        wt.run(DT, args.steps)
        b.record(st)
        b.synchronize()
        loop_ms += a.elapsed_time(b)
        loop_nf += nf_t[t]
        wt.close()
    loop_value = loop_nf * args.steps / (loop_ms / 1e3)

    hbm_peak, peak_kind = _peaks()
    line = {
        "metric": f"SPH fluid particle-steps/s, batched form ({args.tanks} tanks, {args.precision})",
        "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": warm,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.precision, "data": "synthetic", "form": "batched",
        "config": {"workload": f"batch_dam_break_{args.tanks}", "tanks": args.tanks,
                   "fluid_particles": nf, "particles": int(sum(len(t_) for t_ in tanks)),
                   "tank_particles_range": [2048, 65536], "tank_extent_range_m": [0.3, 1.2],
                   "seed": seed, "dx": DX, "dt": DT, "sound_speed": 20.0, "adapt_sound_speed": False,
                   "parallelism": f"{ws} rank(s), each its own batch of tanks",
                   "l2": "state + lists of the batch exceed the 126 MB L2; no flush needed"},
        "execution": {"graph_steps": 6, "autotuned_shapes": shapes, "scene_build_s": build_s,
                      "launches_per_step": launches / max(1, args.steps),
                      "phase_boundary_cost": phase_overhead(pe, local)},
        "gpu_launches": int(launches), "status": int(status),
        "neighbour_lists": {"used_gb": cap["list_groups_used"] * 16 / 1e9,
                            "pool_gb": cap["list_groups_capacity"] * 16 / 1e9,
                            "pair_weights": pair_weights},
        "per_tank_loop": {"value": loop_value, "unit": UNIT, "tanks_timed": len(sample),
                          "fluid_particles_timed": loop_nf,
                          "how": "single-tank worlds stepped one after another, same steps"},
        "speedup_vs_per_tank_loop": value / ws / loop_value,
        "roofline": {"bound": "hbm", "achieved": STEP_BYTES_FLUID * nf / (ms / args.steps / 1e3) / 1e9,
                     "peak": hbm_peak, "unit": "GB/s", "peak_kind": peak_kind, "traffic": None,
                     "frac": STEP_BYTES_FLUID * nf / (ms / args.steps / 1e3) / 1e9 / hbm_peak,
                     "note": "whole-step algorithmic fluid bytes; FP64/issue bound like the plain step"},
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def learned_leg(workload, local, torch, pe, train_tanks, train_steps, rollout_steps, warm_steps=100):
    """The learned surrogate: trained online on plain rollouts of seeded
    64k-particle tanks (tank extents 0.45..1.0 m), then the bench tank run with
    learned steps judged every 10 steps by the plain SPH density (a window
    whose relative density error exceeds 1% is rerun with the plain step),
    next to the plain f64 run of the same steps."""
    import numpy as np
    from physics_engine_rs import scenes
    from physics_engine_rs import surrogate as S

    prm = pe.WcsphParams.water(1000.0, 20.0, (0.0, 0.0, -9.81))
    prm.adapt_sound_speed = False
    # ---- training ----
    tanks, _ = scenes.batch_dam_break(train_tanks, SEED + 7, 64000, 64000, 0.45, 1.0)
    train = pe.WcsphWorld.from_tanks(prm, tanks, pe.WcsphConfig(device=local))
    del tanks
    sur = S.Surrogate(seed=SEED)
    t0 = time.perf_counter()
    losses = S.train_on_rollouts(sur, train, DT, train_steps, iters_per_step=2, lr=5e-4, stat_steps=20)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    train.close()
    # one-step loss on a 64k tank never trained on: the network against the
    # mean prediction and against persistence (reusing the last plain step's
    # dv/dt, drho/dt)
    held_tanks, _ = scenes.batch_dam_break(1, SEED + 99, 64000, 64000, 0.45, 1.0)
    held = pe.WcsphWorld.from_tanks(prm, held_tanks, pe.WcsphConfig(device=local))
    heldout = S.heldout_comparison(sur, held, DT, steps_before=min(150, train_steps))
    held.close()
    # ---- rollouts on the bench tank ----
    ps, _, nf = build_scene(pe, workload)
    fluid = ps.arrays()["kind"] == 0
    plain = pe.WcsphWorld(ps, prm, pe.WcsphConfig(device=local))
    learned = pe.WcsphWorld(ps, prm, pe.WcsphConfig(device=local))
    del ps
    steps = rollout_steps
    # both worlds leave the lattice start's first steps (never trained on)
    # with untimed plain steps
    if warm_steps:
        plain.run(DT, warm_steps)
        learned.run(DT, warm_steps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain.run(DT, steps)
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0
    sampler = ClockSampler(local)
    sampler.start()
    t0 = time.perf_counter()
    st = S.run_learned(learned, sur, DT, steps, judge_every=10, bound=0.01)
    torch.cuda.synchronize()
    learned_s = time.perf_counter() - t0
    clocks = sampler.stop()
    # ---- error against the plain f64 run ----
    r64, r_l = plain.densities()[fluid], learned.densities()[fluid]
    x64, x_l = plain.positions()[fluid], learned.positions()[fluid]
    rel = np.abs(r_l - r64) / r64
    com64, e64, _ = _device_summary(plain)
    com_l, e_l, _ = _device_summary(learned)
    leg = {
        "value": nf * steps / learned_s, "unit": UNIT, "ms_per_step": learned_s / steps * 1e3,
        "rollout_steps": steps, "plain_steps_before_rollout": warm_steps,
        "dtype": "bf16 network (fp32 accumulation), f64 state",
        "network": "2-hop message passing, MLP width 128 x 2 hidden layers, r_msg = h",
        "judge_every": 10, "fallback_bound": 0.01,
        "training": {"tanks": train_tanks, "particles_per_tank": 64000,
                     "plain_steps": train_steps, "normalisation_steps": 20,
                     "adam_steps": len(losses), "lr": 5e-4, "seconds": train_s,
                     "final_loss": float(np.mean(losses[-20:])) if losses else None},
        "plain_f64": {"ms_per_step": plain_s / steps * 1e3, "value": nf * steps / plain_s},
        "speedup_vs_plain_step": plain_s / learned_s,
        "heldout_one_step_loss": heldout,
        "judge": st, "fallback_rate": st["fallbacks"] / max(1, st["windows"]),
        "error_vs_f64": {"after_steps": warm_steps + steps, "density_rel_max": float(rel.max()),
                         "density_rel_mean": float(rel.mean()),
                         "position_rms_m": float(np.sqrt(((x_l - x64) ** 2).sum(1).mean())),
                         "com_drift_m": float(np.linalg.norm(com_l - com64)),
                         "energy_rel_drift": float((e_l - e64) / abs(e64))},
        "timing": "wall clock around synchronous runs (the learned run synchronises at every judge)",
        "clocks": clocks,
    }
    plain.close()
    learned.close()
    return leg, nf


def run_learned_form(args, ws, rank, local, torch, pe):
    leg, nf = learned_leg(args.workload, local, torch, pe, args.train_tanks, args.train_steps,
                          args.rollout_steps, args.leg_warm_steps)
    line = {
        "metric": "SPH fluid particle-steps/s @1M (learned surrogate, judged every 10 steps)",
        "value": leg["value"], "unit": UNIT, "n_gpus": 1, "steps": leg["rollout_steps"], "warmup": 0,
        "ms_per_step": leg["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": leg["dtype"], "data": "synthetic", "form": "learned",
        "config": {"workload": args.workload, "fluid_particles": nf, "dx": DX, "dt": DT},
    }
    line.update({k: v for k, v in leg.items() if k not in ("value", "unit", "ms_per_step", "dtype")})
    if rank == 0:
        print(json.dumps(line), flush=True)


SOLVER_DT = 1e-3  # PBF / DFSPH: 0.4 dx / (2 g H)^0.5 at dx 0.01 and a 1 m column
SOLVER_DV_CAP = 0.5


def solver_scene(pe, workload, form):
    """The dam-break geometry for the sibling solvers (block two spacings off
    the walls, as in the reference's canonical tanks), with the reference's own
    solver setups: PBF as its canonical tank (scenarios.rs:28-61: poly6/spiky,
    h = 2 dx, 4 iterations, no tensile correction), DFSPH as its canonical tank
    (scenarios.rs:74-116: calibrated mass, recomputed Akinci volumes, 1%
    tolerances, 8 + 8 iterations, XSPH 0.05, warm start) plus the reference's
    cap on the per-iteration pressure velocity change (0.5 m/s): without it the
    reference's DFSPH step diverges on lattice-start blocks of 24^3 and more."""
    (nx, ny, nz), box = WORKLOADS[workload]
    h = 2.0 * DX
    if form == "pbf":
        mass = pe.mass_from_spacing(1000.0, DX, 3)
    else:
        mass = pe.mass_calibrated_to_rest(1000.0, DX, h, 3)
    p = pe.Particles(3, 1000.0, mass, h)
    p.fill_box((2 * DX, 2 * DX, 2 * DX), nx, ny, nz, DX)
    p.jitter_fluid(SEED, JITTER)
    p.fill_box_boundary((0.0, 0.0, 0.0), box, DX, 1)
    g = (0.0, 0.0, -9.81)
    if form == "pbf":
        prm = pe.PbfParams(gravity=g, iterations=4, art_pressure_k=0.0, vorticity_eps=0.0)
    else:
        p.recomputed_akinci_psi()
        prm = pe.DfsphParams(gravity=g, particle_diameter=DX, density_error_tol=0.01, divergence_error_tol=0.01,
                             max_density_iters=8, max_divergence_iters=8, xsph_epsilon=0.05, adaptive_dt=False,
                             warm_start=True, max_velocity_correction=SOLVER_DV_CAP)
    return p, prm, nx * ny * nz


def solver_cpu_baseline(form, steps=2):
    """The oracle's PBF / DFSPH step (CPU restatements pinned by the reference's
    locked tank hashes), single thread, on the 32^3 dam break for `steps` steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    (nx, ny, nz), box = WORKLOADS["dam_break_32k"]
    h = 2.0 * DX
    mass = O.mass_from_spacing(1000.0, DX, 3) if form == "pbf" else O.mass_calibrated_to_rest(1000.0, DX, h, 3)
    s = O.Scene(3, 1000.0, mass, h)
    s.fill_box((2 * DX, 2 * DX, 2 * DX), nx, ny, nz, DX)
    s.jitter_fluid(SEED, JITTER)
    s.fill_box_boundary((0.0, 0.0, 0.0), box, DX, 1)
    if form == "pbf":
        q = O.pbf_default_params()
        q.iterations, q.art_pressure_k, q.vorticity_eps = 4, 0.0, 0.0
        q.gravity[:] = (0.0, 0.0, -9.81)
        w = O.PbfWorld(s, q)
    else:
        s.recompute_psi()
        q = O.dfsph_default_params()
        q.particle_diameter, q.density_error_tol, q.divergence_error_tol = DX, 0.01, 0.01
        q.max_density_iters, q.max_divergence_iters, q.xsph_epsilon, q.adaptive_dt = 8, 8, 0.05, 0
        q.max_velocity_correction = SOLVER_DV_CAP
        q.gravity[:] = (0.0, 0.0, -9.81)
        w = O.DfsphWorld(s, q)
    w.step(SOLVER_DT)
    t0 = time.perf_counter()
    w.run(SOLVER_DT, steps)
    sec = time.perf_counter() - t0
    nf = nx * ny * nz
    name = "PbfWorld::step" if form == "pbf" else "DfsphWorld::step"
    return {"value": nf * steps / sec, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"32^3 dam break (32,768 fluid), {steps} steps of the single-threaded C++ "
                      f"restatement of {name}, -O2 -ffp-contract=off; {sec:.1f} s",
            "host_cpus": os.cpu_count()}


def run_solver_form(args, ws, rank, local, torch, pe):
    """PBF or DFSPH on the dam break: the bit-exact GPU step (the reference's
    solver path), timed with CUDA events on the world's stream."""
    import numpy as np

    form = args.form
    ps, prm, nf = solver_scene(pe, args.workload, form)
    nb = len(ps) - nf
    cfg = pe.WcsphConfig(device=local)
    w = pe.PbfWorld(ps, prm, cfg) if form == "pbf" else pe.DfsphWorld(ps, prm, cfg)
    del ps
    stream = torch.cuda.ExternalStream(w.stream_handle(), device=local)
    w.run(SOLVER_DT, max(args.warmup, 3))
    torch.cuda.synchronize()
    iters = []
    sampler = ClockSampler(local)
    sampler.start()
    w.kernel_launches(reset=True)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier = (lambda: torch.distributed.barrier()) if ws > 1 else (lambda: None)
    barrier()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        w.step(SOLVER_DT)
        if form == "dfsph":
            iters.append(w.last_iterations())
    b.record(stream)
    b.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = a.elapsed_time(b)
    launches = w.kernel_launches()
    clocks = sampler.stop()
    status = w.status()
    ms = max_over_ranks(ms, torch)
    value = job_throughput(nf, args.steps, ms, ws)
    fluid = w.kinds() == 0
    rho = w.densities()[fluid]
    v = w.velocities()[fluid]
    line = {
        "metric": f"SPH fluid particle-steps/s @1M ({form.upper()} step)", "value": value, "unit": UNIT,
        "n_gpus": ws, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "form": form,
        "config": {"workload": args.workload, "fluid_particles": nf, "boundary_particles": nb, "dx": DX,
                   "dt": SOLVER_DT, "h_over_dx": 2.0,
                   "params": {k: getattr(prm, k) for k in type(prm)._FIELDS},
                   "parallelism": f"{ws} independent tank(s), one per GPU",
                   "l2": "state + neighbour lists exceed the 126 MB L2; no flush needed"},
        "gpu_launches": int(launches), "status": int(status),
        "state": {"mean_density_error": float(np.mean(np.abs(rho - 1000.0)) / 1000.0),
                  "v_max": float(np.sqrt((v * v).sum(1).max()))},
        "clocks": clocks,
    }
    if form == "dfsph":
        it = np.array(iters)
        line["solver_iterations_mean"] = {"density": float(it[:, 0].mean()), "divergence": float(it[:, 1].mean())}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = solver_cpu_baseline(form)
    w.close()
    if rank == 0:
        print(json.dumps(line, default=str), flush=True)


def main():
    args = _args()
    ws, rank, local = _dist()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    if args.form in ("f32", "batched", "learned", "pbf", "dfsph"):
        import torch

        torch.cuda.set_device(local)
        if ws > 1:
            import datetime

            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        import physics_engine_rs as pe

        {"f32": run_f32, "batched": run_batched, "learned": run_learned_form, "pbf": run_solver_form,
         "dfsph": run_solver_form}[args.form](
            args, ws, rank, local, torch, pe)
        if ws > 1:
            torch.distributed.destroy_process_group()
        return

    import numpy as np
    import torch

    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import physics_engine_rs as pe

    ps, prm, nf = build_scene(pe, args.workload)
    nb = len(ps) - nf
    world = pe.WcsphWorld(ps, prm, pe.WcsphConfig(device=local))
    del ps
    stream = torch.cuda.ExternalStream(world.stream_handle(), device=local)

    world.run(DT, max(args.warmup, 3))
    # launch shapes picked on this tank by the product's autotuner (block
    # sizes, the list build's tile and CTAs per SM; no shape changes a bit)
    shapes = world.autotune()
    world.run(DT, 2)
    torch.cuda.synchronize()

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    # ---- device-timed region ----
    sampler = ClockSampler(local)
    sampler.start()
    world.set_profiling(True)
    world.profile(reset=True)
    world.kernel_launches(reset=True)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    start.record(stream)
    world.run(DT, args.steps)
    end.record(stream)
    end.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(end)
    launches = world.kernel_launches()
    prof = world.profile(reset=True)
    world.set_profiling(False)
    clocks = sampler.stop()
    status = world.status()
    cap = world.capacity_info()
    ms = max_over_ranks(ms, torch)
    value = job_throughput(nf, args.steps, ms, ws)

    # ---- end-to-end through the public API with host buffers ----
    if args.e2e_steps <= 0:
        args.e2e_steps = 0
    x_h = torch.empty((world.n, 3), dtype=torch.float64, pin_memory=True).numpy()
    v_h = torch.empty((world.n, 3), dtype=torch.float64, pin_memory=True).numpy()
    world.positions(out=x_h)
    world.velocities(out=v_h)

    def e2e_step():
        world.set_positions(x_h)
        world.set_velocities(v_h)
        world.step(DT)
        world.positions(out=x_h)
        world.velocities(out=v_h)

    e2e_step()  # untimed: the first host round trip re-checks the list capacity
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_sec = max(time.perf_counter() - t0, 1e-12)
    e2e_sec = max_over_ranks(e2e_sec, torch)
    e2e = ws * nf * args.e2e_steps / e2e_sec
    io_bytes = 2 * world.n * 24

    hbm_peak, peak_kind = _peaks()
    f_ms, f_n = prof["forces"]
    achieved = FORCE_BYTES_PER_FLUID * nf * f_n / (f_ms / 1e3) / 1e9 if f_ms > 0 else 0.0
    l_ms, l_n = prof["lists"]
    # list pool groups used by one build (16 B each) + per-slot descriptors (uint4 + uint2 + u32)
    list_bytes = cap["list_groups_used"] * 16 + (nf + nb) * (16 + 8 + 4)
    # FP64 axis: visited in-support pairs of the force pass against the
    # device's measured non-fused FP64 issue rate
    _, in_sup = world.neighbour_counts()
    fluid_mask = world.kinds() == 0
    pairs = int(in_sup[fluid_mask].astype(np.int64).sum())
    fp64_peak = fp64_rate(pe, local)
    f_launch_s = f_ms / max(1, f_n) / 1e3
    fp64_achieved = pairs * FORCE_OPS_PER_PAIR / f_launch_s / 1e9 if f_launch_s > 0 else 0.0
    total_prof = sum(v[0] for v in prof.values())
    step_bytes = STEP_BYTES_FLUID * nf + STEP_BYTES_BOUNDARY * nb
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(args.workload, nf, nb, ws),
        "launch_shapes": shapes,
        "gpu_launches": int(launches),
        "status": int(status),
        "phases_ms_per_step": {k: v[0] / max(1, args.steps) for k, v in prof.items()},
        "neighbour_lists": {"used_gb": cap["list_groups_used"] * 16 / 1e9,
                            "pool_gb": cap["list_groups_capacity"] * 16 / 1e9,
                            "union_stage": cap["union_capacity"], "max_union": cap["max_union"],
                            "pair_weights": world.pair_weights()},
        "roofline": {"bound": "hbm", "kernel": "k_forces (force + kick + drift)",
                     "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "peak_kind": peak_kind,
                     "traffic": FORCE_TRAFFIC_PER_FLUID * nf if FORCE_TRAFFIC_PER_FLUID else None,
                     "bytes_per_unit": FORCE_BYTES_PER_FLUID, "units_per_launch": nf,
                     "launch_ms": f_ms / max(1, f_n),
                     "binding": "fp64 (roofline_fp64): the pass is FP64-ALU bound, not HBM bound"},
        "roofline_fp64": {"bound": "fp64", "kernel": "k_forces (force + kick + drift)",
                          "achieved": fp64_achieved, "peak": fp64_peak, "unit": "Gop/s",
                          "frac": fp64_achieved / fp64_peak if fp64_peak else None,
                          "peak_kind": "measured: independent DMUL + DADD issue rate of this device "
                                       "(pe_fluid_probe_fp64_rate; the f64 passes compile without FMA)",
                          "ops_per_pair": FORCE_OPS_PER_PAIR, "pairs_per_launch": pairs,
                          "pairs_per_fluid": pairs / max(1, nf),
                          "ncu_fp64_pipe_active": FORCE_FP64_PIPE_ACTIVE,
                          "note": "pairs are visited (ordered) in-support pairs: the gather evaluates each "
                                  "fluid pair from both sides, the reference's scatter once"},
        # The list build is the largest kernel by time but has no algorithmic
        # work in the step's byte or FLOP model (its ~1,700 candidate tests per
        # fluid particle are the builder's overhead); its DRAM traffic is
        # about the lists it writes, and it is issue bound (no FP64).
        "roofline_lists": {"bound": "issue", "kernel": "k_nlist_both (visit + lower lists)",
                           "achieved": list_bytes / (l_ms / max(1, l_n) / 1e3) / 1e9 if l_ms > 0 else None,
                           "peak": hbm_peak, "unit": "GB/s",
                           "frac": (list_bytes / (l_ms / max(1, l_n) / 1e3) / 1e9 / hbm_peak) if l_ms > 0 else None,
                           "peak_kind": peak_kind, "bytes_per_launch": list_bytes,
                           "launch_ms": l_ms / max(1, l_n), "ncu_issue_active": LISTS_ISSUE_ACTIVE,
                           "note": "bytes = the list entries and descriptors written per build; issue bound, "
                                   "not HBM bound"},
        "step_roofline": {"algorithmic_bytes_per_step": step_bytes,
                          "achieved_gbs": step_bytes / (ms / args.steps / 1e3) / 1e9,
                          "profiled_ms_per_step": total_prof / max(1, args.steps)},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": io_bytes,
                "d2h_bytes_per_step": io_bytes, "steps": args.e2e_steps,
                "pattern": "set_positions + set_velocities from pinned host buffers, step, "
                           "get_positions + get_velocities (state round-trips through the host)"},
        "clocks": clocks,
    }
    world.close()
    # ---- the other forms of the metric, on the same tank (1 GPU) ----
    if ws == 1 and not args.no_forms:
        forms = {}
        leg, _, _ = f32_leg(args.workload, local, torch, pe, args.f32_timed_steps, max(args.warmup, 3),
                            args.f32_steps)
        forms["f32"] = leg
        leg, _ = learned_leg(args.workload, local, torch, pe, args.leg_train_tanks, args.leg_train_steps,
                             args.leg_rollout_steps, args.leg_warm_steps)
        forms["learned"] = leg
        line["forms"] = forms
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
