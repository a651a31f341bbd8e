#!/usr/bin/env python
"""ns/day of the 23,958-atom PME water box (LangevinMiddle + SETTLE, 2 fs) on B200.

One bench step is one segment of `--segment` MD steps (default 200) run back to back through
Context.step, as in production; L2 is flushed (256 MiB write) between timed segments, outside
the timed region.  Timing uses CUDA events on the Context's own stream; multi-GPU runs are
independent replicas (no collective on the data path) timed as the max over ranks.

--impl reference times the reference algorithm's CPU implementation (the f64 oracle port of
openmm-rs's NonbondedForce/PME/LangevinMiddle/SHAKE path, all host threads) on the same
workload, one MD step per bench step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "openmm-rs_b200"))

WORKLOAD = "water-23958"
DT_PS = 0.002
METRIC = "ns/day @24k-atom PME water box (1 B200) + force RMS rel err vs FP64"
METRIC_LARGE = "ns/day @1,065k-atom PME water box (1 B200) + force RMS rel err vs FP64"


def water_metric():
    return METRIC_LARGE if WORKLOAD == "water-1065000" else METRIC
# Algorithmic FP32 work per in-cutoff pair of the mixed-precision PME pair kernel, FMA = 2,
# MUFU (rsqrt, exp2, rcp) = 1: delta 3, r^2 5, rsqrt + 1/r^2 2, LJ 11, Ewald (r, exp2,
# erfc fit with 7 FMAs, force) 28, f/r sum 1, i and j force accumulation 6 + 6 = 62.
FLOPS_PER_PAIR = 62
# HBM bytes per particle of one integrator launch: read x, v, fixed-point F, rebuild
# reference (4 x 24) plus per-molecule index (16/3), write x, v (2 x 24).
INTEGRATE_BYTES_PER_ATOM = 96 + 16 / 3 + 48


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--segment", type=int, default=200, help="MD steps per bench step")
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--precision", choices=["mixed", "double"], default="mixed")
    p.add_argument("--skip-extras", action="store_true",
                   help="skip the FP64-form, roofline and CPU-baseline legs")
    p.add_argument("--no-equilibrate", action="store_true",
                   help="start from the lattice (short runs for profiler captures)")
    p.add_argument("--workload", choices=["water-23958", "water-1065000", "chains-256",
                                          "chains-learned"],
                   default="water-23958",
                   help="water-1065000: the 22 nm box of 355,000 waters; chains-256: 256 uneven "
                        "implicit-solvent chains batched in one Context; chains-learned: 16 "
                        "chains of 5,000 atoms with learned Born radii vs exact OBC")
    p.add_argument("--no-graph", action="store_true",
                   help="launch kernels one by one instead of from CUDA graphs (profiler "
                        "captures: kernels inside graphs with conditional nodes cannot be "
                        "profiled individually)")
    p.add_argument("--systems", type=int, default=16,
                   help="chains-learned: number of chains (small cases for profiler captures)")
    p.add_argument("--atoms", type=int, default=5000, help="chains-learned: atoms per chain")
    p.add_argument("--pair-cull", type=int, default=-1,
                   help="water boxes without the autotuner (--no-equilibrate): tiles per warp "
                        "run of the culling pair kernel (0 off, -1 the default)")
    p.add_argument("--skin", type=float, default=0.0,
                   help="water boxes without the autotuner (--no-equilibrate): Verlet skin in "
                        "nm (0: the default)")
    return p.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def init_replicas(world, local, backend="nccl"):
    """One process per GPU, each an independent replica: the process group carries only the
    barriers around the timed region and the max-over-ranks timing reduction (a short timeout,
    so ranks that lose each other fail instead of waiting)."""
    if world <= 1:
        return
    import datetime

    import torch
    import torch.distributed as dist

    kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)


def replica_barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(values, world, device):
    """Element-wise maximum of per-rank timings (the job takes as long as its slowest rank)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def close_replicas(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def ns_per_day(md_steps, seconds):
    return md_steps * DT_PS / 1000.0 / seconds * 86400.0


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
               "-lms", "200"]
        if gpu_id:
            cmd += ["-i", gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


_EQUILIBRATED = {}


EQUILIBRATION_STEPS = 2000


def equilibrate(seed, device, steps=None):
    """Untimed: the jittered-lattice start releases ~27 MJ/mol while it relaxes, so the box is
    first brought to 300 K with a strongly coupled bath (20/ps, 4 ps)."""
    import ommb200
    from ommb200 import synth, systems

    steps = EQUILIBRATION_STEPS if steps is None else steps
    if seed not in _EQUILIBRATED:
        w = synth.water_preset(WORKLOAD)
        ctx = ommb200.Context(systems.water_system(w), systems.langevin(friction=20.0, seed=seed),
                              precision="mixed", device=device, use_cuda_graph=USE_GRAPH)
        ctx.set_positions(w.positions)
        ctx.set_velocities_to_temperature(300.0, seed=seed)
        if steps:
            ctx.step(steps)
        st = ctx.get_state(positions=True, velocities=True)
        ctx.close()
        _EQUILIBRATED[seed] = (w, st.positions, st.velocities)
    return _EQUILIBRATED[seed]


def build_context(precision, seed, device):
    import ommb200
    from ommb200 import systems

    w, x, v = equilibrate(seed, device)
    ctx = ommb200.Context(systems.water_system(w), systems.langevin(seed=seed),
                          precision=precision, device=device, use_cuda_graph=USE_GRAPH,
                          pair_cull=PAIR_CULL, neighbor_skin=SKIN)
    ctx.set_positions(x)
    ctx.set_velocities(v)
    TUNED[precision] = ctx.autotune(200) if TUNE else None
    return w, ctx


TUNE = True
TUNED = {}
USE_GRAPH = True
PAIR_CULL = -1
SKIN = 0.0


def time_segments(ctx, torch, segments, md_steps, flush):
    """Device time (ms) of `segments` Context.step(md_steps) calls, flushing L2 between."""
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    total = 0.0
    for _ in range(segments):
        flush.zero_()
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        ctx.step(md_steps)
        stop.record(stream)
        stop.synchronize()
        total += start.elapsed_time(stop)
    return total


def time_e2e(ctx, torch, n_atoms, segments, md_steps, flush):
    """End to end through the public API: pinned host inputs uploaded, MD segment, positions,
    velocities and energies read back, every bench step."""
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    st = ctx.get_state(positions=True, velocities=True)
    pos = torch.from_numpy(st.positions.copy()).pin_memory()
    vel = torch.from_numpy(st.velocities.copy()).pin_memory()
    total = 0.0
    for _ in range(segments):
        flush.zero_()
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        ctx.set_positions_from_pointer(pos.data_ptr())
        ctx.set_velocities_from_pointer(vel.data_ptr())
        ctx.step(md_steps)
        ctx.get_state_into(pos.data_ptr(), vel.data_ptr(), energy=True)
        stop.record(stream)
        stop.synchronize()
        total += start.elapsed_time(stop)
    h2d = 2 * 24 * n_atoms
    d2h = 2 * 24 * n_atoms + 8
    return total, h2d, d2h


def kernel_profile(ctx, md_steps):
    """Per-kernel device time from CUDA events recorded around every launch on the Context's
    stream (non-graph launch path), over `md_steps` MD steps."""
    ctx.set_profiling(True)
    ctx.step(md_steps)
    times = ctx.kernel_times()
    ctx.set_profiling(False)
    return times


def cpu_baseline(w, x0, threads, gpu_forces):
    """The oracle port of the reference path timed on the host: force evaluation (all given
    threads) + LangevinMiddle/SHAKE steps of the same box from positions `x0`, bounded to
    ~10 s of CPU work.  Its first force evaluation is also the FP64 reference for the GPU
    forces computed at `x0`."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np

    import oracle as O

    t0 = time.perf_counter()
    f, e = O.nonbonded(x0, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                       method="PME", cutoff=0.9, ewald_tolerance=5e-4, box=w.box,
                       threads=threads)
    first = time.perf_counter() - t0
    err = None
    if gpu_forces is not None:
        err = float(np.sqrt(((gpu_forces - f) ** 2).sum() / (f ** 2).sum()))
    x, v = x0.copy(), np.zeros_like(x0)
    steps, spent = 0, 0.0
    budget = 10.0
    while spent < budget and steps < 50:
        t0 = time.perf_counter()
        f, _ = O.nonbonded(x, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                           method="PME", cutoff=0.9, ewald_tolerance=5e-4, box=w.box,
                           threads=threads)
        rc, x, v = O.lfmiddle_step(x, v, f, w.masses(), DT_PS, 300.0, 1.0,
                                   O.gaussian_noise(1, 0, steps, w.n_atoms),
                                   constraints=w.constraints(), tolerance=1e-5, mode=0)
        spent += time.perf_counter() - t0
        steps += 1
        if rc != 0:
            break
    return {"value": ns_per_day(steps, spent), "unit": "ns/day", "cores": threads,
            "kind": "port",
            "sample": f"{steps} MD steps of the {w.n_atoms}-atom box (f64 oracle: PME force "
                      f"evaluation + LangevinMiddle/SHAKE), {spent:.1f} s; first force "
                      f"evaluation {first:.2f} s", "energy": e}, err


def nve_drift(w, x, v, device, precision, ps=100.0, sample_ps=0.5, settle_ps=10.0, blocks=10):
    """Total-energy drift without a thermostat (LangevinMiddle at zero friction and temperature,
    which is velocity Verlet with SETTLE) over `ps` picoseconds at 2 fs, after `settle_ps` more
    picoseconds at 1/ps coupling from the given state: the least-squares slope of
    E_pot + E_kin sampled every `sample_ps`, with its standard error from the slope of `blocks`
    block means (neighbouring samples are correlated, block means much less)."""
    import numpy as np

    import ommb200
    from ommb200 import systems

    settle = ommb200.Context(systems.water_system(w), systems.langevin(friction=1.0, seed=7),
                             precision=precision, device=device)
    settle.set_positions(x)
    settle.set_velocities(v)
    settle.step(int(round(settle_ps / DT_PS)))
    st = settle.get_state(positions=True, velocities=True)
    settle.close()
    ctx = ommb200.Context(systems.water_system(w),
                          systems.langevin(temperature=0.0, friction=0.0, seed=1),
                          precision=precision, device=device)
    ctx.set_positions(st.positions)
    ctx.set_velocities(st.velocities)
    every = int(round(sample_ps / DT_PS))
    t, e = [], []
    for k in range(int(round(ps / sample_ps)) + 1):
        st = ctx.get_state(energy=True)
        t.append(k * sample_ps)
        e.append(st.potential_energy + st.kinetic_energy)
        if k * sample_ps < ps:
            ctx.step(every)
    ctx.close()
    t, e = np.array(t), np.array(e)
    slope = float(np.polyfit(t, e, 1)[0]) * 1000.0  # kJ/mol/ns
    per = len(e) // blocks
    tb = t[:per * blocks].reshape(blocks, per).mean(1)
    eb = e[:per * blocks].reshape(blocks, per).mean(1)
    fit = np.polyfit(tb, eb, 1)
    resid = eb - np.polyval(fit, tb)
    stderr = float(np.sqrt((resid ** 2).sum() / (blocks - 2) / ((tb - tb.mean()) ** 2).sum())) * 1000.0
    dof = 3 * w.n_atoms - 3 * w.n_waters  # rigid waters: 6 degrees of freedom each
    return {"precision": precision, "ps": ps, "settle_ps": settle_ps, "samples": len(e),
            "kj_mol_per_ns": slope, "slope_stderr_kj_mol_per_ns": stderr,
            "kj_mol_per_ns_per_dof": slope / dof, "slope_stderr_per_dof": stderr / dof,
            "energy_rms_fluctuation_kj_mol": float(np.std(e - np.polyval(np.polyfit(t, e, 1), t))),
            "dof": dof}


def cpu_one_core(w, x0):
    """The oracle's PME force evaluation on one host thread (the reference is single-threaded),
    as ns/day if every MD step cost one such evaluation."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    t0 = time.perf_counter()
    O.nonbonded(x0, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(), method="PME",
                cutoff=0.9, ewald_tolerance=5e-4, box=w.box, threads=1)
    sec = time.perf_counter() - t0
    return {"value": ns_per_day(1, sec), "unit": "ns/day", "cores": 1, "kind": "port",
            "sample": f"one f64 PME force evaluation in {sec:.2f} s"}


def profiled_traffic(name, tiles_now):
    """DRAM bytes per launch of a kernel from the committed ncu summary `profiles/<name>.md`
    (lines `traffic_bytes_per_launch: B` and `tiles_at_capture: T`), scaled to the current
    launch by its tile count (the traffic is the tile entries and the particles they name)."""
    try:
        text = (ROOT / "profiles" / f"{name}.md").read_text()
    except OSError:
        return None
    vals = {}
    for key in ("traffic_bytes_per_launch", "tiles_at_capture"):
        for line in text.splitlines():
            if line.strip("`").startswith(key + ":"):
                vals[key] = float(line.strip("`").split(":")[1])
    if "traffic_bytes_per_launch" not in vals:
        return None
    scale = tiles_now / vals["tiles_at_capture"] if vals.get("tiles_at_capture") else 1.0
    return vals["traffic_bytes_per_launch"] * scale


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np

    import oracle as O
    from ommb200 import synth

    w = synth.water_preset(WORKLOAD)
    threads = O.max_threads()
    x, v = w.positions.copy(), np.zeros_like(w.positions)

    def md_step(k):
        nonlocal x, v
        f, _ = O.nonbonded(x, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                           method="PME", cutoff=0.9, ewald_tolerance=5e-4, box=w.box,
                           threads=threads)
        rc, x, v = O.lfmiddle_step(x, v, f, w.masses(), DT_PS, 300.0, 1.0,
                                   O.gaussian_noise(1, 0, k, w.n_atoms),
                                   constraints=w.constraints(), tolerance=1e-5, mode=0)
        if rc != 0:
            raise RuntimeError(f"reference constraint solver failed ({rc})")

    for k in range(args.warmup):
        md_step(k)
    t0 = time.perf_counter()
    for k in range(args.steps):
        md_step(args.warmup + k)
    secs = time.perf_counter() - t0
    value = ns_per_day(args.steps, secs)
    out = {
        "impl": "reference", "metric": water_metric(), "value": value, "unit": "ns/day",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_atoms": w.n_atoms, "box_nm": float(w.box[0][0]),
                   "dt_ps": DT_PS, "method": "PME cutoff 0.9 nm tol 5e-4, grid by the "
                                             "tolerance rule",
                   "md_steps_per_bench_step": 1, "threads": threads},
        "cpu_baseline": {"value": value, "unit": "ns/day", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} MD steps, f64 oracle port of the reference "
                                   "CPU path (PME + LangevinMiddle/SHAKE)"},
        "e2e": {"value": value, "unit": "ns/day", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    global EQUILIBRATION_STEPS, TUNE, WORKLOAD, USE_GRAPH, PAIR_CULL, SKIN
    USE_GRAPH = not args.no_graph
    PAIR_CULL, SKIN = args.pair_cull, args.skin
    if args.workload.startswith("water"):
        WORKLOAD = args.workload
    if args.no_equilibrate:
        EQUILIBRATION_STEPS = 0
        TUNE = False
    if args.workload == "chains-256":
        main_chains(args)
        return
    if args.workload == "chains-learned":
        main_learned(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    import numpy as np
    import torch

    import ommb200

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    init_replicas(world, local)
    seed = 1000 + rank
    w, ctx = build_context(args.precision, seed, local)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    st0 = ctx.get_state(positions=True, forces=True, energy=True)
    x0, gpu_forces, e_gpu = st0.positions, st0.forces, st0.potential_energy
    time_segments(ctx, torch, args.warmup, args.segment, flush)

    def barrier():
        replica_barrier(world)
        torch.cuda.synchronize()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    barrier()
    rebuilds0 = ctx.nlist_stats()["rebuilds"]
    prunes0 = ctx.nlist_prune_stats()["prunes"]
    sampler = ClockSampler(uuid)
    torch.cuda.nvtx.range_push("timed")  # profiler captures can select the timed region
    ms = time_segments(ctx, torch, args.steps, args.segment, flush)
    torch.cuda.nvtx.range_pop()
    clocks = sampler.stop()
    rebuilds_timed = ctx.nlist_stats()["rebuilds"] - rebuilds0
    prunes_timed = ctx.nlist_prune_stats()["prunes"] - prunes0
    barrier()
    e2e_ms, h2d, d2h = time_e2e(ctx, torch, w.n_atoms, args.steps, args.segment, flush)
    barrier()
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], world, f"cuda:{local}")
    md_steps = args.steps * args.segment
    value = world * ns_per_day(md_steps, ms / 1000.0)
    tiles_timed = ctx.nlist_stats()["tiles"]
    e2e_value = world * ns_per_day(md_steps, e2e_ms / 1000.0)

    extras = {}
    roofline = None
    cpu = None
    launches = None
    if rank == 0 and not args.skip_extras:
        prof_steps = 100
        cull0 = ctx.pair_cull_stats()
        times = kernel_profile(ctx, prof_steps)
        cull1 = ctx.pair_cull_stats()
        pairs = ctx.count_pairs()
        pair_ms, pair_n = times.get("pair", (0.0, 1))
        t_pair = pair_ms / max(pair_n, 1) / 1000.0
        fp32_peak = ommb200.measure_fp32_peak(local)
        achieved = pairs * FLOPS_PER_PAIR / t_pair / 1e12 if t_pair > 0 else None
        culled = cull1["cull_tiles"] > 0
        kernel = ("pair_kernel_cull<Ewald> (packed FP32, entries culled at the current "
                  "positions, runs of %d tiles)" % cull1["cull_tiles"] if culled
                  else "pair_kernel_x2<Ewald> (packed FP32)")
        roofline = {"bound": "fp32", "kernel": kernel,
                    "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": (achieved / fp32_peak) if achieved else None,
                    "peak_source": "measured FP32 FMA throughput of this GPU "
                                   "(ommb200_measure_fp32_peak); MEASURED_PEAKS.json has no "
                                   "FP32 figure",
                    "algorithmic": f"{pairs} in-cutoff pairs x {FLOPS_PER_PAIR} flops per launch",
                    "avg_launch_ms": 1000.0 * t_pair,
                    "traffic": None,
                    "traffic_source": "profiles/%s_%s.md (one ncu capture, scaled by tiles)"
                                      % ("pair_kernel_cull" if culled else "pair_kernel", WORKLOAD)}
        peaks = measured_peaks()
        hbm = peaks.get("hbm_gbs")
        integ_ms, integ_n = times.get("integrate", (0.0, 1))
        if integ_ms > 0 and hbm:
            gbs = w.n_atoms * INTEGRATE_BYTES_PER_ATOM / (integ_ms / integ_n / 1000.0) / 1e9
            extras["integrate_roofline"] = {"bound": "hbm", "achieved": gbs, "peak": hbm,
                                            "unit": "GB/s", "frac": gbs / hbm,
                                            "note": "of measured; latency-bound at this size"}
        if hbm:
            # reciprocal-space spreading and gathering against the HBM roofline: spreading
            # reads position (24 B), charge (8 B) and slot (4 B) per atom and adds 8 B per grid
            # point; gathering reads the same per atom plus 4 B per grid point and adds 24 B of
            # fixed-point force per atom
            g_pts = int(np.prod(ctx.get_pme_parameters()[1]))
            pme_bytes = {"pme_spread": 36 * w.n_atoms + 8 * g_pts,
                         "pme_gather": 60 * w.n_atoms + 4 * g_pts}
            pme_roof = {}
            for k, nbytes in pme_bytes.items():
                k_ms, k_n = times.get(k, (0.0, 0))
                if k_ms > 0 and k_n:
                    gbs = nbytes / (k_ms / k_n / 1000.0) / 1e9
                    pme_roof[k.replace("pme_", "")] = {
                        "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                        "algorithmic_bytes": nbytes, "avg_launch_ms": k_ms / k_n}
            layout = ctx.pme_layout()
            form = ("atomic spread (64-atom CTAs staged in shared memory); gather " +
                    ("brick-owned (one CTA per 14^3 grid brick, %d bricks)" % layout["bricks"]
                     if layout["bricks_in_use"] else "eight lanes per particle"))
            extras["pme_roofline"] = dict(pme_roof, note="of measured HBM copy bandwidth",
                                          forms=form)
        per_step = {k: (v[0] / v[1], v[1] / prof_steps) for k, v in times.items()}
        extras["kernel_ms_per_md_step"] = {k: round(v[0] * v[1], 5) for k, v in per_step.items()}
        # our kernels per MD step: rebuild condition 1, prune condition 1 (pruned list), pair 1,
        # PME (spread, the three transform kernels, gather: 5; or spread, convert, convolve,
        # gather: 4 beside cuFFT; + the stencil kernel of the brick gather), exceptions 1,
        # integrate 1 (it also writes the pair kernel's packed coordinates); on rebuild steps the
        # 8 rebuild kernels, the pack of the new slots and the brick gather's ranges; the 2
        # prune kernels on prune steps; one counter kernel per graph launch of 20 steps
        pruned = ctx.nlist_prune_stats()["margin_nm"] > 0
        bricks = ctx.pme_layout()["bricks_in_use"]
        per_md = (1 + (1 if pruned else 0) + 1 + (5 if "pme_transform" in times else 4)
                  + (1 if bricks else 0) + 1 + 1)
        launches = (md_steps * per_md + (9 + (1 if bricks else 0)) * rebuilds_timed
                    + 2 * prunes_timed + args.steps * (args.segment // 20))
        extras["pairs_in_cutoff"] = pairs
        nl = ctx.nlist_stats()
        roofline["traffic"] = profiled_traffic(
            ("pair_kernel_cull_" if culled else "pair_kernel_") + WORKLOAD, nl["tiles"])
        # self tiles are 32 x 32 pair slots, neighbour tiles 2 x 16 x 16 (halves of block I)
        # or 32 x 32 (whole blocks), as the autotuner chose
        per_tile = 512 if ctx.tuning()["tile_entries"] == 16 else 1024
        slots = nl["blocks"] * 1024 + (nl["tiles"] - nl["blocks"]) * per_tile
        if culled:  # the slots the culling kernel evaluated: 512 per round
            nl["listed_pair_efficiency"] = pairs / max(1, slots)
            nl["cull_rounds_per_launch"] = (cull1["rounds"] - cull0["rounds"]) / max(1, pair_n)
            slots = 512 * nl["cull_rounds_per_launch"]
        nl["pair_efficiency"] = pairs / max(1, slots)
        nl["md_steps_per_rebuild"] = md_steps / max(1, rebuilds_timed)  # timed region only
        nl.update(ctx.nlist_prune_stats())
        nl["md_steps_per_prune"] = md_steps / max(1, prunes_timed) if pruned else None
        extras["nlist"] = nl
        # FP64-on-GPU form of the same kernels
        _, ctx64 = build_context("double", seed, local)
        time_segments(ctx64, torch, 1, args.segment, flush)
        n64 = max(2, args.steps // 4)
        ms64 = time_segments(ctx64, torch, n64, args.segment, flush)
        v64 = ns_per_day(n64 * args.segment, ms64 / 1000.0)
        ctx64.close()
        extras["fp64_form"] = {"value": v64, "unit": "ns/day", "mixed_over_fp64": value / world / v64}
        if world == 1:
            threads = os.cpu_count() or 1
            cpu, err = cpu_baseline(w, x0, threads, gpu_forces)
            extras["force_rms_rel_err_vs_fp64_oracle"] = err
            extras["energy_rel_err_vs_fp64_oracle"] = abs(e_gpu - cpu.pop("energy")) / abs(e_gpu)
            extras["host_cpu"] = {"nproc": os.cpu_count(), "model": _cpu_model()}
            extras["cpu_baseline_1_core"] = cpu_one_core(w, x0)
        if WORKLOAD == "water-23958":  # 2 x 110 ps of dynamics: the headline box only
            st_eq = ctx.get_state(positions=True, velocities=True)
            mixed = nve_drift(w, st_eq.positions, st_eq.velocities, local, "mixed")
            fp64 = nve_drift(w, st_eq.positions, st_eq.velocities, local, "double")
            extras["nve_drift"] = {"mixed": mixed, "fp64": fp64}
    out = {
        "metric": water_metric(), "value": value, "unit": "ns/day", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "ms_per_md_step": ms / md_steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32" if args.precision == "mixed" else "fp64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_atoms": w.n_atoms, "box_nm": float(w.box[0][0]),
                   "method": "PME cutoff 0.9 nm, Ewald tol 5e-4, grid %d^3, order 5"
                             % ctx.get_pme_parameters()[1][0],
                   "integrator": "LangevinMiddle 300 K, 1/ps, 2 fs, SETTLE",
                   "precision": args.precision + " (FP32 pair/spline math, int64 fixed-point "
                                "forces, FP64 integration and constraints)",
                   "md_steps_per_bench_step": args.segment,
                   "l2": "flushed (256 MiB write) between timed bench steps; MD steps inside a "
                         "bench step run back to back",
                   "parallelism": f"replicas x{world}",
                   "autotuned": TUNED.get(args.precision), "tiles": tiles_timed},
        "e2e": {"value": e2e_value, "unit": "ns/day", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clocks,
        "roofline": roofline,
        "cpu_baseline": cpu,
    }
    out.update(extras)
    ctx.close()
    close_replicas(world)
    if rank == 0:
        print(json.dumps(out), flush=True)


# FP32 work per pair of the Coulomb (NoCutoff) pair kernel: the Ewald count above with the
# 28-flop screened term replaced by the 2-flop bare Coulomb term.
FLOPS_PER_PAIR_COULOMB = FLOPS_PER_PAIR - 28 + 2
# GB pair term of pass 2 on top of the shared distance and force work (FMA = 2, MUFU = 1):
# 3 MUFU (rcp, ex2, rsqrt) + 13 multiplies/adds + 6 FMAs (two of them the dE/dR sums)
FLOPS_PER_PAIR_GB2 = 3 + 13 + 2 * 6
CHAIN_DT_PS = 0.001


def chain_oracle_step(O, ch, x, v, threads, k):
    """One f64 oracle MD step of one chain: NonbondedForce (NoCutoff, 1-2/1-3 exclusions, 1-4
    exceptions), GBSAOBCForce, bonds, angles, then LangevinMiddle."""
    n = ch.n_atoms
    excl = sorted({(i, i + 1) for i in range(n - 1)} | {(i, i + 2) for i in range(n - 2)})
    exc = [(i, j, 0.0, ch.sigma, 0.0) for i, j in excl]
    exc += [(i, i + 3, ch.charges[i] * ch.charges[i + 3], ch.sigma, ch.epsilon)
            for i in range(n - 3)]
    f, _ = O.nonbonded(x, ch.charges, [ch.sigma] * n, [ch.epsilon] * n, exc, method="NoCutoff",
                       threads=threads)
    f = f + O.gbsa_obc(x, ch.charges, ch.radii, [ch.gb_scale] * n, solvent_dielectric=78.5,
                       solute_dielectric=1.0)[0]
    f = f + O.harmonic_bonds(x, ch.bonds())[0] + O.harmonic_angles(x, ch.angles())[0]
    import numpy as np

    _, x, v = O.lfmiddle_step(x, v, f, np.full(n, ch.mass), CHAIN_DT_PS, 300.0, 1.0,
                              O.gaussian_noise(1, 0, k, n), mode=0)
    return x, v


def chains_cpu(chs, threads, budget=10.0):
    """The oracle's MD step time for the whole batch, extrapolated from chains stepped within
    `budget` seconds by the batch's sum of n^2 (all terms but the bonded ones are O(n^2))."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np

    import oracle as O

    spent, sample_n2, done = 0.0, 0.0, 0
    for ch in chs:
        x, v = ch.positions.copy(), np.zeros_like(ch.positions)
        t0 = time.perf_counter()
        chain_oracle_step(O, ch, x, v, threads, 0)
        spent += time.perf_counter() - t0
        sample_n2 += float(ch.n_atoms) ** 2
        done += 1
        if spent > budget:
            break
    total_n2 = sum(float(c.n_atoms) ** 2 for c in chs)
    return spent * total_n2 / sample_n2, done, spent


def main_chains(args):
    """256 independent implicit-solvent chains (200-2,000 atoms each) in one BatchContext:
    MD steps per second of the whole batch, against one Context per chain stepped in turn
    (the reference's way to run many systems) and the oracle on the host."""
    import numpy as np
    import torch

    import ommb200
    from ommb200 import synth, systems

    rank, world, local = dist_env()
    if args.impl == "reference":
        if rank != 0:
            return
        chs = synth.chain_batch(256, 200, 2000, seed=7)
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        threads = O.max_threads()
        secs = []
        for k in range(args.warmup + args.steps):
            sec, done, spent = chains_cpu(chs, threads, budget=5.0)
            secs.append(sec)
        sec = statistics.median(secs[args.warmup:])
        value = 1.0 / sec
        print(json.dumps({
            "impl": "reference", "metric": "MD steps/s of the 256-chain batch", "value": value,
            "unit": "batch steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * sec, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "chains-256", "threads": threads},
            "cpu_baseline": {"value": value, "unit": "batch steps/s", "cores": threads,
                             "kind": "port", "sample": f"{done} chains per bench step, "
                             "extrapolated by sum of n^2"},
            "e2e": {"value": value, "unit": "batch steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    torch.cuda.set_device(local)
    init_replicas(world, local)
    chs = synth.chain_batch(256, 200, 2000, seed=7)
    sizes = np.array([c.n_atoms for c in chs])
    seed = 1000 + rank
    ctx = ommb200.BatchContext([systems.chain_system(c) for c in chs],
                               systems.langevin(step_size=CHAIN_DT_PS, seed=seed),
                               precision=args.precision, device=local,
                               use_cuda_graph=not args.no_graph)
    ctx.set_positions(np.concatenate([c.positions for c in chs]))
    ctx.set_velocities_to_temperature(300.0, seed=seed)
    ctx.step(500)  # untimed: relax the random-walk start
    tuned = ctx.autotune(100)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    seg = args.segment
    time_segments(ctx, torch, args.warmup, seg, flush)
    replica_barrier(world)
    torch.cuda.synchronize()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    ms = time_segments(ctx, torch, args.steps, seg, flush)
    clocks = sampler.stop()
    e2e_ms, h2d, d2h = time_e2e(ctx, torch, int(sizes.sum()), args.steps, seg, flush)
    replica_barrier(world)
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], world, f"cuda:{local}")
    md_steps = args.steps * seg
    value = world * md_steps / (ms / 1000.0)
    extras = {}
    cpu = None
    if rank == 0 and not args.skip_extras:
        prof = 20
        times = kernel_profile(ctx, prof)
        extras["kernel_ms_per_md_step"] = {k: round(v[0] / prof, 5) for k, v in times.items()}
        n_excl = int((2 * sizes - 3).sum())
        pairs = int((sizes * (sizes - 1) // 2).sum()) - n_excl
        fp32_peak = ommb200.measure_fp32_peak(local)
        if "pair" in times:  # a separate nonbonded pair kernel
            kname, flops = "pair_kernel<float, Coulomb>", pairs * FLOPS_PER_PAIR_COULOMB
            algo = f"{pairs} pairs x {FLOPS_PER_PAIR_COULOMB} flops per launch"
            pair_ms, pair_n = times["pair"]
        else:  # the Coulomb/LJ terms run inside GB pass 2 over every pair of each chain
            all_pairs = int((sizes * (sizes - 1) // 2).sum())
            kname = "gb_pass<float, 2> with the NoCutoff nonbonded terms"
            flops = pairs * FLOPS_PER_PAIR_COULOMB + all_pairs * FLOPS_PER_PAIR_GB2
            algo = (f"{pairs} nonbonded pairs x {FLOPS_PER_PAIR_COULOMB} + {all_pairs} GB pairs "
                    f"x {FLOPS_PER_PAIR_GB2} flops per launch")
            pair_ms, pair_n = times.get("gb_pairs", (0.0, 1))
        t_pair = pair_ms / max(pair_n, 1) / 1000.0
        achieved = flops / t_pair / 1e12 if t_pair > 0 else None
        extras["roofline"] = {
            "bound": "fp32", "kernel": kname, "achieved": achieved,
            "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": achieved / fp32_peak if achieved else None,
            "algorithmic": algo, "avg_launch_ms": 1000.0 * t_pair, "traffic": None}
        # one Context per chain, stepped in turn: a sample of the first 32 chains
        sample = chs[:32]
        total = 0.0
        for k, ch in enumerate(sample):
            one = ommb200.Context(systems.chain_system(ch),
                                  systems.langevin(step_size=CHAIN_DT_PS, seed=seed),
                                  precision=args.precision, device=local)
            one.set_positions(ch.positions)
            one.set_velocities_to_temperature(300.0, seed=seed)
            one.step(seg)
            total += time_segments(one, torch, 1, seg, flush)
            one.close()
        per_step_sep = total / seg * len(chs) / len(sample)
        extras["separate_contexts"] = {
            "ms_per_batch_step": per_step_sep,
            "batch_speedup": per_step_sep / (ms / md_steps),
            "sample": f"{len(sample)} of {len(chs)} chains, each its own Context, scaled by count"}
        threads = os.cpu_count() or 1
        sec, done, spent = chains_cpu(chs, threads)
        cpu = {"value": 1.0 / sec, "unit": "batch steps/s", "cores": threads, "kind": "port",
               "sample": f"{done} chains, one f64 oracle MD step each in {spent:.1f} s, "
                         "extrapolated to the batch by sum of n^2"}
        _, kin = ctx.system_energies()
        temps = 2.0 * kin / (3 * sizes * 0.008314462618)
        extras["temperature_k"] = {"mean": float(temps.mean()), "min": float(temps.min()),
                                   "max": float(temps.max())}
    out = {
        "metric": "MD steps/s of the 256-chain batch", "value": value,
        "unit": "batch steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "ms_per_md_step": ms / md_steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32" if args.precision == "mixed" else "fp64", "data": "synthetic",
        "aggregate_ns_per_day": len(chs) * md_steps * CHAIN_DT_PS / 1000.0 / (ms / 1000.0) * 86400.0,
        "gb_evaluations_per_s": len(chs) * value,
        "config": {"workload": "chains-256", "n_systems": len(chs), "n_atoms": int(sizes.sum()),
                   "sizes": "uniform in [200, 2000], seed 7",
                   "method": "NoCutoff NonbondedForce + GBSAOBCForce (78.5 / 1), bonds, angles",
                   "integrator": "LangevinMiddle 300 K, 1/ps, 1 fs",
                   "md_steps_per_bench_step": seg,
                   "l2": "flushed (256 MiB write) between timed bench steps",
                   "parallelism": f"replicas x{world}", "autotuned": tuned},
        "e2e": {"value": world * md_steps / (e2e_ms / 1000.0), "unit": "batch steps/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    out.update(extras)
    ctx.close()
    close_replicas(world)
    if rank == 0:
        print(json.dumps(out), flush=True)


def main_learned(args):
    """16 chains of 5,000 atoms in one BatchContext: MD steps/s with learned Born radii (judge
    and training included) against the same batch with exact OBC radii, and the GB energy and
    force error of the learned radii against the f64 oracle's exact OBC."""
    import numpy as np
    import torch

    import ommb200
    from ommb200 import synth, systems

    rank, world, local = dist_env()
    if args.impl == "reference":
        if rank == 0:
            sys.path.insert(0, str(ROOT / "oracle"))
            import oracle as O

            chs = [synth.chain(args.atoms, seed=70 + k) for k in range(args.systems)]
            threads = O.max_threads()
            sec, done, spent = chains_cpu(chs, threads, budget=10.0)
            print(json.dumps({
                "impl": "reference",
                "metric": f"MD steps/s, {args.systems} x {args.atoms:,}-atom chains (exact OBC)",
                "value": 1.0 / sec, "unit": "batch steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sec,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": "chains-learned", "threads": threads},
                "cpu_baseline": {"value": 1.0 / sec, "unit": "batch steps/s", "cores": threads,
                                 "kind": "port", "sample": f"{done} chains, extrapolated"},
                "e2e": {"value": 1.0 / sec, "unit": "batch steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}), flush=True)
        return
    torch.cuda.set_device(local)
    init_replicas(world, local)
    chs = [synth.chain(args.atoms, seed=70 + k) for k in range(args.systems)]
    n_atoms = sum(c.n_atoms for c in chs)
    x0 = np.concatenate([c.positions for c in chs])
    seed = 1000 + rank
    learned = {"judge_interval": 50, "radius_tolerance": 0.01, "train_steps": 10}

    def make(lr):
        ctx = ommb200.BatchContext(
            [systems.chain_system(c, learned_radii=lr, gb_force_group=1) for c in chs],
            systems.langevin(step_size=CHAIN_DT_PS, seed=seed), precision=args.precision,
            device=local, use_cuda_graph=not args.no_graph)
        ctx.set_positions(x0)
        ctx.set_velocities_to_temperature(300.0, seed=seed)
        return ctx

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    seg = args.segment
    exact = make(None)
    exact.step(500)
    time_segments(exact, torch, args.warmup, seg, flush)
    ms_exact = time_segments(exact, torch, args.steps, seg, flush)
    exact_kernels = None
    if rank == 0 and not args.skip_extras:
        exact_kernels = {k: round(v[0] / 50, 5) for k, v in kernel_profile(exact, 50).items()}
    exact.close()
    ctx = make(learned)
    ctx.step(1000)  # untimed: the first judges fix the normalisation and train the network
    time_segments(ctx, torch, args.warmup, seg, flush)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    stats0 = ctx.learned_radii_stats()
    replica_barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(uuid)
    ms = time_segments(ctx, torch, args.steps, seg, flush)
    clocks = sampler.stop()
    stats1 = ctx.learned_radii_stats()
    e2e_ms, h2d, d2h = time_e2e(ctx, torch, n_atoms, args.steps, seg, flush)
    replica_barrier(world)
    ms, e2e_ms, ms_exact = max_over_ranks([ms, e2e_ms, ms_exact], world, f"cuda:{local}")
    md_steps = args.steps * seg
    value = world * md_steps / (ms / 1000.0)
    extras = {}
    cpu = None
    if rank == 0 and not args.skip_extras:
        times = kernel_profile(ctx, 50)
        extras["kernel_ms_per_md_step"] = {k: round(v[0] / 50, 5) for k, v in times.items()}
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        st = ctx.get_state(positions=True, forces=True)
        gb_f = ctx.get_state(forces=True, groups=1 << 1).forces
        pot, _ = ctx.system_energies(groups=1 << 1)
        errs_e, f_num, f_den = [], 0.0, 0.0
        t0 = time.perf_counter()
        for k, (c, pos, f) in enumerate(zip(chs, ctx.split(st.positions), ctx.split(gb_f))):
            n = c.n_atoms
            f_ref, e_ref, _ = O.gbsa_obc(pos, c.charges, c.radii, np.full(n, c.gb_scale),
                                         solvent_dielectric=78.5)
            errs_e.append(abs(pot[k] - e_ref) / (n / 1000.0))
            f_num += float(((f - f_ref) ** 2).sum())
            f_den += float((f_ref ** 2).sum())
        oracle_s = time.perf_counter() - t0
        extras["learned_accuracy_vs_f64_exact_obc"] = {
            "gb_energy_err_kj_mol_per_1000_atoms": {"mean": float(np.mean(errs_e)),
                                                    "max": float(np.max(errs_e))},
            "gb_force_rms_rel_err": (f_num / f_den) ** 0.5,
            "oracle_seconds": oracle_s}
        threads = os.cpu_count() or 1
        sec, done, spent = chains_cpu(chs, threads, budget=10.0)
        cpu = {"value": 1.0 / sec, "unit": "batch steps/s", "cores": threads, "kind": "port",
               "sample": f"{done} chains, one f64 oracle MD step each (exact OBC) in "
                         f"{spent:.1f} s, extrapolated to the batch by sum of n^2"}
    d = {k: stats1[k] - stats0[k] for k in ("judges", "learned_steps", "exact_steps")}
    out = {
        "metric": f"MD steps/s, {args.systems} x {args.atoms:,}-atom chains, learned Born radii",
        "value": value, "unit": "batch steps/s (summed over replicas)", "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "ms_per_md_step": ms / md_steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32+bf16" if args.precision == "mixed" else "fp64+bf16", "data": "synthetic",
        "exact_obc": {"value": world * md_steps / (ms_exact / 1000.0), "unit": "batch steps/s",
                      "ms_per_md_step": ms_exact / md_steps},
        "learned_over_exact": ms_exact / ms,
        "learned_radii_timed": {**d, "last_radius_error": stats1["last_radius_error"],
                                "active": stats1["active"]},
        "config": {"workload": "chains-learned", "n_systems": len(chs), "n_atoms": n_atoms,
                   "method": "NoCutoff NonbondedForce + GBSAOBCForce (78.5 / 1), bonds, angles",
                   "learned_radii": learned, "integrator": "LangevinMiddle 300 K, 1/ps, 1 fs",
                   "md_steps_per_bench_step": seg,
                   "l2": "flushed (256 MiB write) between timed bench steps"},
        "e2e": {"value": world * md_steps / (e2e_ms / 1000.0), "unit": "batch steps/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if exact_kernels is not None and "kernel_ms_per_md_step" in extras:
        # the Born-radii work each mode does per MD step: the exact descreening passes, or the
        # learned lists, features, network and forces plus the judges' exact passes and training
        lk = extras["kernel_ms_per_md_step"]
        radii = ("gb_descreening", "gb_descreening_forces")
        exact_ms = sum(exact_kernels.get(k, 0.0) for k in radii)
        learned_ms = sum(v for k, v in lk.items() if k.startswith("lr_") or k in radii)
        out["exact_obc"]["kernel_ms_per_md_step"] = exact_kernels
        out["born_radii_work"] = {"exact_ms_per_md_step": exact_ms,
                                  "learned_ms_per_md_step": learned_ms,
                                  "exact_over_learned": exact_ms / learned_ms if learned_ms else None}
    out.update(extras)
    ctx.close()
    close_replicas(world)
    if rank == 0:
        print(json.dumps(out), flush=True)


def _cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


if __name__ == "__main__":
    main()
