"""Benchmark: MIC timesteps per second of the mixed-precision GPU path beside
the plain FP64 GPU path.

Workload (default): the synthetic 401x401 planetesimal (2,560,000 markers,
4x4 per cell; 140 km box, 50 km rock body in sticky air; rock viscosity
log-uniform per marker in 1e17-1e23 Pa s).  A step is one whole timestep of
simulation_loop (src/Erebus.jl:6370-7235).  The line's `value` is the
mixed-precision path (FGMRES in FP64 preconditioned by lagged multifrontal
LU factors applied in FP32; ErebusSolverOptions.krylov); the plain FP64 path
(direct LU of every new matrix plus FP64 refinement) is timed over the same
timesteps from the same initial state and reported under "fp64", with the
ratio.  Both solve every system to the same 1e-13 scaled residual.  With N
GPUs (torchrun) every rank advances its own planetesimal (replicas; the path
has no exchange step) and `value` is all ranks' timesteps over the slowest
rank's device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload planetesimal_141] [--precision fp64|mixed]

The line also carries "adjoint": gradients per second of the heat-path
adjoint (20 timesteps forward and reversed, checkpoints every 5) on the
141x141 adjoint workload at mechanical rest.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "MIC timesteps/sec (mixed-prec vs FP64 GPU, rel err<=1e-8)"
UNIT = "timesteps/s"
WORKLOAD = "planetesimal_401"
# solver options of each precision mode (ErebusSolverOptions fields)
MODES = {"fp64": {}, "mixed": {"krylov": 1, "precond_fp32": 1},
         "fp32-factors": {"factor_fp32": 1}, "krylov-fp64": {"krylov": 1}}


def load_pkg():
    import importlib.util
    if "erebus_b200" in sys.modules:
        return sys.modules["erebus_b200"]
    pkg_dir = os.path.join(ROOT, "erebus.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "erebus_b200", os.path.join(pkg_dir, "__init__.py"),
        submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["erebus_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    return O


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def config_dict(pkg, name, extra=None):
    c = pkg.CONFIGS[name]
    d = {"workload": name, "grid": "%dx%d basic nodes" % (c["N"], c["N"]),
         "markers_per_cell": "%dx%d" % (c["mpc"], c["mpc"]),
         "l2": "inputs larger than L2: the Stokes-Darcy factor storage (GBs) is read by "
               "every triangular solve and the marker arrays (>100 MB) are streamed every "
               "timestep"}
    if extra:
        d.update(extra)
    return d


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), "--query-gpu=" + q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() in ("active", "1"):
                        reasons.add(nm)
            except Exception:
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp64_peak():
    """Measured FP64 dense throughput of this GPU: cuBLAS DGEMM (torch.matmul,
    8192^3), best of 3, TFLOP/s."""
    import torch
    n = 8192
    a = torch.rand(n, n, dtype=torch.float64, device="cuda")
    b = torch.rand(n, n, dtype=torch.float64, device="cuda")
    a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1000.0) / 1e12


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    return rank, world, local


def max_over_ranks(x, world):
    """The largest of the ranks' values (device times): the job's time."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, ms_per_rank, world):
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / (max_over_ranks(ms_per_rank, world) / 1000.0)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def oracle_sample(pkg, O, name, steps, warmup):
    """The oracle (C restatement of the reference's timestep with OpenMP on
    the marker loops the reference threads, SuperLU solves) on the host
    cores: `warmup` untimed timesteps, then `steps` timed ones.  Returns
    (timesteps/s, seconds, first timed timestep)."""
    st = pkg.make_state(name)
    o = O.Oracle(st)
    for ts in range(1, warmup + 1):
        o.step(ts)
    t0 = time.perf_counter()
    for ts in range(warmup + 1, warmup + steps + 1):
        o.step(ts)
    el = time.perf_counter() - t0
    return steps / el, el, warmup + 1


def cpu_sample_plan(name):
    """The bounded sample of a workload the CPU legs time: (timed steps,
    warm-up steps, description).  At 401x401 one oracle timestep takes
    minutes, so the sample is timestep 1 alone, which has one thermochemical
    iteration where the timed GPU timesteps have three: the sample flatters
    the CPU side."""
    if name == "planetesimal_401":
        return 1, 0, ("timestep 1 of the same workload (one thermochemical iteration; "
                      "later timesteps take three, so this favours the CPU)")
    if name == "planetesimal_141":
        return 2, 1, "timesteps 2-3 of the same workload after 1 untimed"
    return 3, 1, "timesteps 2-4 of the same workload after 1 untimed"


def cpu_baseline(pkg, O, name):
    steps, warm, what = cpu_sample_plan(name)
    v, el, _ = oracle_sample(pkg, O, name, steps, warm)
    return {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": "%s: oracle restatement of the reference (Julia is not available), "
                      "OpenMP on the marker loops the reference threads, SuperLU direct "
                      "solves with nested-dissection ordering, %.1f s" % (what, el)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    pkg = load_pkg()
    O = load_oracle()
    # each step is a bounded sample of the workload (cpu_sample_plan); the
    # requested --steps / --warmup are recorded beside it
    steps, warm, what = cpu_sample_plan(args.workload)
    v, el, first = oracle_sample(pkg, O, args.workload, steps, warm)
    cores = os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
            "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": 1000 * el / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(pkg, args.workload),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "%s (requested %d timed, %d warm-up); oracle "
                                       "restatement of the reference (Julia is not "
                                       "available) with SuperLU solves, OpenMP on the "
                                       "marker loops the reference threads"
                                       % (what, args.steps, args.warmup)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def algorithmic_bytes(n, nodes):
    """Bytes each marker phase must move once (per launch of the phase), for
    n markers and `nodes` P nodes."""
    return {
        # read 16 marker fields (129 B) + write 7 derived (56 B); ~217 B per
        # P node of normalised outputs
        "markers_to_nodes": 185 * n + 217 * nodes,
        "rk4": 97 * n,
        "nodes_to_markers": 137 * n,
        "reaction": 73 * n,
    }


def measure_adjoint(pkg, world, reps=3, n_steps=20, every=5):
    """Gradients per second of erebus_adjoint_heat on the 141x141 adjoint
    workload (4x4 markers per cell, porosity U(0.05, 0.25)) at mechanical
    rest: each gradient is n_steps timesteps forward plus the reverse sweep,
    from the same initial state (re-uploaded, untimed)."""
    import torch
    from erebus_b200.adjoint import at_rest
    name = "planetesimal_141_adjoint"
    st = at_rest(pkg.make_state(name))
    sim = pkg.Simulation(st)
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    ev = lambda: torch.cuda.Event(enable_timing=True)
    sim.adjoint_heat(n_steps, every)          # warm-up: plans and tape
    sim.upload()
    e0, e1 = ev(), ev()
    torch.cuda.synchronize()
    e0.record(stream)
    for ts in range(1, n_steps + 1):
        sim.step(ts)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    times = []
    for _ in range(reps):
        sim.upload()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        J, g, gr, ast = sim.adjoint_heat(n_steps, every)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    sim.close()
    ms = max_over_ranks(sum(times) / reps, world)
    return {"metric": "adjoint grads/sec", "value": world * 1000.0 / ms,
            "unit": "gradients/s", "ms_per_gradient": ms,
            "forward_ms": fwd_ms, "reverse_overhead": ms / fwd_ms,
            "gradients": reps,
            "J": J, "dJ_dratio_al": gr, "max_abs_dJ_dphim": float(np.abs(g).max()),
            "adjoint_solves": ast.adjoint_solves,
            "config": {"workload": name, "grid": "141x141 basic nodes",
                       "markers": int(ast.markers), "markers_per_cell": "4x4",
                       "timesteps": n_steps, "checkpoint_every": every,
                       "objective": "mean basic-node temperature inside the body after the "
                                    "last timestep",
                       "parameters": "per-marker porosity and the 26Al/27Al ratio",
                       "state": "mechanical rest: G = 0, reactions off (the adjoint's scope)"}}


def measure_ensemble(pkg, world, rank, bodies, steps, warmup, wave):
    """Aggregate timesteps/s of an ensemble of planetesimals of uneven sizes
    (erebus_b200.ensemble: radius U(20, 100) km, grid side 61-201, per-body
    porosity, 26Al/27Al and viscosity), advanced `wave` bodies at a time,
    each body on its own host thread and stream.  Per wave: `warmup` untimed
    timesteps, then `steps` timed ones; the time of a wave is from an event
    before its first timed step to the last body's end event."""
    import torch
    from erebus_b200.ensemble import Ensemble, ensemble_states
    done, ms_total, sides = 0, 0.0, []
    for w0 in range(0, bodies, wave):
        nb = min(wave, bodies - w0)
        states = ensemble_states(nb, seed=42 + 1000 * rank, first=w0)
        sides += [st.p.Nx for st in states]
        ens = Ensemble(states)
        try:
            ens.run(warmup)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.cuda.synchronize()
            ens.run(steps, start_step=warmup + 1)
            ends = []
            for h in ens.streams():
                e = torch.cuda.Event(enable_timing=True)
                e.record(torch.cuda.ExternalStream(h))
                ends.append(e)
            torch.cuda.synchronize()
            ms_total += max(e0.elapsed_time(e) for e in ends)
            done += nb * steps
        finally:
            ens.close()
    ms = max_over_ranks(ms_total, world)
    return {"metric": "ensemble timesteps/sec (aggregate over bodies)",
            "value": world * done / (ms / 1000.0), "unit": "timesteps/s",
            "bodies": bodies * world, "steps_per_body": steps, "warmup": warmup,
            "ms": ms, "wave": wave, "grid_sides": [min(sides), max(sides)],
            "config": {"workload": "ensemble", "radius_km": [20, 100],
                       "grid_side": "61-201, linear in the radius", "markers_per_cell": "4x4",
                       "per_body": "porosity U(0.05, 0.3), 26Al/27Al U(1e-5, 5e-5), "
                                   "rock viscosity log-uniform 1e18-1e21 Pa s",
                       "execution": "one host thread and stream per body; solver kernels "
                                    "of all bodies on one shared stream",
                       "precision": "fp64"}}


def time_mode(pkg, args, mode, world, rank, local, clocks=False):
    """One precision mode on the workload: `warmup` untimed timesteps, then
    `steps` timed ones bracketed by a barrier and a device synchronisation,
    timed with CUDA events on the library's stream (max over ranks), with
    the device phase timer on."""
    import torch
    st = pkg.make_state(args.workload)
    sim = pkg.Simulation(st)
    sim.set_solver_options(**MODES[mode])
    for ts in range(1, args.warmup + 1):
        sim.step(ts)
    f0 = {k: sim.factor_stats(i) for i, k in enumerate(("hydro", "thermal", "gravity"))}
    sim.enable_phase_timing(True)
    l0 = sim.kernel_launches()
    y0 = sim.host_syncs()
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ck = Clocks(local) if clocks and rank == 0 else None
    barrier(world)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed:" + mode)   # lets ncu capture the timed region alone
    e0.record(stream)
    stats = []
    for ts in range(args.warmup + 1, args.warmup + args.steps + 1):
        stats.append(sim.step(ts))
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier(world)
    ck = ck.stop() if ck else None
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world)
    out = {"ms": ms_max, "value": world * args.steps / (ms_max / 1000.0), "stats": stats,
           "launches": sim.kernel_launches() - l0, "host_syncs": sim.host_syncs() - y0,
           "phases": sim.phase_times(),
           "fstats": {k: sim.factor_stats(i)
                      for i, k in enumerate(("hydro", "thermal", "gravity"))},
           "clocks": ck, "marknum": st.marknum}
    out["factorizations"] = {k: out["fstats"][k].factorizations - f0[k].factorizations
                             for k in f0}
    out["krylov_iterations"] = {k: out["fstats"][k].krylov_iterations -
                                f0[k].krylov_iterations for k in f0}
    sim.close()
    return out


def phase_table(marknum, nodes, phases):
    ab = algorithmic_bytes(marknum, nodes)
    per = {}
    for k, (t, c) in phases.items():
        if c:
            ent = {"ms_total": round(t, 3), "launches": c, "ms_per_launch": t / c}
            if k in ab:
                ent["GBps"] = ab[k] / (t / c / 1000.0) / 1e9
            per[k] = ent
    return per


# DRAM traffic per launch of the dominant kernels, from ncu captures of the
# same kernels (dram__bytes_read.sum + dram__bytes_write.sum), keyed by
# (workload, kernel, factor precision); the profiles/ summaries give the
# commands.  Absent entries are reported as null.
NCU_TRAFFIC = {
    ("planetesimal_141", "k_mf_factor", "fp64"): 5.43e9,
}
# The triangular solve reads every factor tile once, so its traffic grows with
# the factor bytes: captured at 141x141 (k_mf_solve<double>: 0.80 GB against
# 0.79 GB of factors; k_mf_solve<float>: 0.4085 GB against 0.3932 GB), the
# ratio scales the factor bytes of any workload to a per-launch figure.
NCU_SOLVE_TRAFFIC_RATIO = {"fp64": 0.80 / 0.79, "fp32": 0.4085 / 0.3932}


def roofline(args, res, hbm, hbm_src, f64):
    """Roofline of the headline mode's dominant kernel: the Stokes-Darcy
    factorisation (k_mf_factor: FP64 tile flops against the DGEMM peak
    measured in this run) or its triangular solves (k_mf_solve: factor bytes
    read per solve against the measured HBM copy bandwidth), whichever takes
    more device time."""
    per, fh = res["per"], res["fstats"]["hydro"]
    fac = per.get("hydro_factor", {}).get("ms_total", 0.0)
    sol = per.get("hydro_precond", {}).get("ms_total", 0.0)
    prec = "fp64" if args.precision == "fp64" else "fp32"
    if fac >= sol and fac > 0:
        ms = per["hydro_factor"]["ms_per_launch"]
        tf = fh.flops / (ms / 1000.0) / 1e12
        tr = NCU_TRAFFIC.get((args.workload, "k_mf_factor", "fp64"))
        return {"bound": "fp64", "kernel": "k_mf_factor", "phase": "hydro_factor",
                "achieved": tf, "peak": f64, "unit": "TFLOP/s", "frac": tf / f64,
                "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 (torch.matmul)",
                "traffic": tr, "flops_per_launch": fh.flops, "launches": per["hydro_factor"]["launches"],
                "ms_per_launch": ms,
                "note": "FP64 flops of the 64x64 tile algorithm (padding included) per "
                        "factorisation over its event-timed duration"}
    ms = per["hydro_precond"]["ms_per_launch"]
    gbs = fh.solve_bytes / (ms / 1000.0) / 1e9
    tr = NCU_SOLVE_TRAFFIC_RATIO[prec] * fh.solve_bytes
    return {"bound": "hbm", "kernel": "k_mf_solve", "phase": "hydro_precond",
            "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
            "peak_source": hbm_src, "traffic": tr,
            "traffic_source": "ncu capture at 141x141, DRAM bytes / factor bytes "
                              "scaled to this launch's factor bytes",
            "bytes_per_launch": fh.solve_bytes,
            "launches": per["hydro_precond"]["launches"], "ms_per_launch": ms,
            "note": "factor bytes one forward plus backward triangular solve reads (%s "
                    "factors) over its event-timed duration" % prec}


def measure_e2e(pkg, args, mode, world):
    """End to end through the public API: every step, the whole marker and
    grid state is uploaded from pinned host arrays, advanced one timestep and
    copied back (erebus_step_host; part of the copy-back overlaps the
    timestep)."""
    import torch
    st2 = pkg.make_state(args.workload).pinned()
    sim2 = pkg.Simulation(st2)
    sim2.set_solver_options(**MODES[mode])
    # the same timesteps as the device-resident arm: warm-up on the device,
    # then args.steps timesteps through erebus_step_host
    for ts in range(1, args.warmup + 1):
        sim2.step(ts)
    sim2.download()
    h2d = sum(a[: st2.marknum].nbytes for k, a in st2.m.items() if k != "etasolidm_m") + \
        sum(a.nbytes for a in st2.grid.values())
    if st2.p.per_marker_eta:
        h2d += st2.m["etasolidm_m"][: st2.marknum].nbytes
    stream2 = torch.cuda.ExternalStream(sim2.stream_handle())
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ne2e = args.steps
    barrier(world)
    torch.cuda.synchronize()
    e2.record(stream2)
    for ts in range(args.warmup + 1, args.warmup + 1 + ne2e):
        sim2.step_host(ts)
    e3.record(stream2)
    torch.cuda.synchronize()
    ms = max_over_ranks(e2.elapsed_time(e3), world)
    sim2.close()
    return {"value": world * ne2e / (ms / 1000.0), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(h2d), "steps": ne2e,
            "precision": mode}


def run_ours(args):
    rank, world, local = dist_setup(args.gpus)
    pkg = load_pkg()
    head = args.precision
    res = {}
    for mode in (["fp64", head] if head != "fp64" else ["fp64"]):
        res[mode] = time_mode(pkg, args, mode, world, rank, local, clocks=(mode == head))
    e2e = measure_e2e(pkg, args, head, world)
    adj = None if args.no_adjoint else measure_adjoint(pkg, world)
    ens = None if args.no_ensemble else measure_ensemble(pkg, world, rank, 16, 5, 2, 16)
    if rank == 0:
        hbm, src = peaks()
        f64 = fp64_peak()
        nodes = (pkg.CONFIGS[args.workload]["N"] + 1) ** 2
        for mode, r in res.items():
            r["per"] = phase_table(r["marknum"], nodes, r["phases"])
        h = res[head]
        roof = roofline(args, h, hbm, src, f64)
        cpu = None
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(pkg, load_oracle(), args.workload)
        fp = res["fp64"]

        def summary(mode, r):
            return {"value": r["value"], "ms_per_step": r["ms"] / args.steps,
                    "titer_per_step": [s.titer for s in r["stats"]],
                    "factorizations": r["factorizations"],
                    "krylov_iterations": r["krylov_iterations"],
                    "hydro_solves": sum(s.hydro_solves for s in r["stats"]),
                    "worst_rel_residual": max(s.worst_rel_residual for s in r["stats"]),
                    "solver_options": MODES[mode], "phases": r["per"],
                    "gpu_launches": r["launches"],
                    "host_syncs_per_step": r["host_syncs"] / args.steps}
        line = {"metric": METRIC, "value": h["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": h["ms"] / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if head == "fp64" else "f64 (preconditioner factors f32)",
                "data": "synthetic",
                "config": config_dict(pkg, args.workload,
                                      {"parallelism": "replicas x%d" % world,
                                       "precision": head,
                                       "solver_options": MODES[head],
                                       "timesteps": [args.warmup + 1,
                                                     args.warmup + args.steps]}),
                "fp64": summary("fp64", fp),
                "mixed_over_fp64": h["value"] / fp["value"],
                "headline": summary(head, h),
                "roofline": roof, "cpu_baseline": cpu, "clocks": h["clocks"], "e2e": e2e,
                "gpu_launches": h["launches"], "adjoint": adj, "ensemble": ens}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_marker_phases(args):
    """bench.py --marker-phases K: the marker phases alone on the workload's
    initial state (no linear solve, so no factor storage is allocated; a
    small device footprint for profiling), K rounds of markers_to_nodes,
    the reaction, nodes_to_markers and RK4 advection under a synthetic rigid
    rotation of the grid (about one cell per timestep at the box edge, so
    the markers move and are sorted again every round).  Prints per-phase
    device times and algorithmic GB/s."""
    rank, world, local = dist_setup(args.gpus)
    import torch
    pkg = load_pkg()
    st = pkg.make_state(args.workload)
    g, p = st.g, st.p
    dt = p.dt_longest
    om = g.dx / (0.5 * p.xsize) / dt
    ny1, nx1 = g.Ny1, g.Nx1
    xs_vx = np.arange(nx1) * g.dx
    ys_vx = -g.dy / 2 + np.arange(ny1) * g.dy
    xs_vy = -g.dx / 2 + np.arange(nx1) * g.dx
    ys_vy = np.arange(ny1) * g.dy
    st.grid["vx"][...] = -om * (ys_vx[:, None] - g.ycenter) + 0 * xs_vx[None, :]
    st.grid["vy"][...] = om * (xs_vy[None, :] - g.xcenter) + 0 * ys_vy[:, None]
    st.grid["vxf"][...] = st.grid["vx"]
    st.grid["vyf"][...] = st.grid["vy"]
    st.grid["tk2"][...] = p.tkm0[0]
    sim = pkg.Simulation(st)
    sim.enable_phase_timing(True)
    torch.cuda.synchronize()
    for k in range(args.marker_phases):
        ts = 2 + k
        sim.markers_to_nodes(st.timesum)
        sim.thermochemical_reaction(dt, ts, 1)
        sim.nodes_to_markers(dt, ts)
        sim.advect_rk4(dt)
    torch.cuda.synchronize()
    ph = sim.phase_times()
    sim.close()
    if rank == 0:
        per = phase_table(st.marknum, g.Nx1 * g.Ny1, ph)
        print(json.dumps({"workload": args.workload, "markers": st.marknum,
                          "rounds": args.marker_phases, "phases": per}), flush=True)
    return 0


def run_ensemble(args):
    """bench.py --workload ensemble: the ensemble line alone (default 256
    bodies, 20 timed timesteps each after 3 untimed ones, 32 bodies at a
    time)."""
    rank, world, local = dist_setup(args.gpus)
    pkg = load_pkg()
    clocks = Clocks(local) if rank == 0 else None
    line = measure_ensemble(pkg, world, rank, args.bodies, args.steps or 20, args.warmup,
                            args.wave)
    ck = clocks.stop() if clocks else None
    if rank == 0:
        line.update({"n_gpus": world, "higher_is_better": True, "scaling": "weak",
                     "vs_baseline": None, "dtype": "f64", "data": "synthetic", "clocks": ck})
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 20; ensemble workload: 20 per body)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint gradients/s measurement")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the 16-body ensemble measurement")
    ap.add_argument("--bodies", type=int, default=256,
                    help="ensemble workload: number of planetesimals")
    ap.add_argument("--wave", type=int, default=32,
                    help="ensemble workload: bodies resident at a time")
    ap.add_argument("--workload", default=WORKLOAD,
                    choices=["planetesimal_41", "planetesimal_141", "planetesimal_401",
                             "ensemble"])
    ap.add_argument("--precision", default="mixed", choices=sorted(MODES),
                    help="headline path: mixed (FGMRES with lagged FP32-applied LU "
                         "preconditioner), fp64 (direct LU + FP64 refinement), or "
                         "fp32-factors (FP32 factorisation + FP64 refinement); the FP64 "
                         "path is always timed beside it")
    ap.add_argument("--refactor-iterations", type=int, default=None,
                    help="Krylov modes: refresh the factors after a solve that took more "
                         "iterations than this")
    ap.add_argument("--marker-phases", type=int, default=0,
                    help="run only the marker phases this many times (profiling)")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the multifrontal analysis parameters for the workload by "
                         "timing (erebus_b200.autotune); prints the trials as JSON")
    args = ap.parse_args()
    if args.marker_phases:
        return run_marker_phases(args)
    if args.autotune:
        load_pkg()
        from erebus_b200 import autotune
        prec = "mixed" if args.precision == "mixed" else "fp64"
        return autotune.main(["--workload", args.workload, "--precision", prec])
    if args.refactor_iterations is not None:
        for m in MODES.values():
            if m.get("krylov"):
                m["refactor_iterations"] = args.refactor_iterations
    if args.impl == "reference" and args.workload == "ensemble":
        print(json.dumps({"impl": "reference", "unavailable": "the ensemble workload is "
                          "timed on the GPU only; the CPU oracle takes ~10 s per 141x141 "
                          "timestep, so its arm runs the single-body workloads"}))
        return 0
    if args.workload == "ensemble":
        return run_ensemble(args)
    args.steps = args.steps or 20
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
