"""Autotuner of the multifrontal solver's analysis parameters.

The nested-dissection leaf sizes and the thresholds that decide, per tree
level, whether a CTA takes a whole front or the front's tiles are dealt to
all CTAs (ErebusSolverOptions.mf_leaf_vector, mf_leaf_scalar,
mf_local_factor_ops, mf_local_solve_tiles) trade tree depth against tile work and the fixed cost
of cooperative phases; the best values depend on the grid size.  `tune`
picks them by timing whole timesteps on the device (coordinate descent over
candidate values, each trial from the same initial state), and `main` runs
it from the command line:

    python bench.py --autotune --workload planetesimal_401 [--precision fp64]

(the package directory is erebus.jl_b200, which is not an importable module
name; bench.py loads it as erebus_b200 and calls `main`).
"""
import argparse
import json
import sys
import time

CANDIDATES = {
    "mf_leaf_vector": [16, 24, 32, 48],
    "mf_leaf_scalar": [32, 64, 128, 256],
    "mf_local_factor_ops": [4, 8, 16, 32],
    "mf_local_solve_tiles": [12, 24, 48, 64, 96, 128],
}
DEFAULTS = {"mf_leaf_vector": 32, "mf_leaf_scalar": 64, "mf_local_factor_ops": 8,
            "mf_local_solve_tiles": 64}


def time_config(make_state, opts, steps, warmup):
    """Device milliseconds per timestep of `steps` timesteps after `warmup`
    untimed ones, from a fresh state (CUDA events on the library's stream)."""
    import torch
    from .device import Simulation
    st = make_state()
    sim = Simulation(st)
    try:
        sim.set_solver_options(**opts)
        for ts in range(1, warmup + 1):
            sim.step(ts)
        stream = torch.cuda.ExternalStream(sim.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for ts in range(warmup + 1, warmup + steps + 1):
            sim.step(ts)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps
    finally:
        sim.close()


def tune(make_state, base_opts=None, steps=4, warmup=3, candidates=None, log=print):
    """Coordinate descent over `candidates` (default CANDIDATES), one
    parameter at a time, keeping the fastest value.  Returns (best options,
    list of (options, ms per timestep) trials)."""
    candidates = candidates or CANDIDATES
    best = dict(DEFAULTS)
    base = dict(base_opts or {})
    trials = []
    best_ms = time_config(make_state, {**base, **best}, steps, warmup)
    trials.append((dict(best), best_ms))
    measured = {tuple(sorted(best.items())): best_ms}
    log("start %s: %.3f ms/timestep" % (best, best_ms))
    for name, values in candidates.items():
        for v in values:
            trial = dict(best, **{name: v})
            if tuple(sorted(trial.items())) in measured:   # e.g. the value in force
                continue
            ms = time_config(make_state, {**base, **trial}, steps, warmup)
            measured[tuple(sorted(trial.items()))] = ms
            trials.append((trial, ms))
            log("%s=%d: %.3f ms/timestep" % (name, v, ms))
            if ms < best_ms:
                best, best_ms = trial, ms
    log("best %s: %.3f ms/timestep" % (best, best_ms))
    return best, trials


def main(argv=None):
    from .host import make_state
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="planetesimal_141")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args(argv)
    base = {"krylov": 1, "precond_fp32": 1} if args.precision == "mixed" else {}
    t0 = time.time()
    best, trials = tune(lambda: make_state(args.workload), base, args.steps, args.warmup,
                        log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps({"workload": args.workload, "precision": args.precision,
                      "best": best, "seconds": time.time() - t0,
                      "trials": [{"options": o, "ms_per_timestep": ms} for o, ms in trials]}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
