"""Ensembles of planetesimals of uneven sizes advanced together on one GPU.

Every body is its own device state (a Simulation) stepped by its own host
thread, so the bodies' kernels run on their own CUDA streams and overlap on
the GPU.  The grid-synchronised solver kernels (the multifrontal
factorisations and solves, whose CTAs wait for one another) of all bodies go
to one shared stream (erebus_share_solver_stream), so that two of them are
never in flight together; everything else of different bodies runs
concurrently.  Bodies are independent: the results are those of each body
stepped alone.

This is the ensemble's first form.  The packed work list of all bodies in one
persistent launch per phase is not built.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .device import Simulation
from .host import HostState, define_markers, u01
from .params import config_params


def ensemble_params(n_bodies, seed=42, side_min=61, side_max=201, first=0):
    """Parameters of a synthetic ensemble, one ErebusParams per body.

    Radius U(20, 100) km; grid side linear in the radius from side_min (20 km)
    to side_max (100 km), odd; square box of 2.8 radii (the 140 km / 50 km
    ratio of the single-body workloads); crust from 0.96 radii; 4 x 4 markers
    per cell.  Per body: rock porosity U(0.05, 0.3), 26Al/27Al U(1e-5, 5e-5)
    and rock viscosity log-uniform in 1e18-1e21 Pa s.  The variates come
    from the counter-based generator u01 with the given seed; `first` is the
    index of the first body (for ensembles built in waves).  Other constants
    are those of the single-body workloads."""
    out = []
    for b in range(first, first + n_bodies):
        u = [float(u01(seed, 300 + k, np.uint64(b))) for k in range(4)]
        r = 20e3 + 80e3 * u[0]
        side = int(round(side_min + (r - 20e3) / 80e3 * (side_max - side_min)))
        side += 1 - side % 2
        p = config_params("planetesimal_41")
        p.Nx = p.Ny = side
        p.xsize = p.ysize = 2.8 * r
        p.rplanet, p.rcrust = r, 0.96 * r
        p.ratio_al = 1e-5 + 4e-5 * u[1]
        eta = 10.0 ** (18.0 + 3.0 * u[2])
        p.etasolidm[0] = p.etasolidm[1] = eta
        p.etasolidmm[0] = p.etasolidmm[1] = eta
        p.per_marker_eta = 0
        p.seed = seed + b
        out.append((p, 0.05 + 0.25 * u[3], eta))
    return out


def ensemble_states(n_bodies, seed=42, **kw):
    """HostStates of the synthetic ensemble with their initial markers."""
    states = []
    for p, phi, eta in ensemble_params(n_bodies, seed=seed, **kw):
        st = HostState(p)
        states.append(define_markers(st, ("const", phi), ("const", eta)))
    return states


class Ensemble:
    """Bodies stepped concurrently, one host thread and one stream each."""

    def __init__(self, states):
        self.sims = []
        try:
            for st in states:
                sim = Simulation(st)
                sim.share_solver_stream(True)
                self.sims.append(sim)
        except Exception:
            self.close()
            raise

    def run(self, n_steps, start_step=1, workers=None):
        """Advances every body by n_steps timesteps; returns the per-body lists
        of ErebusStepStats."""
        def body(k):
            sim = self.sims[k]
            return [sim.step(ts) for ts in range(start_step, start_step + n_steps)]

        with ThreadPoolExecutor(max_workers=workers or len(self.sims)) as ex:
            return list(ex.map(body, range(len(self.sims))))

    def download(self):
        for sim in self.sims:
            sim.download()

    def streams(self):
        return [sim.stream_handle() for sim in self.sims]

    def close(self):
        for sim in self.sims:
            sim.close()
        self.sims = []
