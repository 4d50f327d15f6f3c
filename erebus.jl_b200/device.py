"""ctypes binding of liberebus_b200.so and the device-side simulation.

`Simulation` owns one device state.  Its methods are the per-phase drop-ins
of the reference's timestep (simulation_loop, src/Erebus.jl:6370-7235) and
`step`, which runs a whole timestep.  Every call goes through the C ABI of
include/erebus_b200.h; a non-zero status raises `ErebusError`.  There is no
CPU path: without the library or a CUDA device the constructor raises.
"""
import ctypes
import os

import numpy as np

from .abi import (STATUS_NAMES, ErebusAdjointStats, ErebusFactorStats, ErebusGridHost,
                  ErebusMarkersHost,
                  ErebusParams, ErebusSolverOptions, ErebusSolveStats, ErebusStepStats,
                  ErebusSumsHost)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liberebus_b200.so")

EXPORTS = [
    "erebus_default_params", "erebus_default_solver_options", "erebus_check_params",
    "erebus_create", "erebus_destroy", "erebus_set_solver_options", "erebus_last_error",
    "erebus_grid_layout",
    "erebus_upload_markers", "erebus_download_markers", "erebus_upload_grid",
    "erebus_download_grid", "erebus_download_sums", "erebus_set_time", "erebus_get_time",
    "erebus_markers_to_nodes", "erebus_gravity", "erebus_thermochemical_reaction",
    "erebus_hydromech_pass", "erebus_thermal_solve", "erebus_nodes_to_markers",
    "erebus_advect_rk4", "erebus_replenish", "erebus_step", "erebus_export_hydromech",
    "erebus_apply_hydromech", "erebus_kernel_launches", "erebus_host_syncs",
    "erebus_factor_stats",
    "erebus_snapshot_begin", "erebus_snapshot_wait", "erebus_adjoint_heat",
    "erebus_step_host", "erebus_share_solver_stream",
]


class ErebusError(RuntimeError):
    def __init__(self, fn, code, msg=""):
        super().__init__("%s failed: %s (%d) %s" % (fn, STATUS_NAMES.get(code, "?"), code, msg))
        self.code = code


_lib = None


def load_library(path=LIB_PATH):
    """Loads liberebus_b200.so (raises OSError when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError("liberebus_b200.so not built: run erebus.jl_b200/build.py")
    L = ctypes.CDLL(path)
    P, I, I32, I64, D = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int32, ctypes.c_int64,
                         ctypes.c_double)
    PP = ctypes.POINTER(ctypes.c_void_p)
    pI64 = ctypes.POINTER(ctypes.c_int64)
    pD = ctypes.POINTER(ctypes.c_double)
    pI32 = ctypes.POINTER(ctypes.c_int32)
    sigs = {
        "erebus_default_params": [ctypes.POINTER(ErebusParams), I32, I32],
        "erebus_default_solver_options": [ctypes.POINTER(ErebusSolverOptions)],
        "erebus_check_params": [ctypes.POINTER(ErebusParams)],
        "erebus_create": [ctypes.POINTER(ErebusParams), I64, PP],
        "erebus_grid_layout": [ctypes.POINTER(ErebusParams), pI64, pI64],
        "erebus_share_solver_stream": [P, I32],
        "erebus_destroy": [P],
        "erebus_set_solver_options": [P, ctypes.POINTER(ErebusSolverOptions)],
        "erebus_factor_stats": [P, I32, ctypes.POINTER(ErebusFactorStats)],
        "erebus_upload_markers": [P, ctypes.POINTER(ErebusMarkersHost), I64],
        "erebus_download_markers": [P, ctypes.POINTER(ErebusMarkersHost), pI64],
        "erebus_upload_grid": [P, ctypes.POINTER(ErebusGridHost)],
        "erebus_download_grid": [P, ctypes.POINTER(ErebusGridHost)],
        "erebus_download_sums": [P, ctypes.POINTER(ErebusSumsHost)],
        "erebus_snapshot_begin": [P, ctypes.POINTER(ErebusGridHost),
                                  ctypes.POINTER(ErebusMarkersHost)],
        "erebus_snapshot_wait": [P, pI64, pD, pD],
        "erebus_adjoint_heat": [P, I32, I32, I32, pD, pD, pD,
                                ctypes.POINTER(ErebusAdjointStats)],
        "erebus_step_host": [P, I32, ctypes.POINTER(ErebusMarkersHost), I64,
                             ctypes.POINTER(ErebusGridHost), ctypes.POINTER(ErebusMarkersHost),
                             pI64, ctypes.POINTER(ErebusGridHost),
                             ctypes.POINTER(ErebusStepStats)],
        "erebus_set_time": [P, D, D],
        "erebus_get_time": [P, pD, pD],
        "erebus_markers_to_nodes": [P, D],
        "erebus_gravity": [P, ctypes.POINTER(ErebusSolveStats)],
        "erebus_thermochemical_reaction": [P, D, I32, I32],
        "erebus_hydromech_pass": [P, pD, I32, pI32, ctypes.POINTER(ErebusSolveStats)],
        "erebus_thermal_solve": [P, D, I32, pD, ctypes.POINTER(ErebusSolveStats)],
        "erebus_nodes_to_markers": [P, D, I32],
        "erebus_advect_rk4": [P, D],
        "erebus_replenish": [P, I32, pI64],
        "erebus_step": [P, I32, ctypes.POINTER(ErebusStepStats)],
        "erebus_export_hydromech": [P, D, pI64, P, P, P, P],
        "erebus_apply_hydromech": [P, D, P, P],
        "erebus_kernel_launches": [P, pI64],
        "erebus_host_syncs": [P, pI64],
        "erebus_get_stream": [P, PP],
        "erebus_enable_phase_timing": [P, I32],
        "erebus_phase_times": [P, pD, pI64, I32],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = I
    L.erebus_last_error.argtypes = [P]
    L.erebus_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


class Simulation:
    """One planetesimal resident on the GPU.

    `host` is a HostState (erebus_b200.host) whose arrays are uploaded at
    construction and refreshed by `download()`.  Timestep counters and dt /
    timesum are those of simulation_loop."""

    def __init__(self, host, capacity=None):
        self.L = load_library()
        self.host = host
        self.p = host.p
        cap = int(capacity or host.capacity)
        self.capacity = cap
        h = ctypes.c_void_p()
        self._check("erebus_create", self.L.erebus_create(ctypes.byref(self.p), cap,
                                                          ctypes.byref(h)), None)
        self.h = h
        self.upload()

    def _check(self, fn, rc, h="self"):
        if rc != 0:
            msg = ""
            if h == "self" and getattr(self, "h", None):
                msg = (self.L.erebus_last_error(self.h) or b"").decode()
            raise ErebusError(fn, rc, msg)

    def close(self):
        if getattr(self, "h", None):
            self.L.erebus_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- data movement ----------------------------------------------------------
    def upload(self):
        st = self.host
        self._check("erebus_upload_markers", self.L.erebus_upload_markers(
            self.h, ctypes.byref(st.markers_struct()), st.marknum))
        self._check("erebus_upload_grid", self.L.erebus_upload_grid(
            self.h, ctypes.byref(st.grid_struct())))
        self._check("erebus_set_time", self.L.erebus_set_time(self.h, st.dt, st.timesum))

    def download(self):
        """Copies markers, grid and dt/timesum back into the HostState."""
        st = self.host
        n = ctypes.c_int64()
        self._check("erebus_download_markers", self.L.erebus_download_markers(
            self.h, ctypes.byref(st.markers_struct()), ctypes.byref(n)))
        st.marknum = n.value
        self._check("erebus_download_grid", self.L.erebus_download_grid(
            self.h, ctypes.byref(st.grid_struct())))
        dt, ts = ctypes.c_double(), ctypes.c_double()
        self._check("erebus_get_time", self.L.erebus_get_time(self.h, ctypes.byref(dt),
                                                              ctypes.byref(ts)))
        st.dt, st.timesum = dt.value, ts.value
        return st

    def download_sums(self):
        st = self.host
        self._check("erebus_download_sums", self.L.erebus_download_sums(
            self.h, ctypes.byref(st.sums_struct())))
        return st.sums

    def snapshot_begin(self, buffers):
        """Starts an asynchronous copy of the state (markers, grid, marknum,
        dt, timesum) into `buffers`, a HostState of the same geometry, and
        returns at once; steps may follow while the copy runs.  Buffers made
        with HostState(..., pinned=True) let the copy overlap the steps.
        The snapshot is the input of save_state (E:5718-5960)."""
        self._check("erebus_snapshot_begin", self.L.erebus_snapshot_begin(
            self.h, ctypes.byref(buffers.grid_struct()),
            ctypes.byref(buffers.markers_struct())))
        self._snapshot = buffers

    def snapshot_wait(self):
        """Waits for the copy started by `snapshot_begin`; returns its buffers
        with marknum, dt and timesum as they were when it began."""
        n, dt, ts = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        self._check("erebus_snapshot_wait", self.L.erebus_snapshot_wait(
            self.h, ctypes.byref(n), ctypes.byref(dt), ctypes.byref(ts)))
        b, self._snapshot = self._snapshot, None
        b.marknum, b.dt, b.timesum = n.value, dt.value, ts.value
        return b

    def share_solver_stream(self, on=True):
        """Queue this state's grid-synchronised solver kernels on the stream
        shared by all states that opted in (erebus_share_solver_stream), for
        states stepped concurrently from several threads."""
        self._check("erebus_share_solver_stream",
                    self.L.erebus_share_solver_stream(self.h, 1 if on else 0))

    def set_solver_options(self, **kw):
        o = ErebusSolverOptions()
        self.L.erebus_default_solver_options(ctypes.byref(o))
        for k, v in kw.items():
            setattr(o, k, v)
        self._check("erebus_set_solver_options",
                    self.L.erebus_set_solver_options(self.h, ctypes.byref(o)))

    # -- phases (reference function groups) ----------------------------------
    def markers_to_nodes(self, timesum):
        """E:6376-6604 (compute_marker_properties!, marker_to_*_nodes!,
        compute_*_node_properties!, insulating boundary on tk1)."""
        self._check("erebus_markers_to_nodes", self.L.erebus_markers_to_nodes(self.h, timesum))

    def gravity(self):
        """E:6610-6614 (assemble_gravitational_lse!, solve,
        process_gravitational_solution!)."""
        s = ErebusSolveStats()
        self._check("erebus_gravity", self.L.erebus_gravity(self.h, ctypes.byref(s)))
        return s

    def thermochemical_reaction(self, dt, timestep, titer):
        """perform_thermochemical_reaction! (E:2558-2694)."""
        self._check("erebus_thermochemical_reaction",
                    self.L.erebus_thermochemical_reaction(self.h, dt, timestep, titer))

    def hydromech_pass(self, dt, iplast):
        """One plastic pass (E:6678-6869); returns (dt, converged, stats)."""
        d = ctypes.c_double(dt)
        conv = ctypes.c_int32(0)
        s = ErebusSolveStats()
        self._check("erebus_hydromech_pass", self.L.erebus_hydromech_pass(
            self.h, ctypes.byref(d), iplast, ctypes.byref(conv), ctypes.byref(s)))
        return d.value, bool(conv.value), s

    def thermal_solve(self, dt, timestep):
        """E:6887-6927; returns (max|DT|, stats)."""
        m = ctypes.c_double()
        s = ErebusSolveStats()
        self._check("erebus_thermal_solve", self.L.erebus_thermal_solve(
            self.h, dt, timestep, ctypes.byref(m), ctypes.byref(s)))
        return m.value, s

    def nodes_to_markers(self, dt, timestep):
        """E:6945-7019 (marker viscosity, stress, temperature, porosity,
        melt composition)."""
        self._check("erebus_nodes_to_markers",
                    self.L.erebus_nodes_to_markers(self.h, dt, timestep))

    def advect_rk4(self, dt):
        """E:7026-7059 (velocities, rotation, move_markers_rk4!,
        backtrace_pressures_rk4!)."""
        self._check("erebus_advect_rk4", self.L.erebus_advect_rk4(self.h, dt))

    def replenish(self, timestep):
        """replenish_markers! (E:5586-5698); returns the new marker count."""
        n = ctypes.c_int64()
        self._check("erebus_replenish", self.L.erebus_replenish(self.h, timestep,
                                                                ctypes.byref(n)))
        self.host.marknum = n.value
        return n.value

    def step(self, timestep):
        """One whole timestep (E:6370-7235); returns ErebusStepStats."""
        s = ErebusStepStats()
        self._check("erebus_step", self.L.erebus_step(self.h, timestep, ctypes.byref(s)))
        return s

    def step_host(self, timestep):
        """One timestep on the HostState's arrays (erebus_step_host): they
        are uploaded, advanced and copied back in one call; returns
        ErebusStepStats and updates marknum, dt and timesum of the host."""
        h = self.host
        # the ctypes views are rebuilt only when an array object changed
        key = tuple(id(a) for a in h.m.values()) + tuple(id(a) for a in h.grid.values())
        if getattr(self, "_views_key", None) != key:
            self._views = (h.markers_struct(), h.grid_struct())
            self._views_key = key
        ms, gs = self._views
        n = ctypes.c_int64()
        s = ErebusStepStats()
        self._check("erebus_step_host", self.L.erebus_step_host(
            self.h, timestep, ctypes.byref(ms), h.marknum, ctypes.byref(gs), ctypes.byref(ms),
            ctypes.byref(n), ctypes.byref(gs), ctypes.byref(s)))
        h.marknum = n.value
        h.dt, h.timesum = s.dt, s.timesum
        return s

    def adjoint_heat(self, n_steps, checkpoint_every=5, first_timestep=1):
        """Runs n_steps timesteps and returns (J, dJ/dphim, dJ/dratio_al,
        ErebusAdjointStats): J is the mean of the 4-P-node average of tk2
        over the basic nodes inside the body after the last step; the
        gradients come from the reverse sweep of erebus_adjoint_heat (states
        at mechanical rest only; see include/erebus_b200.h)."""
        J, dr = ctypes.c_double(), ctypes.c_double()
        st = ErebusAdjointStats()
        g = np.zeros(self.capacity)
        self._check("erebus_adjoint_heat", self.L.erebus_adjoint_heat(
            self.h, first_timestep, n_steps, checkpoint_every, ctypes.byref(J),
            g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(dr),
            ctypes.byref(st)))
        return J.value, g[: st.markers].copy(), dr.value, st

    def export_hydromech(self, dt):
        """The assembled Stokes-Darcy system as COO (rows, cols, vals) and R."""
        nnz = ctypes.c_int64()
        self._check("erebus_export_hydromech", self.L.erebus_export_hydromech(
            self.h, dt, ctypes.byref(nnz), None, None, None, None))
        n = nnz.value
        rows = np.zeros(n, np.int64)
        cols = np.zeros(n, np.int64)
        vals = np.zeros(n)
        R = np.zeros(6 * self.host.g.Nx1 * self.host.g.Ny1)
        self._check("erebus_export_hydromech", self.L.erebus_export_hydromech(
            self.h, dt, ctypes.byref(nnz), rows.ctypes.data, cols.ctypes.data,
            vals.ctypes.data, R.ctypes.data))
        return rows, cols, vals, R

    def factor_stats(self, system):
        """ErebusFactorStats of system 0 (Stokes-Darcy), 1 (heat) or 2 (gravity)."""
        o = ErebusFactorStats()
        self._check("erebus_factor_stats",
                    self.L.erebus_factor_stats(self.h, system, ctypes.byref(o)))
        return o

    def kernel_launches(self):
        n = ctypes.c_int64()
        self._check("erebus_kernel_launches",
                    self.L.erebus_kernel_launches(self.h, ctypes.byref(n)))
        return n.value

    def host_syncs(self):
        """Host waits on this state's streams since creation."""
        n = ctypes.c_int64()
        self._check("erebus_host_syncs", self.L.erebus_host_syncs(self.h, ctypes.byref(n)))
        return n.value

    PHASES = ["markers_to_nodes", "gravity", "reaction", "hydro_assemble", "hydro_factor",
              "hydro_solve", "hydro_post", "thermal_assemble", "thermal_factor",
              "thermal_solve", "nodes_to_markers", "rk4", "backtrace", "replenish",
              "scatter_merge", "hydro_precond"]

    def enable_phase_timing(self, on=True):
        self._check("erebus_enable_phase_timing",
                    self.L.erebus_enable_phase_timing(self.h, 1 if on else 0))

    def phase_times(self):
        """{phase: (total ms, launches)} from the device event timer."""
        n = len(self.PHASES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int64 * n)()
        self._check("erebus_phase_times", self.L.erebus_phase_times(self.h, ms, cnt, n))
        return {k: (ms[i], cnt[i]) for i, k in enumerate(self.PHASES)}

    def stream_handle(self):
        """The cudaStream_t (as an int) this state's work runs on."""
        v = ctypes.c_void_p()
        self._check("erebus_get_stream", self.L.erebus_get_stream(self.h, ctypes.byref(v)))
        return v.value or 0


def run_simulation(host, n_steps, start_step=1, callback=None, output_path=None,
                   savematstep=10):
    """The reference's simulation_loop over `n_steps` timesteps on the GPU.
    Returns the list of ErebusStepStats.

    With `output_path`, the state after every timestep divisible by
    `savematstep` is written as output_<timestep>.npz (save_state,
    E:7106-7235): the snapshot is copied out on a second stream while the
    next timestep runs, and a writer thread saves it."""
    from concurrent.futures import ThreadPoolExecutor

    from .host import HostState
    from .output import save_state

    sim = Simulation(host)
    out = []
    pool = ThreadPoolExecutor(max_workers=1) if output_path is not None else None
    buffers, pending, written = None, None, None
    try:
        for ts in range(start_step, start_step + n_steps):
            s = sim.step(ts)
            out.append(s)
            if pending is not None:
                written = pool.submit(save_state, output_path, pending, sim.snapshot_wait())
                pending = None
            if callback:
                callback(ts, s)
            if output_path is not None and ts % savematstep == 0:
                if written is not None:
                    written.result()
                if buffers is None:
                    buffers = HostState(host.p, host.capacity, pinned=True)
                sim.snapshot_begin(buffers)
                pending = ts
            if s.timesum > host.p.endtime:
                break
        if pending is not None:
            written = pool.submit(save_state, output_path, pending, sim.snapshot_wait())
        if written is not None:
            written.result()
        sim.download()
    finally:
        if pool is not None:
            pool.shutdown()
        sim.close()
    return out
