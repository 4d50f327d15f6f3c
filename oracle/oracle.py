"""CPU oracle driver for the Erebus.jl timestep hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline, never by the product.

`Oracle.step` runs one timestep of simulation_loop (src/Erebus.jl:6370-7235)
over a HostState: the marker and stencil phases run in the C restatement
(erebus_oracle.c, built into liboracle.so next to this file) and the three
linear systems, assembled there in CSC form exactly as the reference
assembles them, are solved with SuperLU (scipy.sparse.linalg.splu) in place
of UMFPACK, which is not available here.  Parity of this restatement is
pinned to re-expressions of the reference's own unit tests
(test/runtests.jl); Julia cannot run here, so no output of the reference
itself is available.
"""
import ctypes
import importlib.util
import os
import subprocess
import sys
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liboracle.so")


def load_package():
    """The erebus.jl_b200 package (its directory name is not an identifier)."""
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


def build(force=False):
    src = os.path.join(HERE, "erebus_oracle.c")
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= os.path.getmtime(src)):
        return LIB
    subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        P, I64, D, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
        sig = {
            "oracle_markers_to_nodes": (I, [P, P, I64, P, P, D]),
            "oracle_thermochemical_reaction": (I, [P, P, I64, P, P, D, I, I]),
            "oracle_assemble_gravity": (I64, [P, P, P, P, P, P]),
            "oracle_process_gravity": (I, [P, P, P]),
            "oracle_bulk_viscosity": (I, [P, P]),
            "oracle_assemble_hydromech": (I64, [P, P, D, P, P, P, P]),
            "oracle_process_hydromech": (I, [P, P, P]),
            "oracle_compute_aphi": (D, [P, P, D]),
            "oracle_fluid_velocities": (I, [P, P]),
            "oracle_displacement_timestep": (D, [P, P, D, D]),
            "oracle_stress_strainrate": (I, [P, P, D]),
            "oracle_symmetrize": (I, [P, P]),
            "oracle_nodal_adjustment": (I, [P, P, D, I, P, P]),
            "oracle_finalize_plastic": (D, [P, P, D, I]),
            "oracle_shear_heating": (I, [P, P]),
            "oracle_adiabatic_heating": (I, [P, P]),
            "oracle_assemble_thermal": (I64, [P, P, D, P, P, P, P]),
            "oracle_nodes_to_markers": (I, [P, P, I64, P, P, D, I]),
            "oracle_velocities": (I, [P, P]),
            "oracle_rotation_rate": (I, [P, P]),
            "oracle_move_markers_rk4": (I, [P, P, I64, P, D]),
            "oracle_backtrace_pressures": (I, [P, P, D]),
            "oracle_replenish": (I64, [P, P, I64, I64, P, P, I]),
            "oracle_u01": (D, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
            # pointwise hooks for the re-expressed reference unit tests
            "oracle_fix_grid": (None, [P, I, D, D, P, P]),
            "oracle_weights_grid": (None, [P, I, D, D, P, P, P]),
            "oracle_ktotal": (D, [D, D, D]),
            "oracle_total": (D, [D, D, D]),
            "oracle_etaf_inv_kphi": (D, [P, D, D, D]),
            "oracle_Q_radiogenic": (D, [D, D, D, D, D]),
            "oracle_radioactive_heating": (None, [P, D, P, P]),
            "oracle_dtreaction": (D, [P, D, D]),
            "oracle_rhocpfluid": (D, [P, D]),
            "oracle_ksolid": (D, [P, D]),
            "oracle_kfluid": (D, [P, D]),
            "oracle_gibbs": (D, [P, D, D, D, D, D, D]),
            "oracle_rel_enthalpy": (D, [P, D, D]),
            "oracle_reaction_constant": (D, [P, D, D, D]),
            "oracle_scatter_only": (None, [P, P, I64, P]),
            "oracle_node_properties": (None, [P, P, P]),
            "oracle_insulating_bc": (None, [P, P]),
            "oracle_subgrid_stress": (I, [P, P, I64, P, P, D]),
            "oracle_subgrid_temperature": (I, [P, P, I64, P, P, D]),
            "oracle_thermodynamic_xfer": (None, [P, P, P]),
            "oracle_melt_composition": (None, [P, P, I64, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def _p(x):
    return ctypes.cast(ctypes.pointer(x), ctypes.c_void_p)


def _a(arr):
    return arr.ctypes.data_as(ctypes.c_void_p)


def finalize_thermochemical_iteration_pass(p, maxDT, dt, titer):
    """finalize_thermochemical_iteration_pass (E:4187-4197): at the first
    thermochemical iteration, dt shrinks so that the largest temperature
    change is DTmax."""
    if titer == 1 and maxDT > p.DTmax:
        dt *= p.DTmax * (1.0 / maxDT)
    return dt


def thermochemical_iteration_outcome(p, DMP, pf, pf0, titer):
    """compute_thermochemical_iteration_outcome (E:4216-4223): the
    iteration stops once the fluid pressure changed by less than pferrmax
    and either two iterations were taken or no marker reacted."""
    pferr = float(np.max(np.abs(pf - pf0)))
    dmpmax = float(np.max(np.abs(DMP)))
    return pferr < p.pferrmax and (titer > 2 or dmpmax <= 0.0)


class Oracle:
    """One planetesimal advanced by the CPU restatement.

    The HostState passed in is updated in place.  `timers` accumulates wall
    time per phase."""

    def __init__(self, st):
        self.st = st
        self.L = lib()
        g = st.g
        self.np = g.Nx1 * g.Ny1
        n6 = 6 * self.np
        self.coo_h = (np.zeros(12 * n6, np.int64), np.zeros(12 * n6, np.int64),
                      np.zeros(12 * n6, np.float64))
        self.coo_t = (np.zeros(6 * self.np, np.int64), np.zeros(6 * self.np, np.int64),
                      np.zeros(6 * self.np, np.float64))
        self.R = np.zeros(n6)
        self.RT = np.zeros(self.np)
        self.RP = np.zeros(self.np)
        self.mdis = np.zeros(g.Nxm * g.Nym)
        self.mnum = np.zeros(g.Nxm * g.Nym, np.int64)
        self.YERRNOD = np.zeros(1)
        self.timers = {}
        self._refresh()

    def _refresh(self):
        st = self.st
        self.P = st.p
        self.M = st.markers_struct()
        self.G = st.grid_struct()
        self.S = st.sums_struct()
        self.pP, self.pM, self.pG, self.pS = _p(self.P), _p(self.M), _p(self.G), _p(self.S)

    def _t(self, key, t0):
        self.timers[key] = self.timers.get(key, 0.0) + time.perf_counter() - t0

    # -- systems -------------------------------------------------------------
    def _csc(self, n, coo, dim):
        r, c, v = coo
        return sp.csc_matrix((v[:n], (r[:n], c[:n])), shape=(dim, dim))

    def gravity_system(self):
        n = self.L.oracle_assemble_gravity(self.pP, self.pG, _a(self.coo_t[0]),
                                           _a(self.coo_t[1]), _a(self.coo_t[2]),
                                           _a(self.RP))
        return self._csc(n, self.coo_t, self.np), self.RP.copy()

    def hydromech_system(self, dt):
        n = self.L.oracle_assemble_hydromech(self.pP, self.pG, dt, _a(self.coo_h[0]),
                                             _a(self.coo_h[1]), _a(self.coo_h[2]),
                                             _a(self.R))
        return self._csc(n, self.coo_h, 6 * self.np), self.R.copy()

    def thermal_system(self, dt):
        n = self.L.oracle_assemble_thermal(self.pP, self.pG, dt, _a(self.coo_t[0]),
                                           _a(self.coo_t[1]), _a(self.coo_t[2]),
                                           _a(self.RT))
        return self._csc(n, self.coo_t, self.np), self.RT.copy()

    def solve(self, A, b):
        """Direct solve with the rows scaled by their absolute sums first.

        This is the default row scaling of UMFPACK (UMFPACK_SCALE_SUM), the
        solver the reference reaches through LinearSolve / `\\` (E:6612,
        E:6736-6748, E:6925).  Without it the Stokes-Darcy pressures at
        sticky-air nodes, whose rows carry coefficients ~1e-1 next to Darcy
        rows of ~1e23, are only determined to ~1e7 Pa by a backward-stable
        solve and differ between orderings.

        UMFPACK itself is not available; SuperLU (scipy.sparse.linalg.splu,
        partial pivoting) stands in for it.  Its fill-reducing ordering is a
        nested dissection of the node grid (recursive bisection of the node
        rectangle by one-node-wide separators, all unknowns of a node kept
        together), applied as a symmetric permutation with SuperLU's own
        column ordering off: on these 2-D 9-point couplings it gives less
        fill than COLAMD (48-58M against 73M factor entries at 201 x 201) and
        halves the time.  As UMFPACK does by default (UMFPACK_IRSTEP = 2),
        up to two steps of iterative refinement follow the solve."""
        rs = np.asarray(abs(A).sum(axis=1)).ravel()
        rs[rs == 0.0] = 1.0
        D = sp.diags(1.0 / rs)
        As = (D @ A).tocsc()
        bs = D @ b
        perm = self._nd_permutation(A.shape[0])
        F = spla.splu(As[perm][:, perm].tocsc(), permc_spec="NATURAL")
        x = np.empty_like(bs)
        x[perm] = F.solve(bs[perm])
        bn = np.linalg.norm(bs)
        for _ in range(2):
            r = bs - As @ x
            if not np.linalg.norm(r) > 1e-15 * bn:
                break
            d = np.empty_like(bs)
            d[perm] = F.solve(r[perm])
            x += d
        return x

    def _nd_permutation(self, n):
        """Unknown order of the nested dissection for a system of n unknowns
        on the (Ny1, Nx1) P-node grid (n / nodes unknowns per node, node-major
        as the assembly numbers them)."""
        cache = self.__dict__.setdefault("_perms", {})
        if n not in cache:
            g = self.st.g
            ny, nx = g.Ny1, g.Nx1
            dof = n // (ny * nx)
            order = []

            def split(i0, i1, j0, j1):
                h, w = i1 - i0, j1 - j0
                if h <= 0 or w <= 0:
                    return
                if h * w <= 16:
                    for j in range(j0, j1):
                        order.extend(range(j * ny + i0, j * ny + i1))
                    return
                if w >= h:
                    m = (j0 + j1) // 2
                    split(i0, i1, j0, m)
                    split(i0, i1, m + 1, j1)
                    order.extend(range(m * ny + i0, m * ny + i1))
                else:
                    m = (i0 + i1) // 2
                    split(i0, m, j0, j1)
                    split(m + 1, i1, j0, j1)
                    order.extend(j * ny + m for j in range(j0, j1))

            split(0, ny, 0, nx)
            nodes = np.asarray(order, dtype=np.int64)
            assert nodes.size == ny * nx
            cache[n] = (nodes[:, None] * dof + np.arange(dof)[None, :]).ravel()
        return cache[n]

    # -- phases ----------------------------------------------------------------
    def markers_to_nodes(self, timesum):
        self.L.oracle_markers_to_nodes(self.pP, self.pM, self.st.marknum, self.pG,
                                       self.pS, timesum)

    def gravity(self):
        A, b = self.gravity_system()
        SP = np.ascontiguousarray(self.solve(A, b))
        self.L.oracle_process_gravity(self.pP, _a(SP), self.pG)

    def hydromech_pass(self, dt, iplast):
        """One plastic pass (E:6678-6869); returns (dt, converged)."""
        L = self.L
        grid = self.st.grid
        t0 = time.perf_counter()
        L.oracle_bulk_viscosity(self.pP, self.pG)
        A, b = self.hydromech_system(dt)
        self._t("hydro_assemble", t0)
        t0 = time.perf_counter()
        S = np.ascontiguousarray(self.solve(A, b))
        self._t("hydro_solve", t0)
        t0 = time.perf_counter()
        L.oracle_process_hydromech(self.pP, _a(S), self.pG)
        aphimax = L.oracle_compute_aphi(self.pP, self.pG, dt)
        L.oracle_fluid_velocities(self.pP, self.pG)
        dt = L.oracle_displacement_timestep(self.pP, self.pG, dt, aphimax)
        L.oracle_stress_strainrate(self.pP, self.pG, dt)
        L.oracle_compute_aphi(self.pP, self.pG, dt)
        L.oracle_symmetrize(self.pP, self.pG)
        ynpl = ctypes.c_int(0)
        conv = L.oracle_nodal_adjustment(self.pP, self.pG, dt, iplast,
                                         _a(self.YERRNOD), ctypes.byref(ynpl))
        if not conv:
            dt = L.oracle_finalize_plastic(self.pP, self.pG, dt, iplast)
        self._t("hydro_post", t0)
        return dt, bool(conv)

    def thermal(self, dt, timestep):
        """E:6887-6927; returns max|DT|."""
        L, grid = self.L, self.st.grid
        L.oracle_shear_heating(self.pP, self.pG)
        if timestep == 1:
            grid["pr0"][:] = grid["pr"]
            grid["pf0"][:] = grid["pf"]
            grid["ps0"][:] = grid["ps"]
        L.oracle_adiabatic_heating(self.pP, self.pG)
        A, b = self.thermal_system(dt)
        ST = self.solve(A, b)
        grid["tk2"][:] = ST.reshape(grid["tk2"].shape, order="F")
        grid["DT"][:] = grid["tk2"] - grid["tk1"]
        return float(np.max(np.abs(grid["DT"])))

    def step(self, timestep):
        """One timestep of simulation_loop (E:6370-7235).  Returns a stats
        dict; st.dt / st.timesum / st.marknum are updated."""
        st, L, p = self.st, self.L, self.P
        grid = st.grid
        stats = {"titer": 0, "iplast_total": 0}
        t0 = time.perf_counter()
        self.markers_to_nodes(st.timesum)
        self._t("markers_to_nodes", t0)
        t0 = time.perf_counter()
        self.gravity()
        self._t("gravity", t0)
        dt = min(st.dt * p.dtcoefup, p.dt_longest)
        for titer in range(1, p.titermax + 1):
            stats["titer"] = titer
            t0 = time.perf_counter()
            if p.reaction_active:
                L.oracle_thermochemical_reaction(self.pP, self.pM, st.marknum, self.pG,
                                                 self.pS, dt, timestep, titer)
            self._t("reaction", t0)
            grid["ETA00"][:] = grid["ETA"]
            grid["YNY00"][:] = grid["YNY"]
            if timestep == 1:
                grid["BETAPHI"][:] = 0.0
            grid["pr0"][:] = grid["pr"]
            grid["pf0"][:] = grid["pf"]
            for iplast in range(1, p.titermax + 1):
                stats["iplast_total"] += 1
                dt, conv = self.hydromech_pass(dt, iplast)
                if conv:
                    break
            t0 = time.perf_counter()
            maxDT = self.thermal(dt, timestep)
            dt = finalize_thermochemical_iteration_pass(p, maxDT, dt, titer)
            done = thermochemical_iteration_outcome(p, grid["DMP"], grid["pf"], grid["pf0"],
                                                    titer)
            self._t("thermal", t0)
            if done:
                break
        t0 = time.perf_counter()
        L.oracle_nodes_to_markers(self.pP, self.pM, st.marknum, self.pG, self.pS,
                                  dt, timestep)
        self._t("nodes_to_markers", t0)
        t0 = time.perf_counter()
        L.oracle_velocities(self.pP, self.pG)
        L.oracle_rotation_rate(self.pP, self.pG)
        L.oracle_move_markers_rk4(self.pP, self.pM, st.marknum, self.pG, dt)
        L.oracle_backtrace_pressures(self.pP, self.pG, dt)
        self._t("advect", t0)
        t0 = time.perf_counter()
        n = L.oracle_replenish(self.pP, self.pM, st.marknum, st.capacity,
                               _a(self.mdis), _a(self.mnum), timestep)
        self._t("replenish", t0)
        if n < 0:
            raise RuntimeError("marker capacity exceeded in replenish")
        st.marknum = int(n)
        st.dt = dt
        st.timesum += dt
        stats.update(dt=dt, timesum=st.timesum, marknum=st.marknum,
                     maxT=float(grid["tk2"].max()))
        return stats
