"""Host-side state: numpy arrays in the reference's layouts, and the
synthetic marker initialiser.

Node arrays are Fortran-ordered numpy arrays of shape (Ny, Nx) (basic) or
(Ny1, Nx1) (Vx, Vy, P), so that `A[i-1, j-1]` is the reference's `A[i, j]`
and the memory is the reference's column-major layout.  Markers are 1-D
arrays of length `capacity`; `marknum` of them are in use.
"""
import ctypes

import numpy as np

from .abi import (GRID_FIELDS, MARKER_FIELDS, SUM_FIELDS, ErebusGridHost,
                  ErebusMarkersHost, ErebusSumsHost)

BASIC_GRID = ["ETA", "ETA0", "GGG", "EXY", "SXY", "SXY0", "wyx", "COH", "TEN",
              "FRI", "YNY", "ETA5", "ETA00", "YNY5", "YNY00", "YNY_inv_ETA",
              "DSXY", "DSY"]
BOOL_GRID = ["YNY", "YNY5", "YNY00"]
BASIC_SUMS = ["ETA0SUM", "ETASUM", "GGGSUM", "SXYSUM", "COHSUM", "TENSUM",
              "FRISUM", "WTSUM"]


class Geometry:
    """Derived grid quantities (src/constants.jl:25-124)."""

    def __init__(self, p):
        self.Nx, self.Ny = p.Nx, p.Ny
        self.Nx1, self.Ny1 = p.Nx + 1, p.Ny + 1
        self.dx = p.xsize / (p.Nx - 1)
        self.dy = p.ysize / (p.Ny - 1)
        self.Nxm = (p.Nx - 1) * p.Nxmc
        self.Nym = (p.Ny - 1) * p.Nymc
        self.dxm = p.xsize / self.Nxm
        self.dym = p.ysize / self.Nym
        self.xcenter = p.xsize / 2
        self.ycenter = p.ysize / 2
        self.start_marknum = self.Nxm * self.Nym


def _splitmix64(z):
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def u01(seed, stream, idx):
    """Counter-based uniform variates in [0, 1) (splitmix64 of seed, stream
    and index); identical to the device and C implementations."""
    idx = np.asarray(idx, dtype=np.uint64)
    s = _splitmix64(np.uint64(stream) ^ _splitmix64(idx))
    z = _splitmix64(np.uint64(seed) ^ s)
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def grid_layout(p):
    """Byte offsets of the grid arrays in one block, and the block size: each
    array at the next multiple of 256 bytes after the previous one (the
    layout of erebus_grid_layout, in which erebus_step_host copies the grid in
    one transfer)."""
    nb, npn = p.Nx * p.Ny, (p.Nx + 1) * (p.Ny + 1)
    off, o = {}, 0
    for name in GRID_FIELDS:
        n = nb if name in BASIC_GRID else npn
        b = n if name in BOOL_GRID else 8 * n
        off[name] = o
        o += (b + 255) // 256 * 256
    return off, o


class HostState:
    """Numpy arrays for one planetesimal, plus ctypes views of them.

    With `pinned`, the marker and grid arrays live in page-locked host memory
    (allocated through torch), which lets device copies run asynchronously."""

    def __init__(self, p, capacity=None, pinned=False):
        self.p = p
        self.g = g = Geometry(p)
        if capacity is None:
            capacity = int(g.start_marknum * 1.25) + 1024
        self.capacity = int(capacity)
        self.marknum = 0
        self._pins = []
        zeros = self._pinned_zeros if pinned else (
            lambda shape, dtype, order="C": np.zeros(shape, dtype=dtype, order=order))
        self.m = {}
        for name in MARKER_FIELDS:
            dt = np.int64 if name == "tm" else np.float64
            self.m[name] = zeros(self.capacity, dt)
        self.grid = self._grid_block(pinned)
        self.sums = {}
        for name in SUM_FIELDS:
            shape = (g.Ny, g.Nx) if name in BASIC_SUMS else (g.Ny1, g.Nx1)
            self.sums[name] = np.zeros(shape, dtype=np.float64, order="F")
        self.dt = p.dt_longest          # setup_dynamic_simulation_parameters
        self.timesum = p.start_time     # (E:55-70)

    def _grid_block(self, pinned):
        """Grid arrays as views of one zeroed block in the grid_layout."""
        g = self.g
        off, total = grid_layout(self.p)
        if pinned:
            import torch
            t = torch.zeros(total, dtype=torch.uint8, pin_memory=True)
            self._pins.append(t)
            block = t.numpy()
        else:
            block = np.zeros(total, dtype=np.uint8)
        grid = {}
        for name in GRID_FIELDS:
            shape = (g.Ny, g.Nx) if name in BASIC_GRID else (g.Ny1, g.Nx1)
            dt = np.dtype(np.uint8 if name in BOOL_GRID else np.float64)
            n = shape[0] * shape[1]
            grid[name] = block[off[name]: off[name] + n * dt.itemsize].view(dt).reshape(
                shape, order="F")
        return grid

    def pinned(self):
        """A copy of this state in page-locked host memory (grid in one
        block), for asynchronous transfers."""
        o = HostState(self.p, self.capacity, pinned=True)
        for k, v in self.m.items():
            o.m[k][...] = v
        for k, v in self.grid.items():
            o.grid[k][...] = v
        for k, v in self.sums.items():
            o.sums[k][...] = v
        o.marknum, o.dt, o.timesum = self.marknum, self.dt, self.timesum
        return o

    def _pinned_zeros(self, shape, dtype, order="C"):
        import torch
        dtype = np.dtype(dtype)
        n = int(np.prod(shape))
        t = torch.zeros(max(n, 1) * dtype.itemsize, dtype=torch.uint8, pin_memory=True)
        self._pins.append(t)
        return t.numpy()[: n * dtype.itemsize].view(dtype).reshape(shape, order=order)

    # -- ctypes views -----------------------------------------------------
    @staticmethod
    def _ptr(a, ctype):
        return a.ctypes.data_as(ctypes.POINTER(ctype))

    def markers_struct(self):
        s = ErebusMarkersHost()
        for name, ctype in ErebusMarkersHost._fields_:
            if name == "etasolidm_m" and not self.p.per_marker_eta:
                setattr(s, name, ctypes.cast(None, ctype))
                continue
            setattr(s, name, self._ptr(self.m[name], ctype._type_))
        return s

    def grid_struct(self):
        s = ErebusGridHost()
        for name, ctype in ErebusGridHost._fields_:
            setattr(s, name, self._ptr(self.grid[name], ctype._type_))
        return s

    def sums_struct(self):
        s = ErebusSumsHost()
        for name, ctype in ErebusSumsHost._fields_:
            setattr(s, name, self._ptr(self.sums[name], ctype._type_))
        return s

    def copy(self):
        o = HostState.__new__(HostState)
        o.p, o.g, o.capacity, o.marknum = self.p, self.g, self.capacity, self.marknum
        o._pins = []
        o.m = {k: v.copy() for k, v in self.m.items()}
        o.grid = {k: v.copy(order="F") for k, v in self.grid.items()}
        o.sums = {k: v.copy(order="F") for k, v in self.sums.items()}
        o.dt, o.timesum = self.dt, self.timesum
        return o

    def markers_view(self):
        """Marker arrays trimmed to marknum."""
        return {k: v[: self.marknum] for k, v in self.m.items()}


def define_markers(st, phi_law=None, eta_law=None, randomized=None):
    """Initial marker set (define_markers!, src/Erebus.jl:593-668).

    Markers sit on the regular marker sub-grid, column-major, with uniform
    jitter of +-1/2 spacing when `randomized`; rock markers inside
    `rplanet` (crust beyond `rcrust`), sticky air outside.  The variates
    come from the counter-based generator `u01` (the reference draws them
    from a MersenneTwister).  `phi_law` / `eta_law` override the initial
    rock porosity ("const", v) / ("uniform", lo, hi) and the per-marker
    solid viscosity ("const", v) / ("loguniform", lo, hi)."""
    p, g = st.p, st.g
    if randomized is None:
        randomized = bool(p.random_markers)
    n = g.Nxm * g.Nym
    if n > st.capacity:
        raise ValueError("marker capacity too small for the initial set")
    idx = np.arange(n, dtype=np.uint64)
    jm = np.arange(n) // g.Nym + 1
    im = np.arange(n) % g.Nym + 1
    xm = g.dxm / 2 + (jm - 1) * g.dxm
    ym = g.dym / 2 + (im - 1) * g.dym
    if randomized:
        xm = xm + (u01(p.seed, 100, idx) - 0.5) * g.dxm
        ym = ym + (u01(p.seed, 101, idx) - 0.5) * g.dym
    rmark = np.sqrt((xm - g.xcenter) ** 2 + (ym - g.ycenter) ** 2)
    rock = rmark < p.rplanet
    tm = np.where(rock, np.where(rmark > p.rcrust, 2, 1), 3).astype(np.int64)
    t0 = tm - 1
    tab = lambda name: np.asarray(list(getattr(p, name)))[t0]
    phim = np.where(rock, p.phim0, p.phimin)
    if randomized:
        phim = np.where(rock, phim + p.phim0 * (u01(p.seed, 102, idx) - 0.5), phim)
    xw0 = np.where(rock, tab("XWsolidm_init"), 0.0)
    if randomized:
        xw0 = np.where(rock, xw0 + tab("XWsolidm_init") * (u01(p.seed, 103, idx) - 0.5), xw0)
    if phi_law is not None:
        if phi_law[0] == "const":
            phim = np.where(rock, phi_law[1], phim)
        else:
            lo, hi = phi_law[1], phi_law[2]
            phim = np.where(rock, lo + (hi - lo) * u01(p.seed, 104, idx), phim)
    etas = tab("etasolidm")
    if eta_law is not None and eta_law[0] != "const":
        lo, hi = np.log10(eta_law[1]), np.log10(eta_law[2])
        etas = np.where(rock, 10.0 ** (lo + (hi - lo) * u01(p.seed, 105, idx)), etas)
    m = st.m
    for k in m:
        m[k][:] = 0
    m["xm"][:n], m["ym"][:n], m["tm"][:n] = xm, ym, tm
    m["phim"][:n] = phim
    m["etavpm"][:n] = etas if p.per_marker_eta else tab("etasolidm")
    m["etasolidm_m"][:n] = etas
    m["XWsolidm0"][:n] = xw0
    air = ~rock
    m["rhototalm"][:n] = np.where(air, tab("rhosolidm"), 0.0)
    m["rhocptotalm"][:n] = np.where(air, tab("rhocpsolidm"), 0.0)
    m["etatotalm"][:n] = np.where(air, tab("etasolidm"), 0.0)
    m["hrtotalm"][:n] = np.where(air, tab("start_hrsolidm"), 0.0)
    m["ktotalm"][:n] = np.where(air, tab("ksolidm"), 0.0)
    m["tkm"][:n] = tab("tkm0")
    m["inv_gggtotalm"][:n] = 1.0 / tab("gggsolidm")
    m["fricttotalm"][:n] = tab("frictsolidm")
    m["cohestotalm"][:n] = tab("cohessolidm")
    m["tenstotalm"][:n] = tab("tenssolidm")
    m["rhofluidcur"][:n] = tab("rhofluidm")
    m["alphasolidcur"][:n] = tab("alphasolidm")
    m["alphafluidcur"][:n] = tab("alphafluidm")
    # simulation_loop E:6189-6190
    m["XWsolidm"][:n] = m["XWsolidm0"][:n]
    m["phinewm"][:n] = m["phim"][:n]
    st.marknum = n
    return st


def make_state(name_or_params, capacity=None):
    """HostState of a named synthetic workload (see params.CONFIGS), or of
    an explicit parameter set, with its initial markers."""
    from .params import CONFIGS, config_params
    if isinstance(name_or_params, str):
        p = config_params(name_or_params)
        c = CONFIGS[name_or_params]
        st = HostState(p, capacity)
        return define_markers(st, c["phi"], c["eta"])
    st = HostState(name_or_params, capacity)
    return define_markers(st)
