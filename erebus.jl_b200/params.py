"""Runtime parameter sets (the reference's compile-time constants).

`default_params` returns the values of src/constants.jl (C:1-447) for a given
grid; `config_params` returns the synthetic planetesimal workloads (a 140 km
box with a 50 km rock body in sticky air) at 41x41, 141x141 and 401x401
basic nodes.  Everything here is host-side configuration.
"""
import math

from .abi import ErebusParams

YEARLENGTH = 365.25 * 24 * 3600          # C:325


def _set3(p, name, values):
    arr = getattr(p, name)
    for k, v in enumerate(values):
        arr[k] = float(v)


def default_params(Nx=15, Ny=15):
    """ErebusParams holding src/constants.jl (C:1-447) on an Nx x Ny grid.

    The geometry (xsize, rplanet, ...) is that of src/constants.jl (a 14 km
    box); callers resize it for other workloads."""
    p = ErebusParams()
    p.Nx, p.Ny = int(Nx), int(Ny)
    p.Nxmc = p.Nymc = 4                                   # C:104-106
    p.xsize = p.ysize = 14_000.0                          # C:15-19
    p.rplanet, p.rcrust, p.psurface = 5_000.0, 4_800.0, 1.0e3   # C:8-12
    _set3(p, "rhosolidm", [3300.0, 3300.0, 1.0])          # C:146-186
    _set3(p, "rhofluidm", [1000.0, 1000.0, 1.0])
    _set3(p, "etasolidm", [1e19, 1e19, 1e16])
    _set3(p, "etasolidmm", [1e19, 1e19, 1e16])
    _set3(p, "etafluidm", [1e12, 1e12, 1e-3])
    _set3(p, "etafluidmm", [1e-3, 1e-3, 1e-3])
    _set3(p, "rhocpsolidm", [3.3e6, 3.3e6, 3.0e6])
    _set3(p, "rhocpfluidm", [1.0e6, 1.0e6, 3.0e6])
    _set3(p, "alphasolidm", [3.0e-5, 3.0e-5, 0.0])
    _set3(p, "alphafluidm", [5.0e-5, 5.0e-5, 0.0])
    _set3(p, "ksolidm", [3.0, 3.0, 3000.0])
    _set3(p, "kfluidm", [50.0, 50.0, 3000.0])
    _set3(p, "start_hrsolidm", [0.0, 0.0, 0.0])
    _set3(p, "start_hrfluidm", [0.0, 0.0, 0.0])
    _set3(p, "gggsolidm", [1e10, 1e10, 1e10])
    _set3(p, "frictsolidm", [0.6, 0.6, 0.0])
    _set3(p, "cohessolidm", [1e8, 1e8, 1e8])
    _set3(p, "tenssolidm", [6e7, 6e7, 6e7])
    _set3(p, "kphim0", [1e-13, 1e-13, 1e-17])
    _set3(p, "tkm0", [170.0, 170.0, 170.0])
    _set3(p, "XWsolidm_init", [0.5, 0.5, float("nan")])
    p.marker_property_mode = 9                            # C:188
    p.reaction_rate_coeff_mode = 1                        # C:271
    p.etaphikoef = 1.0                                    # C:190
    p.hr_al, p.hr_fe = 1, 0                               # C:2-4
    p.t_half_al = 717_000.0 * 31_540_000.0                # C:196
    p.ratio_al, p.E_al, p.f_al = 5.0e-5, 5.0470e-13, 1.9e23
    p.t_half_fe = 2_620_000.0 * 31_540_000.0
    p.ratio_fe, p.E_fe, p.f_fe = 1.0e-6, 4.34e-13, 1.957e24
    p.tmsolidphase, p.tmfluidphase, p.Lf = 1416.0, 273.0, 333.55e3
    p.phim0, p.phimin = 0.2, 1.0e-4                       # C:222-227
    p.phimax = 1.0 - p.phimin
    p.RG, p.MH2O, p.MD = 8.314, 0.018, 0.120              # C:230-245
    p.rhoDs, p.rhoWs, p.rhoH2Of, p.rhoH2Ofi = 3300.0, 2600.0, 1000.0, 917.0
    p.dHWD, p.dSWD = 40000.0, 60.0
    p.pfcoeff, p.pferrmax = 0.5, 1.0e5
    p.reaction_active = 1
    p.dtreaction = 1.0e10
    p.log_completion_rate = math.log(0.01)
    p.A_I, p.b_I, p.c_I = 1.0e-11, 2.5e-4, 543.0
    p.Sxo_B, p.Tscl_B, p.To_B = 2.0e-11, 10.0, 293.0
    p.Sxo_T, p.To_T, p.Ea_T = 2.0e-11, 293.0, 63.8e3
    p.bcleft = p.bcright = p.bctop = p.bcbottom = -1.0    # C:283-300
    p.bcfleft = p.bcfright = p.bcftop = p.bcfbottom = -1.0
    p.strainrate = 0.0
    p.G, p.Kcont = 6.672e-11, 1.0e20                      # C:137-143
    p.dt_longest, p.dtcoefdn, p.dtcoefup = 1.0e11, 0.5, 1.2   # C:316-320
    p.dtstep, p.nplast = 200, 100_000
    p.dxymax, p.DTmax = 0.05, 20.0
    p.dsubgridt = p.dsubgrids = 0.0
    p.start_time = 2.25e6 * YEARLENGTH
    p.endtime = 15.0e6 * YEARLENGTH
    p.etamin, p.etamax = 1e12, 1e23
    p.titermax = 10_000
    p.random_markers = 1
    p.yerrmax, p.etawt, p.dphimax = 1e2, 0.0, 100.01
    p.seed = 42
    p.per_marker_eta = 0
    return p


# Synthetic planetesimal workloads: name -> (basic grid side, markers per
# cell, porosity law, rock viscosity law).
CONFIGS = {
    "planetesimal_41": dict(N=41, mpc=4, phi=("const", 0.1), eta=("const", 1e19)),
    "planetesimal_141": dict(N=141, mpc=5, phi=("uniform", 0.05, 0.25),
                             eta=("loguniform", 1e18, 1e20)),
    "planetesimal_401": dict(N=401, mpc=4, phi=("const", 0.1),
                             eta=("loguniform", 1e17, 1e23)),
    "planetesimal_141_adjoint": dict(N=141, mpc=4, phi=("uniform", 0.05, 0.25),
                                     eta=("const", 1e19)),
}


def config_params(name):
    """Parameters of a synthetic planetesimal workload.

    Shared physics: 140 km x 140 km box, rock body of radius 50 km (crust
    from 48 km) centred in sticky air (density 1, viscosity 1e17 Pa s), rock
    permeability 1e-13 m^2 at the reference porosity 0.1 with Kozeny-Carman
    scaling, fluid viscosity 1e-3 Pa s, fluid density 1000, 170 K, 26Al/27Al
    = 5e-5, self-gravity, free-slip.  Constants the workload does not state
    keep their src/constants.jl values."""
    c = CONFIGS[name]
    p = default_params(c["N"], c["N"])
    p.Nxmc = p.Nymc = c["mpc"]
    p.xsize = p.ysize = 140_000.0
    p.rplanet, p.rcrust = 50_000.0, 48_000.0
    _set3(p, "etafluidm", [1e-3, 1e-3, 1e-3])
    _set3(p, "etafluidmm", [1e-3, 1e-3, 1e-3])
    p.etasolidm[2] = p.etasolidmm[2] = 1e17
    p.phim0 = 0.1
    p.per_marker_eta = 1 if c["eta"][0] != "const" else 0
    if c["eta"][0] == "const":
        p.etasolidm[0] = p.etasolidm[1] = c["eta"][1]
        p.etasolidmm[0] = p.etasolidmm[1] = c["eta"][1]
    return p


def params_dict(p):
    """Plain dict of a parameter set (for logs and JSON)."""
    out = {}
    for name, ctype in p._fields_:
        v = getattr(p, name)
        if hasattr(v, "__len__"):
            v = list(v)
        out[name] = v
    return out
