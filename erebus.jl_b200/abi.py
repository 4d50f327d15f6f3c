"""ctypes mirror of include/erebus_b200.h (the library's C ABI).

The field lists follow the header exactly; tests/test_abi.py re-parses the
header and checks names, order and sizes.
"""
from ctypes import (POINTER, Structure, c_char_p, c_double, c_int, c_int32,
                    c_int64, c_uint8, c_uint64, c_void_p)


class ErebusParams(Structure):
    """Runtime parameter set replacing src/constants.jl (C:1-447)."""
    _fields_ = [
        ("Nx", c_int32), ("Ny", c_int32), ("Nxmc", c_int32), ("Nymc", c_int32),
        ("xsize", c_double), ("ysize", c_double), ("rplanet", c_double),
        ("rcrust", c_double), ("psurface", c_double), ("rhosolidm", c_double * 3),
        ("rhofluidm", c_double * 3), ("etasolidm", c_double * 3),
        ("etasolidmm", c_double * 3), ("etafluidm", c_double * 3),
        ("etafluidmm", c_double * 3), ("rhocpsolidm", c_double * 3),
        ("rhocpfluidm", c_double * 3), ("alphasolidm", c_double * 3),
        ("alphafluidm", c_double * 3), ("ksolidm", c_double * 3),
        ("kfluidm", c_double * 3), ("start_hrsolidm", c_double * 3),
        ("start_hrfluidm", c_double * 3), ("gggsolidm", c_double * 3),
        ("frictsolidm", c_double * 3), ("cohessolidm", c_double * 3),
        ("tenssolidm", c_double * 3), ("kphim0", c_double * 3), ("tkm0", c_double * 3),
        ("XWsolidm_init", c_double * 3), ("marker_property_mode", c_int32),
        ("reaction_rate_coeff_mode", c_int32), ("etaphikoef", c_double),
        ("hr_al", c_int32), ("hr_fe", c_int32), ("t_half_al", c_double),
        ("ratio_al", c_double), ("E_al", c_double), ("f_al", c_double),
        ("t_half_fe", c_double), ("ratio_fe", c_double), ("E_fe", c_double),
        ("f_fe", c_double), ("tmsolidphase", c_double), ("tmfluidphase", c_double),
        ("Lf", c_double), ("phim0", c_double), ("phimin", c_double),
        ("phimax", c_double), ("RG", c_double), ("MH2O", c_double), ("MD", c_double),
        ("rhoDs", c_double), ("rhoWs", c_double), ("rhoH2Of", c_double),
        ("rhoH2Ofi", c_double), ("dHWD", c_double), ("dSWD", c_double),
        ("pfcoeff", c_double), ("pferrmax", c_double), ("reaction_active", c_int32),
        ("_pad0", c_int32), ("dtreaction", c_double),
        ("log_completion_rate", c_double), ("A_I", c_double), ("b_I", c_double),
        ("c_I", c_double), ("Sxo_B", c_double), ("Tscl_B", c_double),
        ("To_B", c_double), ("Sxo_T", c_double), ("To_T", c_double),
        ("Ea_T", c_double), ("bcleft", c_double), ("bcright", c_double),
        ("bctop", c_double), ("bcbottom", c_double), ("bcfleft", c_double),
        ("bcfright", c_double), ("bcftop", c_double), ("bcfbottom", c_double),
        ("strainrate", c_double), ("G", c_double), ("Kcont", c_double),
        ("dt_longest", c_double), ("dtcoefdn", c_double), ("dtcoefup", c_double),
        ("dtstep", c_int32), ("nplast", c_int32), ("dxymax", c_double),
        ("DTmax", c_double), ("dsubgridt", c_double), ("dsubgrids", c_double),
        ("start_time", c_double), ("endtime", c_double), ("etamin", c_double),
        ("etamax", c_double), ("titermax", c_int32), ("random_markers", c_int32),
        ("yerrmax", c_double), ("etawt", c_double), ("dphimax", c_double),
        ("seed", c_uint64), ("per_marker_eta", c_int32), ("_pad1", c_int32),
    ]


class ErebusMarkersHost(Structure):
    """Host views of the marker SoA (src/Erebus.jl:426-552)."""
    _fields_ = [
        ("xm", POINTER(c_double)), ("ym", POINTER(c_double)), ("tm", POINTER(c_int64)),
        ("tkm", POINTER(c_double)), ("sxxm", POINTER(c_double)),
        ("sxym", POINTER(c_double)), ("etavpm", POINTER(c_double)),
        ("phim", POINTER(c_double)), ("phinewm", POINTER(c_double)),
        ("pfm0", POINTER(c_double)), ("XWsolidm", POINTER(c_double)),
        ("XWsolidm0", POINTER(c_double)), ("rhototalm", POINTER(c_double)),
        ("rhocptotalm", POINTER(c_double)), ("etatotalm", POINTER(c_double)),
        ("hrtotalm", POINTER(c_double)), ("ktotalm", POINTER(c_double)),
        ("tkm_rhocptotalm", POINTER(c_double)),
        ("etafluidcur_inv_kphim", POINTER(c_double)),
        ("inv_gggtotalm", POINTER(c_double)), ("fricttotalm", POINTER(c_double)),
        ("cohestotalm", POINTER(c_double)), ("tenstotalm", POINTER(c_double)),
        ("rhofluidcur", POINTER(c_double)), ("alphasolidcur", POINTER(c_double)),
        ("alphafluidcur", POINTER(c_double)), ("etasolidm_m", POINTER(c_double)),
    ]


class ErebusGridHost(Structure):
    """Host views of the staggered-grid arrays (src/Erebus.jl:147-415)."""
    _fields_ = [
        ("ETA", POINTER(c_double)), ("ETA0", POINTER(c_double)),
        ("GGG", POINTER(c_double)), ("EXY", POINTER(c_double)),
        ("SXY", POINTER(c_double)), ("SXY0", POINTER(c_double)),
        ("wyx", POINTER(c_double)), ("COH", POINTER(c_double)),
        ("TEN", POINTER(c_double)), ("FRI", POINTER(c_double)),
        ("YNY", POINTER(c_uint8)), ("ETA5", POINTER(c_double)),
        ("ETA00", POINTER(c_double)), ("YNY5", POINTER(c_uint8)),
        ("YNY00", POINTER(c_uint8)), ("YNY_inv_ETA", POINTER(c_double)),
        ("DSXY", POINTER(c_double)), ("DSY", POINTER(c_double)),
        ("RHOX", POINTER(c_double)), ("RHOFX", POINTER(c_double)),
        ("KX", POINTER(c_double)), ("PHIX", POINTER(c_double)),
        ("vx", POINTER(c_double)), ("vxf", POINTER(c_double)),
        ("RX", POINTER(c_double)), ("qxD", POINTER(c_double)),
        ("gx", POINTER(c_double)), ("RHOY", POINTER(c_double)),
        ("RHOFY", POINTER(c_double)), ("KY", POINTER(c_double)),
        ("PHIY", POINTER(c_double)), ("vy", POINTER(c_double)),
        ("vyf", POINTER(c_double)), ("RY", POINTER(c_double)),
        ("qyD", POINTER(c_double)), ("gy", POINTER(c_double)),
        ("RHO", POINTER(c_double)), ("RHOCP", POINTER(c_double)),
        ("ALPHA", POINTER(c_double)), ("ALPHAF", POINTER(c_double)),
        ("HR", POINTER(c_double)), ("HA", POINTER(c_double)),
        ("HS", POINTER(c_double)), ("ETAP", POINTER(c_double)),
        ("GGGP", POINTER(c_double)), ("EXX", POINTER(c_double)),
        ("SXX", POINTER(c_double)), ("SXX0", POINTER(c_double)),
        ("tk1", POINTER(c_double)), ("tk2", POINTER(c_double)),
        ("DT", POINTER(c_double)), ("DT0", POINTER(c_double)),
        ("vxp", POINTER(c_double)), ("vyp", POINTER(c_double)),
        ("vxpf", POINTER(c_double)), ("vypf", POINTER(c_double)),
        ("pr", POINTER(c_double)), ("pf", POINTER(c_double)),
        ("ps", POINTER(c_double)), ("pr0", POINTER(c_double)),
        ("pf0", POINTER(c_double)), ("ps0", POINTER(c_double)),
        ("ETAPHI", POINTER(c_double)), ("BETAPHI", POINTER(c_double)),
        ("PHI", POINTER(c_double)), ("APHI", POINTER(c_double)),
        ("FI", POINTER(c_double)), ("DMP", POINTER(c_double)),
        ("DHP", POINTER(c_double)), ("XWS", POINTER(c_double)),
        ("EII", POINTER(c_double)), ("SII", POINTER(c_double)),
        ("DSXX", POINTER(c_double)), ("tk0", POINTER(c_double)),
    ]


class ErebusSumsHost(Structure):
    """Scatter sums of src/Erebus.jl:851-923."""
    _fields_ = [
        ("ETA0SUM", POINTER(c_double)), ("ETASUM", POINTER(c_double)),
        ("GGGSUM", POINTER(c_double)), ("SXYSUM", POINTER(c_double)),
        ("COHSUM", POINTER(c_double)), ("TENSUM", POINTER(c_double)),
        ("FRISUM", POINTER(c_double)), ("WTSUM", POINTER(c_double)),
        ("RHOXSUM", POINTER(c_double)), ("RHOFXSUM", POINTER(c_double)),
        ("KXSUM", POINTER(c_double)), ("PHIXSUM", POINTER(c_double)),
        ("RXSUM", POINTER(c_double)), ("WTXSUM", POINTER(c_double)),
        ("RHOYSUM", POINTER(c_double)), ("RHOFYSUM", POINTER(c_double)),
        ("KYSUM", POINTER(c_double)), ("PHIYSUM", POINTER(c_double)),
        ("RYSUM", POINTER(c_double)), ("WTYSUM", POINTER(c_double)),
        ("RHOSUM", POINTER(c_double)), ("RHOCPSUM", POINTER(c_double)),
        ("ALPHASUM", POINTER(c_double)), ("ALPHAFSUM", POINTER(c_double)),
        ("HRSUM", POINTER(c_double)), ("GGGPSUM", POINTER(c_double)),
        ("SXXSUM", POINTER(c_double)), ("TKSUM", POINTER(c_double)),
        ("PHISUM", POINTER(c_double)), ("DMPSUM", POINTER(c_double)),
        ("DHPSUM", POINTER(c_double)), ("XWSSUM", POINTER(c_double)),
        ("WTPSUM", POINTER(c_double)),
    ]


class ErebusSolveStats(Structure):
    _fields_ = [
        ("iterations", c_int32), ("converged", c_int32), ("rel_residual", c_double),
    ]


class ErebusStepStats(Structure):
    _fields_ = [
        ("titer", c_int32), ("iplast_total", c_int32), ("hydro_solves", c_int32),
        ("thermal_solves", c_int32), ("gravity_solves", c_int32), ("factorizations", c_int32),
        ("marknum", c_int64), ("dt", c_double), ("timesum", c_double),
        ("maxT", c_double), ("worst_rel_residual", c_double),
    ]


class ErebusFactorStats(Structure):
    _fields_ = [
        ("direct_solver", c_int32), ("fronts", c_int32), ("levels", c_int32),
        ("factorizations", c_int32), ("fp64_refactorizations", c_int32),
        ("krylov_iterations", c_int32),
        ("unknowns", c_int64), ("storage_bytes", c_int64),
        ("flops", c_double), ("solve_bytes", c_double),
    ]


class ErebusAdjointStats(Structure):
    _fields_ = [
        ("steps", c_int32), ("checkpoints", c_int32), ("adjoint_solves", c_int32),
        ("factorizations", c_int32), ("markers", c_int64), ("J", c_double),
        ("body_nodes", c_double),
    ]


class ErebusSolverOptions(Structure):
    _fields_ = [
        ("hydro_rtol", c_double), ("thermal_rtol", c_double),
        ("gravity_rtol", c_double), ("max_refinements", c_int32),
        ("reuse_factors", c_int32), ("direct_solver", c_int32), ("factor_fp32", c_int32),
        ("krylov", c_int32), ("precond_fp32", c_int32), ("krylov_restart", c_int32),
        ("refactor_iterations", c_int32), ("mf_leaf_vector", c_int32),
        ("mf_leaf_scalar", c_int32), ("mf_local_factor_ops", c_int32),
        ("mf_local_solve_tiles", c_int32), ("mf_block_substitution", c_int32),
    ]


MARKER_FIELDS = [f[0] for f in ErebusMarkersHost._fields_]
GRID_FIELDS = [f[0] for f in ErebusGridHost._fields_]
SUM_FIELDS = [f[0] for f in ErebusSumsHost._fields_]

# Status codes (EREBUS_* in the header).
OK, EINVAL, ECUDA, ENOMEM, ECAPACITY, ENOCONV, ENONFINITE, ENODEVICE = range(8)
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ENOMEM",
                4: "ECAPACITY", 5: "ENOCONV", 6: "ENONFINITE", 7: "ENODEVICE"}
