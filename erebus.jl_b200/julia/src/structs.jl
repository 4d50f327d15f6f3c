# Generated by gen_structs.py from the ctypes mirror of
# include/erebus_b200.h; do not edit by hand.

struct ErebusParams
    Nx::Cint
    Ny::Cint
    Nxmc::Cint
    Nymc::Cint
    xsize::Float64
    ysize::Float64
    rplanet::Float64
    rcrust::Float64
    psurface::Float64
    rhosolidm::NTuple{3, Float64}
    rhofluidm::NTuple{3, Float64}
    etasolidm::NTuple{3, Float64}
    etasolidmm::NTuple{3, Float64}
    etafluidm::NTuple{3, Float64}
    etafluidmm::NTuple{3, Float64}
    rhocpsolidm::NTuple{3, Float64}
    rhocpfluidm::NTuple{3, Float64}
    alphasolidm::NTuple{3, Float64}
    alphafluidm::NTuple{3, Float64}
    ksolidm::NTuple{3, Float64}
    kfluidm::NTuple{3, Float64}
    start_hrsolidm::NTuple{3, Float64}
    start_hrfluidm::NTuple{3, Float64}
    gggsolidm::NTuple{3, Float64}
    frictsolidm::NTuple{3, Float64}
    cohessolidm::NTuple{3, Float64}
    tenssolidm::NTuple{3, Float64}
    kphim0::NTuple{3, Float64}
    tkm0::NTuple{3, Float64}
    XWsolidm_init::NTuple{3, Float64}
    marker_property_mode::Cint
    reaction_rate_coeff_mode::Cint
    etaphikoef::Float64
    hr_al::Cint
    hr_fe::Cint
    t_half_al::Float64
    ratio_al::Float64
    E_al::Float64
    f_al::Float64
    t_half_fe::Float64
    ratio_fe::Float64
    E_fe::Float64
    f_fe::Float64
    tmsolidphase::Float64
    tmfluidphase::Float64
    Lf::Float64
    phim0::Float64
    phimin::Float64
    phimax::Float64
    RG::Float64
    MH2O::Float64
    MD::Float64
    rhoDs::Float64
    rhoWs::Float64
    rhoH2Of::Float64
    rhoH2Ofi::Float64
    dHWD::Float64
    dSWD::Float64
    pfcoeff::Float64
    pferrmax::Float64
    reaction_active::Cint
    _pad0::Cint
    dtreaction::Float64
    log_completion_rate::Float64
    A_I::Float64
    b_I::Float64
    c_I::Float64
    Sxo_B::Float64
    Tscl_B::Float64
    To_B::Float64
    Sxo_T::Float64
    To_T::Float64
    Ea_T::Float64
    bcleft::Float64
    bcright::Float64
    bctop::Float64
    bcbottom::Float64
    bcfleft::Float64
    bcfright::Float64
    bcftop::Float64
    bcfbottom::Float64
    strainrate::Float64
    G::Float64
    Kcont::Float64
    dt_longest::Float64
    dtcoefdn::Float64
    dtcoefup::Float64
    dtstep::Cint
    nplast::Cint
    dxymax::Float64
    DTmax::Float64
    dsubgridt::Float64
    dsubgrids::Float64
    start_time::Float64
    endtime::Float64
    etamin::Float64
    etamax::Float64
    titermax::Cint
    random_markers::Cint
    yerrmax::Float64
    etawt::Float64
    dphimax::Float64
    seed::UInt64
    per_marker_eta::Cint
    _pad1::Cint
end

struct ErebusMarkersHost
    xm::Ptr{Float64}
    ym::Ptr{Float64}
    tm::Ptr{Int64}
    tkm::Ptr{Float64}
    sxxm::Ptr{Float64}
    sxym::Ptr{Float64}
    etavpm::Ptr{Float64}
    phim::Ptr{Float64}
    phinewm::Ptr{Float64}
    pfm0::Ptr{Float64}
    XWsolidm::Ptr{Float64}
    XWsolidm0::Ptr{Float64}
    rhototalm::Ptr{Float64}
    rhocptotalm::Ptr{Float64}
    etatotalm::Ptr{Float64}
    hrtotalm::Ptr{Float64}
    ktotalm::Ptr{Float64}
    tkm_rhocptotalm::Ptr{Float64}
    etafluidcur_inv_kphim::Ptr{Float64}
    inv_gggtotalm::Ptr{Float64}
    fricttotalm::Ptr{Float64}
    cohestotalm::Ptr{Float64}
    tenstotalm::Ptr{Float64}
    rhofluidcur::Ptr{Float64}
    alphasolidcur::Ptr{Float64}
    alphafluidcur::Ptr{Float64}
    etasolidm_m::Ptr{Float64}
end

struct ErebusGridHost
    ETA::Ptr{Float64}
    ETA0::Ptr{Float64}
    GGG::Ptr{Float64}
    EXY::Ptr{Float64}
    SXY::Ptr{Float64}
    SXY0::Ptr{Float64}
    wyx::Ptr{Float64}
    COH::Ptr{Float64}
    TEN::Ptr{Float64}
    FRI::Ptr{Float64}
    YNY::Ptr{UInt8}
    ETA5::Ptr{Float64}
    ETA00::Ptr{Float64}
    YNY5::Ptr{UInt8}
    YNY00::Ptr{UInt8}
    YNY_inv_ETA::Ptr{Float64}
    DSXY::Ptr{Float64}
    DSY::Ptr{Float64}
    RHOX::Ptr{Float64}
    RHOFX::Ptr{Float64}
    KX::Ptr{Float64}
    PHIX::Ptr{Float64}
    vx::Ptr{Float64}
    vxf::Ptr{Float64}
    RX::Ptr{Float64}
    qxD::Ptr{Float64}
    gx::Ptr{Float64}
    RHOY::Ptr{Float64}
    RHOFY::Ptr{Float64}
    KY::Ptr{Float64}
    PHIY::Ptr{Float64}
    vy::Ptr{Float64}
    vyf::Ptr{Float64}
    RY::Ptr{Float64}
    qyD::Ptr{Float64}
    gy::Ptr{Float64}
    RHO::Ptr{Float64}
    RHOCP::Ptr{Float64}
    ALPHA::Ptr{Float64}
    ALPHAF::Ptr{Float64}
    HR::Ptr{Float64}
    HA::Ptr{Float64}
    HS::Ptr{Float64}
    ETAP::Ptr{Float64}
    GGGP::Ptr{Float64}
    EXX::Ptr{Float64}
    SXX::Ptr{Float64}
    SXX0::Ptr{Float64}
    tk1::Ptr{Float64}
    tk2::Ptr{Float64}
    DT::Ptr{Float64}
    DT0::Ptr{Float64}
    vxp::Ptr{Float64}
    vyp::Ptr{Float64}
    vxpf::Ptr{Float64}
    vypf::Ptr{Float64}
    pr::Ptr{Float64}
    pf::Ptr{Float64}
    ps::Ptr{Float64}
    pr0::Ptr{Float64}
    pf0::Ptr{Float64}
    ps0::Ptr{Float64}
    ETAPHI::Ptr{Float64}
    BETAPHI::Ptr{Float64}
    PHI::Ptr{Float64}
    APHI::Ptr{Float64}
    FI::Ptr{Float64}
    DMP::Ptr{Float64}
    DHP::Ptr{Float64}
    XWS::Ptr{Float64}
    EII::Ptr{Float64}
    SII::Ptr{Float64}
    DSXX::Ptr{Float64}
    tk0::Ptr{Float64}
end

struct ErebusSumsHost
    ETA0SUM::Ptr{Float64}
    ETASUM::Ptr{Float64}
    GGGSUM::Ptr{Float64}
    SXYSUM::Ptr{Float64}
    COHSUM::Ptr{Float64}
    TENSUM::Ptr{Float64}
    FRISUM::Ptr{Float64}
    WTSUM::Ptr{Float64}
    RHOXSUM::Ptr{Float64}
    RHOFXSUM::Ptr{Float64}
    KXSUM::Ptr{Float64}
    PHIXSUM::Ptr{Float64}
    RXSUM::Ptr{Float64}
    WTXSUM::Ptr{Float64}
    RHOYSUM::Ptr{Float64}
    RHOFYSUM::Ptr{Float64}
    KYSUM::Ptr{Float64}
    PHIYSUM::Ptr{Float64}
    RYSUM::Ptr{Float64}
    WTYSUM::Ptr{Float64}
    RHOSUM::Ptr{Float64}
    RHOCPSUM::Ptr{Float64}
    ALPHASUM::Ptr{Float64}
    ALPHAFSUM::Ptr{Float64}
    HRSUM::Ptr{Float64}
    GGGPSUM::Ptr{Float64}
    SXXSUM::Ptr{Float64}
    TKSUM::Ptr{Float64}
    PHISUM::Ptr{Float64}
    DMPSUM::Ptr{Float64}
    DHPSUM::Ptr{Float64}
    XWSSUM::Ptr{Float64}
    WTPSUM::Ptr{Float64}
end

struct ErebusSolveStats
    iterations::Cint
    converged::Cint
    rel_residual::Float64
end

struct ErebusStepStats
    titer::Cint
    iplast_total::Cint
    hydro_solves::Cint
    thermal_solves::Cint
    gravity_solves::Cint
    factorizations::Cint
    marknum::Int64
    dt::Float64
    timesum::Float64
    maxT::Float64
    worst_rel_residual::Float64
end

struct ErebusFactorStats
    direct_solver::Cint
    fronts::Cint
    levels::Cint
    factorizations::Cint
    fp64_refactorizations::Cint
    krylov_iterations::Cint
    unknowns::Int64
    storage_bytes::Int64
    flops::Float64
    solve_bytes::Float64
end

struct ErebusAdjointStats
    steps::Cint
    checkpoints::Cint
    adjoint_solves::Cint
    factorizations::Cint
    markers::Int64
    J::Float64
    body_nodes::Float64
end

struct ErebusSolverOptions
    hydro_rtol::Float64
    thermal_rtol::Float64
    gravity_rtol::Float64
    max_refinements::Cint
    reuse_factors::Cint
    direct_solver::Cint
    factor_fp32::Cint
    krylov::Cint
    precond_fp32::Cint
    krylov_restart::Cint
    refactor_iterations::Cint
    mf_leaf_vector::Cint
    mf_leaf_scalar::Cint
    mf_local_factor_ops::Cint
    mf_local_solve_tiles::Cint
    mf_block_substitution::Cint
end

const MARKER_FIELDS = (:xm, :ym, :tm, :tkm, :sxxm, :sxym, :etavpm, :phim, :phinewm, :pfm0, :XWsolidm, :XWsolidm0, :rhototalm, :rhocptotalm, :etatotalm, :hrtotalm, :ktotalm, :tkm_rhocptotalm, :etafluidcur_inv_kphim, :inv_gggtotalm, :fricttotalm, :cohestotalm, :tenstotalm, :rhofluidcur, :alphasolidcur, :alphafluidcur, :etasolidm_m)
const GRID_FIELDS = (:ETA, :ETA0, :GGG, :EXY, :SXY, :SXY0, :wyx, :COH, :TEN, :FRI, :YNY, :ETA5, :ETA00, :YNY5, :YNY00, :YNY_inv_ETA, :DSXY, :DSY, :RHOX, :RHOFX, :KX, :PHIX, :vx, :vxf, :RX, :qxD, :gx, :RHOY, :RHOFY, :KY, :PHIY, :vy, :vyf, :RY, :qyD, :gy, :RHO, :RHOCP, :ALPHA, :ALPHAF, :HR, :HA, :HS, :ETAP, :GGGP, :EXX, :SXX, :SXX0, :tk1, :tk2, :DT, :DT0, :vxp, :vyp, :vxpf, :vypf, :pr, :pf, :ps, :pr0, :pf0, :ps0, :ETAPHI, :BETAPHI, :PHI, :APHI, :FI, :DMP, :DHP, :XWS, :EII, :SII, :DSXX, :tk0)
const SUM_FIELDS = (:ETA0SUM, :ETASUM, :GGGSUM, :SXYSUM, :COHSUM, :TENSUM, :FRISUM, :WTSUM, :RHOXSUM, :RHOFXSUM, :KXSUM, :PHIXSUM, :RXSUM, :WTXSUM, :RHOYSUM, :RHOFYSUM, :KYSUM, :PHIYSUM, :RYSUM, :WTYSUM, :RHOSUM, :RHOCPSUM, :ALPHASUM, :ALPHAFSUM, :HRSUM, :GGGPSUM, :SXXSUM, :TKSUM, :PHISUM, :DMPSUM, :DHPSUM, :XWSSUM, :WTPSUM)
