# CLI equivalent of Erebus.run_simulation (src/Erebus.jl:7251-7303) whose
# timestep loop runs on the B200 library:
#
#     julia --project=<environment with Erebus, ChainRulesCore, ArgParse> \
#           run_simulation_b200.jl <output_path> [--show_timer false] [--mixed true]
#
# The reference package sets the run up exactly as its simulation_loop does
# (setup_* allocators, define_markers!, the initial save_state); each
# iteration of the `for timestep` loop (E:6370-7235) is then one
# ErebusB200.step! on the device, and every savematstep timesteps the state is
# copied back and written with the reference's own save_state (JLD2), so the
# output is read by generate_plots.jl unchanged.  The argument names of the
# setup functions' results below are the reference's own (they are its API).
using ArgParse, Dates, Logging
using Erebus
include(joinpath(@__DIR__, "src", "ErebusB200.jl"))
using .ErebusB200

const E = Erebus

# results of the reference's setup functions, in their return order
const GRID_SETUP = (
    :ETA, :ETA0, :GGG, :EXY, :SXY, :SXY0, :wyx, :COH,
    :TEN, :FRI, :YNY, :RHOX, :RHOFX, :KX, :PHIX, :vx,
    :vxf, :RX, :qxD, :gx, :RHOY, :RHOFY, :KY, :PHIY,
    :vy, :vyf, :RY, :qyD, :gy, :RHO, :RHOCP, :ALPHA,
    :ALPHAF, :HR, :HA, :HS, :ETAP, :GGGP, :EXX, :SXX,
    :SXX0, :tk1, :tk2, :DT, :DT0, :vxp, :vyp, :vxpf,
    :vypf, :pr, :pf, :ps, :pr0, :pf0, :ps0, :ETAPHI,
    :BETAPHI, :PHI, :APHI, :FI, :DMP, :DHP, :XWS,
)
const GRID_HELPERS = (
    :ETA5, :ETA00, :YNY5, :YNY00, :YNY_inv_ETA, :DSXY, :DSY, :EII,
    :SII, :DSXX, :tk0,
)
const MARKER_SETUP = (
    :xm, :ym, :tm, :tkm, :sxxm, :sxym, :etavpm, :phim,
    :phinewm, :pfm0, :XWsolidm, :XWsolidm0,
)
const MARKER_HELPERS = (
    :rhototalm, :rhocptotalm, :etatotalm, :hrtotalm, :ktotalm, :tkm_rhocptotalm, :etafluidcur_inv_kphim, :inv_gggtotalm,
    :fricttotalm, :cohestotalm, :tenstotalm, :rhofluidcur, :alphasolidcur, :alphafluidcur,
)
# define_markers! arguments (E:6166-6186)
const DEFINE_MARKERS_ARGS = (
    :xm, :ym, :tm, :phim, :etavpm, :rhototalm, :rhocptotalm, :etatotalm,
    :hrtotalm, :ktotalm, :tkm, :inv_gggtotalm, :fricttotalm, :cohestotalm, :tenstotalm, :rhofluidcur,
    :alphasolidcur, :alphafluidcur, :XWsolidm0,
)
# save_state arrays after (output_path, timestep, dt, timesum, marknum)
const SAVE_STATE_ARRAYS = (
    :ETA, :ETA0, :GGG, :EXY, :SXY, :SXY0, :wyx, :COH,
    :TEN, :FRI, :YNY, :RHOX, :RHOFX, :KX, :PHIX, :vx,
    :vxf, :RX, :qxD, :gx, :RHOY, :RHOFY, :KY, :PHIY,
    :vy, :vyf, :RY, :qyD, :gy, :RHO, :RHOCP, :ALPHA,
    :ALPHAF, :HR, :HA, :HS, :ETAP, :GGGP, :EXX, :SXX,
    :SXX0, :tk1, :tk2, :vxp, :vyp, :vxpf, :vypf, :pr,
    :pf, :ps, :pr0, :pf0, :ps0, :ETAPHI, :BETAPHI, :PHI,
    :APHI, :FI, :ETA5, :ETA00, :YNY5, :YNY00, :YNY_inv_ETA, :DSXY,
    :EII, :SII, :DSXX, :DMP, :DHP, :XWS, :XWsolidm0, :xm,
    :ym, :tm, :tkm, :sxxm, :sxym, :etavpm, :phim, :rhototalm,
    :rhocptotalm, :etatotalm, :hrtotalm, :ktotalm, :tkm_rhocptotalm, :etafluidcur_inv_kphim, :inv_gggtotalm, :fricttotalm,
    :cohestotalm, :tenstotalm, :rhofluidcur, :alphasolidcur, :alphafluidcur,
)

function parse_commandline()
    s = ArgParseSettings()
    @add_arg_table! s begin
        "output_path"
            help = "output path for simulation data"
            required = true
        "--show_timer"
            help = "show timing results?"
            arg_type = Bool
            default = false
        "--mixed"
            help = "mixed-precision Krylov solves (lagged FP32-applied LU preconditioner)"
            arg_type = Bool
            default = false
    end
    return parse_args(s)
end

_trim(v::AbstractVector, n) = v[1:n]
_trim(a, n) = a

function save(output_path, timestep, dt, timesum, marknum, A)
    E.save_state(output_path, timestep, dt, timesum, marknum,
                 (_trim(A[k], marknum) for k in SAVE_STATE_ARRAYS)...)
end

function simulation_loop_b200(output_path; mixed::Bool=false)
    timestep, dt, timesum, marknum, hrsolidm, hrfluidm, YERRNOD =
        E.setup_dynamic_simulation_parameters()
    A = Dict{Symbol,Any}()
    merge!(A, Dict(zip(GRID_SETUP, E.setup_staggered_grid_properties())))
    merge!(A, Dict(zip(GRID_HELPERS, E.setup_staggered_grid_properties_helpers())))
    mdis, mnum = E.setup_marker_geometry_helpers()
    merge!(A, Dict(zip(MARKER_SETUP, E.setup_marker_properties(marknum))))
    merge!(A, Dict(zip(MARKER_HELPERS, E.setup_marker_properties_helpers(marknum))))
    E.define_markers!((A[k] for k in DEFINE_MARKERS_ARGS)...)
    A[:XWsolidm] .= A[:XWsolidm0]
    A[:phinewm] .= A[:phim]
    save(output_path, 0, dt, timesum, marknum, A)

    p = ErebusB200.params_from_module(E)
    capacity = ceil(Int, 1.25 * marknum) + 1024
    s = ErebusB200.create(p, capacity)
    mixed && ErebusB200.set_solver_options!(s; krylov=1, precond_fp32=1)
    # marker vectors at the capacity, so that replenishment's new markers
    # come back in place (the reference push!es them)
    m = Dict{Symbol,Any}()
    for k in ErebusB200.MARKER_FIELDS
        haskey(A, k) || continue
        resize!(A[k], capacity)
        m[k] = A[k]
    end
    g = Dict{Symbol,Any}(k => A[k] for k in ErebusB200.GRID_FIELDS)
    ErebusB200.upload_markers!(s, m, marknum)
    ErebusB200.upload_grid!(s, g)
    ErebusB200.set_time!(s, dt, timesum)
    for timestep = E.start_step:1:E.n_steps
        t0 = now()
        st = ErebusB200.step!(s, timestep)
        dt, timesum, marknum = st.dt, st.timesum, st.marknum
        if timestep % E.savematstep == 0
            marknum = ErebusB200.download_markers!(s, m)
            ErebusB200.download_grid!(s, g)
            save(output_path, timestep, dt, timesum, marknum, A)
        end
        @info "timestep $timestep computed in $(Dates.canonicalize(Dates.CompoundPeriod(now() - t0)))"
        @info "markers in use = $marknum, max T = $(st.maxT) K, thermochemical iterations $(st.titer)"
        timesum > E.endtime && break
    end
    ErebusB200.destroy!(s)
    return nothing
end

function run_simulation_b200()
    args = parse_commandline()
    output_path = args["output_path"]
    mkpath(output_path)
    io = open(joinpath(output_path, "Erebus_run.log"), "w+")
    global_logger(SimpleLogger(io))
    @info "=========== Erebus simulation run (B200 timestep) ==========="
    @info "writing results to $output_path"
    t1 = now()
    simulation_loop_b200(output_path; mixed=args["mixed"])
    @info "total run time = $(Dates.canonicalize(Dates.CompoundPeriod(now() - t1)))"
    close(io)
end

if abspath(PROGRAM_FILE) == @__FILE__
    run_simulation_b200()
end
