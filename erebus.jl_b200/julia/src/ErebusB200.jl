"""
    ErebusB200

Julia binding of liberebus_b200, the B200 implementation of Erebus.jl's
per-timestep marker-in-cell hot path (`simulation_loop`,
src/Erebus.jl:6370-7235).  Every entry point of include/erebus_b200.h is
wrapped here with `ccall`; the host arrays keep the reference's own layouts
(column-major `Matrix{Float64}`, `Matrix{Bool}` as bytes, marker `Vector`s
with `tm::Vector{Int}`), so the arrays `simulation_loop` allocates are passed
as they are.  The library owns all device memory; host arrays stay owned by
the caller and must stay rooted (`GC.@preserve`) around each call, which the
wrappers below do.

`heat_objective` is differentiable through `ChainRulesCore.rrule`, backed by
the library's hand-written adjoint (`erebus_adjoint_heat`).

The library path defaults to liberebus_b200.so in the directory that holds
this Julia package (erebus.jl_b200/); set `EREBUS_B200_LIB` to use another
build.
"""
module ErebusB200

import ChainRulesCore

export ErebusError, State, default_params, params_from_module, create, destroy!,
       set_solver_options!, upload_markers!, upload_grid!, download_markers!,
       download_grid!, markers_to_nodes!, gravity!, thermochemical_reaction!,
       hydromech_pass!, thermal_solve!, nodes_to_markers!, advect_rk4!, replenish!,
       step!, step_host!, heat_objective, factor_stats, markers_to_nodes_noalloc!

const liberebus = get(ENV, "EREBUS_B200_LIB",
                      normpath(joinpath(@__DIR__, "..", "..", "liberebus_b200.so")))

include("structs.jl")

# ---- status codes and errors (EREBUS_* in the header) -----------------------
const STATUS = Dict{Int32,String}(0 => "OK", 1 => "EINVAL", 2 => "ECUDA", 3 => "ENOMEM",
                                  4 => "ECAPACITY", 5 => "ENOCONV", 6 => "ENONFINITE",
                                  7 => "ENODEVICE")

"""Raised when an entry point returns a non-zero status (the reference throws
a `String` where it detects an error; the library reports codes)."""
struct ErebusError <: Exception
    fn::String
    code::Int32
    msg::String
end
Base.showerror(io::IO, e::ErebusError) =
    print(io, e.fn, " failed: ", get(STATUS, e.code, "status $(e.code)"),
          isempty(e.msg) ? "" : ": " * e.msg)

"""The device state of one planetesimal (an `erebus_state*`)."""
mutable struct State
    ptr::Ptr{Cvoid}
    capacity::Int64
    nodes::Int64          # P nodes, (Ny + 1) * (Nx + 1)
end

s_nodes(s::State) = s.nodes

last_error(h::Ptr{Cvoid}) =
    h == C_NULL ? "" : unsafe_string(ccall((:erebus_last_error, liberebus), Cstring,
                                           (Ptr{Cvoid},), h))

function check(fn::AbstractString, h, rc::Integer)
    rc == 0 && return nothing
    throw(ErebusError(String(fn), Int32(rc), last_error(h isa State ? h.ptr : h)))
end

# ---- parameters ----------------------------------------------------------------
"""ErebusParams with the values of src/constants.jl for an Nx x Ny grid."""
function default_params(Nx::Integer, Ny::Integer)
    p = Ref{ErebusParams}()
    check("erebus_default_params", C_NULL,
          ccall((:erebus_default_params, liberebus), Cint, (Ptr{ErebusParams}, Int32, Int32),
                p, Nx, Ny))
    return p[]
end

# ErebusParams fields whose src/constants.jl names are spelled differently
const CONSTANT_NAMES = Dict(:Lf => :Lᶠ, :MH2O => :MH₂O, :rhoDs => :ρDˢ, :rhoWs => :ρWˢ,
                            :rhoH2Of => :ρH₂Oᶠ, :rhoH2Ofi => :ρH₂Oᶠⁱ, :dHWD => :ΔHWD,
                            :dSWD => :ΔSWD, :dtreaction => :Δtreaction)

_pvalue(::Type{T}, v) where {T<:Real} = T(v)
_pvalue(::Type{NTuple{N,T}}, v) where {N,T} = ntuple(i -> T(v[i]), N)

"""
    params_from_module(M::Module = Main.Erebus)

ErebusParams holding the module globals of the reference (src/constants.jl,
read as `M.<name>`), for the grid and physics the reference was loaded with.
Fields with no counterpart there (the per-marker viscosity switch, the
seed) keep the library's defaults."""
function params_from_module(M::Module)
    base = default_params(getfield(M, :Nx), getfield(M, :Ny))
    vals = map(fieldnames(ErebusParams)) do f
        T = fieldtype(ErebusParams, f)
        name = get(CONSTANT_NAMES, f, f)
        isdefined(M, name) ? _pvalue(T, getfield(M, name)) : getfield(base, f)
    end
    p = ErebusParams(vals...)
    check("erebus_check_params", C_NULL,
          ccall((:erebus_check_params, liberebus), Cint, (Ref{ErebusParams},), p))
    return p
end

function default_solver_options()
    o = Ref{ErebusSolverOptions}()
    check("erebus_default_solver_options", C_NULL,
          ccall((:erebus_default_solver_options, liberebus), Cint,
                (Ptr{ErebusSolverOptions},), o))
    return o[]
end

# ---- lifecycle -----------------------------------------------------------------
"""Creates the device state (replaces the setup_* allocators, E:55-592)."""
function create(p::ErebusParams, capacity::Integer)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check("erebus_create", C_NULL,
          ccall((:erebus_create, liberebus), Cint, (Ref{ErebusParams}, Int64, Ptr{Ptr{Cvoid}}),
                p, capacity, h))
    s = State(h[], Int64(capacity), Int64(p.Nx + 1) * Int64(p.Ny + 1))
    finalizer(destroy!, s)
    return s
end

function destroy!(s::State)
    if s.ptr != C_NULL
        ccall((:erebus_destroy, liberebus), Cint, (Ptr{Cvoid},), s.ptr)
        s.ptr = C_NULL
    end
    return nothing
end

"""Solver controls; keywords are ErebusSolverOptions fields, e.g.
`set_solver_options!(s; krylov = 1, precond_fp32 = 1)` for the
mixed-precision Krylov mode."""
function set_solver_options!(s::State; kw...)
    o = default_solver_options()
    vals = map(f -> haskey(kw, f) ? fieldtype(ErebusSolverOptions, f)(kw[f]) : getfield(o, f),
               fieldnames(ErebusSolverOptions))
    check("erebus_set_solver_options", s,
          ccall((:erebus_set_solver_options, liberebus), Cint,
                (Ptr{Cvoid}, Ref{ErebusSolverOptions}), s.ptr, ErebusSolverOptions(vals...)))
end

function factor_stats(s::State, system::Integer)
    o = Ref{ErebusFactorStats}()
    check("erebus_factor_stats", s,
          ccall((:erebus_factor_stats, liberebus), Cint, (Ptr{Cvoid}, Int32,
                                                           Ptr{ErebusFactorStats}),
                s.ptr, system, o))
    return o[]
end

# ---- host views ------------------------------------------------------------------
_ptr(::Type{Ptr{T}}, a::AbstractArray) where {T} = Ptr{T}(pointer(a))
_ptr(::Type{Ptr{T}}, ::Nothing) where {T} = Ptr{T}(C_NULL)

"""ErebusMarkersHost pointing into the marker vectors `m` (a NamedTuple or
Dict keyed by the reference's names: xm, ym, tm, tkm, ...).  `etasolidm_m`
may be absent (per-marker viscosity off)."""
function markers_struct(m)
    ErebusMarkersHost(map(f -> _ptr(fieldtype(ErebusMarkersHost, f), get(m, f, nothing)),
                          MARKER_FIELDS)...)
end

"""ErebusGridHost pointing into the node arrays `g` (keyed by the
reference's names: ETA, ETA0, GGG, ..., tk0)."""
grid_struct(g) = ErebusGridHost(map(f -> _ptr(fieldtype(ErebusGridHost, f), g[f]),
                                    GRID_FIELDS)...)

sums_struct(sm) = ErebusSumsHost(map(f -> _ptr(fieldtype(ErebusSumsHost, f), sm[f]),
                                     SUM_FIELDS)...)

function upload_markers!(s::State, m, marknum::Integer)
    GC.@preserve m check("erebus_upload_markers", s,
        ccall((:erebus_upload_markers, liberebus), Cint,
              (Ptr{Cvoid}, Ref{ErebusMarkersHost}, Int64), s.ptr, markers_struct(m), marknum))
end

function upload_grid!(s::State, g)
    GC.@preserve g check("erebus_upload_grid", s,
        ccall((:erebus_upload_grid, liberebus), Cint, (Ptr{Cvoid}, Ref{ErebusGridHost}),
              s.ptr, grid_struct(g)))
end

"""Copies the markers back (the vectors must hold `capacity` entries, as
replenishment appends markers); returns marknum."""
function download_markers!(s::State, m)
    n = Ref{Int64}(0)
    GC.@preserve m check("erebus_download_markers", s,
        ccall((:erebus_download_markers, liberebus), Cint,
              (Ptr{Cvoid}, Ref{ErebusMarkersHost}, Ptr{Int64}), s.ptr, markers_struct(m), n))
    return n[]
end

function download_grid!(s::State, g)
    GC.@preserve g check("erebus_download_grid", s,
        ccall((:erebus_download_grid, liberebus), Cint, (Ptr{Cvoid}, Ref{ErebusGridHost}),
              s.ptr, grid_struct(g)))
end

function set_time!(s::State, dt::Real, timesum::Real)
    check("erebus_set_time", s,
          ccall((:erebus_set_time, liberebus), Cint, (Ptr{Cvoid}, Float64, Float64),
                s.ptr, dt, timesum))
end

# ---- the reference's phases (same semantics as the Julia functions) ----------------
"""calculate_radioactive_heating, compute_marker_properties!, the four
marker_to_*_nodes!, compute_*_node_properties! and
apply_insulating_boundary_conditions! (E:6376-6604)."""
markers_to_nodes!(s::State, timesum::Real) =
    check("erebus_markers_to_nodes", s,
          ccall((:erebus_markers_to_nodes, liberebus), Cint, (Ptr{Cvoid}, Float64),
                s.ptr, timesum))

"""assemble_gravitational_lse!, LP \\ RP, process_gravitational_solution!
(E:6610-6614)."""
function gravity!(s::State)
    st = Ref{ErebusSolveStats}()
    check("erebus_gravity", s, ccall((:erebus_gravity, liberebus), Cint,
                                     (Ptr{Cvoid}, Ptr{ErebusSolveStats}), s.ptr, st))
    return st[]
end

"""perform_thermochemical_reaction! (E:2558-2694)."""
thermochemical_reaction!(s::State, dt::Real, timestep::Integer, titer::Integer) =
    check("erebus_thermochemical_reaction", s,
          ccall((:erebus_thermochemical_reaction, liberebus), Cint,
                (Ptr{Cvoid}, Float64, Int32, Int32), s.ptr, dt, timestep, titer))

"""One plastic pass (E:6678-6869); returns (dt, converged, solve stats)."""
function hydromech_pass!(s::State, dt::Real, iplast::Integer)
    d = Ref{Float64}(dt)
    conv = Ref{Int32}(0)
    st = Ref{ErebusSolveStats}()
    check("erebus_hydromech_pass", s,
          ccall((:erebus_hydromech_pass, liberebus), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Int32, Ptr{Int32}, Ptr{ErebusSolveStats}),
                s.ptr, d, iplast, conv, st))
    return d[], conv[] != 0, st[]
end

"""Shear and adiabatic heating, assemble_thermal_lse!, the heat solve and DT
(E:6887-6927); returns max|DT|."""
function thermal_solve!(s::State, dt::Real, timestep::Integer)
    mx = Ref{Float64}(0.0)
    st = Ref{ErebusSolveStats}()
    check("erebus_thermal_solve", s,
          ccall((:erebus_thermal_solve, liberebus), Cint,
                (Ptr{Cvoid}, Float64, Int32, Ptr{Float64}, Ptr{ErebusSolveStats}),
                s.ptr, dt, timestep, mx, st))
    return mx[]
end

"""Marker viscosity, stress, temperature, porosity and melt composition
(E:6945-7019)."""
nodes_to_markers!(s::State, dt::Real, timestep::Integer) =
    check("erebus_nodes_to_markers", s,
          ccall((:erebus_nodes_to_markers, liberebus), Cint, (Ptr{Cvoid}, Float64, Int32),
                s.ptr, dt, timestep))

"""compute_velocities!, compute_rotation_rate!, move_markers_rk4!,
backtrace_pressures_rk4! (E:7026-7059)."""
advect_rk4!(s::State, dt::Real) =
    check("erebus_advect_rk4", s,
          ccall((:erebus_advect_rk4, liberebus), Cint, (Ptr{Cvoid}, Float64), s.ptr, dt))

"""replenish_markers! (E:5586-5698); returns the new marknum."""
function replenish!(s::State, timestep::Integer)
    n = Ref{Int64}(0)
    check("erebus_replenish", s,
          ccall((:erebus_replenish, liberebus), Cint, (Ptr{Cvoid}, Int32, Ptr{Int64}),
                s.ptr, timestep, n))
    return n[]
end

"""One iteration of the `for timestep` loop (E:6370-7235) on the device
state; returns ErebusStepStats (dt, timesum, marknum, iterations, ...)."""
function step!(s::State, timestep::Integer)
    st = Ref{ErebusStepStats}()
    check("erebus_step", s, ccall((:erebus_step, liberebus), Cint,
                                  (Ptr{Cvoid}, Int32, Ptr{ErebusStepStats}),
                                  s.ptr, timestep, st))
    return st[]
end

"""One timestep on host arrays: upload `m`/`g`, step, copy the state back
into the same arrays.  The drop-in for the body of the reference's timestep
loop; returns ErebusStepStats."""
function step_host!(s::State, timestep::Integer, m, marknum::Integer, g)
    n = Ref{Int64}(0)
    st = Ref{ErebusStepStats}()
    GC.@preserve m g begin
        ms, gs = markers_struct(m), grid_struct(g)
        check("erebus_step_host", s,
              ccall((:erebus_step_host, liberebus), Cint,
                    (Ptr{Cvoid}, Int32, Ref{ErebusMarkersHost}, Int64, Ref{ErebusGridHost},
                     Ref{ErebusMarkersHost}, Ptr{Int64}, Ref{ErebusGridHost},
                     Ptr{ErebusStepStats}),
                    s.ptr, timestep, ms, marknum, gs, ms, n, gs, st))
    end
    return st[]
end

# ---- diagnostics and helpers (no reference counterpart) ------------------------------
"""Byte offsets of the grid arrays in one block (each at the next 256-byte
boundary) and the block size: host grids laid out so move in one transfer."""
function grid_layout(p::ErebusParams)
    off = zeros(Int64, length(GRID_FIELDS))
    total = Ref{Int64}(0)
    check("erebus_grid_layout", C_NULL,
          ccall((:erebus_grid_layout, liberebus), Cint, (Ref{ErebusParams}, Ptr{Int64},
                                                          Ptr{Int64}), p, off, total))
    return off, total[]
end

share_solver_stream!(s::State, on::Bool=true) =
    check("erebus_share_solver_stream", s,
          ccall((:erebus_share_solver_stream, liberebus), Cint, (Ptr{Cvoid}, Int32),
                s.ptr, on ? 1 : 0))

function download_sums!(s::State, sm)
    GC.@preserve sm check("erebus_download_sums", s,
        ccall((:erebus_download_sums, liberebus), Cint, (Ptr{Cvoid}, Ref{ErebusSumsHost}),
              s.ptr, sums_struct(sm)))
end

function get_time(s::State)
    dt, t = Ref{Float64}(0), Ref{Float64}(0)
    check("erebus_get_time", s, ccall((:erebus_get_time, liberebus), Cint,
                                      (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}), s.ptr, dt, t))
    return dt[], t[]
end

"""The Stokes-Darcy matrix (COO, 0-based) and right-hand side that
assemble_hydromechanical_lse! (E:3089-3572) builds for the current state."""
function export_hydromech(s::State, dt::Real)
    n = 6 * Int64(s_nodes(s))
    rows, cols, vals = zeros(Int64, 12n), zeros(Int64, 12n), zeros(Float64, 12n)
    R = zeros(Float64, n)
    nnz = Ref{Int64}(0)
    check("erebus_export_hydromech", s,
          ccall((:erebus_export_hydromech, liberebus), Cint,
                (Ptr{Cvoid}, Float64, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Float64},
                 Ptr{Float64}), s.ptr, dt, nnz, rows, cols, vals, R))
    k = nnz[]
    return rows[1:k], cols[1:k], vals[1:k], R
end

"""y = L x with the Stokes-Darcy matrix of the current state."""
function apply_hydromech!(s::State, dt::Real, x::Vector{Float64}, y::Vector{Float64})
    check("erebus_apply_hydromech", s,
          ccall((:erebus_apply_hydromech, liberebus), Cint,
                (Ptr{Cvoid}, Float64, Ptr{Float64}, Ptr{Float64}), s.ptr, dt, x, y))
end

function kernel_launches(s::State)
    n = Ref{Int64}(0)
    check("erebus_kernel_launches", s, ccall((:erebus_kernel_launches, liberebus), Cint,
                                             (Ptr{Cvoid}, Ptr{Int64}), s.ptr, n))
    return n[]
end

function host_syncs(s::State)
    n = Ref{Int64}(0)
    check("erebus_host_syncs", s, ccall((:erebus_host_syncs, liberebus), Cint,
                                        (Ptr{Cvoid}, Ptr{Int64}), s.ptr, n))
    return n[]
end

function get_stream(s::State)
    st = Ref{Ptr{Cvoid}}(C_NULL)
    check("erebus_get_stream", s, ccall((:erebus_get_stream, liberebus), Cint,
                                        (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}), s.ptr, st))
    return st[]
end

enable_phase_timing!(s::State, on::Bool=true) =
    check("erebus_enable_phase_timing", s,
          ccall((:erebus_enable_phase_timing, liberebus), Cint, (Ptr{Cvoid}, Int32),
                s.ptr, on ? 1 : 0))

const PHASES = (:markers_to_nodes, :gravity, :reaction, :hydro_assemble, :hydro_factor,
                :hydro_solve, :hydro_post, :thermal_assemble, :thermal_factor, :thermal_solve,
                :nodes_to_markers, :rk4, :backtrace, :replenish, :scatter_merge,
                :hydro_precond)

"""Per-phase device milliseconds and launch counts since timing was enabled."""
function phase_times(s::State)
    n = length(PHASES)
    ms, cnt = zeros(Float64, n), zeros(Int64, n)
    check("erebus_phase_times", s, ccall((:erebus_phase_times, liberebus), Cint,
                                         (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int64}, Int32),
                                         s.ptr, ms, cnt, n))
    return Dict(PHASES[i] => (ms[i], cnt[i]) for i in 1:n)
end

# ---- snapshots ---------------------------------------------------------------------
"""Starts copying the state into `g`/`m` (page-locked host arrays for the
copy to overlap the next timestep); `snapshot_wait!` returns (marknum, dt,
timesum) once the copy is complete.  The arrays then feed the reference's
save_state (E:5718-5960).  The caller keeps `g` and `m` rooted until
`snapshot_wait!` has returned."""
function snapshot_begin!(s::State, g, m)
    check("erebus_snapshot_begin", s,
          ccall((:erebus_snapshot_begin, liberebus), Cint,
                (Ptr{Cvoid}, Ref{ErebusGridHost}, Ref{ErebusMarkersHost}),
                s.ptr, grid_struct(g), markers_struct(m)))
end

function snapshot_wait!(s::State)
    n, dt, t = Ref{Int64}(0), Ref{Float64}(0), Ref{Float64}(0)
    check("erebus_snapshot_wait", s,
          ccall((:erebus_snapshot_wait, liberebus), Cint,
                (Ptr{Cvoid}, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}), s.ptr, n, dt, t))
    return n[], dt[], t[]
end

# ---- allocation-free pass ------------------------------------------------------------
"""The marker -> node pass on caller-owned device buffers (device pointers in
`md`/`gd`, an ErebusMarkersHost / ErebusGridHost of device addresses, e.g.
from CUDA.jl arrays), allocating nothing; `stream` is a cudaStream_t."""
markers_to_nodes_noalloc!(p::ErebusParams, md::ErebusMarkersHost, marknum::Integer,
                          gd::ErebusGridHost, timesum::Real, stream::Ptr{Cvoid}=C_NULL) =
    check("erebus_markers_to_nodes_noalloc", C_NULL,
          ccall((:erebus_markers_to_nodes_noalloc, liberebus), Cint,
                (Ref{ErebusParams}, Ref{ErebusMarkersHost}, Int64, Ref{ErebusGridHost},
                 Float64, Ptr{Cvoid}), p, md, marknum, gd, timesum, stream))

# ---- adjoint ---------------------------------------------------------------------------
"""
    heat_objective(s, m, marknum, g, phim, n_steps; checkpoint_every = 5)

J after `n_steps` timesteps from the host state (`m`, `g`) with the marker
porosities `phim`: the mean over the basic nodes inside the body of the
4-P-node average of tk2.  Differentiable with respect to `phim` (and the
26Al/27Al ratio, through the gradient the rrule returns) for states at
mechanical rest (the scope of erebus_adjoint_heat)."""
function heat_objective(s::State, m, marknum::Integer, g, phim::AbstractVector{Float64},
                        n_steps::Integer; checkpoint_every::Integer=5)
    J, _, _ = heat_objective_and_gradient(s, m, marknum, g, phim, n_steps;
                                          checkpoint_every=checkpoint_every)
    return J
end

function heat_objective_and_gradient(s::State, m, marknum::Integer, g,
                                     phim::AbstractVector{Float64}, n_steps::Integer;
                                     checkpoint_every::Integer=5)
    m[:phim][1:marknum] .= phim[1:marknum]
    m[:phinewm][1:marknum] .= phim[1:marknum]
    upload_markers!(s, m, marknum)
    upload_grid!(s, g)
    J, dr = Ref{Float64}(0), Ref{Float64}(0)
    dphim = zeros(Float64, s.capacity)
    st = Ref{ErebusAdjointStats}()
    check("erebus_adjoint_heat", s,
          ccall((:erebus_adjoint_heat, liberebus), Cint,
                (Ptr{Cvoid}, Int32, Int32, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                 Ptr{ErebusAdjointStats}),
                s.ptr, 1, n_steps, checkpoint_every, J, dphim, dr, st))
    return J[], dphim[1:marknum], dr[]
end

function ChainRulesCore.rrule(::typeof(heat_objective), s::State, m, marknum::Integer, g,
                              phim::AbstractVector{Float64}, n_steps::Integer;
                              checkpoint_every::Integer=5)
    J, dphim, _ = heat_objective_and_gradient(s, m, marknum, g, phim, n_steps;
                                              checkpoint_every=checkpoint_every)
    nt = ChainRulesCore.NoTangent()
    pullback(dJ) = (nt, nt, nt, nt, nt, dJ .* dphim, nt)
    return J, pullback
end

end # module ErebusB200
