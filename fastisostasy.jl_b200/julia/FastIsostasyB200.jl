# FastIsostasyB200.jl -- Julia `ccall` shim over libfastiso_b200.so (include/fastiso_b200.h).
#
# Builds a B200 handle from a FastIsostasy `Simulation` (the reference's own constructors
# prepare every input: rigidity, effective viscosity, R, masks, reference state, ice
# history) and runs `run!` / `init_integrator` + `step!` semantics on the GPU.  Julia
# matrices are column-major with dimension 1 = x, which is the C ABI's layout, so arrays
# are passed without a transpose.  Not exercised by the test suite, which runs without Julia.
module FastIsostasyB200

using FastIsostasy

const LIB = get(ENV, "FASTISO_B200_LIB", joinpath(@__DIR__, "..", "lib", "libfastiso_b200.so"))

const FI_FORM_FP32 = Int32(0)
const FI_FORM_FP64 = Int32(1)

# field ids (fi_set_field / fi_get_field)
const F = (litho_rigidity = 0, effective_viscosity = 1, pseudodiff_scaling = 2, maskactive = 3,
           u_ref = 4, ue_ref = 5, dz_ss_ref = 6, z_b_ref = 7, u = 8, ue = 9, dudt = 10, dz_ss = 11,
           H_ice = 12, z_ss = 13, z_b = 14, H_af = 21, maskgrounded = 22, maskocean = 23, H_water = 24,
           columnanom_seawater = 25, tau = 26, u_eq = 27)

# fi_config, field for field (isbits: Julia lays it out as C does)
mutable struct FiConfig
    nx::Int32; ny::Int32
    Wx::Float64; Wy::Float64
    mE::Float64; r_pole::Float64; g::Float64; seconds_per_year::Float64
    rho_ice::Float64; rho_water::Float64; rho_seawater::Float64
    rho_litho::Float64; rho_uppermantle::Float64; litho_poissonratio::Float64
    lithosphere::Int32; lithosphere_column::Int32; sea_surface::Int32
    z_bsl::Float64
    bc_viscous_border::Float64; bc_elastic_border::Float64; bc_sea_surface_border::Float64
    ice_mode::Int32; ice_flat_bc::Int32
    t0::Float64; t1::Float64; reltol::Float64; abstol::Float64; dt_sparse_diagnostics::Float64
    max_steps::Int64
    form::Int32; device::Int32
    sealevel_load::Int32; bsl_mode::Int32; bsl_update::Int32
    volume_contribution::Int32; density_contribution::Int32; adjustment_contribution::Int32
    bsl_ref_A::Float64
    mantle::Int32; alg::Int32
    dt_min::Float64
end

FiConfig() = FiConfig(zeros(Int32, 2)..., zeros(12)..., zeros(Int32, 3)..., zeros(4)..., zeros(Int32, 2)...,
                      zeros(5)..., Int64(0), Int32(0), Int32(0), zeros(Int32, 6)..., 0.0, Int32(0), Int32(0), 0.0)

mutable struct B200Simulation
    sim::Any
    h::Ptr{Cvoid}
end

function check(rc::Cint, h::Ptr{Cvoid}, what)
    rc == 0 && return nothing
    msg = h == C_NULL ? "" : unsafe_string(ccall((:fi_last_error, LIB), Cstring, (Ptr{Cvoid},), h))
    error("$what failed ($rc): $msg")
end

set_field!(b::B200Simulation, id::Integer, X::AbstractMatrix) =
    check(ccall((:fi_set_field, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Csize_t),
                b.h, id, Array{Float64}(X), length(X)), b.h, "fi_set_field")

function getfield_b200(b::B200Simulation, id::Integer)
    d = b.sim.domain
    X = Matrix{Float64}(undef, d.nx, d.ny)
    check(ccall((:fi_get_field, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Csize_t), b.h, id, X, length(X)),
          b.h, "fi_get_field")
    return X
end

"""
    B200Simulation(sim, t_span; form = :fp32, device = 0, tiles = nothing, fft_schedules = Dict())

A GPU twin of `sim` over `t_span` (form :fp32 runs the laterally-variable ELVA path;
:fp64 also the ELRA, rigid-mantle and laterally-constant Maxwell rheologies), the
same tuple given to `Simulation`: the same inputs, run by libfastiso_b200.so.  `tiles =
(h_rows, B_cols)` and `fft_schedules = Dict(L => [radices...])` pass tuned settings
(fastiso_b200's `tuning/b200.json`) to fi_set_tiles / fi_set_fft_schedule.
"""
function B200Simulation(sim, t_span; form = :fp32, device = 0, tiles = nothing, fft_schedules = Dict())
    d, c, se, sl, bcs = sim.domain, sim.c, sim.solidearth, sim.sealevel, sim.bcs
    cfg = FiConfig()
    ccall((:fi_config_default, LIB), Cvoid, (Ref{FiConfig}, Int32, Int32, Float64, Float64), cfg, d.nx, d.ny,
          d.Wx, d.Wy)
    cfg.mE, cfg.r_pole, cfg.g, cfg.seconds_per_year = c.mE, c.r_pole, c.g, c.seconds_per_year
    cfg.rho_ice, cfg.rho_water, cfg.rho_seawater = c.rho_ice, c.rho_water, c.rho_seawater
    cfg.rho_litho, cfg.rho_uppermantle = se.rho_litho, se.rho_uppermantle
    cfg.litho_poissonratio = se.litho_poissonratio
    cfg.lithosphere = se.lithosphere isa RigidLithosphere ? Int32(1) :
                      se.lithosphere isa LaterallyConstantLithosphere ? Int32(2) : Int32(0)
    cfg.mantle = se.mantle isa RelaxedMantle ? Int32(1) : se.mantle isa RigidMantle ? Int32(2) : Int32(0)
    dq = sim.opts.diffeq
    cfg.alg = dq.dt_min isa Real ? Int32(1) : Int32(0)          # Euler with dt_min, else BS3
    cfg.dt_min = dq.dt_min isa Real ? Float64(dq.dt_min) : 0.0
    cfg.sealevel_load = sl.load isa InteractiveSealevelLoad ? Int32(1) : Int32(0)
    cfg.bsl_mode = sl.bsl isa ConstantOceanSurfaceBSL ? Int32(1) : sl.bsl isa PiecewiseConstantBSL ? Int32(2) :
                   sl.bsl isa ImposedBSL ? Int32(3) : Int32(0)
    cfg.bsl_update = sl.update_bsl isa ExternalBSLUpdate ? Int32(1) : Int32(0)
    cfg.volume_contribution = sl.volume_contribution isa FastIsostasy.NoVolumeContribution ? Int32(0) : Int32(1)
    cfg.density_contribution = sl.density_contribution isa FastIsostasy.NoDensityContribution ? Int32(0) : Int32(1)
    cfg.adjustment_contribution = sl.adjustment_contribution isa FastIsostasy.GoelzerAdjustmentContribution ?
                                  Int32(1) : Int32(0)
    sl.bsl isa CombinedBSL && error("CombinedBSL is not supported")
    cfg.z_bsl = Float64(sl.bsl.ref.z)
    cfg.bsl_ref_A = Float64(sl.bsl.ref.A)
    cfg.lithosphere_column = se.lithosphere_column isa CompressibleLithosphereColumn ? Int32(1) : Int32(0)
    cfg.sea_surface = sl.surface isa LaterallyVariableSeaSurface ? Int32(1) : Int32(0)
    cfg.bc_viscous_border = bcs.viscous_displacement.x_border
    cfg.bc_elastic_border = bcs.elastic_displacement.x_border
    cfg.bc_sea_surface_border = bcs.sea_surface_perturbation.x_border
    it = bcs.ice_thickness
    timeinterp = it isa TimeInterpolatedIceThickness
    cfg.ice_mode = timeinterp ? Int32(0) : Int32(1)
    cfg.t0, cfg.t1 = Float64(t_span[1]), Float64(t_span[2])
    cfg.form = form == :fp32 ? FI_FORM_FP32 : FI_FORM_FP64
    cfg.device = device
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:fi_create, LIB), Cint, (Ref{FiConfig}, Ref{Ptr{Cvoid}}), cfg, h), C_NULL, "fi_create")
    b = B200Simulation(sim, h[])
    finalizer(x -> ccall((:fi_destroy, LIB), Cvoid, (Ptr{Cvoid},), x.h), b)
    if tiles !== nothing && form == :fp32
        check(ccall((:fi_set_tiles, LIB), Cint, (Ptr{Cvoid}, Int32, Int32), b.h, tiles[1], tiles[2]),
              b.h, "fi_set_tiles")
    end
    for (L, r) in fft_schedules
        rr = Vector{Int32}(r)
        check(ccall((:fi_set_fft_schedule, LIB), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Int32}),
                    b.h, L, length(rr), rr), b.h, "fi_set_fft_schedule")
    end
    set_field!(b, F.litho_rigidity, se.litho_rigidity)
    set_field!(b, F.effective_viscosity, se.effective_viscosity)
    set_field!(b, F.pseudodiff_scaling, se.pseudodiff_scaling)
    set_field!(b, F.maskactive, Float64.(se.maskactive))
    set_field!(b, F.u_ref, sim.ref.u)
    set_field!(b, F.ue_ref, sim.ref.ue)
    set_field!(b, F.z_b_ref, sim.ref.z_b)
    set_field!(b, F.tau, se.tau)
    if sl.bsl isa PiecewiseConstantBSL
        z = Vector{Float64}(sl.bsl.ref.z_vec)
        A = Vector{Float64}([FastIsostasy.interpolate(zz, sl.bsl.ref.A_itp) for zz in z])
        check(ccall((:fi_set_ocean_surface_table, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}),
                    b.h, length(z), z, A), b.h, "fi_set_ocean_surface_table")
    elseif sl.bsl isa ImposedBSL
        t, z = Vector{Float64}(sl.bsl.t_vec), Vector{Float64}(sl.bsl.z_vec)
        check(ccall((:fi_set_bsl_history, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}),
                    b.h, length(t), t, z), b.h, "fi_set_bsl_history")
    end
    if timeinterp
        t = Vector{Float64}(it.t_vec)
        H = cat((Array{Float64}(X) for X in it.H_vec)...; dims = 3)
        check(ccall((:fi_set_ice_history, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}),
                    b.h, length(t), t, H), b.h, "fi_set_ice_history")
    end
    rm, GE = FastIsostasy.get_greenintegrand_coeffs(Float64)
    check(ccall((:fi_set_elastic_table, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}),
                b.h, length(rm), Vector{Float64}(rm), Vector{Float64}(GE)), b.h, "fi_set_elastic_table")
    check(ccall((:fi_init, LIB), Cint, (Ptr{Cvoid},), b.h), b.h, "fi_init")
    return b
end

"""run!(b): integrate t_span and fill b.sim.nout with u, ue, dudt and dz_ss at nout.t."""
function run!(b::B200Simulation)
    tout = Vector{Float64}(b.sim.nout.t)
    d = b.sim.domain
    n, k = d.nx * d.ny, length(tout)
    ot = zeros(k); U = zeros(n * k); UE = zeros(n * k); DU = zeros(n * k); DZ = zeros(n * k)
    check(ccall((:fi_run, LIB), Cint,
                (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                b.h, k, tout, ot, U, UE, DU, DZ), b.h, "fi_run")
    sl(A, i) = reshape(A[(i - 1) * n + 1:i * n], d.nx, d.ny)
    return (t = ot, u = [sl(U, i) for i in 1:k], ue = [sl(UE, i) for i in 1:k],
            dudt = [sl(DU, i) for i in 1:k], dz_ss = [sl(DZ, i) for i in 1:k])
end

"""init_integrator(b) and step!(b, dt): step!(integrator, dt, true) for coupling."""
function init_integrator(b::B200Simulation)
    ts = Vector{Float64}(b.sim.nout.t)
    check(ccall((:fi_init_integrator, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}), b.h, length(ts), ts),
          b.h, "fi_init_integrator")
    return b
end

step!(b::B200Simulation, dt::Real) =
    check(ccall((:fi_step, LIB), Cint, (Ptr{Cvoid}, Float64), b.h, dt), b.h, "fi_step")

"""Set the ice thickness of an externally updated load (coupling)."""
set_ice!(b::B200Simulation, H::AbstractMatrix) = set_field!(b, F.H_ice, H)

current_u(b::B200Simulation) = getfield_b200(b, F.u)

"""
    B200Ensemble(members::Vector{B200Simulation})

Members (FP32 form, each after init_integrator) advanced together by the persistent
ensemble kernel; `step!(e, dt)` is step!(integrator_m, dt, true) for every member and
returns the members' status codes (a failing member does not stop the others).
"""
mutable struct B200Ensemble
    members::Vector{B200Simulation}
    h::Ptr{Cvoid}
end

function B200Ensemble(members::Vector{B200Simulation})
    hs = [m.h for m in members]
    e = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:fi_ensemble_create, LIB), Cint, (Ptr{Ptr{Cvoid}}, Int32, Ref{Ptr{Cvoid}}), hs, length(hs), e)
    rc == 0 || error("fi_ensemble_create failed ($rc)")
    ens = B200Ensemble(members, e[])
    finalizer(x -> ccall((:fi_ensemble_destroy, LIB), Cvoid, (Ptr{Cvoid},), x.h), ens)
    return ens
end

function step!(e::B200Ensemble, dt::Real)
    status = zeros(Int32, length(e.members))
    rc = ccall((:fi_ensemble_step, LIB), Cint, (Ptr{Cvoid}, Float64, Ptr{Int32}), e.h, dt, status)
    rc == 0 || error("fi_ensemble_step failed ($rc)")
    return status
end

end  # module
