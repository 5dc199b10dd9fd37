# GeoDynamoB200.jl -- ccall shim that puts libgdb200.so (B200, sm_100a) behind
# GeoDynamo.jl's transform, nonlinear and time-step functions.
#
# Usage from a GeoDynamo.jl session (as a package, so that loading
# ChainRulesCore also loads the reverse-mode rule of ext/):
#     using Pkg; Pkg.develop(path = joinpath(path_to_repo, "geodynamo.jl_b200", "julia", "GeoDynamoB200"))
#     using GeoDynamoB200
#     GeoDynamoB200.install!(GeoDynamo)          # overloads the methods below
# or, without the package manager,
#     include(joinpath(path_to_repo, "geodynamo.jl_b200", "julia", "GeoDynamoB200", "src", "GeoDynamoB200.jl"))
#
# Array layouts need no conversion: GeoDynamo's spectral planes
# (nlm, 1, nr) and physical fields (nlat, nlon, nr) are column-major, which is
# the library's host layout (lm fastest / theta fastest).  Every call borrows
# the arrays for its duration (GC.@preserve) and reports errors by throwing,
# as the reference does.
module GeoDynamoB200

const LIB = normpath(joinpath(@__DIR__, "..", "..", "..", "libgdb200.so"))

# gd_config (include/gdb200.h)
struct GDConfig
    lmax::Cint; mmax::Cint; nlat::Cint; nlon::Cint; nr::Cint; kl::Cint
    rratio::Cdouble; ekman::Cdouble; rayleigh::Cdouble; prandtl::Cdouble; magnetic_prandtl::Cdouble
    dt::Cdouble; implicit_theta::Cdouble
    ab_mode::Cint; bc_mode::Cint; fd_mode::Cint; precision::Cint; magnetic::Cint
    composition::Cint; schmidt::Cdouble
    segments::Cint; geometry::Cint; r_outer::Cdouble
    segment_nr::Ptr{Cint}
end

mutable struct Handle
    ptr::Ptr{Cvoid}
end

const FIELD = Dict(:u_tor => 0, :u_pol => 1, :b_tor => 2, :b_pol => 3, :temp => 4, :comp => 5)

lasterror(h::Handle) = unsafe_string(ccall((:gd_last_error, LIB), Cstring, (Ptr{Cvoid},), h.ptr))
check(h::Handle, st::Cint) = st == 0 ? nothing : error("libgdb200 status $st: $(lasterror(h))")

function create(cfg::GDConfig; device::Integer = 0)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    st = ccall((:gd_create, LIB), Cint, (Ref{GDConfig}, Cint, Ref{Ptr{Cvoid}}), cfg, device, out)
    st == 0 || error("gd_create failed with status $st")
    h = Handle(out[])
    finalizer(x -> ccall((:gd_destroy, LIB), Cint, (Ptr{Cvoid},), x.ptr), h)
    return h
end

# One handle per (transform config, nr, precision), built from GeoDynamo's
# parameters (src/parameters.jl:14-76) on first use.
const HANDLES = Dict{Tuple{UInt,Int,Int},Handle}()

function handle_for(GD, config, nr::Integer; precision::Integer = 0, composition::Bool = false)
    key = (objectid(config), Int(nr), Int(precision) + 2 * Int(composition))
    get!(HANDLES, key) do
        # a ball (geometry = :ball) steps with the boundary-row operator (bc_mode 2):
        # the reference's own operator holds 1/r at r = 0
        ball = GD.geometry === :ball
        cfg = GDConfig(config.lmax, config.mmax, config.nlat, config.nlon, nr, GD.i_KL,
                       GD.d_rratio, GD.d_E, GD.d_Ra, GD.d_Pr, GD.d_Pm, GD.d_timestep, GD.d_implicit,
                       0, ball ? 2 : 0, 0, precision, GD.i_B, composition ? 1 : 0, composition ? GD.d_Sc : 1.0, 0,
                       ball ? 1 : 0, ball ? GD.d_R_outer : 1.0, C_NULL)
        create(cfg)
    end
end

# The mixed-precision step's velocity chain at FP64 accuracy (gd_set_fp64_stages
# with GD_STAGE_VEL_PRODUCTS | GD_STAGE_VEL_ANALYSIS and either the DMMA
# synthesis, GD_STAGE_VEL_SYNTH = 1, or the int8-slice synthesis on the tensor
# cores, GD_STAGE_VEL_SYNTH_I8 = 8, with `digits` 7-bit digits per operand).
function velocity_chain_fp64!(h::Handle; int8::Bool = true, digits::Integer = 6)
    int8 && check(h, ccall((:gd_set_int8_digits, LIB), Cint, (Ptr{Cvoid}, Cint), h.ptr, digits))
    mask = (int8 ? 8 : 1) | 2 | 4
    check(h, ccall((:gd_set_fp64_stages, LIB), Cint, (Ptr{Cvoid}, Cint), h.ptr, mask))
    return h
end

# shtnskit_spectral_to_physical! (src/shtnskit_field_functions.jl:11)
function spectral_to_physical!(h::Handle, spec, phys)
    re = parent(spec.data_real); im = parent(spec.data_imag); g = parent(phys.data)
    GC.@preserve re im g check(h, ccall((:gd_spectral_to_physical, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, 1, re, im, g))
    return phys
end

# shtnskit_physical_to_spectral! (:131)
function physical_to_spectral!(h::Handle, phys, spec)
    re = parent(spec.data_real); im = parent(spec.data_imag); g = parent(phys.data)
    GC.@preserve re im g check(h, ccall((:gd_physical_to_spectral, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, 1, g, re, im))
    return spec
end

# shtnskit_vector_synthesis!(tor, pol, vec) (:252): only theta/phi are written
function vector_synthesis!(h::Handle, tor, pol, vec)
    tr = parent(tor.data_real); ti = parent(tor.data_imag)
    pr = parent(pol.data_real); pi = parent(pol.data_imag)
    vt = parent(vec.θ_component.data); vp = parent(vec.φ_component.data)
    GC.@preserve tr ti pr pi vt vp check(h, ccall((:gd_vector_synthesis, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, tr, ti, pr, pi, vt, vp))
    return vec
end

# shtnskit_vector_analysis!(vec, tor, pol) (:291)
function vector_analysis!(h::Handle, vec, tor, pol)
    tr = parent(tor.data_real); ti = parent(tor.data_imag)
    pr = parent(pol.data_real); pi = parent(pol.data_imag)
    vt = parent(vec.θ_component.data); vp = parent(vec.φ_component.data)
    GC.@preserve tr ti pr pi vt vp check(h, ccall((:gd_vector_analysis, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, vt, vp, tr, ti, pr, pi))
    return tor, pol
end

# ball_physical_to_spectral! / ball_vector_analysis! (src/Ball/Ball.jl:214-245):
# the analyses, then the first radial level set to 0 for l >= 1 on the device
function ball_physical_to_spectral!(h::Handle, phys, spec)
    re = parent(spec.data_real); im = parent(spec.data_imag); g = parent(phys.data)
    GC.@preserve re im g check(h, ccall((:gd_ball_physical_to_spectral, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, 1, g, re, im))
    return spec
end

function ball_vector_analysis!(h::Handle, vec, tor, pol)
    tr = parent(tor.data_real); ti = parent(tor.data_imag)
    pr = parent(pol.data_real); pi = parent(pol.data_imag)
    vt = parent(vec.θ_component.data); vp = parent(vec.φ_component.data)
    GC.@preserve tr ti pr pi vt vp check(h, ccall((:gd_ball_vector_analysis, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, vt, vp, tr, ti, pr, pi))
    return tor, pol
end

# compute_temperature_nonlinear!(temp, vel, oc) (src/thermal.jl:149): the
# Dirichlet values and sources of temp go to the handle, then one call
# (gd_compute_temperature_nonlinear) fills temp.nonlinear, applies the boundary
# rows to temp.spectral and writes the temperature grid.
function temperature_nonlinear!(h::Handle, temp, vel)
    scalar_bc_types!(h, FIELD[:temp], temp)
    bv = Matrix{Float64}(permutedims(temp.boundary_values))   # [nlm, 2] = C's [2][nlm]
    src = Vector{Float64}(temp.internal_sources)
    GC.@preserve bv src check(h, ccall((:gd_set_temperature_bc, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, bv, src))
    tr = parent(temp.spectral.data_real); ti = parent(temp.spectral.data_imag)
    ut = parent(vel.velocity.θ_component.data); up = parent(vel.velocity.φ_component.data)
    nr = parent(temp.nonlinear.data_real); ni = parent(temp.nonlinear.data_imag)
    tg = parent(temp.temperature.data)
    GC.@preserve tr ti ut up nr ni tg check(h, ccall((:gd_compute_temperature_nonlinear, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, tr, ti, ut, up, nr, ni, tg))
    return temp
end

# bc_type_inner / bc_type_outer of a scalar field (1 fixed value, 2 flux) to the handle
function scalar_bc_types!(h::Handle, field::Integer, f)
    ti = Vector{Cint}(f.bc_type_inner); to = Vector{Cint}(f.bc_type_outer)
    GC.@preserve ti to check(h, ccall((:gd_set_scalar_bc_types, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cint}, Ptr{Cint}), h.ptr, field, ti, to))
end

# compute_composition_nonlinear!(comp, vel, oc) (src/compositional.jl:219): the
# boundary types, values (or fluxes) and sources of comp go to the handle, then
# gd_compute_composition_nonlinear fills comp.nonlinear, applies the boundary
# conditions to comp.spectral and writes the composition grid.
function composition_nonlinear!(h::Handle, comp, vel)
    scalar_bc_types!(h, FIELD[:comp], comp)
    bv = Matrix{Float64}(permutedims(comp.boundary_values))
    src = Vector{Float64}(comp.internal_sources)
    GC.@preserve bv src check(h, ccall((:gd_set_composition_bc, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, bv, src))
    cr = parent(comp.spectral.data_real); ci = parent(comp.spectral.data_imag)
    ut = parent(vel.velocity.θ_component.data); up = parent(vel.velocity.φ_component.data)
    nr = parent(comp.nonlinear.data_real); ni = parent(comp.nonlinear.data_imag)
    cg = parent(comp.composition.data)
    GC.@preserve cr ci ut up nr ni cg check(h, ccall((:gd_compute_composition_nonlinear, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, cr, ci, ut, up, nr, ni, cg))
    return comp
end

# compute_velocity_nonlinear!(fields, temp, comp, mag, domain) (src/velocity.jl:312):
# the Lorentz term reads mag's current and field grids (C_NULL without mag).
function velocity_nonlinear!(h::Handle, fields, mag)
    tr = parent(fields.toroidal.data_real); ti = parent(fields.toroidal.data_imag)
    pr = parent(fields.poloidal.data_real); pi = parent(fields.poloidal.data_imag)
    nt = parent(fields.nl_toroidal.data_real); nti = parent(fields.nl_toroidal.data_imag)
    np = parent(fields.nl_poloidal.data_real); npi = parent(fields.nl_poloidal.data_imag)
    ut = parent(fields.velocity.θ_component.data); up = parent(fields.velocity.φ_component.data)
    grids = mag === nothing ? (C_NULL, C_NULL, C_NULL, C_NULL) :
        (pointer(parent(mag.current.θ_component.data)), pointer(parent(mag.current.φ_component.data)),
         pointer(parent(mag.magnetic.θ_component.data)), pointer(parent(mag.magnetic.φ_component.data)))
    GC.@preserve tr ti pr pi nt nti np npi ut up mag check(h, ccall((:gd_compute_velocity_nonlinear, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
         Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
         Ptr{Cdouble}),
        h.ptr, tr, ti, pr, pi, grids..., nt, nti, np, npi, ut, up))
    return fields
end

# compute_magnetic_nonlinear!(mag, vel, oc, ic, rot) (src/magnetic.jl:131)
function magnetic_nonlinear!(h::Handle, mag, vel)
    tr = parent(mag.toroidal.data_real); ti = parent(mag.toroidal.data_imag)
    pr = parent(mag.poloidal.data_real); pi = parent(mag.poloidal.data_imag)
    ut = parent(vel.velocity.θ_component.data); up = parent(vel.velocity.φ_component.data)
    nt = parent(mag.nl_toroidal.data_real); nti = parent(mag.nl_toroidal.data_imag)
    np = parent(mag.nl_poloidal.data_real); npi = parent(mag.nl_poloidal.data_imag)
    bt = parent(mag.magnetic.θ_component.data); bp = parent(mag.magnetic.φ_component.data)
    jt = parent(mag.current.θ_component.data); jp = parent(mag.current.φ_component.data)
    GC.@preserve tr ti pr pi ut up nt nti np npi bt bp jt jp check(h, ccall((:gd_compute_magnetic_nonlinear, LIB),
        Cint, (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
               Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
               Ptr{Cdouble}),
        h.ptr, tr, ti, pr, pi, ut, up, nt, nti, np, npi, bt, bp, jt, jp))
    return mag
end

# Device copies of SHTnsImplicitMatrices (src/timestep.jl:489-496) for
# build_rhs_cnab2! / solve_implicit_step!, made by gd_create_timestepping_matrices
# from the reference struct's own parameters: theta is stored; 1/dt is the
# l = 0 system diagonal plus theta times the l = 0 operator diagonal; the
# diffusivity is (L_0 - L_1) diagonal x r^2 / 2 at the outer node
# (L_l = nu (lap - l(l+1)/r^2)).  Cached per matrices object.
mutable struct DeviceMatrices
    ptr::Ptr{Cvoid}
    h::Handle
end
const MATRICES = IdDict{Any,DeviceMatrices}()

function device_matrices(h::Handle, M, nr::Integer, KL::Integer)
    get!(MATRICES, M) do
        i0 = M.lookup[0]; i1 = M.lookup[1]
        r = zeros(nr); check(h, ccall((:gd_grid, LIB), Cint, (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
                                      h.ptr, C_NULL, C_NULL, r))
        L0 = M.linear_matrices[i0].data; L1 = M.linear_matrices[i1].data; S0 = M.system_matrices[i0].data
        theta = M.theta
        dt = 1.0 / (S0[KL + 1, nr] + theta * L0[KL + 1, nr])
        nu = (L0[KL + 1, nr] - L1[KL + 1, nr]) * r[nr]^2 / 2
        out = Ref{Ptr{Cvoid}}(C_NULL)
        check(h, ccall((:gd_create_timestepping_matrices, LIB), Cint,
                       (Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Ref{Ptr{Cvoid}}), h.ptr, nu, dt, theta, out))
        d = DeviceMatrices(out[], h)
        finalizer(x -> ccall((:gd_destroy_timestepping_matrices, LIB), Cint, (Ptr{Cvoid},), x.ptr), d)
        d
    end
end

# build_rhs_cnab2!(rhs, un, nl, nl_prev, dt, matrices) (src/timestep.jl:610)
function build_rhs_cnab2!(h::Handle, dm::DeviceMatrices, rhs, un, nl, nl_prev, dt::Float64)
    a = map(parent, (un.data_real, un.data_imag, nl.data_real, nl.data_imag, nl_prev.data_real, nl_prev.data_imag,
                     rhs.data_real, rhs.data_imag))
    GC.@preserve a check(h, ccall((:gd_build_rhs_cnab2, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
         Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, dm.ptr, dt, a...))
    return rhs
end

# solve_implicit_step!(sol, rhs, matrices) (src/timestep.jl:692)
function solve_implicit_step!(h::Handle, dm::DeviceMatrices, sol, rhs)
    a = map(parent, (rhs.data_real, rhs.data_imag, sol.data_real, sol.data_imag))
    GC.@preserve a check(h, ccall((:gd_solve_implicit_step, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, dm.ptr, a...))
    return sol
end

upload!(h::Handle, f::Symbol, field) = (re = parent(field.data_real); im = parent(field.data_imag);
    GC.@preserve re im check(h, ccall((:gd_upload_spectral, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, FIELD[f], re, im)))
download!(h::Handle, f::Symbol, field) = (re = parent(field.data_real); im = parent(field.data_imag);
    GC.@preserve re im check(h, ccall((:gd_download_spectral, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, FIELD[f], re, im)))

# step_once! (scripts/bench_timestepping.jl:6-18) on the device: upload the
# five spectral fields, run nsteps graph-replayed steps, copy the fields back.
function step!(h::Handle, state; nsteps::Integer = 1)
    fields = ((:u_tor, state.velocity.toroidal), (:u_pol, state.velocity.poloidal),
              (:b_tor, state.magnetic.toroidal), (:b_pol, state.magnetic.poloidal),
              (:temp, state.temperature.spectral))
    for (f, x) in fields; upload!(h, f, x); end
    check(h, ccall((:gd_step, LIB), Cint, (Ptr{Cvoid}, Cint), h.ptr, nsteps))
    for (f, x) in fields; download!(h, f, x); end
    return state
end

# ts_scheme (src/simulation.jl:1054-1300): :cnab2, :eab2 or :erk2 for the steps of h.
const SCHEME = Dict(:cnab2 => 0, :eab2 => 1, :erk2 => 2)
set_scheme!(h::Handle, scheme::Symbol) =
    check(h, ccall((:gd_set_scheme, LIB), Cint, (Ptr{Cvoid}, Cint), h.ptr, SCHEME[scheme]))

# Reverse mode.  evolve_magnetic(h, re, im, nsteps; field = :b_pol) sets one
# magnetic component of h's state, runs nsteps model steps (gd_step) and
# returns that component afterwards; its ChainRulesCore rrule lives in
# ext/GeoDynamoB200ChainRulesCoreExt.jl and is loaded with ChainRulesCore.
# magnetic_pullback(h, :b_pol, nsteps, λre, λim) -> (gre, gim) is the
# vector-Jacobian product of those steps (gd_magnetic_pullback; planes
# (nlm, nr), as the field data).  In the reference's step the magnetic field
# evolves by its implicit operator alone, the same for every step and state,
# so the pullback needs no checkpoints of the forward run.
function evolve_magnetic(h::Handle, re::AbstractArray{Float64}, im::AbstractArray{Float64}, nsteps::Integer;
                         field::Symbol = :b_pol)
    r = Array{Float64}(re); i = Array{Float64}(im)
    GC.@preserve r i check(h, ccall((:gd_upload_spectral, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, FIELD[field], r, i))
    check(h, ccall((:gd_step, LIB), Cint, (Ptr{Cvoid}, Cint), h.ptr, nsteps))
    GC.@preserve r i check(h, ccall((:gd_download_spectral, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, FIELD[field], r, i))
    return r, i
end

function magnetic_pullback(h::Handle, f::Symbol, nsteps::Integer, lre::AbstractArray{Float64},
                           lim::AbstractArray{Float64})
    gre = similar(lre); gim = similar(lim)
    GC.@preserve lre lim gre gim check(h, ccall((:gd_magnetic_pullback, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, FIELD[f], nsteps, lre, lim, gre, gim))
    return gre, gim
end

# evolve_temperature(h, re, im, nsteps; checkpoint_every = 20) sets the
# temperature of h's state, runs nsteps model steps keeping a device snapshot
# every checkpoint_every steps (gd_temperature_forward) and returns the
# temperature afterwards; its rrule (the extension) pulls the cotangent back
# with gd_temperature_pullback, which recomputes the velocity grids of each
# segment from its snapshot (checkpoint and recompute).  FP64 handles, CNAB2.
function evolve_temperature(h::Handle, re::AbstractArray{Float64}, im::AbstractArray{Float64}, nsteps::Integer;
                            checkpoint_every::Integer = 20)
    r = Array{Float64}(re); i = Array{Float64}(im)
    GC.@preserve r i check(h, ccall((:gd_upload_spectral, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, FIELD[:temp], r, i))
    check(h, ccall((:gd_temperature_forward, LIB), Cint, (Ptr{Cvoid}, Cint, Cint), h.ptr, nsteps, checkpoint_every))
    GC.@preserve r i check(h, ccall((:gd_download_spectral, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, FIELD[:temp], r, i))
    return r, i
end

function temperature_pullback(h::Handle, lre::AbstractArray{Float64}, lim::AbstractArray{Float64})
    gre = similar(lre); gim = similar(lim)
    GC.@preserve lre lim gre gim check(h, ccall((:gd_temperature_pullback, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, lre, lim, gre, gim))
    return gre, gim
end

# evolve_velocity(h, (tre, tim), (pre, pim), nsteps) sets the velocity
# potentials of h's state, runs nsteps model steps and returns them afterwards;
# its rrule (the extension) pulls the cotangents back with
# gd_velocity_pullback.  The literal step's velocity depends on itself alone
# and linearly (its nonlinear term is the Coriolis term), so no checkpoints.
function evolve_velocity(h::Handle, tor::Tuple, pol::Tuple, nsteps::Integer)
    tr = Array{Float64}(tor[1]); ti = Array{Float64}(tor[2])
    pr = Array{Float64}(pol[1]); pi = Array{Float64}(pol[2])
    for (f, a, b) in ((:u_tor, tr, ti), (:u_pol, pr, pi))
        GC.@preserve a b check(h, ccall((:gd_upload_spectral, LIB), Cint,
            (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, FIELD[f], a, b))
    end
    check(h, ccall((:gd_step, LIB), Cint, (Ptr{Cvoid}, Cint), h.ptr, nsteps))
    for (f, a, b) in ((:u_tor, tr, ti), (:u_pol, pr, pi))
        GC.@preserve a b check(h, ccall((:gd_download_spectral, LIB), Cint,
            (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, FIELD[f], a, b))
    end
    return (tr, ti), (pr, pi)
end

function velocity_pullback(h::Handle, nsteps::Integer, ltor::Tuple, lpol::Tuple)
    out = [similar(Array{Float64}(ltor[1])) for _ in 1:4]
    a = [Array{Float64}(x) for x in (ltor[1], ltor[2], lpol[1], lpol[2])]
    GC.@preserve a out check(h, ccall((:gd_velocity_pullback, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
         Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, nsteps, a[1], a[2], a[3], a[4], out[1], out[2], out[3], out[4]))
    return (out[1], out[2]), (out[3], out[4])
end

# The checkpointed run's pullback with respect to the temperature and the
# velocity potentials at its start (gd_temperature_pullback_full):
# ((gTre, gTim), (gtor_re, gtor_im), (gpol_re, gpol_im)).
function temperature_pullback_full(h::Handle, lre::AbstractArray{Float64}, lim::AbstractArray{Float64})
    out = [similar(lre) for _ in 1:6]
    GC.@preserve lre lim out check(h, ccall((:gd_temperature_pullback_full, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
         Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, lre, lim, out[1], out[2], out[3], out[4], out[5], out[6]))
    return (out[1], out[2]), (out[3], out[4]), (out[5], out[6])
end

# Transpose of spectral_to_physical! (gd_spectral_to_physical_adjoint).
function spectral_to_physical_adjoint!(h::Handle, phys_bar, spec_bar)
    g = parent(phys_bar.data); re = parent(spec_bar.data_real); im = parent(spec_bar.data_imag)
    GC.@preserve re im g check(h, ccall((:gd_spectral_to_physical_adjoint, LIB), Cint,
        (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}), h.ptr, 1, g, re, im))
    return spec_bar
end

function energies(h::Handle)
    ek = Ref{Cdouble}(0); em = Ref{Cdouble}(0)
    check(h, ccall((:gd_energy, LIB), Cint, (Ptr{Cvoid}, Ref{Cdouble}, Ref{Cdouble}), h.ptr, ek, em))
    return ek[], em[]
end

"""
    install!(GD::Module; precision = 0)

Overload GeoDynamo's transform, nonlinear and CNAB2 entry points so existing
callers (step_once!, apply_master_implicit_step!) run on the B200 library.
precision = 1 selects the mixed-precision transforms (the nonlinear and CNAB2
functions on host arrays always compute in FP64).
"""
function install!(GD::Module; precision::Integer = 0)
    @eval GD begin
        function shtnskit_spectral_to_physical!(spec::SHTnsSpectralField{Float64}, phys::SHTnsPhysicalField{Float64})
            h = $handle_for($GD, spec.config, size(parent(spec.data_real), 3); precision = $precision)
            $spectral_to_physical!(h, spec, phys)
        end
        function shtnskit_physical_to_spectral!(phys::SHTnsPhysicalField{Float64}, spec::SHTnsSpectralField{Float64})
            h = $handle_for($GD, spec.config, size(parent(spec.data_real), 3); precision = $precision)
            $physical_to_spectral!(h, phys, spec)
        end
        function shtnskit_vector_synthesis!(tor::SHTnsSpectralField{Float64}, pol::SHTnsSpectralField{Float64},
                                            vec::SHTnsVectorField{Float64})
            h = $handle_for($GD, tor.config, size(parent(tor.data_real), 3); precision = $precision)
            $vector_synthesis!(h, tor, pol, vec)
        end
        function shtnskit_vector_analysis!(vec::SHTnsVectorField{Float64}, tor::SHTnsSpectralField{Float64},
                                           pol::SHTnsSpectralField{Float64})
            h = $handle_for($GD, tor.config, size(parent(tor.data_real), 3); precision = $precision)
            $vector_analysis!(h, vec, tor, pol)
        end
        function compute_temperature_nonlinear!(temp::SHTnsTemperatureField{Float64}, vel, oc::RadialDomain;
                                                geometry::Symbol = get_parameters().geometry)
            h = $handle_for($GD, temp.spectral.config, size(parent(temp.spectral.data_real), 3))
            $temperature_nonlinear!(h, temp, vel)
        end
        function compute_composition_nonlinear!(comp::SHTnsCompositionField{Float64}, vel, oc::RadialDomain;
                                                geometry::Symbol = get_parameters().geometry)
            h = $handle_for($GD, comp.spectral.config, size(parent(comp.spectral.data_real), 3); composition = true)
            $composition_nonlinear!(h, comp, vel)
        end
        function compute_velocity_nonlinear!(fields::SHTnsVelocityFields{Float64}, temp, comp, mag,
                                             oc::RadialDomain)
            h = $handle_for($GD, fields.toroidal.config, size(parent(fields.toroidal.data_real), 3))
            $velocity_nonlinear!(h, fields, mag)
        end
        function compute_magnetic_nonlinear!(mag::SHTnsMagneticFields{Float64}, vel, oc::RadialDomain,
                                             ic::RadialDomain, rotation_rate::Float64 = 0.0; geometry::Symbol = :shell)
            h = $handle_for($GD, mag.toroidal.config, size(parent(mag.toroidal.data_real), 3))
            $magnetic_nonlinear!(h, mag, vel)
        end
        function build_rhs_cnab2!(rhs::SHTnsSpectralField{Float64}, un::SHTnsSpectralField{Float64},
                                  nl::SHTnsSpectralField{Float64}, nl_prev::SHTnsSpectralField{Float64},
                                  dt::Float64, M::SHTnsImplicitMatrices{Float64})
            nr = size(parent(un.data_real), 3)
            h = $handle_for($GD, un.config, nr)
            $build_rhs_cnab2!(h, $device_matrices(h, M, nr, i_KL), rhs, un, nl, nl_prev, dt)
        end
        function solve_implicit_step!(sol::SHTnsSpectralField{Float64}, rhs::SHTnsSpectralField{Float64},
                                      M::SHTnsImplicitMatrices{Float64})
            nr = size(parent(rhs.data_real), 3)
            h = $handle_for($GD, rhs.config, nr)
            $solve_implicit_step!(h, $device_matrices(h, M, nr, i_KL), sol, rhs)
        end
    end
    if isdefined(GD, :GeoDynamoBall)
        B = getfield(GD, :GeoDynamoBall)
        @eval B begin
            function ball_physical_to_spectral!(phys::$GD.SHTnsPhysicalField{Float64},
                                                spec::$GD.SHTnsSpectralField{Float64})
                h = $handle_for($GD, spec.config, size(parent(spec.data_real), 3); precision = $precision)
                $ball_physical_to_spectral!(h, phys, spec)
            end
            function ball_vector_analysis!(vec::$GD.SHTnsVectorField{Float64}, tor::$GD.SHTnsSpectralField{Float64},
                                           pol::$GD.SHTnsSpectralField{Float64})
                h = $handle_for($GD, tor.config, size(parent(tor.data_real), 3); precision = $precision)
                $ball_vector_analysis!(h, vec, tor, pol)
            end
        end
    end
    return nothing
end

end # module
