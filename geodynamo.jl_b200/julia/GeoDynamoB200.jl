# GeoDynamoB200.jl -- ccall shim that puts libgdb200.so (B200, sm_100a) behind
# GeoDynamo.jl's transform, nonlinear and time-step functions.
#
# Usage from a GeoDynamo.jl session:
#     include(joinpath(path_to_repo, "geodynamo.jl_b200", "julia", "GeoDynamoB200.jl"))
#     using .GeoDynamoB200
#     GeoDynamoB200.install!(GeoDynamo)          # overloads the methods below
#
# Array layouts need no conversion: GeoDynamo's spectral planes
# (nlm, 1, nr) and physical fields (nlat, nlon, nr) are column-major, which is
# the library's host layout (lm fastest / theta fastest).  Every call borrows
# the arrays for its duration (GC.@preserve) and reports errors by throwing,
# as the reference does.
module GeoDynamoB200

const LIB = normpath(joinpath(@__DIR__, "..", "libgdb200.so"))

# gd_config (include/gdb200.h)
struct GDConfig
    lmax::Cint; mmax::Cint; nlat::Cint; nlon::Cint; nr::Cint; kl::Cint
    rratio::Cdouble; ekman::Cdouble; rayleigh::Cdouble; prandtl::Cdouble; magnetic_prandtl::Cdouble
    dt::Cdouble; implicit_theta::Cdouble
    ab_mode::Cint; bc_mode::Cint; fd_mode::Cint; precision::Cint; magnetic::Cint
end

mutable struct Handle
    ptr::Ptr{Cvoid}
end

const FIELD = Dict(:u_tor => 0, :u_pol => 1, :b_tor => 2, :b_pol => 3, :temp => 4)

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

function handle_for(GD, config, nr::Integer; precision::Integer = 0)
    key = (objectid(config), Int(nr), Int(precision))
    get!(HANDLES, key) do
        cfg = GDConfig(config.lmax, config.mmax, config.nlat, config.nlon, nr, GD.i_KL,
                       GD.d_rratio, GD.d_E, GD.d_Ra, GD.d_Pr, GD.d_Pm, GD.d_timestep, GD.d_implicit,
                       0, 0, 0, precision, GD.i_B)
        create(cfg)
    end
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

# Reverse mode.  magnetic_pullback(h, :b_pol, nsteps, λre, λim) -> (gre, gim):
# the vector-Jacobian product of nsteps steps with respect to a magnetic
# component at their start (gd_magnetic_pullback; planes (nlm, nr), as the
# field data).  A ChainRulesCore rule for the step, for objectives of the
# magnetic field, is then
#     function ChainRulesCore.rrule(::typeof(magnetic_steps), h, bpol_re, bpol_im, nsteps)
#         out = magnetic_steps(h, bpol_re, bpol_im, nsteps)
#         pullback(Δ) = (NoTangent(), NoTangent(),
#                        magnetic_pullback(h, :b_pol, nsteps, Δ[1], Δ[2])..., NoTangent())
#         return out, pullback
#     end
# (written here as a comment: ChainRulesCore is not a dependency of this shim).
function magnetic_pullback(h::Handle, f::Symbol, nsteps::Integer, lre::AbstractArray{Float64},
                           lim::AbstractArray{Float64})
    gre = similar(lre); gim = similar(lim)
    GC.@preserve lre lim gre gim check(h, ccall((:gd_magnetic_pullback, LIB), Cint,
        (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
        h.ptr, FIELD[f], nsteps, lre, lim, gre, gim))
    return gre, gim
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

Overload GeoDynamo's transform entry points so existing callers (step_once!,
compute_*_nonlinear!) run on the B200 library.  precision = 1 selects the
mixed-precision transforms.
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
    end
    return nothing
end

end # module
