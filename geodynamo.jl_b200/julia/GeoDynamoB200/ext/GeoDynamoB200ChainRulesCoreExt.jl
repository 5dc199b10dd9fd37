# Reverse-mode rules of GeoDynamoB200.evolve_magnetic, evolve_temperature and
# evolve_velocity, loaded when
# ChainRulesCore is: the pullback of nsteps model steps with respect to the
# magnetic component they start from is the library's hand-written transposed
# propagator (gd_magnetic_pullback: per step the transposed band solve and the
# transposed band product of the implicit operator, with the boundary
# projections of bc_mode 1 and 2).
module GeoDynamoB200ChainRulesCoreExt

using ChainRulesCore
using GeoDynamoB200

function ChainRulesCore.rrule(::typeof(GeoDynamoB200.evolve_magnetic), h::GeoDynamoB200.Handle,
                              re::AbstractArray{Float64}, im::AbstractArray{Float64}, nsteps::Integer;
                              field::Symbol = :b_pol)
    out = GeoDynamoB200.evolve_magnetic(h, re, im, nsteps; field = field)
    function evolve_magnetic_pullback(Δ)
        d = unthunk(Δ)
        dre = d[1] isa AbstractZero ? zeros(size(re)) : Array{Float64}(unthunk(d[1]))
        dim = d[2] isa AbstractZero ? zeros(size(im)) : Array{Float64}(unthunk(d[2]))
        gre, gim = GeoDynamoB200.magnetic_pullback(h, field, nsteps, dre, dim)
        return NoTangent(), NoTangent(), gre, gim, NoTangent()
    end
    return out, evolve_magnetic_pullback
end

# evolve_temperature: the pullback of the checkpointed run, the velocity grids of
# each segment recomputed from its snapshot (gd_temperature_pullback).
function ChainRulesCore.rrule(::typeof(GeoDynamoB200.evolve_temperature), h::GeoDynamoB200.Handle,
                              re::AbstractArray{Float64}, im::AbstractArray{Float64}, nsteps::Integer;
                              checkpoint_every::Integer = 20)
    out = GeoDynamoB200.evolve_temperature(h, re, im, nsteps; checkpoint_every = checkpoint_every)
    function evolve_temperature_pullback(Δ)
        d = unthunk(Δ)
        dre = d[1] isa AbstractZero ? zeros(size(re)) : Array{Float64}(unthunk(d[1]))
        dim = d[2] isa AbstractZero ? zeros(size(im)) : Array{Float64}(unthunk(d[2]))
        gre, gim = GeoDynamoB200.temperature_pullback(h, dre, dim)
        return NoTangent(), NoTangent(), gre, gim, NoTangent()
    end
    return out, evolve_temperature_pullback
end

# evolve_velocity: the pullback of the steps just run with respect to the velocity
# potentials they started from (gd_velocity_pullback).
function ChainRulesCore.rrule(::typeof(GeoDynamoB200.evolve_velocity), h::GeoDynamoB200.Handle,
                              tor::Tuple, pol::Tuple, nsteps::Integer)
    out = GeoDynamoB200.evolve_velocity(h, tor, pol, nsteps)
    z(x, like) = x isa AbstractZero ? zeros(size(like)) : Array{Float64}(unthunk(x))
    function evolve_velocity_pullback(Δ)
        d = unthunk(Δ)
        dt = d[1] isa AbstractZero ? (zeros(size(tor[1])), zeros(size(tor[2]))) : unthunk(d[1])
        dp = d[2] isa AbstractZero ? (zeros(size(pol[1])), zeros(size(pol[2]))) : unthunk(d[2])
        gt, gp = GeoDynamoB200.velocity_pullback(h, nsteps, (z(dt[1], tor[1]), z(dt[2], tor[2])),
                                                 (z(dp[1], pol[1]), z(dp[2], pol[2])))
        return NoTangent(), NoTangent(), Tangent{typeof(tor)}(gt...), Tangent{typeof(pol)}(gp...), NoTangent()
    end
    return out, evolve_velocity_pullback
end

end # module
