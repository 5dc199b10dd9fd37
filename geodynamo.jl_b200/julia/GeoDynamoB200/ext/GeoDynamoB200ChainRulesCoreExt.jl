# Reverse-mode rule of GeoDynamoB200.evolve_magnetic, loaded when
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

end # module
