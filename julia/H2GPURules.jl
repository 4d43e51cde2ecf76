# H2GPURules.jl -- a differentiable steady solve for Julia's AD systems: a ChainRulesCore rrule
# around the library's adjoint (h2g_adjoint), the counterpart of h2_b200.adjoint.HotspotNorm (a
# torch.autograd.Function).  Include after H2GPU.jl in a session that has ChainRulesCore.
#
#   J(hsrc, lnλ) = (Σ_c w_c θ_c^p)^(1/p),   A(λ0 .* exp.(lnλ)) θ = b(hsrc)   (steady, PBiCGSTAB! + RB-GS)
#
# The pullback returns dJ/dhsrc and dJ/dlnλ per cell from one adjoint (transpose) solve; the
# forward solve of the rule is the same GPU PBiCGSTAB! the reference calls with par="gpu".
module H2GPURules

using ChainRulesCore
using ..H2GPU: Handle, H2GBC, set_fields!, set_hsrc!, set_theta!, calrhs!, pbicgstab!, get_theta!,
               adjoint_gradient

export hotspot_norm

"""Fixed data of the objective: a handle with the grid set, the base conductivity λ0, the mask,
the starting temperature θ0, the boundary set (six H2GBC), the weights w and the exponent p."""
struct HotspotProblem
    h::Handle
    λ0::Array{Float64,3}
    mask::Array{Float64,3}
    θ0::Array{Float64,3}
    bcs::Vector{H2GBC}
    w::Array{Float64,3}
    p::Float64
    tol::Float64
end

function prepare!(P::HotspotProblem, hsrc, lnλ)
    set_fields!(P.h, P.λ0 .* exp.(lnλ), P.mask)
    set_hsrc!(P.h, hsrc)
    set_theta!(P.h, P.θ0)
    calrhs!(P.h, P.bcs, true)          # b = -(hsrc·V + boundary terms), steady (calRHS!)
end

"""J(hsrc, lnλ): the forward solve only."""
function hotspot_norm(P::HotspotProblem, hsrc, lnλ)
    prepare!(P, hsrc, lnλ)
    conv, _, _ = pbicgstab!(P.h; tol=P.tol, smoother=:gs)
    conv || error("hotspot_norm: the forward solve did not converge")
    θ = similar(P.θ0)
    get_theta!(θ, P.h)
    return sum(P.w .* θ .^ P.p)^(1 / P.p)
end

function ChainRulesCore.rrule(::typeof(hotspot_norm), P::HotspotProblem, hsrc, lnλ)
    prepare!(P, hsrc, lnλ)
    J, gh, gl = adjoint_gradient(P.h, P.w, P.p; tol=P.tol)
    pullback(ΔJ) = (NoTangent(), NoTangent(), ΔJ .* gh, ΔJ .* gl)   # tangents of (f, P, hsrc, lnλ)
    return J, pullback
end

end # module H2GPURules
