# H2GPU.jl -- Julia binding of the B200 solver library (libh2g.so, include/h2g.h) for Heat3ds.
#
# Copy this file next to the reference's sources and apply julia/par_gpu.patch: heat3ds.jl then
# includes it and accepts par="gpu", and NonUniform.PBiCGSTAB!/CG! forward to the methods below
# when par == "gpu" (src/NonUniform.jl:115-126 and 248-259 are the signatures mirrored here).
# Every entry point passes the reference's own arrays: Array{Float64,3} column-major with guard
# layers (MX, MY, MZ) = (NX+2, NY+2, NZ+2) and Vector{Float64} ZC, ΔZ (MZ entries) and HC (6).
# The library copies host arrays in and out; it allocates and owns its device memory.
module H2GPU

using Printf

export PBiCGSTAB!, CG!, solveSOR!, Handle, adjoint_gradient, version

const libh2g = get(ENV, "H2G_LIB", "libh2g.so")

# h2g_result (include/h2g.h)
struct H2GResult
    isconverged::Cint
    itr::Cint
    outer::Cint
    status::Cint
    res0::Cdouble
    res::Cdouble
    launches::Clonglong
end
H2GResult() = H2GResult(0, 0, 0, 0, 0.0, 0.0, 0)

# h2g_bc: one face of a BoundaryConditionSet (src/boundary_conditions.jl:15-31)
struct H2GBC
    type::Cint            # 0 isothermal, 1 heat flux, 2 convection (src/common.jl:20-24)
    temperature::Cdouble
    heat_flux::Cdouble
    htc::Cdouble
    ambient::Cdouble
end

const PRECISION = Dict(:fp64 => 0, :mixed => 1, :mixed_ir => 2)
const H2G_OK, H2G_NOT_CONVERGED, H2G_BREAKDOWN, H2G_NONFINITE = 0, 1, 2, 3
const HARD_ERRORS = (4, 5, 6, 7)      # BAD_ARG, CUDA_ERROR, TIMEOUT, UNSUPPORTED

version() = unsafe_string(ccall((:h2g_version, libh2g), Cstring, ()))
last_error() = unsafe_string(ccall((:h2g_last_error, libh2g), Cstring, ()))

function check(st::Integer)
    st in HARD_ERRORS && error("h2g: status $st: $(last_error())")
    return st
end

smoother_code(s::Symbol) =
    s === :gs ? 1 : s === :none ? 0 : throw(ArgumentError("Unsupported smoother: $s. Use :none or :gs"))

# ---- the drop-in solvers: same arguments, keywords and return tuple as NonUniform's ------------
function solve!(fn::Symbol, wk, Δh, Δt, ZC, ΔZ, HC; tol, maxItr, smoother, verbose, is_steady, precision)
    code = smoother_code(smoother)
    MX, MY, MZ = size(wk.θ)
    out = Ref(H2GResult())
    # ρ and cp are read only when the grid is transient (is_steady = false)
    st = if fn === :cg
        ccall((:h2g_CG, libh2g), Cint,
              (Cint, Cint, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
               Ptr{Cdouble}, Cdouble, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
               Cdouble, Cint, Cint, Cint, Cint, Cint, Ptr{Cdouble}, Ref{H2GResult}),
              MX, MY, MZ, wk.θ, wk.b, wk.λ, wk.mask, wk.ρ, wk.cp, Δh[1], Δh[2], Δt, ZC, ΔZ, HC,
              tol, maxItr, code, verbose, is_steady, PRECISION[precision], C_NULL, out)
    else
        ccall((:h2g_PBiCGSTAB, libh2g), Cint,
              (Cint, Cint, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
               Ptr{Cdouble}, Cdouble, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
               Cdouble, Cint, Cint, Cint, Cint, Cint, Ptr{Cdouble}, Ref{H2GResult}),
              MX, MY, MZ, wk.θ, wk.b, wk.λ, wk.mask, wk.ρ, wk.cp, Δh[1], Δh[2], Δt, ZC, ΔZ, HC,
              tol, maxItr, code, verbose, is_steady, PRECISION[precision], C_NULL, out)
    end
    check(st)
    r = out[]
    return r.isconverged != 0, Int(r.itr), r.res0
end

"""PBiCGSTAB! on the B200 (src/NonUniform.jl:248-350): θ updated in place, returns
(isconverged, itr, res0).  `precision` = :fp64 (the reference's arithmetic), :mixed or :mixed_ir."""
PBiCGSTAB!(wk, Δh, Δt, ZC, ΔZ, HC; tol=1e-6, maxItr=20_000, smoother::Symbol=:none, par::String="gpu",
           verbose::Bool=false, is_steady::Bool=false, precision::Symbol=:fp64) =
    solve!(:pbicgstab, wk, Δh, Δt, ZC, ΔZ, HC; tol, maxItr, smoother, verbose, is_steady, precision)

"""CG! on the B200 (src/NonUniform.jl:115-226), same conventions."""
CG!(wk, Δh, Δt, ZC, ΔZ, HC; tol=1e-6, maxItr=20_000, smoother::Symbol=:none, par::String="gpu",
    verbose::Bool=false, is_steady::Bool=false, precision::Symbol=:fp64) =
    solve!(:cg, wk, Δh, Δt, ZC, ΔZ, HC; tol, maxItr, smoother, verbose, is_steady, precision)

"""solveSOR! (src/NonUniform.jl:1004-1051) in FP64: returns the reference's iteration count
(negative when not converged); the residual lines go to F as the reference writes them."""
function solveSOR!(θ, λ, b, mask, ρ, cp, Δh, Δt, ω, ZC, ΔZ, HC, F, tol; maxItr=20_000, is_steady=false)
    MX, MY, MZ = size(θ)
    hist = zeros(maxItr)
    out = Ref(H2GResult())
    st = ccall((:h2g_SolveSOR, libh2g), Cint,
               (Cint, Cint, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                Ptr{Cdouble}, Cdouble, Cdouble, Cdouble, Cdouble, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                Cdouble, Cint, Cint, Cint, Ptr{Cdouble}, Ref{H2GResult}),
               MX, MY, MZ, θ, b, λ, mask, ρ, cp, Δh[1], Δh[2], Δt, ω, ZC, ΔZ, HC, tol, maxItr, 1, is_steady,
               hist, out)
    check(st)
    r = out[]
    for n in 1:min(Int(r.itr), maxItr)
        F === nothing || println(F, lpad(n, 10), " ", format_e(hist[n]))
    end
    return r.isconverged != 0 ? Int(r.itr) : -Int(r.itr)
end

format_e(x) = @sprintf("%24.14E", x)    # the reference's residual line format

# ---- a resident handle: fields uploaded once, many solves (time steps, gradients) ----------------
mutable struct Handle
    ptr::Ptr{Cvoid}
    shape::NTuple{3,Int}
    function Handle(MX, MY, MZ; precision::Symbol=:fp64)
        p = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:h2g_create, libh2g), Cint, (Cint, Cint, Cint, Cint, Ref{Ptr{Cvoid}}),
                    MX, MY, MZ, PRECISION[precision], p))
        h = new(p[], (MX, MY, MZ))
        finalizer(h) do x
            x.ptr == C_NULL || ccall((:h2g_destroy, libh2g), Cint, (Ptr{Cvoid},), x.ptr)
            x.ptr = C_NULL
        end
        return h
    end
end

set_grid!(h::Handle, ZC, ΔZ, Δh, Δt, HC, is_steady) =
    check(ccall((:h2g_set_grid, libh2g), Cint,
                (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Cdouble, Cdouble, Cdouble, Ptr{Cdouble}, Cint),
                h.ptr, ZC, ΔZ, Δh[1], Δh[2], Δt, HC, is_steady))
set_fields!(h::Handle, λ, mask, ρ=nothing, cp=nothing) =
    check(ccall((:h2g_set_fields, libh2g), Cint, (Ptr{Cvoid}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
                h.ptr, λ, mask, ρ === nothing ? C_NULL : ρ, cp === nothing ? C_NULL : cp))
set_rhs!(h::Handle, b) = check(ccall((:h2g_set_rhs, libh2g), Cint, (Ptr{Cvoid}, Ptr{Cdouble}), h.ptr, b))
set_theta!(h::Handle, θ) = check(ccall((:h2g_set_theta, libh2g), Cint, (Ptr{Cvoid}, Ptr{Cdouble}), h.ptr, θ))
get_theta!(θ, h::Handle) = check(ccall((:h2g_get_theta, libh2g), Cint, (Ptr{Cvoid}, Ptr{Cdouble}), h.ptr, θ))
set_hsrc!(h::Handle, hsrc) = check(ccall((:h2g_set_hsrc, libh2g), Cint, (Ptr{Cvoid}, Ptr{Cdouble}), h.ptr, hsrc))
calrhs!(h::Handle, bcs::Vector{H2GBC}, zero_b::Bool) =
    check(ccall((:h2g_calrhs, libh2g), Cint, (Ptr{Cvoid}, Ptr{H2GBC}, Cint), h.ptr, bcs, zero_b))

function pbicgstab!(h::Handle; tol=1e-6, maxItr=20_000, smoother::Symbol=:gs, verbose::Bool=false)
    out = Ref(H2GResult())
    check(ccall((:h2g_pbicgstab, libh2g), Cint,
                (Ptr{Cvoid}, Cdouble, Cint, Cint, Cint, Ptr{Cdouble}, Ref{H2GResult}),
                h.ptr, tol, maxItr, smoother_code(smoother), verbose, C_NULL, out))
    r = out[]
    return r.isconverged != 0, Int(r.itr), r.res0
end

"""main()'s time loop (src/heat3ds.jl:123-151) on the device: nt steps of calRHS! (b rebuilt from
zero each step) and PBiCGSTAB!/CG! from the previous θ.  Returns the per-step statistics
(θmin, θmax, ‖θ‖₂, iterations, final residual) as a 5×nt matrix."""
function transient!(h::Handle, bcs::Vector{H2GBC}, nt::Integer; method::Symbol=:pbicgstab, tol=1e-6,
                    maxItr=20_000, smoother::Symbol=:gs, verbose::Bool=false)
    stats = zeros(5, nt)
    out = Ref(H2GResult())
    check(ccall((:h2g_transient, libh2g), Cint,
                (Ptr{Cvoid}, Ptr{H2GBC}, Cint, Cint, Cdouble, Cint, Cint, Cint, Ptr{Cdouble}, Ref{H2GResult}),
                h.ptr, bcs, nt, method === :cg ? 1 : 0, tol, maxItr, smoother_code(smoother), verbose, stats, out))
    return stats
end

"""J = (Σ w θ^p)^(1/p) of the handle's steady solution and its gradients with respect to the heat
source (dJ/dhsrc) and to ln λ per cell (dJ/dlnλ): a forward and one adjoint (transpose) solve."""
function adjoint_gradient(h::Handle, w::Array{Float64,3}, p::Real; tol=1e-10, maxItr=20_000,
                          smoother::Symbol=:gs)
    J = Ref{Cdouble}(0.0)
    gh = zeros(size(w))
    gl = zeros(size(w))
    check(ccall((:h2g_adjoint, libh2g), Cint,
                (Ptr{Cvoid}, Ptr{Cdouble}, Cdouble, Cdouble, Cint, Cint, Ref{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble},
                 Ptr{Cvoid}, Ptr{Cvoid}),
                h.ptr, w, p, tol, maxItr, smoother_code(smoother), J, gh, gl, C_NULL, C_NULL))
    return J[], gh, gl
end

# ---- CalcRK! on arrays that already live in device memory, without allocating -------------------
"""CalcRK! (src/NonUniform.jl:372-434) on device pointers owned by the caller (CuArrays of
CUDA.jl): r = b - Aθ over the interior and ‖r‖₂, with no device allocation.  `stream` is the
stream the caller's kernels run on (CUDA.stream().handle), so the call is ordered after them; it
synchronises that stream before returning."""
function calcrk_noalloc!(r_d, θ_d, b_d, λ_d, m_d, ρ_d, cp_d, ZC, ΔZ, Δh, Δt, HC, is_steady, stream,
                         MX, MY, MZ)
    res = Ref{Cdouble}(0.0)
    check(ccall((:h2g_calcrk_noalloc, libh2g), Cint,
                (Cint, Cint, Cint, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid},
                 Ptr{Cvoid}, Cdouble, Cdouble, Cdouble, Ptr{Cdouble}, Cint, Ptr{Cvoid}, Ref{Cdouble}, Ptr{Cvoid}),
                MX, MY, MZ, θ_d, b_d, λ_d, m_d, ρ_d, cp_d, ZC, ΔZ, Δh[1], Δh[2], Δt, HC, is_steady, r_d, res, stream))
    return res[]
end

end # module H2GPU
