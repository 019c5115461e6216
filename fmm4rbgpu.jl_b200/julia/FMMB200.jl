# FMMB200.jl -- the Julia binding of libfmmb200.so: a drop-in `FMMB200(eta, N0, n)`
# algorithm for FMM4RBGPU.jl's
#     update_particles_field!(particles, alg; lambda)     (src/update_particles_field.jl:66)
# plus a non-mutating `fmm_fields` with a ChainRulesCore.rrule whose pullback is
# the library's hand-written adjoint.
#
# Usage (next to `using FMM4RBGPU`):
#     include("FMMB200.jl"); using .FMMB200Binding
#     update_particles_field!(beam, FMMB200(0.5, 125, 4); lambda=1.0)
#     update_particles_field!(beam, FMMB200(0.5, 125, 4; precision=:mixed); lambda=1.0)
#     update_particles_field!(beam, FMMB200(eta=0.5, N0=125, n=4); lambda=1.0)
#
# The module is called FMMB200Binding so that the name FMMB200 is free for the
# algorithm constructor (a module binds its own name inside itself).
#
# Every call is synchronous; a nonzero status from the library is raised as an
# ErrorException carrying fmmb200_last_error (the reference's error behaviour).
module FMMB200Binding

using FMM4RBGPU: Particles
import FMM4RBGPU: update_particles_field!
using ChainRulesCore

export FMMB200, FMMB200Alg, fmm_fields, update_particles_field!

const libfmmb200 = get(ENV, "FMMB200_LIB", joinpath(@__DIR__, "..", "lib", "libfmmb200.so"))

"""
    FMMB200Alg{T}(n, N0, eta, precision)

The B200 FMM: interpolation degree `n` (1..10), leaf size `N0`, admissibility
`eta` -- the fields of `FMMGPU` (src/update_particles_field.jl:15-19) --
and `precision` `:fp64` (the plain path) or `:mixed`.  Build it with `FMMB200`.
"""
Base.@kwdef struct FMMB200Alg{T}
    n::Int
    N0::Int
    eta::T
    precision::Symbol = :fp64
end

"""
    FMMB200(eta, N0, n; precision=:fp64)
    FMMB200(; n, N0, eta, precision=:fp64)

The algorithm selector of the field-evaluation call, in the positional order
`(eta, N0, n)` or by keyword like `FMMGPU(eta=..., N0=..., n=...)` (README.md:55).
"""
FMMB200(eta::Real, N0::Integer, n::Integer; precision::Symbol=:fp64) =
    FMMB200Alg(n=Int(n), N0=Int(N0), eta=eta, precision=precision)
FMMB200(; n::Integer, N0::Integer, eta::Real, precision::Symbol=:fp64) = FMMB200(eta, N0, n; precision=precision)

_prec(alg) = alg.precision === :mixed ? Int32(1) : alg.precision === :fp64 ? Int32(0) :
    throw(ArgumentError("precision must be :fp64 or :mixed"))

"A library context (device memory, stream, saved forward state)."
mutable struct Context
    ptr::Ptr{Cvoid}
    function Context(device::Integer=0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:fmmb200_create, libfmmb200), Cint, (Ptr{Ptr{Cvoid}}, Cint), r, device)
        st == 0 || error("fmmb200_create failed with status $st (no CUDA device?)")
        c = new(r[])
        finalizer(c) do c
            c.ptr == C_NULL || ccall((:fmmb200_destroy, libfmmb200), Cint, (Ptr{Cvoid},), c.ptr)
            c.ptr = C_NULL
        end
        return c
    end
end

_error(ctx::Context, st::Cint) = ErrorException(
    "libfmmb200 status $st: " * unsafe_string(ccall((:fmmb200_last_error, libfmmb200), Cstring, (Ptr{Cvoid},), ctx.ptr)))

function _check(ctx::Context, st::Cint)
    st == 0 || throw(_error(ctx, st))
    return nothing
end

const _DEFAULT = Ref{Union{Nothing,Context}}(nothing)
const _DEFAULT_LOCK = ReentrantLock()
default_context() = lock(_DEFAULT_LOCK) do
    something(_DEFAULT[], (_DEFAULT[] = Context(0)))
end

# Contexts that hold a forward saved for a pullback.  A context holds one saved
# forward at a time, so each differentiated call takes one from this pool (making
# one only when the pool is empty) and its pullback puts it back after the
# adjoint has run; a loop of forward + pullback reuses the same context and its
# device buffers.  A context whose pullback never runs is freed by its finalizer.
const _POOL = Context[]
const _POOL_LOCK = ReentrantLock()
_acquire() = lock(_POOL_LOCK) do
    isempty(_POOL) ? Context(0) : pop!(_POOL)
end
_release(ctx::Context) = lock(_POOL_LOCK) do
    push!(_POOL, ctx)
    nothing
end

"""
    update_particles_field!(particles::Particles{Float64}, alg::FMMB200Alg; lambda)

Overwrites `particles.efields` / `particles.bfields` with the space-charge fields
(original particle order); positions and momenta are not modified.
"""
function update_particles_field!(p::Particles{Float64}, alg::FMMB200Alg; lambda)
    ctx = default_context()
    GC.@preserve p begin
        st = ccall((:fmmb200_update_particles_field, libfmmb200), Cint,
                   (Ptr{Cvoid}, Int64, Float64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                    Int32, Int64, Float64, Float64, Int32),
                   ctx.ptr, p.npar, p.charge,
                   pointer(reinterpret(Float64, p.positions)), pointer(reinterpret(Float64, p.momenta)),
                   pointer(reinterpret(Float64, p.efields)), pointer(reinterpret(Float64, p.bfields)),
                   alg.n, alg.N0, Float64(alg.eta), Float64(lambda), _prec(alg))
    end
    _check(ctx, st)
    return nothing
end

function _forward!(ctx, pos::Matrix{Float64}, mom::Matrix{Float64}, alg, charge, lambda, save::Bool)
    size(pos, 1) == 3 && size(pos) == size(mom) || throw(DimensionMismatch("pos, mom must be 3 x N"))
    N = size(pos, 2)
    E = similar(pos)
    B = similar(pos)
    st = ccall((:fmmb200_forward, libfmmb200), Cint,
               (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Float64, Float64, Int32, Int64, Float64, Int32,
                Ptr{Float64}, Int32, Ptr{Float64}, Ptr{Float64}),
               ctx.ptr, N, pos, mom, Float64(charge), Float64(lambda), alg.n, alg.N0, Float64(alg.eta),
               _prec(alg), C_NULL, Int32(save), E, B)
    _check(ctx, st)
    return E, B
end

"""
    (E, B) = fmm_fields(pos, mom, alg; charge=-1.0, lambda=1.0)

Non-mutating field evaluation of 3 x N position / momentum matrices (the memory
of a Vector{SVector{3,Float64}}).  Differentiable through `ChainRulesCore.rrule`.
"""
fmm_fields(pos::Matrix{Float64}, mom::Matrix{Float64}, alg::FMMB200Alg; charge=-1.0, lambda=1.0) =
    _forward!(default_context(), pos, mom, alg, charge, lambda, false)

function ChainRulesCore.rrule(::typeof(fmm_fields), pos::Matrix{Float64}, mom::Matrix{Float64},
                              alg::FMMB200Alg; charge=-1.0, lambda=1.0)
    ctx = _acquire()  # the saved forward lives in this context until the pullback runs
    E, B = try
        _forward!(ctx, pos, mom, alg, charge, lambda, true)
    catch
        _release(ctx)
        rethrow()
    end
    released = Ref(false)
    function fmm_fields_pullback(Δ)
        released[] && error("fmm_fields pullback called twice: the saved forward is gone")
        ΔE, ΔB = unthunk(Δ[1]), unthunk(Δ[2])
        gE = ΔE isa AbstractZero ? zeros(size(pos)) : Matrix{Float64}(ΔE)
        gB = ΔB isa AbstractZero ? zeros(size(pos)) : Matrix{Float64}(ΔB)
        gx = similar(pos)
        gu = similar(pos)
        st = ccall((:fmmb200_backward, libfmmb200), Cint,
                   (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), ctx.ptr, gE, gB, gx, gu)
        err = st == 0 ? nothing : _error(ctx, st)  # read before another call can take ctx
        released[] = true
        _release(ctx)
        err === nothing || throw(err)
        return NoTangent(), gx, gu, NoTangent()
    end
    return (E, B), fmm_fields_pullback
end

end # module
