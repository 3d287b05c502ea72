"""
    SparseMatrixAlgorithmsB200

Drop-in replacements for the solve-free interior eigensolvers of
MathiasTensor/sparse_matrix_algorithms, running on a B200 through libsma's C ABI
(`include/sma.h`).  Same names, positional arguments, keyword arguments, defaults and
return values as

    chebyshev_poly_real_symm_sparse(Ain::SparseMatrixCSC, emin, emax; ...)   # chebyshev_subspace_iteration.jl:667
    chebyshev_poly_real_symm_sparse(matvec!, n, emin, emax; matblock, ...)  # chebyshev_subspace_iteration.jl:771
    polfed(A::MatrixFreeRealSymOp, nev, degree; ...)                         # polfed.jl:1128
    polfed(matvec!, n, nev, degree; matblock!=nothing, kwargs...)           # polfed.jl:1183

Matrix-free operators must act on the GPU: pass a `DeviceCSR(A)`, a `Lap1dDevice(n)`
or a `DeviceMatblock(fptr, user)` (a `@cfunction` enqueuing Y = A X on the given CUDA
stream) as `matblock`/`matblock!`.  A host closure is rejected with an ArgumentError;
it is never run on the CPU.
"""
module SparseMatrixAlgorithmsB200

using SparseArrays
using LinearAlgebra

export chebyshev_poly_real_symm_sparse, polfed, polfed_windows, MatrixFreeRealSymOp, DeviceCSR, Lap1dDevice,
       AndersonDevice, XXZDevice, DeviceMatblock, gershgorin_bounds, lanczos_bounds,
       jackson_kernel, cheb_delta_coeffs, cheb_window_coeffs, cheb_smooth_window_coeffs,
       kpm_moments, kpm_count, slice_spectrum

const libsma = get(ENV, "SMA_LIBRARY", joinpath(@__DIR__, "..", "libsma.so"))

# ------------------------------------------------------------------ C structs (sma.h)
mutable struct ChebOpts
    smin::Float64; smax::Float64; has_bounds::Int64; sigma::Float64
    m0::Int64; degree::Int64; maxiter::Int64; tol::Float64; res_gate::Float64
    jackson::Int64; debug::Int64; two_hit::Int64; seed::Int64; window_type::Int64
    matrix_free::Int64; precision::Int64; lock::Int64; reserved::NTuple{7,Int64}
end
ChebOpts() = ChebOpts(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, ntuple(_ -> 0, 7))

mutable struct PolfedOpts
    s::Int64; smin::Float64; smax::Float64; has_bounds::Int64; sigma::Float64
    emin::Float64; emax::Float64; tol::Float64; threaded::Int64; overextract::Int64
    refine::Int64; window_type::Int64; jackson::Int64; mmax::Int64; rtol::Float64
    reorth_passes::Int64; extra_keep::Int64; seed::Int64; show_progress::Int64
    chunk::Int64; precision::Int64; reserved::NTuple{8,Int64}
end
PolfedOpts() = PolfedOpts(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, ntuple(_ -> 0, 8))

mutable struct SliceOpts
    smin::Float64; smax::Float64; has_bounds::Int64; maxiter::Int64; tol::Float64
    res_gate::Float64; jackson::Int64; two_hit::Int64; seed::Int64; window_type::Int64
    precision::Int64; graph::Int64; debug::Int64; reserved::NTuple{8,Int64}
end
SliceOpts() = SliceOpts(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, ntuple(_ -> 0, 8))

const SMA_ERR_ARG, SMA_ERR_NONSYMMETRIC, SMA_ERR_INTERVAL = 1, 2, 3
const SMA_ERR_BOUNDS, SMA_ERR_WINDOW = 8, 9

function check(rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:sma_last_error, libsma), Cstring, ()))
    if rc in (SMA_ERR_ARG, SMA_ERR_NONSYMMETRIC, SMA_ERR_INTERVAL)
        throw(ArgumentError(msg))
    end
    error(msg)   # SMA_ERR_BOUNDS / SMA_ERR_WINDOW are `error(...)` in the reference
end

window_code(w::Symbol) = w === :step ? 0 : w === :delta ? 1 : w === :smooth ? 2 :
    error("Unknown window type: $w")
precision_code(p::Symbol) = p === :fp64 ? 0 : p === :fp32 ? 1 : p === :mixed ? 2 :
    throw(ArgumentError("precision must be :fp64, :fp32 or :mixed"))

# ------------------------------------------------------------------ context
const CTX = Ref{Ptr{Cvoid}}(C_NULL)
function context()
    if CTX[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:sma_ctx_create, libsma), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, h))
        CTX[] = h[]
    end
    return CTX[]
end

# ------------------------------------------------------------------ device operators
abstract type DeviceOperator end

mutable struct DeviceCSR <: DeviceOperator
    handle::Ptr{Cvoid}
    n::Int
end
"""Device copy of a symmetric SparseMatrixCSC (its CSC arrays are its CSR arrays);
`upper=true` keeps only the upper triangle (symmetric half storage: about half the memory,
slower products)."""
function DeviceCSR(A::SparseMatrixCSC{Float64,Int}; check_symmetric::Bool=false, upper::Bool=false)
    n = size(A, 1)
    size(A, 2) == n || throw(ArgumentError("A must be square"))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    if upper  # ccall needs the symbol as a constant
        check(ccall((:sma_op_create_csc_upper, libsma), Cint,
                    (Ptr{Cvoid}, Int64, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}, Int64, Int64, Ref{Ptr{Cvoid}}),
                    context(), n, nnz(A), A.colptr, A.rowval, A.nzval, 1, check_symmetric, h))
    else
        check(ccall((:sma_op_create_csc, libsma), Cint,
                    (Ptr{Cvoid}, Int64, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}, Int64, Int64, Ref{Ptr{Cvoid}}),
                    context(), n, nnz(A), A.colptr, A.rowval, A.nzval, 1, check_symmetric, h))
    end
    op = DeviceCSR(h[], n)
    finalizer(o -> ccall((:sma_op_destroy, libsma), Cint, (Ptr{Cvoid},), o.handle), op)
    return op
end

mutable struct Lap1dDevice <: DeviceOperator
    handle::Ptr{Cvoid}
    n::Int
end
"tridiag(-1,2,-1) as a device stencil (GPU form of lap1d_matblock!, polfed.jl:1209)."
function Lap1dDevice(n::Int)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sma_op_create_lap1d, libsma), Cint, (Ptr{Cvoid}, Int64, Ref{Ptr{Cvoid}}), context(), n, h))
    op = Lap1dDevice(h[], n)
    finalizer(o -> ccall((:sma_op_destroy, libsma), Cint, (Ptr{Cvoid},), o.handle), op)
    return op
end

mutable struct AndersonDevice <: DeviceOperator
    handle::Ptr{Cvoid}
    n::Int
end
"3D Anderson model on an L^3 periodic lattice (on-site energies eps, hopping t) as a device stencil."
function AndersonDevice(L::Int, eps::Vector{Float64}; t::Float64=-1.0)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sma_op_create_anderson, libsma), Cint, (Ptr{Cvoid}, Int64, Ptr{Float64}, Float64, Ref{Ptr{Cvoid}}),
                context(), L, eps, t, h))
    op = AndersonDevice(h[], L^3)
    finalizer(o -> ccall((:sma_op_destroy, libsma), Cint, (Ptr{Cvoid},), o.handle), op)
    return op
end

mutable struct XXZDevice <: DeviceOperator
    handle::Ptr{Cvoid}
    n::Int
end
"Random-field XXZ chain (even L, periodic) in its Sz = 0 sector as a device stencil."
function XXZDevice(L::Int, h::Vector{Float64}; J::Float64=1.0, Δ::Float64=1.0)
    hh = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sma_op_create_xxz, libsma), Cint, (Ptr{Cvoid}, Int64, Float64, Float64, Ptr{Float64}, Ref{Ptr{Cvoid}}),
                context(), L, J, Δ, h, hh))
    op = XXZDevice(hh[], binomial(L, L ÷ 2))
    finalizer(o -> ccall((:sma_op_destroy, libsma), Cint, (Ptr{Cvoid},), o.handle), op)
    return op
end

mutable struct DeviceMatblock <: DeviceOperator
    handle::Ptr{Cvoid}
    n::Int
    keepalive::Any
end
"""
    DeviceMatblock(n, fptr, user)

`fptr = @cfunction(f, Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Int64, Int64, Ptr{Cvoid}))`
with `f(user, X, Y, n, b, ld, stream)` enqueuing Y = A X for row-major n x b device blocks
(leading dimension ld) on the CUDA stream `stream`, returning 0.
"""
function DeviceMatblock(n::Int, fptr::Ptr{Cvoid}, user=nothing)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    uptr = user === nothing ? C_NULL : pointer_from_objref(user)
    check(ccall((:sma_op_create_matblock, libsma), Cint, (Ptr{Cvoid}, Int64, Ptr{Cvoid}, Ptr{Cvoid}, Ref{Ptr{Cvoid}}),
                context(), n, fptr, uptr, h))
    op = DeviceMatblock(h[], n, user)
    finalizer(o -> ccall((:sma_op_destroy, libsma), Cint, (Ptr{Cvoid},), o.handle), op)
    return op
end

"""
    MatrixFreeRealSymOp(n, matvec!)  /  MatrixFreeRealSymOp(n, matvec!, matblock!)

Same constructors as polfed.jl:159-165.  The block action must be a DeviceOperator.
"""
struct MatrixFreeRealSymOp{F,G}
    n::Int
    matvec!::F
    matblock!::G
    dev::DeviceOperator
end
MatrixFreeRealSymOp(n::Int, matvec!) = MatrixFreeRealSymOp(n, matvec!, nothing)
function MatrixFreeRealSymOp(n::Int, matvec!, matblock!)
    dev = matblock! isa DeviceOperator ? matblock! : matvec! isa DeviceOperator ? matvec! :
        throw(ArgumentError("matrix-free operators must act on device blocks (DeviceCSR, Lap1dDevice, DeviceMatblock); host matvec!/matblock! closures are not run"))
    dev.n == n || throw(ArgumentError("operator dimension $(dev.n) != n = $n"))
    return MatrixFreeRealSymOp{typeof(matvec!),typeof(matblock!)}(n, matvec!, matblock!, dev)
end
Base.size(A::MatrixFreeRealSymOp) = (A.n, A.n)

# ------------------------------------------------------------------ results
function take_result(h::Ptr{Cvoid})
    k = Ref{Int64}(0); n = Ref{Int64}(0)
    try
        check(ccall((:sma_result_count, libsma), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int64}), h, k, n))
        λ = Vector{Float64}(undef, k[]); res = Vector{Float64}(undef, k[])
        X = Matrix{Float64}(undef, n[], k[])
        check(ccall((:sma_result_copy, libsma), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                    h, λ, k[] > 0 ? X : C_NULL, res))
        return λ, X, res
    finally
        ccall((:sma_result_free, libsma), Cint, (Ptr{Cvoid},), h)
    end
end

# ------------------------------------------------------------------ coefficients
function jackson_kernel(K::Int)
    g = Vector{Float64}(undef, max(K, 0) + 1)
    check(ccall((:sma_jackson_kernel, libsma), Cint, (Int64, Ptr{Float64}), K, g)); g
end
function cheb_delta_coeffs(σ̂::Float64, K::Int; jackson::Bool=true)
    c = Vector{Float64}(undef, K + 1)
    check(ccall((:sma_cheb_delta_coeffs, libsma), Cint, (Float64, Int64, Int64, Ptr{Float64}), σ̂, K, jackson, c)); c
end
function cheb_window_coeffs(a::Float64, b::Float64, K::Int; jackson::Bool=true)
    c = Vector{Float64}(undef, K + 1)
    check(ccall((:sma_cheb_window_coeffs, libsma), Cint, (Float64, Float64, Int64, Int64, Ptr{Float64}), a, b, K, jackson, c)); c
end
function cheb_smooth_window_coeffs(a::Float64, b::Float64, K::Int; jackson::Bool=true, nsamp::Int=4096, δ::Float64=0.02)
    c = Vector{Float64}(undef, K + 1)
    check(ccall((:sma_cheb_smooth_window_coeffs, libsma), Cint, (Float64, Float64, Int64, Int64, Int64, Float64, Ptr{Float64}),
                a, b, K, jackson, nsamp, δ, c)); c
end
function gershgorin_bounds(A::SparseMatrixCSC{Float64,Int})
    op = DeviceCSR(A); lo = Ref{Float64}(0); hi = Ref{Float64}(0)
    check(ccall((:sma_gershgorin_bounds, libsma), Cint, (Ptr{Cvoid}, Ref{Float64}, Ref{Float64}), op.handle, lo, hi))
    return lo[], hi[]
end

# ------------------------------------------------------------------ Chebyshev
function cheb_opts(; smin, smax, σ, m0, degree, maxiter, tol, res_gate, jackson, debug,
                   two_hit, seed, window_type, matrix_free, precision)
    o = ChebOpts()
    ccall((:sma_cheb_opts_default, libsma), Cvoid, (Ref{ChebOpts},), o)
    if smin !== nothing && smax !== nothing
        o.smin = smin; o.smax = smax; o.has_bounds = 1
    end
    o.sigma = σ; o.m0 = m0; o.degree = degree; o.maxiter = maxiter; o.tol = tol
    o.res_gate = res_gate; o.jackson = jackson; o.debug = debug; o.two_hit = two_hit
    o.seed = seed; o.window_type = window_code(window_type); o.matrix_free = matrix_free
    o.precision = precision_code(precision)
    return o
end

function chebyshev_poly_real_symm_sparse(Ain::SparseMatrixCSC{Float64,Int}, emin::Float64, emax::Float64;
        smin::Union{Float64,Nothing}=nothing, smax::Union{Float64,Nothing}=nothing, σ::Float64=0.0,
        m0::Int=200, degree::Int=80, maxiter::Int=8, tol::Float64=1e-10, res_gate::Float64=1e-6,
        jackson::Bool=true, debug::Bool=false, two_hit::Bool=true, seed::Int=1,
        window_type::Symbol=:step, precision::Symbol=:fp64, lock::Bool=false)
    op = DeviceCSR(Ain)
    o = cheb_opts(; smin, smax, σ, m0, degree, maxiter, tol, res_gate, jackson, debug, two_hit,
                  seed, window_type, matrix_free=0, precision)
    o.lock = lock
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sma_cheb_solve, libsma), Cint, (Ptr{Cvoid}, Float64, Float64, Ref{ChebOpts}, Ref{Ptr{Cvoid}}),
                op.handle, emin, emax, o, h))
    return take_result(h[])
end

function chebyshev_poly_real_symm_sparse(matvec!::F, n::Int, emin::Float64, emax::Float64;
        matblock::Union{G,Nothing}=nothing, smin::Union{Float64,Nothing}=nothing,
        smax::Union{Float64,Nothing}=nothing, σ::Float64=0.0, m0::Int=200, degree::Int=80,
        maxiter::Int=8, tol::Float64=1e-10, res_gate::Float64=1e-6, jackson::Bool=true,
        debug::Bool=false, two_hit::Bool=true, seed::Int=1, window_type::Symbol=:step,
        precision::Symbol=:fp64, lock::Bool=false) where {F,G}
    A = MatrixFreeRealSymOp(n, matvec!, matblock)
    o = cheb_opts(; smin, smax, σ, m0, degree, maxiter, tol, res_gate, jackson, debug, two_hit,
                  seed, window_type, matrix_free=1, precision)
    o.lock = lock
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sma_cheb_solve, libsma), Cint, (Ptr{Cvoid}, Float64, Float64, Ref{ChebOpts}, Ref{Ptr{Cvoid}}),
                A.dev.handle, emin, emax, o, h))
    return take_result(h[])
end

# ------------------------------------------------------------------ POLFED
function polfed(A::MatrixFreeRealSymOp, nev::Int, degree::Int; s::Int=8, smin=nothing, smax=nothing,
        sigma::Float64=0.0, emin::Float64=-Inf, emax::Float64=Inf, tol::Float64=1e-10,
        threaded::Bool=true, overextract::Int=2, refine::Bool=true, window_type::Symbol=:step,
        jackson::Bool=true, mmax::Union{Nothing,Int}=nothing, rtol::Float64=1e-12,
        reorth_passes::Int=1, extra_keep::Int=8, seed::Int=1, show_progress::Bool=true, chunk=64,
        precision::Symbol=:fp64)
    o = PolfedOpts()
    ccall((:sma_polfed_opts_default, libsma), Cvoid, (Ref{PolfedOpts},), o)
    o.s = s
    if smin !== nothing && smax !== nothing
        o.smin = smin; o.smax = smax; o.has_bounds = 1
    end
    o.sigma = sigma; o.emin = emin; o.emax = emax; o.tol = tol; o.threaded = threaded
    o.overextract = overextract; o.refine = refine; o.window_type = window_code(window_type)
    o.jackson = jackson; o.mmax = mmax === nothing ? 0 : mmax; o.rtol = rtol
    o.reorth_passes = reorth_passes; o.extra_keep = extra_keep; o.seed = seed
    o.show_progress = show_progress; o.chunk = chunk; o.precision = precision_code(precision)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sma_polfed_solve, libsma), Cint, (Ptr{Cvoid}, Int64, Int64, Ref{PolfedOpts}, Ref{Ptr{Cvoid}}),
                A.dev.handle, nev, degree, o, h))
    return take_result(h[])
end

function polfed(matvec!::F, n::Int, nev::Int, degree::Int; matblock!::Union{Nothing,G}=nothing, kwargs...) where {F,G}
    Aop = isnothing(matblock!) ? MatrixFreeRealSymOp(n, matvec!) : MatrixFreeRealSymOp(n, matvec!, matblock!)
    return polfed(Aop, nev, degree; kwargs...)
end

# ------------------------------------------------------------------ extensions
"Spectral bounds from GPU Lanczos (the reference has only gershgorin_bounds)."
function lanczos_bounds(op::DeviceOperator; steps::Int=60, seed::Int=7)
    lo = Ref{Float64}(0); hi = Ref{Float64}(0)
    check(ccall((:sma_lanczos_bounds, libsma), Cint, (Ptr{Cvoid}, Int64, Int64, Ref{Float64}, Ref{Float64}),
                op.handle, steps, seed, lo, hi))
    return lo[], hi[]
end

"Stochastic KPM moments mu[1:M] of the spectral density on [smin, smax] (R Rademacher vectors)."
function kpm_moments(op::DeviceOperator, M::Int, R::Int, smin::Float64, smax::Float64; seed::Int=11)
    mu = Vector{Float64}(undef, M)
    check(ccall((:sma_kpm_moments, libsma), Cint, (Ptr{Cvoid}, Int64, Int64, Int64, Float64, Float64, Ptr{Float64}, Ptr{Float64}),
                op.handle, M, R, seed, smin, smax, mu, C_NULL))
    return mu
end

"Eigenvalue count in [emin, emax] predicted by KPM moments of an n x n operator."
function kpm_count(mu::Vector{Float64}, n::Int, smin::Float64, smax::Float64, emin::Float64, emax::Float64; jackson::Bool=true)
    c = Ref{Float64}(0)
    check(ccall((:sma_kpm_count, libsma), Cint, (Ptr{Float64}, Int64, Int64, Float64, Float64, Float64, Float64, Int64, Ref{Float64}),
                mu, length(mu), n, smin, smax, emin, emax, jackson, c))
    return c[]
end

"""
    slice_spectrum(op::DeviceCSR, windows, degrees, m0s; kwargs...) -> (λ, X, res, win)

Batched spectrum slicing: every window (emin, emax) runs Chebyshev subspace iteration with
its own degree and width; all windows are filtered in ONE batched recurrence per iteration.
`win[j]` is the (1-based) window of pair j.
"""
function slice_spectrum(op::DeviceCSR, windows::Vector{Tuple{Float64,Float64}}, degrees::Vector{Int},
        m0s::Vector{Int}; smin=nothing, smax=nothing, maxiter::Int=8, tol::Float64=1e-10,
        res_gate::Float64=1e-6, jackson::Bool=true, two_hit::Bool=true, seed::Int=1,
        window_type::Symbol=:step, precision::Symbol=:fp64, graph::Bool=true)
    o = SliceOpts()
    ccall((:sma_slice_opts_default, libsma), Cvoid, (Ref{SliceOpts},), o)
    if smin !== nothing && smax !== nothing
        o.smin = smin; o.smax = smax; o.has_bounds = 1
    end
    o.maxiter = maxiter; o.tol = tol; o.res_gate = res_gate; o.jackson = jackson
    o.two_hit = two_hit; o.seed = seed; o.window_type = window_code(window_type)
    o.precision = precision_code(precision); o.graph = graph
    emin = first.(windows); emax = last.(windows)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sma_slice_solve, libsma), Cint,
                (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Int64}, Ptr{Int64}, Ref{SliceOpts}, Ref{Ptr{Cvoid}}),
                op.handle, length(windows), emin, emax, Int64.(degrees), Int64.(m0s), o, h))
    k = Ref{Int64}(0); nn = Ref{Int64}(0)
    check(ccall((:sma_result_count, libsma), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int64}), h[], k, nn))
    win = Vector{Int64}(undef, k[])
    k[] > 0 && check(ccall((:sma_result_windows, libsma), Cint, (Ptr{Cvoid}, Ptr{Int64}), h[], win))
    λ, X, res = take_result(h[])
    return λ, X, res, win .+ 1
end

"""
    polfed_windows(op::DeviceCSR, windows, nevs, degrees, mmaxs; kwargs...) -> (λ, X, res, win)

Batched POLFED (an extension; `polfed` solves one window): window w is a POLFED solve with
its own nev, degree and mmax, its filter centred on the window and start seed `seed + w - 1`;
every block step filters all windows' blocks in ONE segmented recurrence.  Keyword
arguments as `polfed` (s, smin, smax, tol, window_type, jackson, precision, ...).  `win[j]`
is the (1-based) window of pair j; each window's pairs follow polfed's return order.
"""
function polfed_windows(op::DeviceCSR, windows::Vector{Tuple{Float64,Float64}}, nevs::Vector{Int},
        degrees::Vector{Int}, mmaxs::Vector{Int}; s::Int=8, smin::Float64, smax::Float64,
        tol::Float64=1e-10, overextract::Int=2, refine::Bool=true, window_type::Symbol=:step,
        jackson::Bool=true, rtol::Float64=1e-12, reorth_passes::Int=1, extra_keep::Int=8,
        seed::Int=1, show_progress::Bool=false, precision::Symbol=:fp64)
    o = PolfedOpts()
    ccall((:sma_polfed_opts_default, libsma), Cvoid, (Ref{PolfedOpts},), o)
    o.s = s; o.smin = smin; o.smax = smax; o.has_bounds = 1; o.tol = tol
    o.overextract = overextract; o.refine = refine; o.window_type = window_code(window_type)
    o.jackson = jackson; o.rtol = rtol; o.reorth_passes = reorth_passes
    o.extra_keep = extra_keep; o.seed = seed; o.show_progress = show_progress
    o.precision = precision_code(precision)
    emin = first.(windows); emax = last.(windows)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:sma_polfed_batch_solve, libsma), Cint,
                (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64},
                 Ref{PolfedOpts}, Ref{Ptr{Cvoid}}),
                op.handle, length(windows), emin, emax, Int64.(nevs), Int64.(degrees), Int64.(mmaxs), o, h))
    k = Ref{Int64}(0); nn = Ref{Int64}(0)
    check(ccall((:sma_result_count, libsma), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int64}), h[], k, nn))
    win = Vector{Int64}(undef, k[])
    k[] > 0 && check(ccall((:sma_result_windows, libsma), Cint, (Ptr{Cvoid}, Ptr{Int64}), h[], win))
    λ, X, res = take_result(h[])
    return λ, X, res, win .+ 1
end

end # module
