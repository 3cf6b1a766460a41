"""
    ParallelKDEB200

Julia binding of libpkde_b200 (the sm_100a `:gradepro` estimator) for ParallelKDE.jl.

Loading this module after ParallelKDE adds a more specific method of
`DensityEstimators.estimate!(::Type{AbstractGradeProEstimator}, ::CuKDE; ...)`
(src/DensityEstimators/DensityEstimators.jl:64-84), so the user API is unchanged:

    using ParallelKDE, ParallelKDEB200
    est = initialize_estimation(data; grid=true, dims=(512, 512), device=:cuda)
    estimate_density!(est, :gradepro; n_bootstraps=64, n_steps=200)
    density = get_density(est)

Keyword arguments are those of the reference (docs/src/estimators/gradepro.md:19-28),
plus `seed` (counter-based bootstrap draws) or `bootstrap_idxs` (explicit n x B draws).
This file is not exercised by the repository's tests (no Julia toolchain there); the
Python binding in ../pkde_b200 drives the same C ABI.
"""
module ParallelKDEB200

using CUDA
using ParallelKDE
using ParallelKDE.DensityEstimators: AbstractGradeProEstimator, AbstractRoTEstimator
import ParallelKDE.DensityEstimators: estimate!

const libpkde = joinpath(@__DIR__, "..", "lib", "libpkde_b200.so")

const PKDE_OK = Cint(0)
const PKDE_EINVAL = Cint(1)
const PKDE_DEVICE_INPUT = UInt32(1)
const PKDE_DEVICE_OUTPUT = UInt32(2)

# include/pkde_b200.h: pkde_grid
struct PkdeGrid
    ndim::Int32
    reserved::Int32
    dims::NTuple{4,Int64}
    lo::NTuple{4,Float64}
    hi::NTuple{4,Float64}
    h::NTuple{4,Float64}
end

# include/pkde_b200.h: pkde_gradepro_params
struct PkdeGradeproParams
    grid::PkdeGrid
    n_bootstraps::Int32
    n_steps::Int32
    bw_step::Float64
    bw_final::NTuple{4,Float64}
    alpha_s::Float64
    alpha_os::Float64
    eps::Float64
end

const CONTEXTS = Dict{Int,Ptr{Cvoid}}()

function context(device::Integer)
    get!(CONTEXTS, device) do
        ctx = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:pkde_create, libpkde), Cint, (Ref{Ptr{Cvoid}}, Cint), ctx, device)
        rc == PKDE_OK || error("pkde_create failed with status $rc")
        ctx[]
    end
end

function check(rc::Cint, ctx::Ptr{Cvoid})
    rc == PKDE_OK && return nothing
    msg = unsafe_string(ccall((:pkde_last_error, libpkde), Cstring, (Ptr{Cvoid},), ctx))
    rc == PKDE_EINVAL && throw(ArgumentError(msg))
    error("libpkde_b200 status $rc: $msg")
end

pad4(v, fill) = ntuple(i -> i <= length(v) ? v[i] : fill, 4)

function grid_struct(grid)
    lo = Array(low_bounds(grid))
    hi = Array(high_bounds(grid))
    h = Array(spacings(grid))
    dims = size(grid)
    PkdeGrid(Int32(length(dims)), Int32(0), pad4(Int64.(dims), Int64(0)), pad4(Float64.(lo), 0.0),
             pad4(Float64.(hi), 0.0), pad4(Float64.(h), 0.0))
end

nanor(x) = x === nothing ? NaN : Float64(x)

"""
    estimate!(::Type{AbstractGradeProEstimator}, kde::CuKDE; grid, kwargs...)

The `device=:cuda` path of `estimate_density!(est, :gradepro)` on libpkde_b200: fills
`kde.density` in place (FP64 computation, stored in the density's element type).
"""
function estimate!(::Type{AbstractGradeProEstimator}, kde::ParallelKDE.KDEs.CuKDE;
                   method::Union{Nothing,Symbol}=nothing, grid, n_bootstraps::Integer=100,
                   n_steps=nothing, bw_step=nothing, bw_final=nothing, alpha_s=nothing,
                   alpha_os=nothing, eps=nothing, seed::Integer=0, bootstrap_idxs=nothing,
                   device::Integer=CUDA.device().handle)
    method === nothing || method == :cuda ||
        throw(ArgumentError("Invalid implementation $method for device IsCUDA()"))
    N = ndims(kde.density)
    g = grid_struct(grid)
    bwf = bw_final === nothing ? ntuple(_ -> NaN, 4) :
          bw_final isa Real ? pad4(fill(Float64(bw_final), N), NaN) : pad4(Float64.(Array(bw_final)), NaN)
    p = PkdeGradeproParams(g, Int32(n_bootstraps), Int32(n_steps === nothing ? 0 : n_steps),
                           nanor(bw_step), bwf, nanor(alpha_s), nanor(alpha_os), nanor(eps))
    data = CuArray{Float64}(kde.data)                 # N x n, column-major
    n = size(data, 2)
    idx = bootstrap_idxs === nothing ? nothing : CuArray{Int32}(bootstrap_idxs)  # n x B, 1-based
    dens = CuArray{Float64}(undef, size(kde.density))
    ctx = context(device)
    stream = CUDA.stream().handle
    rc = ccall((:pkde_gradepro_estimate, libpkde), Cint,
               (Ptr{Cvoid}, Ref{PkdeGradeproParams}, CuPtr{Float64}, Int64, CuPtr{Int32}, UInt64,
                CuPtr{Float64}, Ptr{Int32}, UInt32, Ptr{Cvoid}),
               ctx, p, data, n, idx === nothing ? CuPtr{Int32}(0) : pointer(idx), UInt64(seed),
               dens, C_NULL, PKDE_DEVICE_INPUT | PKDE_DEVICE_OUTPUT, stream)
    check(rc, ctx)
    copyto!(kde.density, dens)
    return nothing
end

"""
    estimate!(::Type{AbstractRoTEstimator}, kde::CuKDE; grid, rule_of_thumb=:scott)

The `device=:cuda` path of `estimate_density!(est, :rot)` (RoTEstimator.jl:117-201) on
libpkde_b200: identity binning, FFT, one propagation by the rule-of-thumb bandwidth minus
h/2, inverse FFT, `abs`.
"""
function estimate!(::Type{AbstractRoTEstimator}, kde::ParallelKDE.KDEs.CuKDE;
                   method::Union{Nothing,Symbol}=nothing, grid, rule_of_thumb::Symbol=:scott,
                   device::Integer=CUDA.device().handle, kwargs...)
    method === nothing || method == :cuda ||
        throw(ArgumentError("Invalid implementation $method for device IsCUDA()"))
    rule = rule_of_thumb === :scott ? Int32(0) : rule_of_thumb === :silverman ? Int32(1) :
           throw(ArgumentError("Rule of thumb $rule_of_thumb not implemented."))
    data = CuArray{Float64}(kde.data)
    dens = CuArray{Float64}(undef, size(kde.density))
    ctx = context(device)
    rc = ccall((:pkde_rot_estimate, libpkde), Cint,
               (Ptr{Cvoid}, Ref{PkdeGrid}, Int32, CuPtr{Float64}, Int64, CuPtr{Float64}, UInt32, Ptr{Cvoid}),
               ctx, grid_struct(grid), rule, data, size(data, 2), dens,
               PKDE_DEVICE_INPUT | PKDE_DEVICE_OUTPUT, CUDA.stream().handle)
    check(rc, ctx)
    copyto!(kde.density, dens)
    return nothing
end

"""
    find_grid_device(data::CuMatrix; dims=nothing, padding=nothing) -> (lo, hi, dims, h)

find_grid (Grids.jl:252-300) with the extrema reduced on the GPU (pkde_find_grid); the
caller builds its CuGrid from the returned ranges.
"""
function find_grid_device(data::CuMatrix{Float64}; dims=nothing, padding=nothing, device::Integer=CUDA.device().handle)
    N = size(data, 1)
    g = Ref(PkdeGrid(Int32(0), Int32(0), (0, 0, 0, 0), (0.0, 0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 0.0)))
    d = dims === nothing ? C_NULL : Int64[dims...]
    pd = padding === nothing ? C_NULL : Float64[padding...]
    ctx = context(device)
    rc = ccall((:pkde_find_grid, libpkde), Cint,
               (Ptr{Cvoid}, Int32, CuPtr{Float64}, Int64, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}, Ref{PkdeGrid},
                UInt32, Ptr{Cvoid}),
               ctx, Int32(N), data, size(data, 2), d, C_NULL, pd, g, PKDE_DEVICE_INPUT, CUDA.stream().handle)
    check(rc, ctx)
    G = g[]
    return (G.lo[1:N], G.hi[1:N], G.dims[1:N], G.h[1:N])
end

"""
    normalize_density!(density::CuArray{Float64}, dx)

get_density(...; normalize=true) (ParallelKDE.jl:189-202) in place on the device, FP64 sum.
"""
function normalize_density!(density::CuArray{Float64}, dx::Real; device::Integer=CUDA.device().handle)
    ctx = context(device)
    rc = ccall((:pkde_normalize_density, libpkde), Cint, (Ptr{Cvoid}, CuPtr{Float64}, Int64, Float64, UInt32, Ptr{Cvoid}),
               ctx, density, length(density), Float64(dx), PKDE_DEVICE_INPUT, CUDA.stream().handle)
    check(rc, ctx)
    return density
end

end # module
