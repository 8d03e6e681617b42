# SPECTreconB200.jl -- Julia host layer over libspectgpu.so (the B200 projector).
#
# Drop-in for the projector hot path of SPECTrecon.jl: the same names and
# argument meaning as src/spectplan.jl, src/project.jl, src/backproject.jl and
# src/ml-os-em.jl, with the bodies replaced by `ccall`s into the C ABI declared
# in include/spect_gpu.h.  Arrays keep Julia's column-major layout, which is
# exactly the layout of the C ABI (image[nx,ny,nz] == float[nz][ny][nx]).
# Errors are rethrown as the reference's `String`s (or DimensionMismatch).
#
# Usage (a maintainer would `include` this file in place of the CPU bodies):
#     ENV["SPECT_B200_LIB"] = "/path/to/libspectgpu.so"
#     plan = SPECTplan(mumap, psfs, dy)            # uploads, precomputes PSF spectra
#     views = project(image, plan)                 # host arrays, synchronous
#     backproject!(image, views, plan; index = 1:2:plan.nview)
#     xhat = osem(x0, ynoisy, background, Ablock(plan, 8); niter = 4)
#
# Ablock(plan, nblocks) returns the reference's Vector{LinearMapAO} (one
# LinearMapAA per subset, src/ml-os-em.jl:70-84), so reference-style code that
# indexes Ab[nb] and applies Ab[nb] * x, Ab[nb]' * y runs unchanged; osem!/mlem!
# recognise maps built here from one plan and run the whole reconstruction as
# one device-resident call, and fall back to the reference's loop otherwise.

module SPECTreconB200

using LinearAlgebra: mul!
using LinearMapsAA: LinearMapAO, LinearMapAA

export SPECTplan, project, project!, backproject, backproject!
export mlem, mlem!, osem, osem!, Ablock, SPECTmap, psf_gauss, autotune!, conv_kernels

const LIB = get(ENV, "SPECT_B200_LIB", joinpath(@__DIR__, "..", "libspectgpu.so"))

const SPECT_OK = Cint(0)
const SPECT_ERR_DIM = Cint(8)

function check(status::Cint)
    status == SPECT_OK && return nothing
    msg = unsafe_string(ccall((:spect_last_error, LIB), Cstring, ()))
    status == SPECT_ERR_DIM && throw(DimensionMismatch(msg))
    throw(msg) # the reference throws Strings ("nx != ny", "asym. psf", ...)
end

mutable struct SPECTplan{T}
    handle::Ptr{Cvoid}
    T::Type{<:AbstractFloat}
    imgsize::NTuple{3, Int}
    px::Int
    pz::Int
    nview::Int
    viewangle::Vector{Float32}
    interpmeth::Symbol
    mode::Symbol
    dy::T
    nthread::Int
end

"""
    SPECTplan(mumap, psfs, dy; T, viewangle, interpmeth, nthread, mode)
Same keywords and validation as src/spectplan.jl:58-137.  `mumap` and `psfs`
are uploaded once; later host edits are not seen (the reference aliases them).
"""
function SPECTplan(
    mumap::Array{<:Real, 3},
    psfs::Array{<:Real, 4},
    dy::Real;
    T::Type{<:AbstractFloat} = promote_type(eltype(mumap), Float32),
    viewangle::AbstractVector{<:Real} = (0:size(psfs, 4) - 1) / size(psfs, 4) * T(2π),
    interpmeth::Symbol = :two,
    nthread::Int = Threads.nthreads(),
    mode::Symbol = :fast,
)
    T === Float32 || throw("the B200 path computes in Float32")
    nx, ny, nz = size(mumap)
    px, pz, _, nview = size(psfs)
    mu = Array{Float32}(mumap)
    ps = Array{Float32}(psfs)
    ang = Vector{Float32}(viewangle)
    im = interpmeth === :one ? Cint(1) : interpmeth === :two ? Cint(2) : Cint(0)
    md = mode === :fast ? Cint(0) : mode === :mem ? Cint(1) : Cint(-1)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:spect_plan_create, LIB), Cint,
        (Ref{Ptr{Cvoid}}, Cint, Cint, Cint, Cint, Cint, Cint, Ptr{Float32}, Ptr{Float32}, Float32,
         Ptr{Float32}, Cint, Cint, Cint, Cint),
        h, nx, ny, nz, px, pz, nview, mu, ps, Float32(dy), ang, im, md, nthread, Threads.nthreads()))
    plan = SPECTplan{Float32}(h[], Float32, (nx, ny, nz), px, pz, nview, ang, interpmeth, mode,
        Float32(dy), nthread)
    finalizer(p -> ccall((:spect_plan_destroy, LIB), Cint, (Ptr{Cvoid},), p.handle), plan)
    return plan
end

_index(index) = Cint.(collect(index) .- 1) # 1-based Julia views -> 0-based C

# the caller's array itself when it already is a dense Float32 Array (no copy)
_f32(a::Array{Float32}) = a
_f32(a::AbstractArray) = Array{Float32}(a)

"""
    project!(views, image, plan; index = 1:plan.nview)   (src/project.jl:143-163)
"""
function project!(
    views::AbstractArray{<:Real, 3},
    image::AbstractArray{<:Real, 3},
    plan::SPECTplan;
    index::AbstractVector{<:Int} = 1:plan.nview,
)
    idx = _index(index)
    size(views) == (plan.imgsize[1], plan.imgsize[3], length(idx)) || throw(DimensionMismatch("views size"))
    out = views isa Array{Float32, 3} ? views : Array{Float32}(undef, size(views))
    check(ccall((:spect_project_host, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Cint}, Cint),
        plan.handle, out, _f32(image), idx, length(idx)))
    out === views || (views .= out)
    return views
end

"""
    project!(view, image, plan, viewidx)  (src/project.jl:11-69)
"""
function project!(view::AbstractMatrix{<:Real}, image::AbstractArray{<:Real, 3}, plan::SPECTplan, viewidx::Int)
    v = reshape(view, size(view, 1), size(view, 2), 1)
    project!(v, image, plan; index = [viewidx])
    return view
end

"""
    project!(view, image, plan, buffer_id, viewidx)  (src/project.jl:77-135); buffer_id is ignored
"""
project!(view::AbstractMatrix{<:Real}, image::AbstractArray{<:Real, 3}, plan::SPECTplan, ::Int, viewidx::Int) =
    project!(view, image, plan, viewidx)

function project(image::AbstractArray{<:Real, 3}, plan::SPECTplan; kwargs...)
    index = get(kwargs, :index, 1:plan.nview)
    views = Array{Float32}(undef, plan.imgsize[1], plan.imgsize[3], length(index))
    return project!(views, image, plan; index)
end

function project(image::AbstractArray{<:Real, 3}, mumap::AbstractArray{<:Real, 3},
    psfs::AbstractArray{<:Real, 4}, dy::Real; interpmeth::Symbol = :two, mode::Symbol = :fast, kwargs...)
    size(mumap) == size(image) || throw(DimensionMismatch("image/mumap size"))
    size(image, 2) == size(psfs, 3) || throw(DimensionMismatch("image/psfs size"))
    return project(image, SPECTplan(Array(mumap), Array(psfs), dy; interpmeth, mode); kwargs...)
end

"""
    backproject!(image, views, plan; index = 1:plan.nview)  (src/backproject.jl:132-162)
"""
function backproject!(
    image::AbstractArray{<:Real, 3},
    views::AbstractArray{<:Real, 3},
    plan::SPECTplan;
    index::AbstractVector{<:Int} = 1:plan.nview,
)
    idx = _index(index)
    size(image) == plan.imgsize || throw(DimensionMismatch("image size"))
    out = image isa Array{Float32, 3} ? image : Array{Float32}(undef, plan.imgsize)
    check(ccall((:spect_backproject_host, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Cint}, Cint),
        plan.handle, out, _f32(views), idx, length(idx)))
    out === image || (image .= out)
    return image
end

function backproject!(image::AbstractArray{<:Real, 3}, view::AbstractMatrix{<:Real}, plan::SPECTplan, viewidx::Int)
    tmp = similar(image, Float32)
    backproject!(tmp, reshape(view, size(view, 1), size(view, 2), 1), plan; index = [viewidx])
    image .= tmp
    return image
end

backproject!(image::AbstractArray{<:Real, 3}, view::AbstractMatrix{<:Real}, plan::SPECTplan, ::Int, viewidx::Int) =
    backproject!(image, view, plan, viewidx)

function backproject(views::AbstractArray{<:Real, 3}, plan::SPECTplan; kwargs...)
    image = zeros(Float32, plan.imgsize)
    return backproject!(image, views, plan; kwargs...)
end

function backproject(views::AbstractArray{<:Real, 3}, mumap::AbstractArray{<:Real, 3},
    psfs::AbstractArray{<:Real, 4}, dy::Real; interpmeth::Symbol = :two, mode::Symbol = :fast, kwargs...)
    size(mumap, 1) == size(views, 1) || throw(DimensionMismatch("nx"))
    size(mumap, 3) == size(views, 2) || throw(DimensionMismatch("nz"))
    return backproject(views, SPECTplan(Array(mumap), Array(psfs), dy; interpmeth, mode); kwargs...)
end

"""
    SPECTmap(plan; index = 1:plan.nview) -> LinearMapAO
The projector of `plan` for the views `index` as a LinearMapAA (the map that
test/adjoint-project.jl:33-35 builds from project!/backproject!), tagged with
the plan so that mlem!/osem! can run it as one device-resident call.
"""
function SPECTmap(plan::SPECTplan; index::AbstractVector{<:Int} = 1:plan.nview, nblocks::Int = 1, block::Int = 1)
    nx, ny, nz = plan.imgsize
    forw!(y, x) = project!(y, x, plan; index)
    back!(x, y) = backproject!(x, y, plan; index)
    idim = (nx, ny, nz)
    odim = (nx, nz, length(index))
    return LinearMapAA(forw!, back!, (prod(odim), prod(idim)); T = plan.T, odim, idim,
        prop = (plan = plan, nblocks = nblocks, block = block))
end

"""
    Ablock(plan, nblocks) -> Vector{LinearMapAO}  (src/ml-os-em.jl:70-84)
One map per subset nb:nblocks:nview, as the reference returns.
"""
function Ablock(plan::SPECTplan, nblocks::Int)
    rem(plan.nview, nblocks) == 0 || throw("nview must be divisible by nblocks!")
    Ab = Vector{LinearMapAO}(undef, nblocks)
    for nb in 1:nblocks
        Ab[nb] = SPECTmap(plan; index = nb:nblocks:plan.nview, nblocks, block = nb)
    end
    return Ab
end

# the plan behind maps built by SPECTmap/Ablock from one plan covering all
# views in the reference's subset order, or nothing
_tagged(A) = A isa LinearMapAO && haskey(A.prop, :plan) ? A.prop : nothing
function _plan_of(Ab::AbstractVector)
    props = map(_tagged, Ab)
    any(isnothing, props) && return nothing
    plan = props[1].plan
    n = length(Ab)
    all(k -> props[k].plan === plan && props[k].nblocks == n && props[k].block == k, 1:n) || return nothing
    return plan
end

function _em_checks(out, x0, ynoisy, background)
    all(>(0), background) || throw("need background > 0")
    size(out) == size(x0) || throw(DimensionMismatch("size out and x0 not match"))
    size(ynoisy) == size(background) || throw(DimensionMismatch("size ynoisy and background"))
end

# the whole OS-EM (nblocks = 1: ML-EM) as one call: sensitivities, iterations
# and the fused EM ratio/update on the device
function _em!(out, x0, ynoisy, background, plan::SPECTplan, nblocks::Int, niter::Int)
    res = out isa Array{Float32, 3} && out !== x0 ? out : Array{Float32}(undef, plan.imgsize)
    check(ccall((:spect_osem_host, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Cint, Cint),
        plan.handle, res, _f32(x0), _f32(ynoisy), _f32(background), nblocks, niter))
    res === out || (out .= res)
    return out
end

# the reference's OS-EM loop (src/ml-os-em.jl:106-131) for any maps
function _em_generic!(out, x0, ynoisy, background, Ab, niter, chat)
    nblocks = length(Ab)
    nx, nz, nview = size(ynoisy)
    asum = [Ab[nb]' * ones(eltype(ynoisy), nx, nz, nview ÷ nblocks) for nb in 1:nblocks]
    for a in asum
        a[a .== 0] .= Inf
    end
    ybar = Array{eltype(ynoisy)}(undef, nx, nz, nview ÷ nblocks)
    yratio = similar(ybar)
    back = similar(x0)
    copyto!(out, x0)
    for iter in 1:niter, nb in 1:nblocks
        chat && (@show iter, nb, extrema(out))
        mul!(ybar, Ab[nb], out)
        @. yratio = (@view ynoisy[:, :, nb:nblocks:nview]) / (ybar + (@view background[:, :, nb:nblocks:nview]))
        mul!(back, Ab[nb]', yratio)
        @. out *= back / asum[nb]
    end
    return out
end

"""
    mlem!(out, x0, ynoisy, background, A; niter = 20)  (src/ml-os-em.jl:21-49)
`A` as in the reference (AbstractArray or LinearMapAO); a map from SPECTmap
(or the plan itself) runs as one device-resident call.
"""
function mlem!(out::AbstractArray, x0::AbstractArray, ynoisy::AbstractArray, background::AbstractArray,
    A::Union{AbstractArray, LinearMapAO}; niter::Int = 20, chat::Bool = false)
    _em_checks(out, x0, ynoisy, background)
    plan = _plan_of([A])
    plan === nothing || return _em!(out, x0, ynoisy, background, plan, 1, niter)
    return _em_generic!(out, x0, ynoisy, background, [A], niter, chat)
end
function mlem!(out::AbstractArray, x0::AbstractArray, ynoisy::AbstractArray, background::AbstractArray,
    A::SPECTplan; niter::Int = 20, chat::Bool = false)
    _em_checks(out, x0, ynoisy, background)
    return _em!(out, x0, ynoisy, background, A, 1, niter)
end
mlem(x0::AbstractArray, args...; kwargs...) = mlem!(similar(x0, Float32), x0, args...; kwargs...)

"""
    osem!(out, x0, ynoisy, background, Ab; niter = 16)  (src/ml-os-em.jl:97-131)
`Ab` as in the reference (a vector of arrays or LinearMapAOs); the maps of
Ablock(plan, nblocks) run as one device-resident call.
"""
function osem!(out::AbstractArray, x0::AbstractArray, ynoisy::AbstractArray, background::AbstractArray,
    Ab::Union{Vector{<:AbstractArray}, Vector{LinearMapAO}}; niter::Int = 16, chat::Bool = false)
    _em_checks(out, x0, ynoisy, background)
    plan = _plan_of(Ab)
    plan === nothing || return _em!(out, x0, ynoisy, background, plan, length(Ab), niter)
    return _em_generic!(out, x0, ynoisy, background, Ab, niter, chat)
end
osem(x0::AbstractArray, args...; kwargs...) = osem!(similar(x0, Float32), x0, args...; kwargs...)

"""
    psf_gauss(; ny, px, pz, fwhm_start, fwhm_end, fwhm, fwhm_x, fwhm_z, T)  (src/psf-gauss.jl:24-55)
"""
function psf_gauss( ; ny::Int = 128, px::Int = 11, pz::Int = px, fwhm_start::Real = 1, fwhm_end::Real = 4,
    fwhm::AbstractVector{<:Real} = range(fwhm_start, fwhm_end, ny),
    fwhm_x::AbstractVector{<:Real} = fwhm, fwhm_z::AbstractVector{<:Real} = fwhm_x,
    T::Type{<:AbstractFloat} = Float32)
    psf = Array{Float32}(undef, px, pz, ny)
    check(ccall((:spect_psf_gauss, LIB), Cint, (Ptr{Float32}, Cint, Cint, Cint, Ptr{Float64}, Ptr{Float64}),
        psf, ny, px, pz, Vector{Float64}(fwhm_x), Vector{Float64}(fwhm_z)))
    return T.(psf)
end

# ---- additions without a counterpart in the reference ------------------------

"""
    autotune!(plan; nindex = plan.nview) -> (forward_ms, adjoint_ms)
Times the launch shapes and, for rank-1 (Gaussian) PSF planes, the direct
separable convolution against the FFT one for calls of `nindex` views, and
keeps the fastest per direction.
"""
function autotune!(plan::SPECTplan; nindex::Int = plan.nview)
    ms = zeros(Float64, 2)
    check(ccall((:spect_plan_autotune, LIB), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}), plan.handle, nindex, ms))
    return (ms[1], ms[2])
end

"""
    conv_kernels(plan) -> (forward = :direct | :fft, adjoint = :direct | :fft)
Which PSF convolution each direction of the plan runs.
"""
function conv_kernels(plan::SPECTplan)
    out = zeros(Cint, 4)
    check(ccall((:spect_plan_conv_kernels, LIB), Cint, (Ptr{Cvoid}, Ptr{Cint}), plan.handle, out))
    name(k) = k == 1 ? :direct : :fft
    return (forward = name(out[3]), adjoint = name(out[4]))
end

end # module
