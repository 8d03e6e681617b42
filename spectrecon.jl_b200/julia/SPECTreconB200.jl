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

module SPECTreconB200

export SPECTplan, project, project!, backproject, backproject!
export mlem, mlem!, osem, osem!, Ablock, psf_gauss, autotune!, conv_kernels

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
    out = Array{Float32}(undef, plan.imgsize[1], plan.imgsize[3], length(idx))
    check(ccall((:spect_project_host, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Cint}, Cint),
        plan.handle, out, Array{Float32}(image), idx, length(idx)))
    views .= out
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
    out = Array{Float32}(undef, plan.imgsize)
    check(ccall((:spect_backproject_host, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Cint}, Cint),
        plan.handle, out, Array{Float32}(views), idx, length(idx)))
    image .= out
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
    Ablock(plan, nblocks)  (src/ml-os-em.jl:70-84): the subsets nb:nblocks:nview
"""
struct Ablock
    plan::SPECTplan
    nblocks::Int
    function Ablock(plan::SPECTplan, nblocks::Int)
        rem(plan.nview, nblocks) == 0 || throw("nview must be divisible by nblocks!")
        new(plan, nblocks)
    end
end
Base.length(Ab::Ablock) = Ab.nblocks

function _em!(out, x0, ynoisy, background, plan::SPECTplan, nblocks::Int, niter::Int)
    all(>(0), background) || throw("need background > 0")
    size(out) == size(x0) || throw(DimensionMismatch("size out and x0 not match"))
    size(ynoisy) == size(background) || throw(DimensionMismatch("size ynoisy and background"))
    res = Array{Float32}(undef, plan.imgsize)
    check(ccall((:spect_osem_host, LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Cint, Cint),
        plan.handle, res, Array{Float32}(x0), Array{Float32}(ynoisy), Array{Float32}(background),
        nblocks, niter))
    out .= res
    return out
end

"""
    mlem!(out, x0, ynoisy, background, plan; niter = 20)  (src/ml-os-em.jl:21-49)
The system matrix is the plan itself (the reference takes the LinearMapAA that wraps it).
"""
mlem!(out, x0, ynoisy, background, A::SPECTplan; niter::Int = 20, chat::Bool = false) =
    _em!(out, x0, ynoisy, background, A, 1, niter)
mlem(x0, args...; kwargs...) = mlem!(similar(x0, Float32), x0, args...; kwargs...)

"""
    osem!(out, x0, ynoisy, background, Ab; niter = 16)  (src/ml-os-em.jl:97-131)
"""
osem!(out, x0, ynoisy, background, Ab::Ablock; niter::Int = 16, chat::Bool = false) =
    _em!(out, x0, ynoisy, background, Ab.plan, Ab.nblocks, niter)
osem(x0, args...; kwargs...) = osem!(similar(x0, Float32), x0, args...; kwargs...)

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
