# Package extension that registers `backend = :b200` in Hammerhead.jl and
# forwards the planar WIDIM path to libhammerhead_b200.so through ccall:
# Hammerhead's own run_piv / run_piv_ensemble drive the device through the
# backend hooks below (piv_correlation_engines, _deform_context,
# apply_predictor, process_windows!, uncertainty_sweep!,
# release_piv_engines!, the ensemble trio); run_piv_b200 and
# run_piv_ensemble_b200 run a whole schedule in one library call.
#
# Not runnable in this repository's environment (no Julia toolchain); it is
# written against the backend-hook contract of docs/src/reference/backends.md
# and src/types.jl:61-111 of the reference, and mirrors what the Python host
# layer (hammerhead.jl_b200/hammerhead_b200) does with the same C ABI.
module HammerheadB200Ext

using Hammerhead
using ChainRulesCore: ChainRulesCore, NoTangent, unthunk
import Hammerhead: _AbstractHammerheadBackend, _resolve_backend, _check_backend_params, _engine_nchunks,
    _supports_fft, _supports_batched_fft, _supports_fp64, PIVParameters, PIVResult, run_piv,
    piv_correlation_engines, process_windows!, uncertainty_sweep!, _deform_context, apply_predictor,
    release_piv_engines!, _correlation_apod, pooled_engines, apodization_window, finalize_uncertainty,
    _plane_accumulator, accumulate_planes!, ensemble_analyze!, _uncertainty_accumulator,
    _uncertainty_scratch, UQ_NSTATS

const LIB = get(ENV, "HAMMERHEAD_B200_LIB", "libhammerhead_b200.so")

struct _B200Backend <: _AbstractHammerheadBackend end
_resolve_backend(::Val{:b200}) = _B200Backend()
_engine_nchunks(::_B200Backend, ::Int) = 1
_supports_fft(::_B200Backend) = true
_supports_batched_fft(::_B200Backend) = true
_supports_fp64(::_B200Backend) = true   # FP64 uncertainty reductions on the device

# hh_validator / hh_pass_desc (include/hammerhead_b200.h), field for field.
struct Validator
    kind::Int32
    neighborhood::Int32
    threshold::Float64
    vmin::Float64
    vmax::Float64
    epsilon::Float64
end
const NOVAL = Validator(0, 0, 0.0, 0.0, 0.0, 0.0)

struct PassDesc
    window::NTuple{2,Int32}
    search::NTuple{2,Int32}
    overlap::NTuple{2,Int32}
    method::Int32
    padding::Int32
    apodization::Int32
    subpixel::Int32
    n_peaks::Int32
    peak_finder::Int32
    uncertainty::Int32
    uod_enable::Int32
    uod_threshold::Float64
    uod_neighborhood::Int32
    replace_outliers::Int32
    min_peak_ratio::Float64
    max_iterations::Int32
    keep_correlation_planes::Int32
    convergence_tol::Float64
    n_validators::Int32
    reserved0::Int32
    validators::NTuple{8,Validator}
end

const SUBPIXEL = Dict(:gauss3 => 0, :gauss9 => 1, :gauss2d => 2, :none => 3)

validator(v::Hammerhead.PeakRatioValidator) = Validator(0, 0, v.threshold, 0.0, 0.0, 0.0)
validator(v::Hammerhead.CorrelationMomentValidator) = Validator(1, 0, v.threshold, 0.0, 0.0, 0.0)
validator(v::Hammerhead.VelocityMagnitudeValidator) = Validator(2, 0, 0.0, v.min, v.max, 0.0)
validator(v::Hammerhead.UniversalOutlierValidator) =
    Validator(3, v.neighborhood_size, v.threshold, 0.0, 0.0, v.epsilon)

function pass_desc(p::PIVParameters)
    vals = map(validator, p.validation)
    length(vals) <= 8 || throw(ArgumentError("backend :b200 supports at most 8 extra validators"))
    vt = ntuple(i -> i <= length(vals) ? vals[i] : NOVAL, 8)
    PassDesc(Int32.(p.window_size), Int32.(p.search_area_size), Int32.(p.overlap),
             p.correlation_method === :phase ? 1 : 0, p.padding, p.apodization === :gauss ? 1 : 0,
             SUBPIXEL[p.subpixel_method], p.n_peaks, p.peak_finder === :exclusion ? 1 : 0,
             p.uncertainty, p.uod_enable, p.uod_threshold, p.uod_neighborhood, p.replace_outliers,
             p.min_peak_ratio, p.max_iterations, p.keep_correlation_planes, p.convergence_tol,
             length(vals), 0, vt)
end

struct Result
    ny::Int32
    nx::Int32
    x::Ptr{Float32}
    y::Ptr{Float32}
    u::Ptr{Float32}
    v::Ptr{Float32}
    peak_ratio::Ptr{Float32}
    correlation_moment::Ptr{Float32}
    uncertainty_u::Ptr{Float32}
    uncertainty_v::Ptr{Float32}
    outliers::Ptr{UInt8}
    mask::Ptr{UInt8}
end

last_error(ctx) = unsafe_string(ccall((:hh_last_error, LIB), Cstring, (Ptr{Cvoid},), ctx))

function check(st, ctx = C_NULL)
    st == 0 && return nothing
    (st == 1 || st == 5) && throw(ArgumentError(last_error(ctx)))
    error("hammerhead_b200: " * last_error(ctx))
end

function _check_backend_params(::_B200Backend, passes)
    d = [pass_desc(p) for p in passes]
    check(ccall((:hh_check_backend_params, LIB), Int32, (Ptr{PassDesc}, Int32), d, length(d)))
end

# Context per workspace: created lazily, destroyed by a finalizer.
mutable struct Context
    ptr::Ptr{Cvoid}
    function Context(device::Integer = 0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:hh_ctx_create, LIB), Int32, (Int32, Ref{Ptr{Cvoid}}), device, r))
        c = new(r[])
        finalizer(c -> ccall((:hh_ctx_destroy, LIB), Cvoid, (Ptr{Cvoid},), c.ptr), c)
        return c
    end
end

# The whole schedule on the device: run_piv(...; backend = :b200) with
# Float32 images (the device path computes in Float32; FP64 only for the
# subpixel logarithms and the uncertainty sums).
function run_piv_b200(imgA::AbstractMatrix{<:Real}, imgB::AbstractMatrix{<:Real},
                      passes::AbstractVector{PIVParameters};
                      predictor_smoothing::Bool = true,
                      mask::Union{Nothing,AbstractMatrix{Bool}} = nothing, mask_threshold::Real = 0.5,
                      ctx::Context = Context())
    _check_backend_params(_B200Backend(), passes)
    size(imgA) == size(imgB) ||
        throw(DimensionMismatch("images must have the same size, got $(size(imgA)) and $(size(imgB))"))
    A = Matrix{Float32}(imgA)
    B = Matrix{Float32}(imgB)
    M = mask === nothing ? C_NULL : Matrix{UInt8}(mask)
    nr, nc = size(A)
    final = last(passes)
    d = [pass_desc(p) for p in passes]
    ny, nx, nj = Ref{Int32}(0), Ref{Int32}(0), Ref{Int64}(0)
    check(ccall((:hh_pass_grid, LIB), Int32,
                (Int64, Int64, Ref{PassDesc}, Ptr{UInt8}, Float64, Ref{Int32}, Ref{Int32}, Ptr{Float32},
                 Ptr{Float32}, Ptr{UInt8}, Ptr{Int32}, Ref{Int64}),
                nr, nc, pass_desc(final), C_NULL, mask_threshold, ny, nx, C_NULL, C_NULL, C_NULL, C_NULL, nj))
    gy, gx = Int(ny[]), Int(nx[])
    x = Vector{Float32}(undef, gx); y = Vector{Float32}(undef, gy)
    f() = Matrix{Float32}(undef, gy, gx)
    u, v, ratio, moment, su, sv = f(), f(), f(), f(), f(), f()
    outl = Matrix{UInt8}(undef, gy, gx); gm = Matrix{UInt8}(undef, gy, gx)
    GC.@preserve A B M x y u v ratio moment su sv outl gm begin
        res = Ref(Result(0, 0, pointer(x), pointer(y), pointer(u), pointer(v), pointer(ratio), pointer(moment),
                         pointer(su), pointer(sv), pointer(outl), pointer(gm)))
        check(ccall((:hh_run_piv, LIB), Int32,
                    (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int64, Int64, Ptr{PassDesc}, Int32, Ptr{UInt8},
                     Float64, Int32, Ref{Result}),
                    ctx.ptr, A, B, nr, nc, d, length(d), M, mask_threshold, predictor_smoothing, res), ctx.ptr)
    end
    return PIVResult(x, y, u, v, ratio, moment, su, sv, BitMatrix(outl .!= 0), BitMatrix(gm .!= 0), final)
end

# ---- the backend hooks: run_piv(A, B, passes; backend = :b200) -----------
#
# Hammerhead's run_piv resolves `backend = :b200` through _resolve_backend
# above and then drives every pass through these private hooks
# (docs/src/reference/backends.md:40-71; the :cuda counterparts are
# ext/HammerheadCUDAExt.jl:105-437):
#   piv_correlation_engines -> one engine per pass configuration (nchunks = 1)
#   _deform_context         -> a handle on the context that holds the pair
#   apply_predictor         -> hh_stage_pair (once per pair: upload + device
#                              B-spline prefilter) + hh_apply_predictor (device
#                              deformation; the warped pair stays on the device)
#   process_windows!        -> hh_process_windows on the staged (warped) pair
#   uncertainty_sweep!      -> hh_process_windows' Wieneke statistics +
#                              hh_finalize_uncertainty
#   release_piv_engines!    -> nothing to release (the context's arena is
#                              reused by the next call)
# and run_piv_ensemble through _plane_accumulator / accumulate_planes! /
# ensemble_analyze! (hh_correlation_planes + hh_analyze_planes; the
# device-resident ensemble is run_piv_ensemble_b200 below).

# The library context of a workspace (one per PIVWorkspace, pooled like an
# engine), or of the process when run_piv gets no workspace.
const _DEFAULT_CTX = Ref{Union{Nothing,Context}}(nothing)
function _b200_context(workspace)
    if workspace === nothing
        _DEFAULT_CTX[] === nothing && (_DEFAULT_CTX[] = Context())
        return _DEFAULT_CTX[]
    end
    return pooled_engines(() -> Context(), workspace, (:b200_context,), 1)[1]
end

# A correlation engine: the pass configuration on a context. Every buffer is
# the context's (grown on demand), so engines are cheap and pure scratch.
struct _B200Engine
    ctx::Context
    params::PIVParameters
    desc::PassDesc
    apod::Matrix{Float32}
end

_correlation_apod(e::_B200Engine) = e.apod

piv_correlation_engines(::_B200Backend, workspace, params::PIVParameters, ::Type{T}, nchunks::Int) where {T} =
    pooled_engines(() -> _B200Engine(_b200_context(workspace), params, pass_desc(params),
                                     apodization_window(Float32, params.window_size, params.apodization)),
                   workspace, (:b200, T, params.correlation_method, params.window_size, params.search_area_size,
                               params.padding, params.apodization, max(params.n_peaks, 2)), nchunks)

release_piv_engines!(::_B200Backend, engines, workspace) = nothing

# The pair held by a context: after apply_predictor it is the deformed pair,
# resident on the device; engines correlate it in place.
struct _B200Pair <: AbstractMatrix{Float32}
    ctx::Context
    nr::Int
    nc::Int
end
Base.size(p::_B200Pair) = (p.nr, p.nc)
Base.getindex(::_B200Pair, ::Int, ::Int) =
    throw(ArgumentError("backend :b200 keeps the deformed images on the device"))

mutable struct _B200Deform
    ctx::Context
    imgsize::Dims{2}
    staged::Bool
end

_deform_context(::_B200Backend, workspace, itpA, itpB, imgsize::Dims{2}, ::Type{T}) where {T} =
    _B200Deform(_b200_context(workspace), imgsize, false)

function _stage!(ctx::Context, imgA::AbstractMatrix, imgB::AbstractMatrix)
    A = Matrix{Float32}(imgA)
    B = Matrix{Float32}(imgB)
    check(ccall((:hh_stage_pair, LIB), Int32, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int64, Int64),
                ctx.ptr, A, B, size(A, 1), size(A, 2)), ctx.ptr)
    return nothing
end

function apply_predictor(::_B200Backend, imgA::AbstractMatrix, imgB::AbstractMatrix, itpA, itpB, predictor,
                         x::AbstractVector, y::AbstractVector, ::Type{T}; ctx = nothing, kwargs...) where {T}
    ny, nx = length(y), length(x)
    predictor === nothing && return imgA, imgB, zeros(T, ny, nx), zeros(T, ny, nx)
    # direct calls without a deform context: the CPU deformation
    ctx === nothing && return apply_predictor(imgA, imgB, itpA, itpB, predictor, x, y, T; kwargs...)
    if !ctx.staged  # once per pair: upload and prefilter on the device
        _stage!(ctx.ctx, imgA, imgB)
        ctx.staged = true
    end
    px, py = predictor.x, predictor.y
    pu = Matrix{Float32}(predictor.u)
    pv = Matrix{Float32}(predictor.v)
    gny, gnx = size(pu)
    ysp = gny > 1 ? Float32(py[2] - py[1]) : 1.0f0
    xsp = gnx > 1 ? Float32(px[2] - px[1]) : 1.0f0
    yy = Vector{Float32}(y)
    xx = Vector{Float32}(x)
    nu = Matrix{Float32}(undef, ny, nx)
    nv = Matrix{Float32}(undef, ny, nx)
    check(ccall((:hh_apply_predictor, LIB), Int32,
                (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int32, Int32, Float32, Float32, Float32, Float32,
                 Ptr{Float32}, Int32, Ptr{Float32}, Int32, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}),
                ctx.ctx.ptr, pu, pv, gny, gnx, Float32(py[1]), ysp, Float32(px[1]), xsp, yy, ny, xx, nx, nu, nv,
                C_NULL, C_NULL), ctx.ctx.ptr)
    r = _B200Pair(ctx.ctx, ctx.imgsize...)
    return r, r, T.(nu), T.(nv)
end

# The pair an engine correlates: the context's resident (deformed) pair, or
# host images of a non-deforming pass, uploaded here.
function _engine_pair!(e::_B200Engine, imgA, imgB, mask)
    imgA isa _B200Pair || _stage!(e.ctx, imgA, imgB)
    if mask === nothing
        check(ccall((:hh_stage_mask, LIB), Int32, (Ptr{Cvoid}, Ptr{UInt8}), e.ctx.ptr, C_NULL), e.ctx.ptr)
    else
        M = Matrix{UInt8}(mask)
        check(ccall((:hh_stage_mask, LIB), Int32, (Ptr{Cvoid}, Ptr{UInt8}), e.ctx.ptr, M), e.ctx.ptr)
    end
    return nothing
end

_job_matrix(jobs) = Int32[j[k] for k in 1:4, j in jobs]  # 4 x njobs, 1-based (gi, gj, rs, cs)

function process_windows!(u, v, peak_ratio, correlation_moment, alt_u, alt_v, uncertainty_u, uncertainty_v, jobs,
                          imgA, imgB, params::PIVParameters, engine::_B200Engine,
                          mask::Union{Nothing,AbstractMatrix{Bool}} = nothing, planes = nothing)
    planes === nothing ||
        throw(ArgumentError("backend :b200 does not support correlation-plane storage yet; use backend = :cpu"))
    jobvec = jobs isa AbstractVector ? jobs : collect(jobs)
    njobs = length(jobvec)
    njobs == 0 && return nothing
    _engine_pair!(engine, imgA, imgB, mask)
    K = max(params.n_peaks, 2)
    J = _job_matrix(jobvec)
    out = Matrix{Float32}(undef, 5 + 2 * (K - 1), njobs)  # packed rows of src/ka_backend.jl:497-506
    want_uq = uncertainty_u !== nothing
    stats = want_uq ? Matrix{Float64}(undef, 2 * UQ_NSTATS, njobs) : nothing
    check(ccall((:hh_process_windows, LIB), Int32,
                (Ptr{Cvoid}, Ref{PassDesc}, Ptr{Int32}, Int64, Ptr{Float32}, Ptr{Int32}, Ptr{Float64}),
                engine.ctx.ptr, engine.desc, J, njobs, out, C_NULL,
                want_uq ? pointer(stats) : Ptr{Float64}(C_NULL)), engine.ctx.ptr)
    T = eltype(u)
    nalt = K - 1
    for m in 1:njobs
        gi, gj = jobvec[m][1], jobvec[m][2]
        u[gi, gj] = out[1, m]
        v[gi, gj] = out[2, m]
        peak_ratio[gi, gj] = out[3, m]
        correlation_moment[gi, gj] = out[4, m]
        if want_uq
            uncertainty_u[gi, gj] = finalize_uncertainty(T, view(stats, 1:UQ_NSTATS, m))
            uncertainty_v[gi, gj] = finalize_uncertainty(T, view(stats, (UQ_NSTATS + 1):(2 * UQ_NSTATS), m))
        end
        if alt_u !== nothing
            found = Int(out[5, m])
            for mm in 2:min(found, params.n_peaks)
                alt_u[gi, gj, mm - 1] = out[5 + (mm - 1), m]
                alt_v[gi, gj, mm - 1] = out[5 + nalt + (mm - 1), m]
            end
        end
    end
    return nothing
end

function uncertainty_sweep!(uncertainty_u, uncertainty_v, jobs, imgA, imgB, params::PIVParameters, apod, mask,
                            engine::_B200Engine)
    jobvec = jobs isa AbstractVector ? jobs : collect(jobs)
    njobs = length(jobvec)
    njobs == 0 && return nothing
    _engine_pair!(engine, imgA, imgB, mask)
    J = _job_matrix(jobvec)
    K = max(params.n_peaks, 2)
    out = Matrix{Float32}(undef, 5 + 2 * (K - 1), njobs)
    stats = Matrix{Float64}(undef, 2 * UQ_NSTATS, njobs)
    check(ccall((:hh_process_windows, LIB), Int32,
                (Ptr{Cvoid}, Ref{PassDesc}, Ptr{Int32}, Int64, Ptr{Float32}, Ptr{Int32}, Ptr{Float64}),
                engine.ctx.ptr, engine.desc, J, njobs, out, C_NULL, stats), engine.ctx.ptr)
    T = eltype(uncertainty_u)
    for m in 1:njobs
        gi, gj = jobvec[m][1], jobvec[m][2]
        uncertainty_u[gi, gj] = finalize_uncertainty(T, view(stats, 1:UQ_NSTATS, m))
        uncertainty_v[gi, gj] = finalize_uncertainty(T, view(stats, (UQ_NSTATS + 1):(2 * UQ_NSTATS), m))
    end
    return nothing
end

# Ensemble trio over the hook entry points: each pair's planes of a pass come
# back from hh_correlation_planes and are summed in pair order on the host
# (accum[j] .+= plane, src/ensemble.jl:317-343); the summed planes are
# analysed by hh_analyze_planes. run_piv_ensemble_b200 keeps the sums on the
# device instead.
struct _B200Planes
    sums::Array{Float32,3}  # (nr, nc, njobs)
end

function _plane_accumulator(engine::_B200Engine, params::PIVParameters, ::Type{T}, njobs::Int) where {T}
    f = params.padding ? 2 : 1
    return _B200Planes(zeros(Float32, f * params.search_area_size[1], f * params.search_area_size[2], njobs))
end
_uncertainty_accumulator(::_B200Engine, ::Type, njobs::Int) = zeros(Float64, 2 * UQ_NSTATS, njobs)
_uncertainty_scratch(::_B200Engine, ::Type) = nothing

function accumulate_planes!(acc::_B200Planes, jobrange::AbstractUnitRange, engine::_B200Engine, imgA, imgB, jobs,
                            params::PIVParameters, mask, uacc = nothing, uscratch = nothing)
    isempty(jobrange) && return nothing
    _engine_pair!(engine, imgA, imgB, mask)
    sub = jobs[jobrange]
    J = _job_matrix(sub)
    nr, nc = size(acc.sums, 1), size(acc.sums, 2)
    pl = Array{Float32,3}(undef, nr, nc, length(sub))
    check(ccall((:hh_correlation_planes, LIB), Int32,
                (Ptr{Cvoid}, Ref{PassDesc}, Ptr{Int32}, Int64, Ptr{Float32}),
                engine.ctx.ptr, engine.desc, J, length(sub), pl), engine.ctx.ptr)
    acc.sums[:, :, jobrange] .+= pl
    if uacc !== nothing
        K = max(params.n_peaks, 2)
        out = Matrix{Float32}(undef, 5 + 2 * (K - 1), length(sub))
        stats = Matrix{Float64}(undef, 2 * UQ_NSTATS, length(sub))
        check(ccall((:hh_process_windows, LIB), Int32,
                    (Ptr{Cvoid}, Ref{PassDesc}, Ptr{Int32}, Int64, Ptr{Float32}, Ptr{Int32}, Ptr{Float64}),
                    engine.ctx.ptr, engine.desc, J, length(sub), out, C_NULL, stats), engine.ctx.ptr)
        uacc[:, jobrange] .+= stats
    end
    return nothing
end

function ensemble_analyze!(acc::_B200Planes, engine::_B200Engine, u, v, peak_ratio, correlation_moment,
                           uncertainty_u, uncertainty_v, planes, alt_u, alt_v, jobs, params::PIVParameters, uacc)
    planes === nothing ||
        throw(ArgumentError("backend :b200 does not support correlation-plane storage yet; use backend = :cpu"))
    njobs = length(jobs)
    K = max(params.n_peaks, 2)
    nr, nc = size(acc.sums, 1), size(acc.sums, 2)
    out = Matrix{Float32}(undef, 5 + 2 * (K - 1), njobs)
    check(ccall((:hh_analyze_planes, LIB), Int32,
                (Ptr{Cvoid}, Ptr{Float32}, Int64, Int32, Int32, Int32, Int32, Int32, Ptr{Float32}, Ptr{Int32}),
                engine.ctx.ptr, acc.sums, njobs, nr, nc, params.n_peaks, params.peak_finder === :exclusion ? 1 : 0,
                SUBPIXEL[params.subpixel_method], out, C_NULL), engine.ctx.ptr)
    T = eltype(u)
    nalt = K - 1
    for (j, job) in enumerate(jobs)
        gi, gj = job[1], job[2]
        if alt_u !== nothing
            for m in 2:min(Int(out[5, j]), params.n_peaks)  # total = shared predictor + residual
                alt_u[gi, gj, m - 1] = u[gi, gj] + out[5 + (m - 1), j]
                alt_v[gi, gj, m - 1] = v[gi, gj] + out[5 + nalt + (m - 1), j]
            end
        end
        u[gi, gj] += out[1, j]
        v[gi, gj] += out[2, j]
        peak_ratio[gi, gj] = out[3, j]
        correlation_moment[gi, gj] = out[4, j]
        if uacc !== nothing
            uncertainty_u[gi, gj] = finalize_uncertainty(T, view(uacc, 1:UQ_NSTATS, j))
            uncertainty_v[gi, gj] = finalize_uncertainty(T, view(uacc, (UQ_NSTATS + 1):(2 * UQ_NSTATS), j))
        end
    end
    return nothing
end

# ---- ensemble (sum-of-correlation) PIV: hh_run_ensemble ------------------
# hh_batch_pair (include/hammerhead_b200.h), field for field.
struct BatchPair
    A::Ptr{Float32}
    B::Ptr{Float32}
    mask::Ptr{UInt8}
    nr::Int64
    nc::Int64
    schedule::Int32
    format::Int32   # 0: Float32 frames
end

# The reducer of a multi-process ensemble, called by the library once per pass
# with the device plane sums and FP64 uncertainty sums of this process's
# pairs; it must leave their sums over all processes in place (for example an
# MPI.Allreduce! on CuArrays wrapping the pointers), ordered on `stream`.
const _REDUCER = Ref{Any}(nothing)

function _reduce_trampoline(user::Ptr{Cvoid}, pass::Int32, planes::Ptr{Float32}, nplanes::Int64,
                            stats::Ptr{Float64}, nstats::Int64, stream::Ptr{Cvoid})::Int32
    try
        _REDUCER[](Int(pass), planes, Int(nplanes), stats, Int(nstats), stream)
        return Int32(0)
    catch err
        @error "ensemble reducer failed" exception = err
        return Int32(1)
    end
end

# run_piv_ensemble(pairs, passes; backend = :b200): Float32 frames of one size;
# `reducer(pass, planes, nplanes, stats, nstats, stream)` when the pairs of the
# ensemble are split over processes (all processes pass the same image size,
# passes, mask and options).
function run_piv_ensemble_b200(pairs::AbstractVector{<:Tuple{AbstractMatrix{<:Real},AbstractMatrix{<:Real}}},
                               passes::AbstractVector{PIVParameters};
                               predictor_smoothing::Bool = true,
                               mask::Union{Nothing,AbstractMatrix{Bool}} = nothing, mask_threshold::Real = 0.5,
                               reducer::Union{Nothing,Function} = nothing, ctx::Context = Context())
    _check_backend_params(_B200Backend(), passes)
    isempty(pairs) && throw(ArgumentError("pairs must not be empty"))
    frames = [(Matrix{Float32}(a), Matrix{Float32}(b)) for (a, b) in pairs]
    nr, nc = size(frames[1][1])
    for (a, b) in frames
        size(a) == size(b) == (nr, nc) ||
            throw(DimensionMismatch("all pairs must share the image size ($nr, $nc), got $(size(a)) and $(size(b))"))
    end
    M = mask === nothing ? C_NULL : Matrix{UInt8}(mask)
    final = last(passes)
    d = [pass_desc(p) for p in passes]
    ny, nx, nj = Ref{Int32}(0), Ref{Int32}(0), Ref{Int64}(0)
    check(ccall((:hh_pass_grid, LIB), Int32,
                (Int64, Int64, Ref{PassDesc}, Ptr{UInt8}, Float64, Ref{Int32}, Ref{Int32}, Ptr{Float32},
                 Ptr{Float32}, Ptr{UInt8}, Ptr{Int32}, Ref{Int64}),
                nr, nc, pass_desc(final), C_NULL, mask_threshold, ny, nx, C_NULL, C_NULL, C_NULL, C_NULL, nj))
    gy, gx = Int(ny[]), Int(nx[])
    x = Vector{Float32}(undef, gx); y = Vector{Float32}(undef, gy)
    f() = Matrix{Float32}(undef, gy, gx)
    u, v, ratio, moment, su, sv = f(), f(), f(), f(), f(), f()
    outl = Matrix{UInt8}(undef, gy, gx); gm = Matrix{UInt8}(undef, gy, gx)
    cb = @cfunction(_reduce_trampoline, Int32,
                    (Ptr{Cvoid}, Int32, Ptr{Float32}, Int64, Ptr{Float64}, Int64, Ptr{Cvoid}))
    GC.@preserve frames M x y u v ratio moment su sv outl gm begin
        bp = [BatchPair(pointer(a), pointer(b), C_NULL, nr, nc, 0, 0) for (a, b) in frames]
        res = Ref(Result(0, 0, pointer(x), pointer(y), pointer(u), pointer(v), pointer(ratio), pointer(moment),
                         pointer(su), pointer(sv), pointer(outl), pointer(gm)))
        if reducer !== nothing
            _REDUCER[] = reducer
            check(ccall((:hh_set_ensemble_reducer, LIB), Int32, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}),
                        ctx.ptr, cb, C_NULL), ctx.ptr)
        end
        try
            check(ccall((:hh_run_ensemble, LIB), Int32,
                        (Ptr{Cvoid}, Ptr{BatchPair}, Int32, Ptr{PassDesc}, Int32, Ptr{UInt8}, Float64, Int32, Int32,
                         Ref{Result}),
                        ctx.ptr, bp, length(bp), d, length(d), M, mask_threshold, predictor_smoothing, 0, res),
                  ctx.ptr)
        finally
            if reducer !== nothing
                ccall((:hh_set_ensemble_reducer, LIB), Int32, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}),
                      ctx.ptr, C_NULL, C_NULL)
                _REDUCER[] = nothing
            end
        end
    end
    return PIVResult(x, y, u, v, ratio, moment, su, sv, BitMatrix(outl .!= 0), BitMatrix(gm .!= 0), final)
end

# ---- autotuning of the correlation kernel's CTA shape ---------------------
# Times the shapes of every equal-area pass class of `passes` on the pair
# (imgA, imgB) and makes the fastest the context's choice; returns
# [(fft_size, window, variant, ms per shape)].
function autotune_b200!(ctx::Context, imgA::AbstractMatrix{<:Real}, imgB::AbstractMatrix{<:Real},
                        passes::AbstractVector{PIVParameters}; reps::Integer = 5)
    A = Matrix{Float32}(imgA)
    B = Matrix{Float32}(imgB)
    size(A) == size(B) || throw(DimensionMismatch("images must have the same size"))
    check(ccall((:hh_stage_pair, LIB), Int32, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int64, Int64),
                ctx.ptr, A, B, size(A, 1), size(A, 2)), ctx.ptr)
    out = Tuple{Int,Int,Int,Vector{Float32}}[]
    for p in passes
        p.search_area_size == p.window_size || continue
        w = p.window_size[1]
        n = p.padding ? 2w : w
        any(o -> o[1] == n && o[2] == w, out) && continue
        ms = zeros(Float32, 5)  # HH_CORR_VARIANTS
        best = Ref{Int32}(0)
        check(ccall((:hh_autotune_correlation, LIB), Int32,
                    (Ptr{Cvoid}, Ref{PassDesc}, Int32, Ptr{Float32}, Ref{Int32}),
                    ctx.ptr, pass_desc(p), reps, ms, best), ctx.ptr)
        push!(out, (n, w, Int(best[]), ms))
    end
    return out
end

# ---- differentiable correlation loss (hh_ncc_loss_grad) -------------------
# A staged pair on a context; P is (gny, gnx, 2) Float32 (u, v) on nodes
# y0 .+ ysp .* (0:gny-1), x0 .+ xsp .* (0:gnx-1).
struct StagedPair
    ctx::Context
    window::Int
    overlap::Int
end

function StagedPair(imgA::AbstractMatrix{<:Real}, imgB::AbstractMatrix{<:Real};
                    window::Integer = 16, overlap::Integer = 8, ctx::Context = Context())
    A = Matrix{Float32}(imgA)
    B = Matrix{Float32}(imgB)
    size(A) == size(B) || throw(DimensionMismatch("images must have the same size"))
    check(ccall((:hh_stage_pair, LIB), Int32, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int64, Int64),
                ctx.ptr, A, B, size(A, 1), size(A, 2)), ctx.ptr)
    return StagedPair(ctx, window, overlap)
end

function _ncc(sp::StagedPair, P::AbstractArray{<:Real,3}, grid::NTuple{4,Real}, want_grad::Bool)
    gny, gnx = size(P, 1), size(P, 2)
    Pf = vcat(vec(Float32.(P[:, :, 1])), vec(Float32.(P[:, :, 2])))  # u then v, column-major planes
    G = want_grad ? similar(Pf) : Float32[]
    L = Ref{Float64}(0)
    check(ccall((:hh_ncc_loss_grad, LIB), Int32,
                (Ptr{Cvoid}, Ptr{Float32}, Int32, Int32, Float32, Float32, Float32, Float32, Int32, Int32, Int32,
                 Ref{Float64}, Ptr{Float32}),
                sp.ctx.ptr, Pf, gny, gnx, grid..., sp.window, sp.overlap, 0, L,
                want_grad ? pointer(G) : Ptr{Float32}(C_NULL)), sp.ctx.ptr)
    return L[], want_grad ? reshape(G, gny, gnx, 2) : nothing
end

"L = -sum of zero-lag NCC over the loss windows of the pair deformed by P."
ncc_loss(sp::StagedPair, P::AbstractArray{<:Real,3}, grid::NTuple{4,Real}) = first(_ncc(sp, P, grid, false))

# The rrule: the adjoint gradient comes from the device in the same call as the loss.
function ChainRulesCore.rrule(::typeof(ncc_loss), sp::StagedPair, P::AbstractArray{<:Real,3}, grid::NTuple{4,Real})
    L, G = _ncc(sp, P, grid, true)
    pullback(dL) = (NoTangent(), NoTangent(), unthunk(dL) .* G, NoTangent())
    return L, pullback
end

end # module
