# CohSearchB200.jl -- Julia binding of libcohsearch_cuda.so (include/cohsearch.h).
#
# Drop-in device dispatch for CoherentSearch.jl: `device_search_region` has the
# inputs and result of `_search_region!` (src/search.jl:1768-1894),
# `device_chunk_metrics` those of `chunk_metrics` (src/search.jl:1740-1755);
# then block ranges (`device_search_range`), the batch over files
# (`device_search_batch`, `set_batch_graph!`), `block_metrics`
# (`device_block_metrics`), `candidate_profile` / `measure_ducy`
# (`device_refold`) and MetricStats / MetricNorm (`set_metricstats!`,
# `block_stats`, `metric_hists`, `set_metricnorm!`).  In `search`
# (src/search.jl:2080-2094) the detection pass's `_search_region!` call becomes
# `set_spectrum!` + `device_search_region` on a handle cached per params.  No
# Julia is installed where this library is built: a host test checks every
# ccall against include/cohsearch.h, and the same C calls run through the
# Python binding (coherentsearch.jl_b200/cohsearch).
module CohSearchB200

const LIB = joinpath(@__DIR__, "..", "lib", "libcohsearch_cuda.so")

const CS_OK = Int32(0)
const CS_ERR_INVALID_ARGUMENT = Int32(1)
const CS_ERR_CAPACITY = Int32(3)
const CS_MAX_DECIM = 16

struct CSParams
    nharms::Int32
    m::Int32
    numbetween::Int32
    ndecim::Int32
    decimations::NTuple{16,Int32}
    hidr::Float64
    threshold::Float64
    boxcar_fsp::Float64
    boxcar_maxfrac::Float64
    boxcar_medmargin::Float64
    precision::Int32
    synth::Int32
end

struct CSCandidate
    freq::Float64
    metric::Float64
    r::Float64
    nharm::Int32
    k::Int32
    trial::Int64
end

# synth: 0 = plain FP32, 1 = BF16 tensor cores, 2 = FP16 tensor cores,
# 3 / 4 = BF16 / FP16 with each amplitude split hi + lo into two operands.
function CSParams(p; synth::Integer=2)
    d = ntuple(i -> i <= length(p.decimations) ? Int32(p.decimations[i]) : Int32(0), 16)
    CSParams(p.nharms, p.m, p.numbetween, length(p.decimations), d, p.hidr, p.threshold,
             p.boxcar_fsp, p.boxcar_maxfrac, p.boxcar_medmargin,
             p.precision === :f64 ? 0 : 1, synth)
end

mutable struct Handle
    ptr::Ptr{Cvoid}
end

function check(st::Int32, h::Ptr{Cvoid})
    st == CS_OK && return
    msg = h == C_NULL ? "" : unsafe_string(ccall((:cs_last_error, LIB), Cstring, (Ptr{Cvoid},), h))
    st == CS_ERR_INVALID_ARGUMENT && throw(ArgumentError(msg))
    error("libcohsearch_cuda status $st: $msg")
end

function Handle(params; device::Integer=0, synth::Integer=2)
    ref = Ref{Ptr{Cvoid}}(C_NULL)
    cp = Ref(CSParams(params; synth=synth))
    check(ccall((:cs_create, LIB), Int32, (Ref{Ptr{Cvoid}}, Ref{CSParams}, Int32), ref, cp, device), C_NULL)
    h = Handle(ref[])
    finalizer(x -> ccall((:cs_destroy, LIB), Int32, (Ptr{Cvoid},), x.ptr), h)
    return h
end

# The FFTFile's mmapped amplitudes go straight to the library (copied to HBM).
function set_spectrum!(h::Handle, amps::Vector{ComplexF32}, N::Integer, dt::Real)
    check(ccall((:cs_set_spectrum, LIB), Int32, (Ptr{Cvoid}, Ptr{ComplexF32}, Int64, Int64, Float64),
                h.ptr, amps, length(amps), N, dt), h.ptr)
end

# Raw detections (freq, metric, r, nharm) as `_search_region!` returns them.
function device_search_region(h::Handle; lofreq, hifreq, lobin=100, blocksize=2048, threshold,
                              exact_all=false)
    cap = 1 << 16
    while true
        out = Vector{CSCandidate}(undef, cap)
        n = Ref{Int64}(0)
        st = ccall((:cs_search, LIB), Int32,
                   (Ptr{Cvoid}, Float64, Float64, Int64, Int64, Float64, Int32, Ptr{CSCandidate}, Int64, Ref{Int64}),
                   h.ptr, lofreq, hifreq, lobin, blocksize, threshold, exact_all, out, cap, n)
        if st == CS_ERR_CAPACITY && n[] > cap
            cap = Int(n[])
            continue
        end
        check(st, h.ptr)
        return out[1:n[]]
    end
end

function device_chunk_metrics(h::Handle, rstart::Real, n::Integer)
    out = Vector{Float64}(undef, n)
    check(ccall((:cs_chunk_metrics, LIB), Int32, (Ptr{Cvoid}, Float64, Int64, Ptr{Float64}),
                h.ptr, rstart, n, out), h.ptr)
    return out
end

# `_search_region!` over blocks [block_begin, block_end) of the band's grid
# (0-based; block_end < 0: through the last block): one GPU's share of a
# sharded band, with trial indices global to the band (cs_search_range).
function device_search_range(h::Handle; lofreq, hifreq, lobin=100, blocksize=2048, threshold,
                             block_begin::Integer, block_end::Integer=-1, exact_all=false)
    cap = 1 << 16
    while true
        out = Vector{CSCandidate}(undef, cap)
        n = Ref{Int64}(0)
        st = ccall((:cs_search_range, LIB), Int32,
                   (Ptr{Cvoid}, Float64, Float64, Int64, Int64, Float64, Int32, Int64, Int64,
                    Ptr{CSCandidate}, Int64, Ref{Int64}),
                   h.ptr, lofreq, hifreq, lobin, blocksize, threshold, exact_all, block_begin, block_end,
                   out, cap, n)
        if st == CS_ERR_CAPACITY && n[] > cap
            cap = Int(n[])
            continue
        end
        check(st, h.ptr)
        return out[1:n[]]
    end
end

struct CSSpectrum
    amps::Ptr{Float32}
    namps::Int64
    N::Int64
    dt::Float64
end

# `search_one` over many spectra with one handle (a DM sweep, src/cli.jl:237-289;
# cs_search_batch).  files: (amps, N, dt) with amps a Vector{ComplexF32} in host
# memory (pinned for full copy/compute overlap), or with on_device=true
# ((device pointer, namps), N, dt), e.g. from a CUDA.jl CuArray.  Returns the
# candidates and, per candidate, the 1-based index of its spectrum.
function device_search_batch(h::Handle, files; lofreq, hifreq, lobin=100, blocksize=2048, threshold,
                             on_device::Bool=false)
    specs = Vector{CSSpectrum}(undef, length(files))
    for (i, f) in enumerate(files)
        if on_device
            (ptr, namps), N, dt = f
            specs[i] = CSSpectrum(Ptr{Float32}(UInt(ptr)), namps, N, dt)
        else
            amps, N, dt = f
            specs[i] = CSSpectrum(Ptr{Float32}(pointer(amps)), length(amps), N, dt)
        end
    end
    cap = 1 << 18
    GC.@preserve files begin
        while true
            out = Vector{CSCandidate}(undef, cap)
            owner = Vector{Int32}(undef, cap)
            n = Ref{Int64}(0)
            st = ccall((:cs_search_batch, LIB), Int32,
                       (Ptr{Cvoid}, Ptr{CSSpectrum}, Int32, Int32, Float64, Float64, Int64, Int64, Float64,
                        Ptr{CSCandidate}, Ptr{Int32}, Int64, Ref{Int64}),
                       h.ptr, specs, length(specs), on_device, lofreq, hifreq, lobin, blocksize, threshold,
                       out, owner, cap, n)
            if st == CS_ERR_CAPACITY && n[] > cap
                cap = Int(n[])
                continue
            end
            check(st, h.ptr)
            return out[1:n[]], owner[1:n[]] .+ 1
        end
    end
end

# Replay a repeated batch of device spectra from one captured CUDA graph
# (cs_set_batch_graph; refill the spectra in place between calls).
set_batch_graph!(h::Handle, enable::Bool=true) =
    check(ccall((:cs_set_batch_graph, LIB), Int32, (Ptr{Cvoid}, Int32), h.ptr, enable), h.ptr)

# `block_metrics(ft, rfund, params; kernel, widths)` (src/search.jl:1061-1079) on
# the device: the coherent-fold S/N at arbitrary trial fundamentals (bins,
# ascending), FP64 throughout; widths empty: the base pass's ladder bank.
function device_block_metrics(h::Handle, rfund::AbstractVector{<:Real}; kernel::Symbol=:fft, widths=Int32[])
    kernel in (:fft, :direct) || throw(ArgumentError("kernel must be :fft or :direct"))
    r = Vector{Float64}(rfund)
    w = Vector{Int32}(widths)
    out = Vector{Float64}(undef, length(r))
    check(ccall((:cs_block_metrics, LIB), Int32,
                (Ptr{Cvoid}, Ptr{Float64}, Int64, Int32, Ptr{Int32}, Int32, Ptr{Float64}),
                h.ptr, r, length(r), kernel === :direct ? 1 : 0, w, length(w), out), h.ptr)
    return out
end

# `candidate_profile` / `measure_ducy` (src/candidate.jl:37-99) for many
# candidates: per candidate the harmonics used (-1: no profile, duty cycle NaN),
# the normalised profile (2H bins; two zero bins for H = 0) and the duty cycle.
function device_refold(h::Handle, r::AbstractVector{<:Real}, nharm::AbstractVector{<:Integer}; m::Integer=64)
    n = length(r)
    length(nharm) == n || throw(ArgumentError("r and nharm differ in length"))
    rr = Vector{Float64}(r)
    nh = Vector{Int32}(nharm)
    H = Vector{Int32}(undef, n)
    prof = Vector{Float64}(undef, 256 * n)
    ducy = Vector{Float64}(undef, n)
    check(ccall((:cs_refold, LIB), Int32,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int32}, Int64, Int32, Ptr{Int32}, Ptr{Float64}, Ptr{Float64}),
                h.ptr, rr, nh, n, m, H, prof, ducy), h.ptr)
    profiles = [H[i] < 0 ? Float64[] : prof[(i - 1) * 256 + 1:(i - 1) * 256 + max(2 * Int(H[i]), 2)] for i in 1:n]
    return H, profiles, ducy
end

# BlockMetricStats record (src/search.jl:1321-1335); block is 1-based.
struct CSBlockStats
    block::Int64
    k::Int32
    Hk::Int32
    nbins::Int32
    pad::Int32
    ngoodbins::Float64
    flo::Float64
    fhi::Float64
    n::Int64
    min::Float64
    median::Float64
    mean::Float64
    std::Float64
    max::Float64
end

# MetricStats collection for the following searches (every trial scored
# exactly; candidates unchanged), with the reference's histogram defaults.
set_metricstats!(h::Handle; enable::Bool=true, hist_lo=0.0, hist_hi=64.0, hist_nb=3200, nwin=16) =
    check(ccall((:cs_set_metricstats, LIB), Int32, (Ptr{Cvoid}, Int32, Float64, Float64, Int32, Int32),
                h.ptr, enable, hist_lo, hist_hi, hist_nb, nwin), h.ptr)

# The last search's BlockMetricStats records, sorted by (block, k).
function block_stats(h::Handle)
    n = Ref{Int64}(0)
    st = ccall((:cs_get_block_stats, LIB), Int32, (Ptr{Cvoid}, Ptr{CSBlockStats}, Int64, Ref{Int64}),
               h.ptr, Ptr{CSBlockStats}(C_NULL), 0, n)
    st == CS_OK || st == CS_ERR_CAPACITY || check(st, h.ptr)
    out = Vector{CSBlockStats}(undef, n[])
    check(ccall((:cs_get_block_stats, LIB), Int32, (Ptr{Cvoid}, Ptr{CSBlockStats}, Int64, Ref{Int64}),
                h.ptr, out, length(out), n), h.ptr)
    return out
end

# The last search's per-(k, window) MetricHistograms: ks; edges (nwin+1, nlev)
# in Hz; counts (nb, nwin, nlev); moments (7, nwin, nlev) = under, over, total,
# sum, sumsq, vmin, vmax (the C arrays' row-major layout, read column-major).
function metric_hists(h::Handle)
    nlev, nwin, nb = Ref{Int32}(0), Ref{Int32}(0), Ref{Int32}(0)
    check(ccall((:cs_get_metric_hists, LIB), Int32,
                (Ptr{Cvoid}, Ref{Int32}, Ref{Int32}, Ref{Int32}, Ptr{Int32}, Ptr{Float64}, Ptr{Int64}, Ptr{Float64}),
                h.ptr, nlev, nwin, nb,
                Ptr{Int32}(C_NULL), Ptr{Float64}(C_NULL), Ptr{Int64}(C_NULL), Ptr{Float64}(C_NULL)), h.ptr)
    L, W, B = Int(nlev[]), Int(nwin[]), Int(nb[])
    ks = Vector{Int32}(undef, L)
    edges = Matrix{Float64}(undef, W + 1, L)
    counts = Array{Int64}(undef, B, W, L)
    moments = Array{Float64}(undef, 7, W, L)
    check(ccall((:cs_get_metric_hists, LIB), Int32,
                (Ptr{Cvoid}, Ref{Int32}, Ref{Int32}, Ref{Int32}, Ptr{Int32}, Ptr{Float64}, Ptr{Int64}, Ptr{Float64}),
                h.ptr, nlev, nwin, nb, ks, edges, counts, moments), h.ptr)
    return ks, edges, counts, moments
end

# MetricNorm for the following searches (build_metricnorm's result): per
# decimation ks[i], window edges edges[:, i] (Hz, nwin+1) and loc/scale[:, i]
# (nwin); a trial is a candidate when (M - loc) / scale > threshold.
# Empty ks clears it.
function set_metricnorm!(h::Handle, ks::AbstractVector{<:Integer}, edges::AbstractMatrix{<:Real},
                         loc::AbstractMatrix{<:Real}, scale::AbstractMatrix{<:Real})
    L = length(ks)
    W = L == 0 ? 0 : size(loc, 1)
    (L == 0 || (size(edges) == (W + 1, L) && size(loc) == (W, L) && size(scale) == (W, L))) ||
        throw(ArgumentError("edges must be (nwin+1, nlev), loc and scale (nwin, nlev)"))
    check(ccall((:cs_set_metricnorm, LIB), Int32,
                (Ptr{Cvoid}, Int32, Int32, Ptr{Int32}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                h.ptr, L, W, Vector{Int32}(ks), Matrix{Float64}(edges), Matrix{Float64}(loc),
                Matrix{Float64}(scale)), h.ptr)
end

end # module
