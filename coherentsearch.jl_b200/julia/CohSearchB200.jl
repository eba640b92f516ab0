# CohSearchB200.jl -- Julia binding of libcohsearch_cuda.so (include/cohsearch.h).
#
# Drop-in device dispatch for CoherentSearch.jl: `device_search_region` has the
# inputs and result of `_search_region!` (src/search.jl:1768-1894), and
# `device_chunk_metrics` those of `chunk_metrics` (src/search.jl:1740-1755).
# A maintainer wires them in as shown in INTEGRATION.md.  No Julia is
# installed where this library is built, so this file is exercised through
# the identical C ABI by the Python binding (coherentsearch.jl_b200/cohsearch).
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

end # module
