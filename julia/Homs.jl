# Homs.jl -- the Julia side of libhoms for HighOrderMRISim.jl.
#
# A maintainer adds this file as src/simulation/kernels/Homs.jl, includes it
# from src/HighOrderMRISim.jl, and adds one branch to simulate_shard
# (src/simulation/Simulate.jl:158-172), beside the array path and the CUDA
# kernel path:
#
#     elseif params["implementation"] == "homs"
#         Homs.run_shard!(obj, hoseqd, sig, Xt, params["sim_method"], parts, excitation_bool;
#                         split = get(params, "homs_precision", "plain") == "split")
#
# Discretisation, get_sim_ranges, initialize_spins_state, the ADC phase
# compensation and the mat/state/raw shaping stay in Julia; only the block
# loop (run_sim_time_iter!, SimulatorCore.jl:96-152) moves into libhoms.
#
# Every struct below mirrors one of include/homs.h field for field (same
# names, order and C types); tests/test_julia_shim.py checks their offsets
# and sizes against the C header.
module Homs

using CUDA

const libhoms = get(ENV, "HOMS_LIBRARY", "libhoms.so")

const HOMS_OK, HOMS_EINVAL, HOMS_ENOMEM, HOMS_EUNSUPPORTED = Cint(0), Cint(1), Cint(2), Cint(3)
const HOMS_ETIMEDOUT, HOMS_ECUDA, HOMS_ECLOSED, HOMS_EBUSY = Cint(4), Cint(5), Cint(6), Cint(7)
const HOMS_F32, HOMS_F64 = Cint(0), Cint(1)
const HOMS_HOST, HOMS_DEVICE = Cint(0), Cint(1)
const HOMS_PLAIN, HOMS_SPLIT = Cint(0), Cint(1)

struct HomsPhantom  # include/homs.h: homs_phantom
    nspins::Int64
    ncoils::Int32
    dtype::Cint
    memory::Cint
    x::Ptr{Cvoid}
    y::Ptr{Cvoid}
    z::Ptr{Cvoid}
    rho::Ptr{Cvoid}
    T1::Ptr{Cvoid}
    T2::Ptr{Cvoid}
    dw::Ptr{Cvoid}
    csm::Ptr{Cvoid}
end

struct HomsSequence  # include/homs.h: homs_sequence
    nnodes::Int64
    dtype::Cint
    memory::Cint
    t::Ptr{Cvoid}
    dt::Ptr{Cvoid}
    gx::Ptr{Cvoid}
    gy::Ptr{Cvoid}
    gz::Ptr{Cvoid}
    b1::Ptr{Cvoid}
    df::Ptr{Cvoid}
    psi::Ptr{Cvoid}
    adc::Ptr{UInt8}
    h::NTuple{16,Ptr{Cvoid}}
    nblocks::Int32
    block_first::Ptr{Int64}
    block_last::Ptr{Int64}
    block_excitation::Ptr{UInt8}
    gamma::Float64
end

struct HomsRunOptions  # include/homs.h: homs_run_options
    method::UInt32
    mode::Cint
    reserved::NTuple{6,Int32}
end

struct HomsState  # include/homs.h: homs_state
    xy::Ptr{Cvoid}
    z::Ptr{Cvoid}
    memory::Cint
end

struct HomsTiming  # include/homs.h: homs_timing
    fused_kernel_ms::Float64
    fused_launches::Int64
    kernel_launches::Int64
end

struct HomsBrainSpec  # include/homs.h: homs_brain_spec
    nx::Int64
    ny::Int64
    nz::Int64
    res::NTuple{3,Float64}
    offcenter::NTuple{3,Float64}
    fieldstrength::Int32
    ncoils::Int32
    memory::Cint
    labels::Ptr{UInt8}
    fieldmap::Ptr{Float64}
    csm::Ptr{Float64}
end

struct HomsBrainOut  # include/homs.h: homs_brain_out
    nspins::Int64
    memory::Cint
    x::Ptr{Float64}
    y::Ptr{Float64}
    z::Ptr{Float64}
    rho::Ptr{Float64}
    T1::Ptr{Float64}
    T2::Ptr{Float64}
    T2s::Ptr{Float64}
    dw::Ptr{Float64}
    csm::Ptr{Float64}
end

struct HomsServerOptions  # include/homs.h: homs_server_options
    device::Cint
    slots::Int32
    max_device_bytes::Int64
    reserved::NTuple{4,Int32}
end

struct HomsRequestTimes  # include/homs.h: homs_request_times
    submitted::Float64
    started::Float64
    finished::Float64
end

# BlochHighOrder(mask) and its Δw flags as the ABI's method word
# (src/simulation/BlochHighOrder.jl:21-43).
homs_flags(m) = UInt32(m.ho0) | UInt32(m.ho1) << 1 | UInt32(m.ho2) << 2 | UInt32(m.ho3) << 3 |
                UInt32(m.Δw_excitation) << 4 | UInt32(m.Δw_precession) << 5

# Status -> exception, with the reference's error types (Simulate.jl:74-99).
function homs_check(st::Integer, ctx::Ptr{Cvoid})
    st == HOMS_OK && return nothing
    msg = ctx == C_NULL ? unsafe_string(ccall((:homs_status_string, libhoms), Cstring, (Cint,), st)) :
          unsafe_string(ccall((:homs_last_error, libhoms), Cstring, (Ptr{Cvoid},), ctx))
    st == HOMS_EINVAL ? throw(ArgumentError(msg)) : error("libhoms: " * msg)
end

devptr(a) = Ptr{Cvoid}(UInt(pointer(a)))

# One context per device and stream, created on first use.
const CONTEXTS = Dict{Tuple{Int,UInt},Ptr{Cvoid}}()
function context()
    dev = CUDA.deviceid(CUDA.device())
    stream = CUDA.stream().handle
    get!(CONTEXTS, (dev, UInt(stream))) do
        ctx = Ref{Ptr{Cvoid}}(C_NULL)
        homs_check(ccall((:homs_context_create, libhoms), Cint, (Cint, Ptr{Cvoid}, Ref{Ptr{Cvoid}}),
                         dev, stream, ctx), C_NULL)
        ctx[]
    end
end

# The whole block loop of one shard on libhoms: the obj, hoseqd, sig and Xt of
# simulate_shard are already on the device (CuArrays).  `parts` are Julia
# UnitRanges over nodes; the ABI takes 0-based inclusive pairs, and the ADC of
# a node shared by two blocks belongs to the earlier one (SimulatorCore.jl:115-118).
function run_shard!(obj, hoseqd, sig, Xt, sim_method, parts, excitation_bool; split::Bool=false)
    T = eltype(obj.x)
    dt = T === Float64 ? HOMS_F64 : HOMS_F32
    s = hoseqd.seqd
    first_ = Int64[first(r) - 1 for r in parts]
    last_ = Int64[last(r) - 1 for r in parts]
    exc = UInt8.(excitation_bool)
    adc = CuArray{UInt8}(s.ADC)
    GC.@preserve obj hoseqd sig Xt first_ last_ exc adc begin
        ph = HomsPhantom(length(obj), size(obj.csm, 2), dt, HOMS_DEVICE, devptr(obj.x), devptr(obj.y),
                         devptr(obj.z), devptr(obj.ρ), devptr(obj.T1), devptr(obj.T2), devptr(obj.Δw),
                         devptr(obj.csm))
        sq = HomsSequence(length(s.t), dt, HOMS_DEVICE, devptr(s.t), devptr(s.Δt), devptr(s.Gx), devptr(s.Gy),
                          devptr(s.Gz), devptr(s.B1), devptr(s.Δf), devptr(s.ϕ), Ptr{UInt8}(UInt(pointer(adc))),
                          ntuple(k -> devptr(getfield(hoseqd, k + 1)), 16), Int32(length(parts)),
                          pointer(first_), pointer(last_), pointer(exc), Float64(γ))
        opts = HomsRunOptions(homs_flags(sim_method), split ? HOMS_SPLIT : HOMS_PLAIN, ntuple(_ -> Int32(0), 6))
        state = HomsState(devptr(Xt.xy), devptr(Xt.z), HOMS_DEVICE)
        ctx = context()
        homs_check(ccall((:homs_simulate, libhoms), Cint,
                         (Ptr{Cvoid}, Ref{HomsPhantom}, Ref{HomsSequence}, Ref{HomsRunOptions}, Ref{HomsState},
                          Ptr{Cvoid}, Cint),
                         ctx, ph, sq, opts, state, devptr(sig), HOMS_DEVICE), ctx)
    end
    return sig
end

# PreparedSimulation (PreparedSimulation.jl:144-258) on libhoms: inputs copied
# to the device once; each run restarts from Mxy = 0, Mz = rho.
mutable struct HomsPlan
    handle::Ptr{Cvoid}
    ctx::Ptr{Cvoid}
end

function prepare(ph::HomsPhantom, sq::HomsSequence, opts::HomsRunOptions)
    ctx = context()
    h = Ref{Ptr{Cvoid}}(C_NULL)
    homs_check(ccall((:homs_plan_create, libhoms), Cint,
                     (Ptr{Cvoid}, Ref{HomsPhantom}, Ref{HomsSequence}, Ref{HomsRunOptions}, Ref{Ptr{Cvoid}}),
                     ctx, ph, sq, opts, h), ctx)
    plan = HomsPlan(h[], ctx)
    finalizer(p -> p.handle == C_NULL || ccall((:homs_plan_destroy, libhoms), Cint, (Ptr{Cvoid},), p.handle), plan)
    return plan
end

function run!(plan::HomsPlan, sig; memory::Cint=HOMS_DEVICE)
    homs_check(ccall((:homs_plan_run, libhoms), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Cvoid}),
                     plan.handle, devptr(sig), memory, C_NULL), plan.ctx)
    return sig
end

function timing(plan::HomsPlan)
    t = Ref{HomsTiming}()
    homs_check(ccall((:homs_plan_timing, libhoms), Cint, (Ptr{Cvoid}, Ref{HomsTiming}), plan.handle, t), plan.ctx)
    return t[]
end

# A phantom kept on the device for many simulations (its arrays and, in split
# mode, its digit operands built once).
mutable struct HomsResident
    handle::Ptr{Cvoid}
    ctx::Ptr{Cvoid}
end

function resident(ph::HomsPhantom, mode::Cint)
    ctx = context()
    h = Ref{Ptr{Cvoid}}(C_NULL)
    homs_check(ccall((:homs_resident_create, libhoms), Cint,
                     (Ptr{Cvoid}, Ref{HomsPhantom}, Cint, Ref{Ptr{Cvoid}}), ctx, ph, mode, h), ctx)
    res = HomsResident(h[], ctx)
    finalizer(r -> r.handle == C_NULL || ccall((:homs_resident_destroy, libhoms), Cint, (Ptr{Cvoid},), r.handle),
              res)
    return res
end

function simulate_resident!(res::HomsResident, sq::HomsSequence, opts::HomsRunOptions, state::HomsState, sig;
                            memory::Cint=HOMS_DEVICE)
    homs_check(ccall((:homs_simulate_resident, libhoms), Cint,
                     (Ptr{Cvoid}, Ptr{Cvoid}, Ref{HomsSequence}, Ref{HomsRunOptions}, Ref{HomsState}, Ptr{Cvoid},
                      Cint), res.ctx, res.handle, sq, opts, state, devptr(sig), memory), res.ctx)
    return sig
end

# The serving loop: simulations queued from any task, run by `slots` workers
# (split-mode requests share one persistent kernel launch per round).  The
# arrays behind a request must stay alive until its ticket has finished.
mutable struct HomsServer
    handle::Ptr{Cvoid}
end

function server(; device::Integer=CUDA.deviceid(CUDA.device()), slots::Integer=4, max_device_bytes::Integer=0)
    opts = HomsServerOptions(Cint(device), Int32(slots), Int64(max_device_bytes), ntuple(_ -> Int32(0), 4))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    homs_check(ccall((:homs_server_create, libhoms), Cint, (Ref{HomsServerOptions}, Ref{Ptr{Cvoid}}), opts, h),
               C_NULL)
    srv = HomsServer(h[])
    finalizer(s -> s.handle == C_NULL || ccall((:homs_server_destroy, libhoms), Cint, (Ptr{Cvoid},), s.handle), srv)
    return srv
end

function server_check(srv::HomsServer, st::Integer, ticket::Int64)
    st == HOMS_OK && return nothing
    msg = unsafe_string(ccall((:homs_server_error, libhoms), Cstring, (Ptr{Cvoid}, Int64), srv.handle, ticket))
    st == HOMS_EINVAL ? throw(ArgumentError(msg)) : error("libhoms: " * msg)
end

function submit!(srv::HomsServer, ph::HomsPhantom, sq::HomsSequence, opts::HomsRunOptions, state::HomsState,
                 sig::Ptr{Cvoid}, memory::Cint)
    t = Ref{Int64}(0)
    homs_check(ccall((:homs_server_submit, libhoms), Cint,
                     (Ptr{Cvoid}, Ref{HomsPhantom}, Ref{HomsSequence}, Ref{HomsRunOptions}, Ref{HomsState},
                      Ptr{Cvoid}, Cint, Ref{Int64}), srv.handle, ph, sq, opts, state, sig, memory, t), C_NULL)
    return t[]
end

function submit!(srv::HomsServer, res::HomsResident, sq::HomsSequence, opts::HomsRunOptions, state::HomsState,
                 sig::Ptr{Cvoid}, memory::Cint)
    t = Ref{Int64}(0)
    homs_check(ccall((:homs_server_submit_resident, libhoms), Cint,
                     (Ptr{Cvoid}, Ptr{Cvoid}, Ref{HomsSequence}, Ref{HomsRunOptions}, Ref{HomsState}, Ptr{Cvoid},
                      Cint, Ref{Int64}), srv.handle, res.handle, sq, opts, state, sig, memory, t), C_NULL)
    return t[]
end

finished(srv::HomsServer, ticket::Int64) =
    ccall((:homs_server_poll, libhoms), Cint, (Ptr{Cvoid}, Int64), srv.handle, ticket) != HOMS_EBUSY

function wait!(srv::HomsServer, ticket::Int64; timeout::Real=600.0)
    st = ccall((:homs_server_wait, libhoms), Cint, (Ptr{Cvoid}, Int64, Cdouble), srv.handle, ticket, timeout)
    server_check(srv, st, ticket)
end

function times(srv::HomsServer, ticket::Int64)
    t = Ref{HomsRequestTimes}()
    server_check(srv, ccall((:homs_server_times, libhoms), Cint, (Ptr{Cvoid}, Int64, Ref{HomsRequestTimes}),
                            srv.handle, ticket, t), ticket)
    return t[]
end

function estimate(srv::HomsServer, ticket::Int64)
    b = Ref{Int64}(0)
    server_check(srv, ccall((:homs_server_estimate, libhoms), Cint, (Ptr{Cvoid}, Int64, Ref{Int64}),
                            srv.handle, ticket, b), ticket)
    return b[]
end

release!(srv::HomsServer, ticket::Int64) =
    ccall((:homs_server_release, libhoms), Cint, (Ptr{Cvoid}, Int64), srv.handle, ticket)

# get_kspace (src/datatypes/HO_Sequence.jl:236-287) on the device: k at every
# interval (nnodes - 1 x 19, column-major: gx, gy, gz, h0..h15) and at the
# query times (nq x 19).  rf_start / rf_sign are the RF breaks and their part
# signs, as KomaMRIBase's get_RF_types gives them.
function kspace!(sq::HomsSequence, rf_start::Vector{Int64}, rf_sign::Vector{Int8}, q_times, k, k_q;
                 memory::Cint=HOMS_DEVICE)
    ctx = context()
    GC.@preserve rf_start rf_sign q_times k k_q begin
        homs_check(ccall((:homs_kspace, libhoms), Cint,
                         (Ptr{Cvoid}, Ref{HomsSequence}, Int32, Ptr{Int64}, Ptr{Int8}, Int64, Ptr{Cvoid}, Ptr{Cvoid},
                          Ptr{Cvoid}, Cint),
                         ctx, sq, Int32(length(rf_start)), pointer(rf_start), pointer(rf_sign), Int64(length(q_times)),
                         devptr(q_times), devptr(k), devptr(k_q), memory), ctx)
    end
    return k, k_q
end

# hophantom_brain's spin arrays from a class volume (src/phantom/hophantom_brain.jl:2-58):
# the count first, then the arrays into the caller's buffers.
function brain_phantom_count(spec::HomsBrainSpec)
    ctx = context()
    n = Ref{Int64}(0)
    homs_check(ccall((:homs_brain_phantom_count, libhoms), Cint, (Ptr{Cvoid}, Ref{HomsBrainSpec}, Ref{Int64}),
                     ctx, spec, n), ctx)
    return n[]
end

function brain_phantom_fill!(spec::HomsBrainSpec, out::HomsBrainOut)
    ctx = context()
    homs_check(ccall((:homs_brain_phantom_fill, libhoms), Cint, (Ptr{Cvoid}, Ref{HomsBrainSpec}, Ref{HomsBrainOut}),
                     ctx, spec, out), ctx)
    return out
end

# csm_Birdcage (src/phantom/csm/Birdcage.jl:21-42): nx x ny x ncoils complex.
function csm_birdcage!(out, nx::Integer, ny::Integer, ncoils::Integer, relative_radius::Real;
                       memory::Cint=HOMS_DEVICE)
    ctx = context()
    homs_check(ccall((:homs_csm_birdcage, libhoms), Cint,
                     (Ptr{Cvoid}, Int64, Int64, Int32, Cdouble, Ptr{Cvoid}, Cint),
                     ctx, Int64(nx), Int64(ny), Int32(ncoils), Float64(relative_radius), devptr(out), memory), ctx)
    return out
end

end  # module Homs
